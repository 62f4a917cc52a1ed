"""Output module ``local`` (igm/outputs/local.py:8-196; the field list and the
``(time, y, x)`` / ``(time, z, y, x)`` layout of igm/outputs/write_ncdf.py:
60-140): at every save time (``state.saveresult``) the fields listed in
``cfg.outputs.local.vars_to_save`` go to ``output_file`` and, with
``write_ts``, the ice volume (km^3) and glaciated area (km^2, thk > 1 m) to
``output_ts_file``.

Same module API as the reference (initialize(cfg, state), run(cfg, state)),
same variable names, long names and units, and the same derived magnitudes
(``velbar_mag``, ``velsurf_mag``, ``velbase_mag``, the Euclidean norm of
getmag, igm/utils/math/getmag.py).  The files are netCDF-3 (64-bit offset),
written with scipy's netCDF writer because netCDF4 / HDF5 libraries are not
available here; every netCDF reader opens them.  Records are appended along
the unlimited ``time`` dimension instead of rewriting the file at each save.
Only the ``netcdf`` entry of ``file_format_list`` is written (``tif`` needs
rasterio/GDAL, absent here; it raises).

Host-side file I/O: the fields are copied to the host once per save.
"""

from __future__ import annotations

import os

import numpy as np

from .state import sync_host

VAR_INFO = {
    "topg": ["Basal Topography", "m"],
    "usurf": ["Surface Topography", "m"],
    "thk": ["Ice Thickness", "m"],
    "icemask": ["Ice mask", "NO UNIT"],
    "smb": ["Surface Mass Balance", "m/y ice eq"],
    "ubar": ["x depth-average velocity of ice", "m/y"],
    "vbar": ["y depth-average velocity of ice", "m/y"],
    "velbar_mag": ["Depth-average velocity magnitude of ice", "m/y"],
    "uvelsurf": ["x surface velocity of ice", "m/y"],
    "vvelsurf": ["y surface velocity of ice", "m/y"],
    "wvelsurf": ["z surface velocity of ice", "m/y"],
    "velsurf_mag": ["Surface velocity magnitude of ice", "m/y"],
    "uvelbase": ["x basal velocity of ice", "m/y"],
    "vvelbase": ["y basal velocity of ice", "m/y"],
    "wvelbase": ["z basal velocity of ice", "m/y"],
    "velbase_mag": ["Basal velocity magnitude of ice", "m/y"],
    "divflux": ["Divergence of the ice flux", "m/y"],
    "strflowctrl": ["arrhenius+1.0*slidingco", "MPa$^{-3}$ a$^{-1}$"],
    "dtopgdt": ["Erosion rate", "m/y"],
    "arrhenius": ["Arrhenius factor", "MPa$^{-3}$ a$^{-1}$"],
    "slidingco": ["Sliding Coefficient", "km MPa$^{-3}$ a$^{-1}$"],
    "meantemp": ["Mean annual surface temperatures", "deg C"],
    "meanprec": ["Mean annual precipitation", "Kg m^(-2) y^(-1)"],
    "velsurfobs_mag": ["Obs. surf. speed of ice", "m/y"],
    "weight_particles": ["weight_particles", "no"],
}
TS_INFO = {"vol": ["Ice volume", "km^3"], "area": ["Glaciated area", "km^2"]}

DEFAULTS = {"file_format_list": ["netcdf"], "output_file": "output.nc",
            "vars_to_save": ["topg", "usurf", "thk", "smb", "velbar_mag", "velsurf_mag", "uvelsurf", "vvelsurf",
                             "wvelsurf"],
            "write_ts": True, "output_ts_file": "output_ts.nc"}


def _host(x):
    if hasattr(x, "detach"):
        return x.detach().float().cpu().numpy()
    return np.asarray(x, dtype=np.float32)


def _opt(cfg, key):
    loc = getattr(getattr(cfg, "outputs", None), "local", None)
    return getattr(loc, key, DEFAULTS[key]) if loc is not None else DEFAULTS[key]


def _mag(u, v):
    u, v = _host(u).astype(np.float64), _host(v).astype(np.float64)
    return np.sqrt(u * u + v * v).astype(np.float32)


def _coords(state, ny, nx):
    dx = float(getattr(state, "dx", 1.0))
    x = _host(state.x) if hasattr(state, "x") else np.arange(nx, dtype=np.float32) * dx
    y = _host(state.y) if hasattr(state, "y") else np.arange(ny, dtype=np.float32) * dx
    return x.astype(np.float32), y.astype(np.float32)


def initialize(cfg, state):
    """local.py:8-41: variable descriptions on the state."""
    state.var_info_ncdf_ex = dict(VAR_INFO)
    state.var_info_ncdf_ts = dict(TS_INFO)


def run(cfg, state):
    """local.py:44-66: on save steps, the derived magnitudes, then the field
    file and the time-series file."""
    if not getattr(state, "saveresult", False):
        return
    sync_host(state)  # a host-resident state: the processes' result copies have landed
    fmts = list(_opt(cfg, "file_format_list"))
    if any(f not in ("netcdf",) for f in fmts):
        raise NotImplementedError(f"output formats {fmts}: only 'netcdf' is written")
    wanted = list(_opt(cfg, "vars_to_save"))
    if "velbar_mag" in wanted and hasattr(state, "ubar"):
        state.velbar_mag = _mag(state.ubar, state.vbar)
    if "velsurf_mag" in wanted and hasattr(state, "uvelsurf"):
        state.velsurf_mag = _mag(state.uvelsurf, state.vvelsurf)
    if "velbase_mag" in wanted and hasattr(state, "uvelbase"):
        state.velbase_mag = _mag(state.uvelbase, state.vvelbase)
    if "netcdf" in fmts:
        update_netcdf_ex(cfg, state)
    if bool(_opt(cfg, "write_ts")):
        update_netcdf_ts(cfg, state)


def update_netcdf_ex(cfg, state):
    """local.py:92-148 / write_ncdf.py:60-140: a (time, y, x) or (time, z, y, x)
    float32 record per listed field present on the state."""
    from scipy.io import netcdf_file
    path = _opt(cfg, "output_file")
    sync_host(state)  # a host-resident state: the processes' result copies have landed
    t = float(getattr(state, "t", 0.0))
    fields = {v: _host(getattr(state, v)) for v in _opt(cfg, "vars_to_save") if hasattr(state, v)}
    info = getattr(state, "var_info_ncdf_ex", VAR_INFO)
    if not getattr(state, "already_called_update_local", False) or not os.path.exists(path):
        ny, nx = _host(state.thk).shape
        x, y = _coords(state, ny, nx)
        with netcdf_file(path, "w", version=2) as nc:
            nc.pyproj_srs = str(getattr(state, "pyproj_srs", ""))
            nc.createDimension("time", None)
            nc.createDimension("y", ny)
            nc.createDimension("x", nx)
            tv = nc.createVariable("time", "f4", ("time",))
            tv.units, tv.long_name, tv.axis = "yr", "time", "T"
            for name, arr, ax in [("y", y, "Y"), ("x", x, "X")]:
                c = nc.createVariable(name, "f4", (name,))
                c.units, c.long_name, c.axis = "m", name, ax
                c[:] = arr
            nzs = [a.shape[0] for a in fields.values() if a.ndim == 3]
            if nzs:
                nc.createDimension("z", nzs[0])
                c = nc.createVariable("z", "f4", ("z",))
                c.units, c.long_name, c.axis = "m", "z", "Z"
                c[:] = np.arange(nzs[0], dtype=np.float32)
            for v, arr in fields.items():
                var = nc.createVariable(v, "f4", ("time", "y", "x") if arr.ndim == 2 else ("time", "z", "y", "x"))
                if v in info:
                    var.long_name, var.units = info[v]
            tv[0] = t
            for v, arr in fields.items():
                nc.variables[v][0] = arr
        state.already_called_update_local = True
        return
    with netcdf_file(path, "a") as nc:
        d = nc.variables["time"].shape[0]
        nc.variables["time"][d] = t
        for v, arr in fields.items():
            if v in nc.variables:
                nc.variables[v][d] = arr


def update_netcdf_ts(cfg, state):
    """local.py:152-196: ice volume sum(thk) dx^2 / 1e9 km^3 and glaciated
    area (thk > 1 m) dx^2 / 1e6 km^2 per save time."""
    from scipy.io import netcdf_file
    path = _opt(cfg, "output_ts_file")
    sync_host(state)
    thk = _host(state.thk).astype(np.float64)
    dx = float(state.dx)
    vol = float(thk.sum() * dx * dx / 1e9)
    area = float((thk > 1).sum() * dx * dx / 1e6)
    t = float(getattr(state, "t", 0.0))
    if not getattr(state, "already_called_update_write_ts", False) or not os.path.exists(path):
        with netcdf_file(path, "w", version=2) as nc:
            nc.createDimension("time", None)
            tv = nc.createVariable("time", "f4", ("time",))
            tv.units, tv.long_name = "yr", "time"
            for name in ("vol", "area"):
                var = nc.createVariable(name, "f4", ("time",))
                var.long_name, var.units = TS_INFO[name]
            tv[0], nc.variables["vol"][0], nc.variables["area"][0] = t, vol, area
        state.already_called_update_write_ts = True
        return
    with netcdf_file(path, "a") as nc:
        d = nc.variables["time"].shape[0]
        nc.variables["time"][d] = t
        nc.variables["vol"][d] = vol
        nc.variables["area"][d] = area
