"""The ``local`` output module (igm/outputs/local.py): field records per save
time and the volume / area time series, read back from the netCDF files.
CPU only (host-resident numpy state)."""

import numpy as np
from scipy.io import netcdf_file

from igm_b200 import outputs
from igm_b200.config import to_cfg
from igm_b200.state import State


def _state(rng, nz=4, ny=7, nx=9):
    st = State()
    st.dx = 100.0
    st.thk = np.maximum(0, rng.normal(50, 40, (ny, nx))).astype(np.float32)
    st.topg = rng.normal(2000, 10, (ny, nx)).astype(np.float32)
    st.usurf = st.topg + st.thk
    st.ubar, st.vbar = (rng.normal(0, 20, (ny, nx)).astype(np.float32) for _ in range(2))
    st.uvelsurf, st.vvelsurf = (rng.normal(0, 20, (ny, nx)).astype(np.float32) for _ in range(2))
    st.W = rng.normal(0, 1, (nz, ny, nx)).astype(np.float32)
    return st


def test_records_and_time_series(tmp_path):
    rng = np.random.default_rng(0)
    f, fts = str(tmp_path / "out.nc"), str(tmp_path / "ts.nc")
    cfg = to_cfg({"outputs": {"local": {"file_format_list": ["netcdf"], "output_file": f,
                                        "vars_to_save": ["topg", "thk", "velbar_mag", "velsurf_mag", "W", "absent"],
                                        "write_ts": True, "output_ts_file": fts}}})
    st = _state(rng)
    outputs.initialize(cfg, st)
    saved = []
    for k, t in enumerate([0.0, 10.0, 20.0]):
        st.t = np.float32(t)
        st.saveresult = True
        st.thk = (st.thk * (1 + 0.1 * k)).astype(np.float32)
        outputs.run(cfg, st)
        saved.append((t, st.thk.copy(), np.sqrt(st.ubar.astype(np.float64) ** 2 + st.vbar.astype(np.float64) ** 2)))
    st.saveresult = False
    outputs.run(cfg, st)  # not a save step: nothing written
    with netcdf_file(f, "r", mmap=False) as nc:
        np.testing.assert_array_equal(nc.variables["time"][:], [0.0, 10.0, 20.0])
        assert nc.variables["thk"].dimensions == ("time", "y", "x")
        assert nc.variables["W"].dimensions == ("time", "z", "y", "x")
        assert "absent" not in nc.variables
        assert nc.variables["velbar_mag"].long_name == b"Depth-average velocity magnitude of ice"
        for d, (t, thk, vm) in enumerate(saved):
            np.testing.assert_array_equal(nc.variables["thk"][d], thk)
            np.testing.assert_allclose(nc.variables["velbar_mag"][d], vm, rtol=1e-6)
        np.testing.assert_array_equal(nc.variables["x"][:], np.arange(9) * 100.0)
    with netcdf_file(fts, "r", mmap=False) as nc:
        for d, (t, thk, _) in enumerate(saved):
            np.testing.assert_allclose(nc.variables["vol"][d], thk.astype(np.float64).sum() * 1e4 / 1e9, rtol=1e-6)
            np.testing.assert_allclose(nc.variables["area"][d], (thk > 1).sum() * 1e4 / 1e6, rtol=1e-6)
