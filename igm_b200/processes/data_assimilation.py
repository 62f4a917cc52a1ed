"""data_assimilation process (igm/processes/data_assimilation/data_assimilation.py:16-71).

Inverts the ice thickness from surface-velocity and thickness observations
through the CNN emulator, as the reference does with its default
configuration: control ``thk``, costs ``velsurf`` + ``thk`` + ``icemask``,
the ``reproject`` + ``penalty`` obstacle constraints, the anisotropic (or
isotropic) regularisation of the bed or of the thickness, ADAM with a
learning rate decaying as step_size decay^(i/100), the emulator retrained on
the Blatter-Pattyn energy of the current geometry after every iteration
(gated by retrain_freq, as in the iceflow process).

One iteration (optimize/update.py:15-103) is a fixed sequence of device
launches with no host synchronisation:

  igm_assim_control mode 0      per control: x_sc = x / sc, x = x_sc sc, fresh moments
  CNN forward (keep activations, thk mask), velsurf / velbar
  igm_assim_flow_direction      (anisotropic regularisation only)
  igm_assim_cost_grad           costs, dC/dthk, dC/d(top-layer U, V)
  igm_divflux + igm_assim_divflux_cost_grad (divfluxobs / divfluxfcz only)
  igm_assim_field_regu          slidingco / arrhenius regularisation and penalty (those controls only)
  CNN backward, data chain only, with igm_cnn_input_gradient
  igm_assim_control mode 1      per control: the gradient of x_sc with its mask
  igm_adam_clipnorm             Keras legacy Adam at iteration i + 1, one variable per control
  igm_assim_control mode 2      per control: x = x_sc sc, reprojection
  igm_divflux_upwind            divflux of the emulated velbar
  rms / std record              device reductions into the history tensor

The cost history and the rms/std record stay on the device until the end of
the loop (``costs.dat`` and ``rms_std_vol.dat`` are written from them then);
the netCDF snapshots every ``output.freq`` iterations and the final
``save_result_in_ncdf`` file are host copies.  The 2-D plots of the
reference (matplotlib) are not drawn.

Supported: control_list within thk, usurf, slidingco (log_slidingco or not),
arrhenius (dim_arrhenius 2); cost_list within velsurf, thk, icemask, usurf,
divfluxobs, divfluxfcz (the flux-divergence terms, with or without
force_zero_sum); fix_opti_normalization_issue, include_low_speed_term and
sole_mask on or off; method ADAM; cook.infer_params off; divflux.method
upwind or centered.  Anything else raises NotImplementedError.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np
import torch

from .. import _lib as L
from .. import kernels as K
from .. import state as S
from . import iceflow as P

_COST_KEYS = ["velsurf", "thk", "icemask", "thk_positive", "thk_regu", "usurf"]  # igm_assim_cost_grad's columns
# total_cost.py:13-71's order of the cost dictionary
_ALL_KEYS = ["velsurf", "thk", "divflux", "usurf", "icemask", "thk_positive", "slidingco_positive",
             "arrhenius_positive", "thk_regu", "slid_regu", "arrh_regu"]
# the controls: emulator input channel (fieldin order thk, usurf, arrhenius, slidingco)
_CHANNEL = {"thk": 0, "usurf": 1, "arrhenius": 2, "slidingco": 3}


def _check_supported(cfg):
    da = cfg.processes.data_assimilation
    o = da.optimization
    bad = []
    ctl = list(da.control_list)
    if not ctl or any(c not in _CHANNEL for c in ctl) or len(set(ctl)) != len(ctl):
        bad.append(f"control_list={ctl} (thk, usurf, slidingco, arrhenius)")
    extra = [c for c in da.cost_list if c not in ("velsurf", "thk", "icemask", "usurf", "divfluxobs", "divfluxfcz")]
    if extra:
        bad.append(f"cost terms {extra} (only velsurf, thk, icemask, usurf, divfluxobs, divfluxfcz)")
    if o.method != "ADAM":
        bad.append(f"optimization.method={o.method!r} (only 'ADAM')")
    if bool(da.cook.infer_params):
        bad.append("cook.infer_params")
    if da.divflux.method not in K.DIVFLUX_METHODS:
        bad.append(f"divflux.method={da.divflux.method!r} (upwind or centered)")
    if da.regularization.to_regularize not in ("topg", "thk"):
        bad.append(f"to_regularize={da.regularization.to_regularize!r}")
    if cfg.processes.iceflow.method != "emulated":
        bad.append("iceflow.method must be 'emulated'")
    if bad:
        raise NotImplementedError("igm_b200 data_assimilation: unsupported configuration: " + "; ".join(bad))


def create_density_matrix(thkobs: np.ndarray, kernel_size: int = 5) -> np.ndarray:
    """utils.py:68-82: number of thickness observations in the
    kernel_size x kernel_size window around each node (zero outside)."""
    m = (~np.isnan(thkobs)).astype(np.float64)
    r = kernel_size // 2
    p = np.pad(m, r)
    c = np.cumsum(np.cumsum(p, 0), 1)
    c = np.pad(c, ((1, 0), (1, 0)))
    k = kernel_size
    ny, nx = m.shape
    return c[k:k + ny, k:k + nx] - c[:ny, k:k + nx] - c[k:k + ny, :nx] + c[:ny, :nx]


def _density_weights(thkobs: np.ndarray, uniformize: bool) -> np.ndarray:
    """optimize/initialize.py:40-46."""
    if not uniformize:
        return np.ones_like(thkobs)
    d = create_density_matrix(thkobs, 5)
    d = np.where(d > 0, 1.0 / np.maximum(d, 1.0), 0.0)
    d = np.where(np.isnan(thkobs), 0.0, d)
    pos = d[d > 0]
    return (d / pos.mean() if pos.size else d).astype(thkobs.dtype)


class _Assim:
    """Device buffers and constants of the assimilation loop."""

    def __init__(self, cfg, state):
        da = cfg.processes.data_assimilation
        thk = S.get(state, "thk")
        ny, nx = thk.shape
        d = thk.device
        self.ny, self.nx, self.n = ny, nx, ny * nx
        self.dx = P._dx(state)
        nan = torch.full((ny, nx), float("nan"), dtype=torch.float32, device=d)
        costs = list(da.cost_list)
        f, r, o = da.fitting, da.regularization, da.optimization
        self.controls = list(da.control_list)
        nc = len(self.controls)
        self.uobs = S.get(state, "uvelsurfobs").contiguous() if "velsurf" in costs else nan
        self.vobs = S.get(state, "vvelsurfobs").contiguous() if "velsurf" in costs else nan
        self.thkobs = S.get(state, "thkobs").contiguous() if "thk" in costs else nan
        self.usurfobs = S.get(state, "usurfobs").contiguous() if "usurf" in costs else None
        self.icemaskobs = S.get(state, "icemaskobs").contiguous()
        self.icemask = S.get(state, "icemask").contiguous() if hasattr(state, "icemask") else self.icemaskobs
        self.dens = S.get(state, "dens_thkobs").contiguous()
        self.cost_list = costs
        nz = int(cfg.processes.iceflow.numerics.Nz)
        self.nz = nz
        f32 = dict(dtype=torch.float32, device=d)
        # the optimizer's variables, one block of n per control (Adam clips each separately)
        self.var, self.grad, self.m, self.v = (torch.empty(nc * self.n, **f32) for _ in range(4))
        self.offsets = (C.c_size_t * (nc + 1))(*[k * self.n for k in range(nc + 1)])
        self.norms = torch.empty(int(L.lib().igm_adam_norms_len(nc, self.offsets)), dtype=torch.float64, device=d)
        self.dU = torch.zeros((1, nz, ny, nx), **f32)
        self.dV = torch.zeros((1, nz, ny, nx), **f32)
        self.g_thk = torch.empty((ny, nx), **f32)
        self.g_us = torch.empty((ny, nx), **f32) if "usurf" in self.controls else None
        self.g_field = {c: torch.empty((ny, nx), **f32) for c in ("slidingco", "arrhenius") if c in self.controls}
        # the emulator's input-field gradient, channels 0 .. the last one a control needs
        self.n_grad = 1 + max(_CHANNEL[c] for c in self.controls)
        self.field_grad = torch.empty((1, self.n_grad, ny, nx), **f32)
        self.partials = torch.empty(148 * 8 * 6, dtype=torch.float64, device=d)
        nit = int(o.nbitmax) + 1
        self.cost_hist = torch.zeros((nit, 6), dtype=torch.float64, device=d)
        self.field_hist = {c: torch.zeros((nit, 6), dtype=torch.float64, device=d) for c in self.g_field}
        self.rms_hist = torch.zeros((nit, 9), dtype=torch.float64, device=d)
        self.stat_partials = torch.empty(148 * 8 * 13, dtype=torch.float64, device=d)
        self.low_partials = torch.empty(3 * 148 * 8 + 1, dtype=torch.float64, device=d)
        # parameters of igm_assim_cost_grad
        p = L.AssimParams()
        p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std = f.velsurfobs_std, f.velsurfobs_thr, f.thkobs_std
        p.regu_thk = r.thk
        area = float((self.icemask > 0.5).sum().item()) * self.dx ** 2  # regu_thk.py:11
        p.gamma = float(r.convexity_weight) * area ** (float(r.convexity_power) - 2.0) if area > 0 else 0.0
        p.aniso_factor = float(r.smooth_anisotropy_factor)
        vo = torch.stack([self.uobs, self.vobs], -1).double()
        rel = torch.linalg.vector_norm(vo, dim=-1) >= float(f.velsurfobs_thr)
        # the means' counts (an absent term has no contributions; its count is kept at 1)
        p.n_vel = max(1.0, float((~torch.isnan(vo) & rel[..., None]).sum().item()))
        p.n_thk = max(1.0, float((~torch.isnan(self.thkobs)).sum().item()))
        p.penalty = int("penalty" in o.obstacle_constraint)
        p.icemask_cost = int("icemask" in costs)
        p.regularize_thk = int(r.to_regularize == "thk")
        p.mask_velsurf = 1
        p.usurf_cost = int("usurf" in costs)
        p.usurfobs_std = float(f.usurfobs_std)
        p.n_usurf = max(1.0, float((self.icemaskobs > 0.5).sum().item()))
        p.no_thk_control = int("thk" not in self.controls)
        p.fix_normalization = int(bool(o.fix_opti_normalization_issue))
        p.sole_mask = int(bool(o.sole_mask))
        self.params = p
        self.log_slidingco = bool(f.log_slidingco)
        pen = bool(p.penalty)
        self.present = {"velsurf": "velsurf" in costs, "thk": "thk" in costs, "usurf": "usurf" in costs,
                        "icemask": pen and bool(p.icemask_cost), "thk_positive": pen and "thk" in self.controls,
                        "slidingco_positive": pen and "slidingco" in self.controls and not self.log_slidingco,
                        "arrhenius_positive": pen and "arrhenius" in self.controls,
                        "thk_regu": "thk" in self.controls, "slid_regu": "slidingco" in self.controls,
                        "arrh_regu": "arrhenius" in self.controls}
        # flux-divergence cost (total_cost.py:23-27: divfluxfcz before divfluxobs)
        self.div_kind = "fcz" if "divfluxfcz" in costs else ("obs" if "divfluxobs" in costs else None)
        self.div_method = str(da.divflux.method)
        self.div_hist = torch.zeros(nit, dtype=torch.float64, device=d)
        self.div_res = None  # (slope, intercept) of cost_divfluxfcz's regression
        if self.div_kind is not None:
            self.D = torch.empty((ny, nx), **f32)
            self.div_scratch = torch.empty((ny, nx), **f32)
            self.div_partials = torch.empty(int(L.lib().igm_assim_divflux_partials_len(148 * 8)),
                                            dtype=torch.float64, device=d)
            self.divfluxobs = S.get(state, "divfluxobs").contiguous() if self.div_kind == "obs" else None
            self.vert_weight = np.asarray(torch.as_tensor(state.vert_weight).cpu(), dtype=np.float64).reshape(-1)
        self.scale = {c: float(getattr(da.scaling, c)) for c in self.controls}
        self.reproject = "reproject" in o.obstacle_constraint
        self.aniso = float(r.smooth_anisotropy_factor)
        self.aniso_sl = float(r.smooth_anisotropy_factor_sl)

    def control_kw(self, c):
        """igm_assim_control's transform, mask and reprojection for control c
        (optimize/update.py:23-27, 58-68, 84-98; sole_mask off)."""
        transform = int(c == "slidingco" and self.log_slidingco)
        mask = (2 if self.params.sole_mask else 0) if c == "slidingco" else 1
        if not self.reproject:
            rep, lower = 0, 0.0
        elif c == "thk":
            rep, lower = 1, 0.0
        elif c == "slidingco":
            rep, lower = 2, 0.0
        elif c == "arrhenius":
            rep, lower = 2, 1.0
        else:
            rep, lower = 0, 0.0
        return dict(transform=transform, mask=mask, reproject=rep, lower=lower,
                    reproject_mask="icemask" in self.cost_list)

    def block(self, t, k):
        return t[k * self.n:(k + 1) * self.n]


def optimize_initialize(cfg, state):
    """optimize/initialize.py:10-69."""
    da = cfg.processes.data_assimilation
    if ("usurf" in da.cost_list) != ("usurf" in da.control_list):
        raise AssertionError("usurf must be in both cost_list and control_list, or in neither")
    thkobs = S.get(state, "thkobs").cpu().numpy()
    if np.all(np.isnan(thkobs)) and "thk" in da.cost_list:
        da.cost_list = [c for c in da.cost_list if c != "thk"]
    if "usurf" in da.control_list and not hasattr(state, "usurfobs"):
        raise ValueError("control usurf needs state.usurfobs")
    thk = S.get(state, "thk")
    if hasattr(state, "thkinit"):
        thk = S.get(state, "thkinit").clone()
    else:
        thk = torch.zeros_like(thk)
    if bool(da.optimization.init_zero_thk):
        thk = thk * 0.0
    S.put(state, "thk", thk.contiguous())
    if "divfluxobs" in da.cost_list and not hasattr(state, "divfluxobs"):
        S.put(state, "divfluxobs", S.get(state, "smb") - S.get(state, "dhdt"))
    dens = _density_weights(thkobs.astype(np.float32), bool(da.fitting.uniformize_thkobs))
    S.put(state, "dens_thkobs", torch.as_tensor(dens, device=thk.device))
    sl = S.get(state, "slidingco")
    S.put(state, "slidingco", torch.where(S.get(state, "icemaskobs") == 2, torch.zeros_like(sl), sl))
    state._igm_assim = _Assim(cfg, state)


def _record_rms(a: _Assim, state, i):
    """compute_rms_std_optimization (utils.py:10-66) into row i of the
    device history (igm_assim_stats): rmsthk, stdthk, rmsvel, stdvel, rmsdiv,
    stddiv, rmsusurf, stdusurf, vol."""
    g = lambda k: S.get(state, k).contiguous() if hasattr(state, k) else None
    vel = hasattr(state, "uvelsurfobs")
    K.assim_stats(S.get(state, "thk"), a.dx, a.icemaskobs, thkobs=g("thkobs"),
                  uvs=g("uvelsurf") if vel else None, vvs=g("vvelsurf") if vel else None,
                  uobs=g("uvelsurfobs"), vobs=g("vvelsurfobs"),
                  divflux=g("divflux") if hasattr(state, "divfluxobs") else None, divfluxobs=g("divfluxobs"),
                  usurf=g("usurf") if hasattr(state, "usurfobs") else None, usurfobs=g("usurfobs"),
                  out=a.rms_hist[i], partials=a.stat_partials)


def optimize_update(cfg, state, cost, i):
    """optimize/update.py:15-103: one ADAM iteration over the controls.
    ``cost`` receives device cost tensors: "all" (double[6], velsurf, thk,
    icemask, thk_positive, thk_regu, usurf), "divflux", "slidingco" and
    "arrhenius" (double[6], [3] the penalty, [4] the regularisation) when
    present."""
    da = cfg.processes.data_assimilation
    o = da.optimization
    a: _Assim = state._igm_assim
    lib, st = L.lib(), L.stream_ptr()
    x = {}
    for k, c in enumerate(a.controls):
        x[c] = S.get(state, c, writable=True).contiguous()  # rewritten in place by the control update below
        K.assim_control(0, x[c], a.scale[c], variable=a.block(a.var, k), m=a.block(a.m, k), v=a.block(a.v, k),
                        **a.control_kw(c))
        S.put(state, c, x[c])
    lr = float(o.step_size) * (float(o.step_size_decay) ** (i / 100)) if o.step_size_decay < 1 else float(o.step_size)
    thk = S.get(state, "thk").contiguous()
    # emulator forward, masked where thk == 0 (emulate.py:116-152), activations kept for the gradient
    model = state.iceflow_model
    f = [thk] + [S.get(state, k).contiguous() for k in ("usurf", "arrhenius", "slidingco")]
    buf = model.buffers(1, a.ny, a.nx, train=True)
    model.prepare_input(f, a.dx, [(0, 0)], a.ny, a.nx, buf)
    U, V = model.forward(buf, 1, a.ny, a.nx, thk_mask=thk, keep_acts=True)
    state.U, state.V = U[0], V[0]
    P.set_derived_velocities(cfg, state, mask=False)
    uvs, vvs = S.get(state, "uvelsurf"), S.get(state, "vvelsurf")
    flow = None
    if a.aniso != 1.0 or ("slidingco" in a.controls and a.aniso_sl != 1.0):
        flow = K.assim_flow_direction(uvs.contiguous(), vvs.contiguous())
        state.flowdirx, state.flowdiry = flow
    # total_cost and its gradient; dC/dvelsurf lands in the top layer of dU, dV (Lagrange basis)
    K.assim_cost_grad(thk, f[1], uvs.contiguous(), vvs.contiguous(), a.uobs, a.vobs, a.thkobs, a.dens, a.icemaskobs,
                      flow if a.aniso != 1.0 else None, a.dx, a.params, partials=a.partials, costs=a.cost_hist[i],
                      g_thk=a.g_thk, g_u=a.dU[0, a.nz - 1], g_v=a.dV[0, a.nz - 1], usurfobs=a.usurfobs,
                      g_us=a.g_us)
    if bool(da.fitting.include_low_speed_term) and "velsurf" in a.cost_list:
        K.assim_low_speed(uvs.contiguous(), vvs.contiguous(), a.uobs, a.vobs, a.dU[0, a.nz - 1], a.dV[0, a.nz - 1],
                          a.cost_hist[i, 0:1], partials=a.low_partials)
    if a.div_kind is not None:
        _divflux_cost(cfg, state, a, thk, i)
    r = da.regularization
    for c, g in a.g_field.items():
        # regu_slidingco / regu_arrhenius and the positivity penalties (total_cost.py:45-54, 63-69)
        aniso = a.aniso_sl if c == "slidingco" else 1.0
        pen = bool(a.params.penalty) and not (c == "slidingco" and a.log_slidingco)
        K.assim_field_regu(S.get(state, c).contiguous(), a.dx, float(getattr(r, c)), aniso,
                           flow if aniso != 1.0 else None, penalty=pen, threshold=1.0 if c == "arrhenius" else 0.0,
                           grad=g, costs=a.field_hist[c][i], partials=a.partials,
                           fix_normalization=bool(a.params.fix_normalization),
                           sole_mask_icemaskobs=a.icemaskobs if a.params.sole_mask else None)
    model.backward(buf, 1, a.ny, a.nx, a.dU, a.dV, field_grad=a.field_grad, param_grads=False)
    direct = {"thk": a.g_thk, "usurf": a.g_us, **a.g_field}
    for k, c in enumerate(a.controls):
        K.assim_control(1, x[c], a.scale[c], icemaskobs=a.icemaskobs, variable=a.block(a.var, k),
                        grad=a.block(a.grad, k), g_direct=direct[c],
                        g_emul=a.field_grad[0, _CHANNEL[c]].reshape(-1), **a.control_kw(c))
    rc = lib.igm_adam_clipnorm(len(a.controls), a.offsets, L.ptr(a.var), L.ptr(a.grad), L.ptr(a.m), L.ptr(a.v),
                               L.ptr(a.norms), lr, 0.9, 0.999, float(o.optimizer_epsilon),
                               float(o.optimizer_clipnorm), i + 1, st)
    L.check(rc, "igm_adam_clipnorm")
    for k, c in enumerate(a.controls):
        K.assim_control(2, x[c], a.scale[c], icemaskobs=a.icemaskobs, variable=a.block(a.var, k),
                        **a.control_kw(c))
        S.put(state, c, x[c])
    if a.reproject and "icemask" in a.cost_list and "thk" not in a.controls:
        # update.py:84-88: thk is masked by the reprojection even when it is not a control
        thk = S.get(state, "thk", writable=True).contiguous()
        K.assim_control(3, thk, 1.0, icemaskobs=a.icemaskobs)
        S.put(state, "thk", thk)
    thk = S.get(state, "thk").contiguous()
    S.put(state, "divflux", K.divflux(S.get(state, "ubar").contiguous(), S.get(state, "vbar").contiguous(), thk,
                                      a.dx, a.div_method))
    cost["all"] = a.cost_hist[i]
    if a.div_kind is not None:
        cost["divflux"] = a.div_hist[i]
    for c in a.g_field:
        cost[c] = a.field_hist[c][i]


def _divflux_cost(cfg, state, a: _Assim, thk, i):
    """cost_divfluxobs / cost_divfluxfcz (cost_terms/cost_divfluxobs.py:9-29,
    cost_divfluxfcz.py:10-38) of the emulated velbar and the current
    thickness: the cost into the history, dC/dthk added to the direct
    gradient, dC/dvelbar spread over the levels of dU, dV.  cost_divfluxfcz
    refits its target (scipy's linregress of divflux on usurf inside the mask,
    on the host) at every 10th iteration, as the reference."""
    da = cfg.processes.data_assimilation
    ub, vb = S.get(state, "ubar").contiguous(), S.get(state, "vbar").contiguous()
    D = K.divflux(ub, vb, thk, a.dx, a.div_method, out=a.D)
    usurf = S.get(state, "usurf").contiguous()
    if a.div_kind == "fcz" and (i % 10 == 0 or a.div_res is None):
        from scipy import stats
        act = (a.icemaskobs > 0.5).cpu().numpy()
        res = stats.linregress(usurf.cpu().numpy()[act], D.cpu().numpy()[act])
        a.div_res = (float(res.slope), float(res.intercept))
        state.res = res
    slope, intercept = a.div_res if a.div_res is not None else (0.0, 0.0)
    K.assim_divflux_cost_grad(a.div_kind, ub, vb, thk, D, a.dx, a.icemaskobs, a.g_thk, a.dU[0], a.dV[0],
                              a.vert_weight, divfluxobs=a.divfluxobs, usurf=usurf if a.div_kind == "fcz" else None,
                              slope=slope, intercept=intercept, std=float(da.fitting.divfluxobs_std),
                              regu=float(da.regularization.divflux),
                              force_zero_sum=bool(da.divflux.get("force_zero_sum", False)), method=a.div_method,
                              mask_thk=thk, scratch=a.div_scratch, partials=a.div_partials, cost=a.div_hist[i:i + 1])


def _cost_table(a: _Assim, n_it):
    """The per-iteration costs in total_cost's order: (keys, [n_it, k] array)."""
    ch = a.cost_hist[:n_it].cpu().numpy()
    cols = {k: ch[:, j] for j, k in enumerate(_COST_KEYS)}
    if a.div_kind is not None:
        cols["divflux"] = a.div_hist[:n_it].cpu().numpy()
    for c, pen, reg in (("slidingco", "slidingco_positive", "slid_regu"), ("arrhenius", "arrhenius_positive",
                                                                          "arrh_regu")):
        if c in a.field_hist:
            fh = a.field_hist[c][:n_it].cpu().numpy()
            cols[pen], cols[reg] = fh[:, 3], fh[:, 4]
    present = dict(a.present, divflux=a.div_kind is not None)
    keys = [k for k in _ALL_KEYS if present.get(k, False)]
    return keys, np.stack([cols[k] for k in keys], axis=1)


def _mag(u, v):
    return torch.sqrt(u * u + v * v)


def _snapshot_fields(cfg, state):
    """The derived fields of output_ncdf.py:20-30, then the listed fields as
    float32 host arrays."""
    da = cfg.processes.data_assimilation
    want = list(da.output.vars_to_save)
    if "velbase_mag" in want:
        state.velbase_mag = _mag(S.get(state, "uvelbase"), S.get(state, "vvelbase"))
    if "velsurf_mag" in want:
        state.velsurf_mag = _mag(S.get(state, "uvelsurf"), S.get(state, "vvelsurf"))
    if "velsurfobs_mag" in want:
        state.velsurfobs_mag = _mag(S.get(state, "uvelsurfobs"), S.get(state, "vvelsurfobs"))
    if "sliding_ratio" in want:
        vs = state.velsurf_mag
        state.sliding_ratio = torch.where(vs > 10, state.velbase_mag / vs, torch.full_like(vs, float("nan")))
    S.sync_host(state)  # a host-resident state: the result copies have landed
    out = {}
    for v in want:
        if hasattr(state, v):
            x = getattr(state, v)
            out[v] = (x.detach().float().cpu().numpy() if isinstance(x, torch.Tensor)
                      else np.asarray(x, dtype=np.float32))
    return out


def _coords(state, ny, nx, dx):
    def host(name, n):
        if hasattr(state, name):
            x = getattr(state, name)
            return (x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)).astype(np.float32)
        return (np.arange(n) * dx).astype(np.float32)
    return host("x", nx), host("y", ny)


def update_ncdf_optimize(cfg, state, it):
    """output_ncdf.py:12-78: one (iterations, y, x) record per listed field
    in optimize.nc (netCDF-3 through scipy)."""
    from scipy.io import netcdf_file
    a: _Assim = state._igm_assim
    fields = _snapshot_fields(cfg, state)
    if it == 0 or not os.path.exists("optimize.nc"):
        x, y = _coords(state, a.ny, a.nx, a.dx)
        with netcdf_file("optimize.nc", "w", version=2) as nc:
            nc.createDimension("iterations", None)
            e = nc.createVariable("iterations", "f4", ("iterations",))
            e.units, e.long_name, e.axis = "None", "iterations", "ITERATIONS"
            for name, arr, ax in [("y", y, "Y"), ("x", x, "X")]:
                nc.createDimension(name, arr.size)
                c = nc.createVariable(name, "f4", (name,))
                c.units, c.long_name, c.axis = "m", name, ax
                c[:] = arr
            for v in fields:
                nc.createVariable(v, "f4", ("iterations", "y", "x"))
            e[0] = it
            for v, arr in fields.items():
                nc.variables[v][0] = arr
        return
    with netcdf_file("optimize.nc", "a") as nc:
        d = nc.variables["iterations"].shape[0]
        nc.variables["iterations"][d] = it
        for v, arr in fields.items():
            if v in nc.variables:
                nc.variables[v][d] = arr


def output_ncdf_optimize_final(cfg, state):
    """output_ncdf.py:81-124: the optimised fields in save_result_in_ncdf."""
    from scipy.io import netcdf_file
    a: _Assim = state._igm_assim
    fields = _snapshot_fields(cfg, state)
    x, y = _coords(state, a.ny, a.nx, a.dx)
    with netcdf_file(cfg.processes.data_assimilation.output.save_result_in_ncdf, "w", version=2) as nc:
        for name, arr, ax in [("y", y, "Y"), ("x", x, "X")]:
            nc.createDimension(name, arr.size)
            c = nc.createVariable(name, "f4", (name,))
            c.units, c.long_name, c.axis = "m", name, ax
            c[:] = arr
        for v, arr in fields.items():
            e = nc.createVariable(v, "f4", ("y", "x"))
            e.standard_name = v
            e[:] = arr


def _write_histories(cfg, state, n_it, glen):
    """prints.py:11-32 (costs.dat) and prints.py:61-82 (rms_std_vol.dat)
    from the device histories; the record lists on the state as in
    utils.py:13-66."""
    a: _Assim = state._igm_assim
    keys, ch = _cost_table(a, n_it)
    rh = a.rms_hist[:n_it].cpu().numpy()
    names = ["rmsthk", "stdthk", "rmsvel", "stdvel", "rmsdiv", "stddiv", "rmsusurf", "stdusurf", "vol"]
    for j, k in enumerate(names):
        setattr(state, k, [float(x) for x in rh[:, j]])
    keys = keys + (["glen"] if glen else [])
    with open("costs.dat", "w") as fh:
        print("   ".join(f"{k:>12}" for k in keys), file=fh)
        for i in range(n_it):
            vals = list(ch[i]) + ([glen[i]] if glen else [])
            print("   ".join(f"{min(float(v), 9999999):>12.4f}" for v in vals), file=fh)
    np.savetxt("rms_std_vol.dat", rh, fmt="%.10f", comments="",
               header="        rmsthk      stdthk       rmsvel       stdvel       rmsdiv       stddiv       "
                      "rmsusurf       stdusurf       vol")


def initialize(cfg, state):
    """data_assimilation.py:16-71."""
    from .. import emulator as E
    _check_supported(cfg)
    P.initialize(cfg, state)
    optimize_initialize(cfg, state)
    da = cfg.processes.data_assimilation
    o = da.optimization
    a: _Assim = state._igm_assim
    glen = []
    n_it = int(o.nbitmax) + 1
    for i in range(n_it):
        cost = {}
        optimize_update(cfg, state, cost, i)
        _record_rms(a, state, i)
        if bool(o.retrain_iceflow_model):
            E.update_iceflow_emulator(cfg, state, i + 1, pertubate=bool(o.pertubate))
            glen.append(state.COST_EMULATOR[-1] if state.COST_EMULATOR else float("nan"))
        if i % int(da.output.freq) == 0 and bool(da.output.save_iterat_in_ncdf):
            update_ncdf_optimize(cfg, state, i)
    state.iceflow_model.check_errors()
    # the bed from the optimised thickness (grounded ice)
    S.put(state, "topg", S.get(state, "usurf") - S.get(state, "thk"))
    if da.output.save_result_in_ncdf != "":
        output_ncdf_optimize_final(cfg, state)
    _write_histories(cfg, state, n_it, glen)
    keys, table = _cost_table(a, n_it)
    state.costs_data_assimilation = [dict(zip(keys, map(float, r))) for r in table]
    S.sync_host(state)


def update(cfg, state):
    pass


def finalize(cfg, state):
    pass
