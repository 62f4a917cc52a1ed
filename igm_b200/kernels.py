"""Typed host wrappers over the C ABI.  Torch tensors are device buffers only:
every computation below is a libigmb200 kernel."""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L


class Workspace:
    """Zero-filled scratch for the reducing kernels (they leave it zeroed).

    One per device/stream; grown on demand.  Calls that share it must be
    ordered on one stream."""

    def __init__(self):
        self.buf = None

    def get(self, grid: L.Grid, device) -> tuple[int, int]:
        need = int(L.lib().igm_workspace_size(C.byref(grid)))
        if need == 0:
            L.check(1, f"igm_workspace_size rejected grid {grid.batch}x{grid.nz}x{grid.ny}x{grid.nx}: "
                       + L.lib().igm_last_error().decode())
        if self.buf is None or self.buf.numel() < need or self.buf.device != torch.device(device):
            self.buf = torch.zeros(max(need, 1 << 16), dtype=torch.uint8, device=device)
        return self.buf.data_ptr(), self.buf.numel()


_WS: dict = {}


def workspace(device) -> Workspace:
    key = str(torch.device(device))
    if key not in _WS:
        _WS[key] = Workspace()
    return _WS[key]


def fields_struct(thk, usurf, arrhenius, slidingco) -> L.Fields:
    f = L.Fields()
    f.thk, f.usurf, f.arrhenius, f.slidingco = (L.ptr(t) for t in (thk, usurf, arrhenius, slidingco))
    return f


def energy(U, V, thk, usurf, arrhenius, slidingco, dx, dzeta, phys=None, grad=False, grad_scale=1.0,
           terms_out=None):
    """Energy sums (device float64 [3]: shear, sliding, gravity) and optionally
    grad_scale * d(sum)/d(U,V).  U, V: [B, Nz, Ny, Nx] or [Nz, Ny, Nx]."""
    squeeze = U.dim() == 3
    if squeeze:
        U, V = U[None], V[None]
        thk, usurf, arrhenius, slidingco = (t[None] for t in (thk, usurf, arrhenius, slidingco))
    B, nz, ny, nx = U.shape
    g = L.make_grid(B, nz, ny, nx, dx, dzeta)
    ph = phys if isinstance(phys, L.Physics) else L.make_physics(phys)
    terms = terms_out if terms_out is not None else torch.empty(3, dtype=torch.float64, device=U.device)
    dU = torch.empty_like(U) if grad else None
    dV = torch.empty_like(V) if grad else None
    wp, wn = workspace(U.device).get(g, U.device)
    f = fields_struct(thk, usurf, arrhenius, slidingco)
    rc = L.lib().igm_energy(L.dtype_code(U.dtype), C.byref(g), C.byref(ph), C.byref(f), L.ptr(U), L.ptr(V),
                            L.ptr(dU), L.ptr(dV), float(grad_scale), L.ptr(terms), wp, wn, L.stream_ptr())
    L.check(rc, "igm_energy")
    if squeeze and grad:
        dU, dV = dU[0], dV[0]
    return terms, dU, dV


def velocity_reduce(U, V, thk, vert_weight, mask=True, want_velomax=True):
    """Masks U, V in place (where thk <= 0) and returns
    (ubar, vbar, uvelbase, vvelbase, uvelsurf, vvelsurf, velomax[1] float32)."""
    squeeze = U.dim() == 3
    if squeeze:
        U4, V4, th = U[None], V[None], thk[None]
    else:
        U4, V4, th = U, V, thk
    B, nz, ny, nx = U4.shape
    outs = [torch.empty((B, ny, nx), dtype=U.dtype, device=U.device) for _ in range(6)]
    vm = torch.empty(1, dtype=torch.float32, device=U.device) if want_velomax else None
    w = (C.c_double * nz)(*[float(x) for x in np.asarray(vert_weight, dtype=np.float64).reshape(-1)[:nz]])
    rc = L.lib().igm_velocity_reduce(L.dtype_code(U.dtype), B, nz, ny, nx, L.ptr(U4), L.ptr(V4), L.ptr(th),
                                     int(bool(mask)), w, *[L.ptr(o) for o in outs], L.ptr(vm), L.stream_ptr())
    L.check(rc, "igm_velocity_reduce")
    if squeeze:
        outs = [o[0] for o in outs]
    return (*outs, vm)


def force_max_velbar(U, V, cap):
    """In place: where |(U, V)| >= cap, (U, V) = cap (U, V) / |(U, V)|
    (igm_force_max_velbar)."""
    if U.shape != V.shape or U.dtype != V.dtype or not (U.is_contiguous() and V.is_contiguous()):
        raise ValueError("force_max_velbar: U and V must be contiguous tensors of one shape and dtype")
    rc = L.lib().igm_force_max_velbar(L.dtype_code(U.dtype), U.numel(), L.ptr(U), L.ptr(V), float(cap),
                                      L.stream_ptr())
    L.check(rc, "igm_force_max_velbar")


def transport_step(ubar, vbar, thk, topg, smb, dx, dt, slope_type="superbee", ratio_density=0.910, sealevel=0.0,
                   want_lsurf=True, want_divflux=True, dt_device=None):
    """Returns (thk_new, usurf, lsurf, divflux) (the last two may be None)."""
    ny, nx = thk.shape
    thk_new = torch.empty_like(thk)
    usurf = torch.empty_like(thk)
    lsurf = torch.empty_like(thk) if want_lsurf else None
    div = torch.empty_like(thk) if want_divflux else None
    rc = L.lib().igm_transport_step(L.dtype_code(thk.dtype), ny, nx, float(dx), L.ptr(ubar), L.ptr(vbar), L.ptr(thk),
                                    L.ptr(thk_new), L.ptr(topg), L.ptr(smb), L.ptr(usurf), L.ptr(lsurf), L.ptr(div),
                                    float(dt), L.ptr(dt_device), L.SLOPE[slope_type], float(ratio_density),
                                    float(sealevel), L.stream_ptr())
    L.check(rc, "igm_transport_step")
    return thk_new, usurf, lsurf, div


def vertical_velocity(U, V, topg, thk, levels, vert_weight, dx, out=None, method="kinematic"):
    """W [Nz, Ny, Nx] of vert_flow version 2, method "kinematic"
    (igm_vertical_velocity) or "incompressibility"
    (igm_vertical_velocity_incompressibility).  levels and vert_weight: the Nz
    values of compute_levels and define_vertical_weight (any array-like)."""
    nz, ny, nx = U.shape
    W = out if out is not None else torch.empty_like(U)
    lv = np.ascontiguousarray(np.asarray(levels, dtype=np.float64).reshape(-1))
    w = np.ascontiguousarray(np.asarray(vert_weight, dtype=np.float64).reshape(-1))
    if lv.size != nz or w.size != nz:
        raise ValueError(f"levels ({lv.size}) and vert_weight ({w.size}) must have Nz = {nz} entries")
    if method not in ("kinematic", "incompressibility"):
        raise ValueError(f"vert_flow method {method!r}")
    name = "igm_vertical_velocity" if method == "kinematic" else "igm_vertical_velocity_incompressibility"
    rc = getattr(L.lib(), name)(L.dtype_code(U.dtype), nz, ny, nx, float(dx), L.ptr(U), L.ptr(V), L.ptr(topg),
                                L.ptr(thk), lv.ctypes.data, w.ctypes.data, L.ptr(W), L.stream_ptr())
    L.check(rc, name)
    return W


def surfaces(thk, topg, ratio_density=0.910, sealevel=0.0):
    lsurf = torch.empty_like(thk)
    usurf = torch.empty_like(thk)
    rc = L.lib().igm_thk_surfaces(L.dtype_code(thk.dtype), thk.numel(), L.ptr(thk), L.ptr(topg), L.ptr(lsurf),
                                  L.ptr(usurf), float(ratio_density), float(sealevel), L.stream_ptr())
    L.check(rc, "igm_thk_surfaces")
    return lsurf, usurf


def smb_simple(usurf, gradabl, gradacc, ela, maxacc, icemask=None, out=None):
    smb = out if out is not None else torch.empty_like(usurf)
    rc = L.lib().igm_smb_simple(L.dtype_code(usurf.dtype), usurf.numel(), L.ptr(usurf), L.ptr(icemask), L.ptr(smb),
                                float(gradabl), float(gradacc), float(ela), float(maxacc), L.stream_ptr())
    L.check(rc, "igm_smb_simple")
    return smb


def cfl_dt(velomax, cfl, dx, step_max, out=None):
    dt = out if out is not None else torch.empty(1, dtype=torch.float32, device=velomax.device)
    rc = L.lib().igm_cfl_dt(L.ptr(velomax), L.ptr(dt), float(cfl), float(dx), float(step_max), L.stream_ptr())
    L.check(rc, "igm_cfl_dt")
    return dt


def absmax2(a, b, out=None):
    vm = out if out is not None else torch.empty(1, dtype=torch.float32, device=a.device)
    rc = L.lib().igm_absmax2(L.dtype_code(a.dtype), a.numel(), L.ptr(a), L.ptr(b), L.ptr(vm), L.stream_ptr())
    L.check(rc, "igm_absmax2")
    return vm


def assim_cost_grad(thk, usurf, uvs, vvs, uobs, vobs, thkobs, dens, icemaskobs, flowdir, dx, params,
                    partials=None, costs=None, g_thk=None, g_u=None, g_v=None, usurfobs=None, g_us=None):
    """Cost terms (device double[6]: velsurf, thk, icemask, thk_positive,
    thk_regu, usurf) and gradients (dC/dthk, dC/duvelsurf, dC/dvvelsurf, and
    dC/dusurf into ``g_us`` when given) of the thk/usurf cost terms
    (igm_assim_cost_grad); ``params`` an _lib.AssimParams, ``flowdir`` (fx,
    fy) [ny-1, nx-1] or None.  The outputs may be given (contiguous [ny, nx]
    views, e.g. the top layer of a [nz, ny, nx] velocity gradient)."""
    ny, nx = thk.shape
    n_parts = 148 * 8
    if partials is None:
        partials = torch.empty(n_parts * 6, dtype=torch.float64, device=thk.device)
    costs = costs if costs is not None else torch.empty(6, dtype=torch.float64, device=thk.device)
    g_thk = g_thk if g_thk is not None else torch.empty_like(thk)
    g_u = g_u if g_u is not None else torch.empty_like(thk)
    g_v = g_v if g_v is not None else torch.empty_like(thk)
    for t in (g_thk, g_u, g_v) + ((g_us,) if g_us is not None else ()):
        if t.shape != thk.shape or not t.is_contiguous() or t.dtype != thk.dtype:
            raise ValueError("assim_cost_grad: gradient outputs must be contiguous [ny, nx] of thk's dtype")
    fx, fy = flowdir if flowdir is not None else (None, None)
    rc = L.lib().igm_assim_cost_grad(L.dtype_code(thk.dtype), ny, nx, float(dx), L.ptr(thk), L.ptr(usurf),
                                     L.ptr(uvs), L.ptr(vvs), L.ptr(uobs), L.ptr(vobs), L.ptr(thkobs), L.ptr(dens),
                                     L.ptr(icemaskobs), L.ptr(fx), L.ptr(fy), L.ptr(usurfobs), C.byref(params),
                                     L.ptr(g_thk), L.ptr(g_u), L.ptr(g_v), L.ptr(g_us), L.ptr(partials),
                                     partials.numel() // 6, L.ptr(costs), L.stream_ptr())
    L.check(rc, "igm_assim_cost_grad")
    return costs, g_thk, g_u, g_v


def assim_field_regu(field, dx, regu, aniso=1.0, flowdir=None, penalty=True, threshold=0.0, grad=None, costs=None,
                     partials=None, fix_normalization=False, sole_mask_icemaskobs=None):
    """The regularisation and positivity penalty of a slidingco / arrhenius
    control (igm_assim_field_regu): returns (costs double[6] with [3] the
    penalty and [4] the regularisation, dC/dfield)."""
    ny, nx = field.shape
    n_parts = 148 * 8
    partials = partials if partials is not None else torch.empty(n_parts * 6, dtype=torch.float64,
                                                                 device=field.device)
    costs = costs if costs is not None else torch.empty(6, dtype=torch.float64, device=field.device)
    grad = grad if grad is not None else torch.empty_like(field)
    fx, fy = flowdir if flowdir is not None else (None, None)
    rc = L.lib().igm_assim_field_regu(L.dtype_code(field.dtype), ny, nx, float(dx), L.ptr(field), L.ptr(fx),
                                      L.ptr(fy), float(regu), float(aniso), int(bool(penalty)), float(threshold),
                                      int(bool(fix_normalization)), L.ptr(sole_mask_icemaskobs),
                                      int(sole_mask_icemaskobs is not None), L.ptr(grad), L.ptr(partials),
                                      partials.numel() // 6, L.ptr(costs),
                                      L.stream_ptr())
    L.check(rc, "igm_assim_field_regu")
    return costs, grad


def assim_low_speed(uvs, vvs, uobs, vobs, g_u, g_v, cost, partials=None):
    """include_low_speed_term (igm_assim_low_speed): adds the term to the
    device double ``cost`` (a 1-element view) and its gradient to g_u, g_v."""
    ny, nx = uvs.shape
    n_parts = 148 * 8
    partials = partials if partials is not None else torch.empty(3 * n_parts + 1, dtype=torch.float64,
                                                                 device=uvs.device)
    rc = L.lib().igm_assim_low_speed(L.dtype_code(uvs.dtype), ny, nx, L.ptr(uvs), L.ptr(vvs), L.ptr(uobs),
                                     L.ptr(vobs), L.ptr(g_u), L.ptr(g_v), L.ptr(partials), (partials.numel() - 1) // 3,
                                     L.ptr(cost), L.stream_ptr())
    L.check(rc, "igm_assim_low_speed")


def assim_flow_direction(uvs, vvs):
    """Flow directions [ny-1, nx-1] of the anisotropic regularisation."""
    ny, nx = uvs.shape
    fx = torch.empty((ny - 1, nx - 1), dtype=uvs.dtype, device=uvs.device)
    fy = torch.empty_like(fx)
    rc = L.lib().igm_assim_flow_direction(L.dtype_code(uvs.dtype), ny, nx, L.ptr(uvs), L.ptr(vvs), L.ptr(fx),
                                          L.ptr(fy), None, L.stream_ptr())
    L.check(rc, "igm_assim_flow_direction")
    return fx, fy


def assim_control(mode, x, scale, icemaskobs=None, variable=None, grad=None, m=None, v=None, g_direct=None,
                  g_emul=None, transform=0, mask=1, reproject=1, reproject_mask=True, lower=0.0):
    """The control update of one assimilation iteration (igm_assim_control)
    for control x: mode 0 variable from x, x from the variable, zero moments;
    mode 1 the variable's gradient dx/dvariable (g_direct + g_emul) with the
    mask (0 none, 1 icemaskobs > 0.5, 2 icemaskobs == 1); mode 2 x from the
    variable and the reprojection (0 none, 1 thk, 2 x >= lower).  transform
    1: x = variable^2 scale.  variable, grad, m, v, g_emul are float32."""
    n = x.numel()
    if g_emul is not None and (g_emul.dtype != torch.float32 or not g_emul.is_contiguous() or g_emul.numel() != n):
        raise ValueError("assim_control: g_emul must be contiguous float32 of x's size")
    p = L.AssimControlParams()
    p.mode, p.transform, p.mask, p.reproject = int(mode), int(transform), int(mask), int(reproject)
    p.reproject_mask, p.scale, p.lower = int(bool(reproject_mask)), float(scale), float(lower)
    rc = L.lib().igm_assim_control(L.dtype_code(x.dtype), n, C.byref(p), L.ptr(x), L.ptr(g_direct), L.ptr(g_emul),
                                   L.ptr(icemaskobs), L.ptr(variable), L.ptr(grad), L.ptr(m), L.ptr(v),
                                   L.stream_ptr())
    L.check(rc, "igm_assim_control")


def assim_stats(thk, dx, icemaskobs, thkobs=None, uvs=None, vvs=None, uobs=None, vobs=None, divflux=None,
                divfluxobs=None, usurf=None, usurfobs=None, out=None, partials=None):
    """The rms/std/volume record of one assimilation iteration (igm_assim_stats):
    device double[9] rmsthk, stdthk, rmsvel, stdvel, rmsdiv, stddiv, rmsusurf,
    stdusurf, vol; an observation given as None gives 0 for its pair."""
    ny, nx = thk.shape
    out = out if out is not None else torch.empty(9, dtype=torch.float64, device=thk.device)
    partials = partials if partials is not None else torch.empty(148 * 8 * 13, dtype=torch.float64,
                                                                 device=thk.device)
    rc = L.lib().igm_assim_stats(L.dtype_code(thk.dtype), ny, nx, float(dx), L.ptr(thk), L.ptr(thkobs), L.ptr(uvs),
                                 L.ptr(vvs), L.ptr(uobs), L.ptr(vobs), L.ptr(icemaskobs), L.ptr(divflux),
                                 L.ptr(divfluxobs), L.ptr(usurf), L.ptr(usurfobs), L.ptr(partials),
                                 partials.numel() // 13, L.ptr(out), L.stream_ptr())
    L.check(rc, "igm_assim_stats")
    return out


DIVFLUX_METHODS = {"upwind": 0, "centered": 1}


def divflux(u, v, h, dx, method="upwind", out=None):
    """compute_divflux (igm_divflux), method "upwind" or "centered"."""
    if method not in DIVFLUX_METHODS:
        raise NotImplementedError(f"divflux method {method!r}")
    ny, nx = h.shape
    out = out if out is not None else torch.empty_like(h)
    rc = L.lib().igm_divflux(L.dtype_code(h.dtype), DIVFLUX_METHODS[method], ny, nx, float(dx), L.ptr(u), L.ptr(v),
                             L.ptr(h), L.ptr(out), L.stream_ptr())
    L.check(rc, "igm_divflux")
    return out


def divflux_upwind(u, v, h, dx, out=None):
    return divflux(u, v, h, dx, "upwind", out)


def assim_divflux_cost_grad(kind, ubar, vbar, thk, D, dx, icemaskobs, g_thk, dU, dV, vert_weight, *, divfluxobs=None,
                            usurf=None, slope=0.0, intercept=0.0, std=1.0, regu=1.0, force_zero_sum=False,
                            method="upwind", mask_thk=None, scratch=None, partials=None, cost=None):
    """The flux-divergence cost (igm_assim_divflux_cost_grad), kind "obs"
    (cost_divfluxobs) or "fcz" (cost_divfluxfcz): returns the device cost
    (double[1]); adds dC/dthk into g_thk and dC/d(ubar, vbar) times the
    vertical weights into dU, dV [nz, ny, nx] (added on the top level,
    assigned below)."""
    ny, nx = thk.shape
    nz = int(dU.shape[-3])
    lib = L.lib()
    n_parts = 148 * 8
    if partials is None:
        partials = torch.empty(int(lib.igm_assim_divflux_partials_len(n_parts)), dtype=torch.float64,
                               device=thk.device)
    else:
        n_parts = (partials.numel() - 3) // 6
    scratch = scratch if scratch is not None else torch.empty_like(thk)
    cost = cost if cost is not None else torch.empty(1, dtype=torch.float64, device=thk.device)
    p = L.DivfluxCostParams()
    p.kind = {"obs": 0, "fcz": 1}[kind]
    p.method = DIVFLUX_METHODS[method]
    p.force_zero_sum = int(bool(force_zero_sum))
    p.divfluxobs_std, p.regu_divflux, p.slope, p.intercept = float(std), float(regu), float(slope), float(intercept)
    w = (C.c_double * nz)(*[float(x) for x in np.asarray(vert_weight, dtype=np.float64).reshape(-1)[:nz]])
    rc = lib.igm_assim_divflux_cost_grad(L.dtype_code(thk.dtype), ny, nx, float(dx), nz, w, L.ptr(ubar), L.ptr(vbar),
                                         L.ptr(thk), L.ptr(D), L.ptr(divfluxobs), L.ptr(usurf), L.ptr(icemaskobs),
                                         L.ptr(mask_thk), C.byref(p), L.ptr(g_thk), L.ptr(dU), L.ptr(dV),
                                         L.ptr(scratch), L.ptr(partials), n_parts, L.ptr(cost), L.stream_ptr())
    L.check(rc, "igm_assim_divflux_cost_grad")
    return cost
