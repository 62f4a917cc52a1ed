"""Data-assimilation kernels through the C ABI: the cost terms and their
gradients against the reference's cost_terms executed on the same inputs
(golden vectors; FP64 to 1e-9, FP32 to 1e-4 relative), the flow directions
against the reference's utils (1e-5), the upwind divergence bit-identical to
the oracle."""

import numpy as np
import pytest
import torch

from igm_b200 import _lib as L
from igm_b200 import kernels as K
from oracle import iceflow_oracle as O
from tests.gpu_util import dev

pytestmark = pytest.mark.gpu


def _params(g, aniso):
    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, 0.0, 3.0, 10.0
    area = float((g["icemaskobs"] > 0.5).sum()) * float(g["dx"]) ** 2
    p.gamma = 0.002 * area ** (1.3 - 2.0)
    p.aniso_factor = 0.2 if aniso else 1.0
    vo = np.stack([g["uobs"], g["vobs"]], -1)
    rel = np.sqrt((vo.astype(np.float64) ** 2).sum(-1)) >= 0.0
    p.n_vel = float((~np.isnan(vo) & rel[..., None]).sum())
    p.n_thk = float((~np.isnan(g["thkobs"])).sum())
    p.penalty, p.icemask_cost, p.regularize_thk = 1, 1, int(bool(g["to_thk"]))
    return p


@pytest.mark.parametrize("tag", ["f64", "f32", "iso_f64", "thk_f64"])
def test_cost_and_gradient_match_reference(golden, tag):
    g = {k[len(tag) + 1:]: v for k, v in golden("assim").items() if k.startswith(tag + "_")}
    aniso = bool(g["aniso"])
    dt = torch.float64 if g["thk"].dtype == np.float64 else torch.float32
    d = {k: dev(g[k], dt) for k in ["thk", "usurf", "uvs", "vvs", "uobs", "vobs", "thkobs", "dens", "icemaskobs"]}
    flow = (dev(g["flowdirx"], dt), dev(g["flowdiry"], dt)) if aniso else None
    costs, gt, gu, gv = K.assim_cost_grad(d["thk"], d["usurf"], d["uvs"], d["vvs"], d["uobs"], d["vobs"],
                                          d["thkobs"], d["dens"], d["icemaskobs"], flow, float(g["dx"]),
                                          _params(g, aniso))
    tol = 1e-9 if dt == torch.float64 else 1e-4
    c = costs.cpu().numpy()[:5]
    ref = [float(g[k]) for k in ["c_vel", "c_thk", "c_ice", "c_pos", "c_reg"]]
    np.testing.assert_allclose(c, ref, rtol=tol, atol=tol * max(abs(x) for x in ref))
    for a, k in [(gt, "g_thk"), (gu, "g_u"), (gv, "g_v")]:
        np.testing.assert_allclose(a.cpu().numpy(), g[k], rtol=tol, atol=tol * np.abs(g[k]).max())


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_flow_direction_matches_reference(golden, tag):
    g = {k[len(tag) + 1:]: v for k, v in golden("assim").items() if k.startswith(tag + "_")}
    dt = torch.float64 if g["thk"].dtype == np.float64 else torch.float32
    fx, fy = K.assim_flow_direction(dev(g["uvs"], dt), dev(g["vvs"], dt))
    np.testing.assert_allclose(fx.cpu().numpy(), g["flowdirx"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(fy.cpu().numpy(), g["flowdiry"], rtol=1e-5, atol=1e-5)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("shape", [(2, 2), (17, 13), (257, 300)])
def test_divflux_upwind_bit_exact(dtype, shape):
    rng = np.random.default_rng(shape[0])
    ny, nx = shape
    h = np.maximum(0, rng.normal(80, 90, (ny, nx)))
    u, v = rng.normal(0, 50, (ny, nx)), rng.normal(0, 50, (ny, nx))
    npd = np.float32 if dtype == torch.float32 else np.float64
    h, u, v = (a.astype(npd) for a in (h, u, v))
    ref = O.divflux_upwind(torch.as_tensor(u), torch.as_tensor(v), torch.as_tensor(h), 50.0)
    out = K.divflux_upwind(dev(u), dev(v), dev(h), 50.0)
    np.testing.assert_array_equal(out.cpu().numpy(), ref.numpy())


STAT_KEYS = ["rmsthk", "stdthk", "rmsvel", "stdvel", "rmsdiv", "stddiv", "rmsusurf", "stdusurf", "vol"]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("present", ["all", "none", "empty_thk"])
def test_stats_match_oracle(dtype, present):
    rng = np.random.default_rng(7)
    ny, nx = 123, 301
    npd = np.float32 if dtype == torch.float32 else np.float64
    r = lambda *a: rng.normal(*a, (ny, nx)).astype(npd)
    thk = np.maximum(0, r(100, 60))
    f = dict(thk=thk, uvs=r(20, 10), vvs=r(0, 10), uobs=r(20, 10), vobs=r(0, 10), div=r(0, 1), divobs=r(0, 1),
             us=r(2000, 100), usobs=r(2000, 100), thkobs=np.where(rng.random((ny, nx)) < 0.05, thk + r(0, 5), np.nan),
             im=(rng.random((ny, nx)) < 0.7).astype(npd))
    f["uobs"][rng.random((ny, nx)) < 0.1] = np.nan
    f["vobs"][rng.random((ny, nx)) < 0.1] = np.nan
    if present == "empty_thk":
        f["thkobs"][:] = np.nan
    t = {k: torch.as_tensor(v) for k, v in f.items()}
    d = {k: dev(v) for k, v in f.items()}
    if present == "none":
        ours = K.assim_stats(d["thk"], 50.0, d["im"]).cpu().numpy()
        ref = O.da_rms_std(t["thk"], None, None, None, None, None, t["im"], 50.0)
    else:
        ours = K.assim_stats(d["thk"], 50.0, d["im"], thkobs=d["thkobs"], uvs=d["uvs"], vvs=d["vvs"],
                             uobs=d["uobs"], vobs=d["vobs"], divflux=d["div"], divfluxobs=d["divobs"], usurf=d["us"],
                             usurfobs=d["usobs"]).cpu().numpy()
        ref = O.da_rms_std(t["thk"], t["thkobs"], t["uvs"], t["vvs"], t["uobs"], t["vobs"], t["im"], 50.0,
                           divflux=t["div"], divfluxobs=t["divobs"], usurf=t["us"], usurfobs=t["usobs"])
    tol = 1e-5 if dtype == torch.float32 else 1e-9
    np.testing.assert_allclose(ours, [ref[k] for k in STAT_KEYS], rtol=tol, atol=tol)


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("method", ["upwind", "centered"])
def test_divflux_methods_match_reference(golden, tag, method):
    """compute_divflux of the reference source, bit for bit."""
    g = golden("divflux")
    dt = torch.float64 if tag == "f64" else torch.float32
    u, v, h = (dev(g[f"{tag}_{k}"], dt) for k in ("u", "v", "thk"))
    out = K.divflux(u, v, h, float(g[f"{tag}_dx"]), method)
    np.testing.assert_array_equal(out.cpu().numpy(), g[f"{tag}_div_{method}"])


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("method", ["upwind", "centered"])
@pytest.mark.parametrize("kind", ["obs", "obs_zs", "fcz", "fcz_zs"])
def test_divflux_cost_terms_match_reference(golden, tag, method, kind):
    """cost_divfluxobs / cost_divfluxfcz of the reference source and their
    gradients w.r.t. ubar, vbar (one level of weight 1, no mask) and thk."""
    g = golden("divflux")
    dt = torch.float64 if tag == "f64" else torch.float32
    key = f"{tag}_{method}_{kind}"
    d = {k: dev(g[f"{tag}_{k}"], dt) for k in ("u", "v", "thk", "usurf", "icemaskobs", "divfluxobs")}
    dx = float(g[f"{tag}_dx"])
    D = K.divflux(d["u"], d["v"], d["thk"], dx, method)
    ny, nx = D.shape
    gt = torch.zeros_like(D)
    dU, dV = torch.zeros((1, ny, nx), dtype=dt, device="cuda"), torch.zeros((1, ny, nx), dtype=dt, device="cuda")
    fcz = kind.startswith("fcz")
    c = K.assim_divflux_cost_grad("fcz" if fcz else "obs", d["u"], d["v"], d["thk"], D, dx, d["icemaskobs"], gt, dU,
                                  dV, [1.0], divfluxobs=None if fcz else d["divfluxobs"],
                                  usurf=d["usurf"] if fcz else None,
                                  slope=float(g[f"{key}_slope"]) if fcz else 0.0,
                                  intercept=float(g[f"{key}_intercept"]) if fcz else 0.0, std=0.7, regu=3.0,
                                  force_zero_sum=kind.endswith("_zs"), method=method)
    tol = 1e-9 if tag == "f64" else 1e-4
    np.testing.assert_allclose(float(c.item()), float(g[f"{key}_cost"]), rtol=tol)
    for a, k in [(gt, "g_h"), (dU[0], "g_u"), (dV[0], "g_v")]:
        ref = g[f"{key}_{k}"]
        np.testing.assert_allclose(a.cpu().numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())


def test_divflux_gradient_levels_and_mask(golden):
    """The velbar gradient spread over the levels with the vertical weights,
    zero where the thk mask is off, added on the top level (which holds the
    surface-velocity gradient) and assigned below."""
    g = golden("divflux")
    d = {k: dev(g[f"f64_{k}"], torch.float64) for k in ("u", "v", "thk", "icemaskobs", "divfluxobs")}
    D = K.divflux(d["u"], d["v"], d["thk"], 100.0, "upwind")
    ny, nx = D.shape
    w = [0.2, 0.5, 0.3]
    mask = d["thk"].clone()
    mask[:, :5] = 0.0
    top_u = torch.rand((ny, nx), dtype=torch.float64, device="cuda")
    dU = torch.full((3, ny, nx), 7.0, dtype=torch.float64, device="cuda")
    dV = torch.full((3, ny, nx), 7.0, dtype=torch.float64, device="cuda")
    dU[2], dV[2] = top_u, top_u
    gt = torch.zeros_like(D)
    K.assim_divflux_cost_grad("obs", d["u"], d["v"], d["thk"], D, 100.0, d["icemaskobs"], gt, dU, dV, w,
                              divfluxobs=d["divfluxobs"], std=0.7, regu=3.0, mask_thk=mask)
    ref_u = torch.as_tensor(g["f64_upwind_obs_g_u"], device="cuda") * (mask > 0)
    ref_v = torch.as_tensor(g["f64_upwind_obs_g_v"], device="cuda") * (mask > 0)
    for k in range(3):
        extra = top_u if k == 2 else 0.0
        torch.testing.assert_close(dU[k], w[k] * ref_u + extra, rtol=1e-9, atol=1e-12)
        torch.testing.assert_close(dV[k], w[k] * ref_v + extra, rtol=1e-9, atol=1e-12)



@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_other_control_terms_match_reference(golden, tag):
    """regu_slidingco (isotropic, anisotropic), regu_arrhenius and the
    slidingco / arrhenius penalties through igm_assim_field_regu; misfit_usurf
    and regu_thk's usurf gradient (bed usurf - thk) through
    igm_assim_cost_grad's usurf output; against the reference source."""
    g = golden("assim_controls")
    dt = torch.float64 if tag == "f64" else torch.float32
    d = {k: dev(g[f"{tag}_{k}"], dt) for k in ("thk", "usurf", "slidingco", "arrhenius", "usurfobs", "icemaskobs")}
    dx = float(g[f"{tag}_dx"])
    tol = 1e-9 if tag == "f64" else 1e-4

    def close(a, ref):
        ref = np.asarray(ref)
        np.testing.assert_allclose(np.asarray(a), ref, rtol=tol, atol=tol * max(np.abs(ref).max(), 1e-30))

    for mode, aniso in (("sliso", 1.0), ("slaniso", 0.3)):
        flow = (dev(g[f"{tag}_{mode}_flowdirx"], dt), dev(g[f"{tag}_{mode}_flowdiry"], dt))
        c, gr = K.assim_field_regu(d["slidingco"], dx, 7.0, aniso, flow if aniso != 1.0 else None, penalty=False)
        close(c[4].item(), g[f"{tag}_{mode}_regu_slidingco"])
        close(gr.cpu().numpy(), g[f"{tag}_{mode}_g_slidingco"])
    c, gr = K.assim_field_regu(d["slidingco"], dx, 0.0, penalty=True, threshold=0.0)
    close(c[3].item(), g[f"{tag}_pen_slidingco"])
    close(gr.cpu().numpy(), g[f"{tag}_g_pen_slidingco"])
    c, gr = K.assim_field_regu(d["arrhenius"], dx, 2.0, penalty=True, threshold=1.0)
    close(c[4].item(), g[f"{tag}_regu_arrhenius"])
    close(c[3].item(), g[f"{tag}_pen_arrhenius"])
    close(gr.cpu().numpy(), g[f"{tag}_g_arrhenius"] + g[f"{tag}_g_pen_arrhenius"])
    # misfit_usurf + regu_thk (topg, isotropic): dC/dusurf
    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, 0.0, 3.0, 10.0
    area = float((g[f"{tag}_icemaskobs"] > 0.5).sum()) * dx ** 2
    p.gamma, p.aniso_factor, p.n_vel, p.n_thk = 0.002 * area ** (1.3 - 2.0), 1.0, 1.0, 1.0
    p.penalty, p.icemask_cost, p.regularize_thk, p.mask_velsurf = 0, 0, 0, 1
    p.usurf_cost, p.usurfobs_std = 1, 1.5
    p.n_usurf = float((g[f"{tag}_icemaskobs"] > 0.5).sum())
    nan = torch.full_like(d["thk"], float("nan"))
    zero = torch.zeros_like(d["thk"])
    g_us = torch.empty_like(d["thk"])
    costs, _, _, _ = K.assim_cost_grad(d["thk"], d["usurf"], zero, zero, nan, nan, nan, zero, d["icemaskobs"], None, dx,
                                       p, usurfobs=d["usurfobs"], g_us=g_us)
    c = costs.cpu().numpy()
    close(c[5], g[f"{tag}_misfit_usurf"])
    close(c[4], g[f"{tag}_regu_thk_topg"])
    close(g_us.cpu().numpy(), g[f"{tag}_g_usurf"] + g[f"{tag}_g_usurf_regu_thk"])



@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["iso", "aniso"])
def test_normalised_regularisations_match_reference(golden, tag, mode):
    """regu_thk (through igm_assim_cost_grad), regu_slidingco and
    regu_arrhenius (igm_assim_field_regu) with fix_opti_normalization_issue,
    against the reference source."""
    g = golden("assim_controls")
    dt = torch.float64 if tag == "f64" else torch.float32
    d = {k: dev(g[f"{tag}_{k}"], dt) for k in ("thk", "usurf", "slidingco", "arrhenius", "icemaskobs")}
    dx = float(g[f"{tag}_dx"])
    key = f"{tag}_norm_{mode}"
    tol = 1e-9 if tag == "f64" else 1e-4
    flow = (dev(g[f"{tag}_slaniso_flowdirx"], dt), dev(g[f"{tag}_slaniso_flowdiry"], dt))

    def close(a, ref):
        ref = np.asarray(ref)
        np.testing.assert_allclose(np.asarray(a), ref, rtol=tol, atol=tol * max(np.abs(ref).max(), 1e-30))

    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, 0.0, 3.0, 10.0
    area = float((g[f"{tag}_icemaskobs"] > 0.5).sum()) * dx ** 2
    p.gamma, p.n_vel, p.n_thk = 0.002 * area ** (1.3 - 2.0), 1.0, 1.0
    p.aniso_factor = 0.2 if mode == "aniso" else 1.0
    p.penalty, p.icemask_cost, p.regularize_thk, p.mask_velsurf, p.fix_normalization = 0, 0, 0, 1, 1
    nan = torch.full_like(d["thk"], float("nan"))
    zero = torch.zeros_like(d["thk"])
    costs, gt, _, _ = K.assim_cost_grad(d["thk"], d["usurf"], zero, zero, nan, nan, nan, zero, d["icemaskobs"],
                                        flow if mode == "aniso" else None, dx, p)
    close(costs.cpu().numpy()[4], g[f"{key}_regu_thk"])
    close(gt.cpu().numpy(), g[f"{key}_g_thk"])
    for field, w, an in (("slidingco", 7.0, 0.3 if mode == "aniso" else 1.0), ("arrhenius", 2.0, 1.0)):
        c, gr = K.assim_field_regu(d[field], dx, w, an, flow if an != 1.0 else None, penalty=False,
                                   fix_normalization=True)
        close(c[4].item(), g[f"{key}_regu_{field}"])
        close(gr.cpu().numpy(), g[f"{key}_g_{field}"])


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("thr", [0.0, 15.0])
def test_low_speed_term_matches_reference(golden, tag, thr):
    """misfit_velsurf with include_low_speed_term: igm_assim_cost_grad's
    velsurf cost and gradient plus igm_assim_low_speed, against the
    reference source."""
    g = golden("assim_controls")
    dt = torch.float64 if tag == "f64" else torch.float32
    d = {k: dev(g[f"{tag}_{k}"], dt) for k in ("thk", "usurf", "uvs", "vvs", "uobs", "vobs", "icemaskobs")}
    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, thr, 3.0, 0.0
    p.gamma, p.aniso_factor, p.n_thk = 0.0, 1.0, 1.0
    vo = np.stack([g[f"{tag}_uobs"], g[f"{tag}_vobs"]], -1).astype(np.float64)
    rel = np.sqrt((vo ** 2).sum(-1)) >= thr
    p.n_vel = float((~np.isnan(vo) & rel[..., None]).sum())
    p.penalty, p.icemask_cost, p.regularize_thk, p.mask_velsurf = 0, 0, 0, 0
    nan = torch.full_like(d["thk"], float("nan"))
    zero = torch.zeros_like(d["thk"])
    costs, _, gu, gv = K.assim_cost_grad(d["thk"], d["usurf"], d["uvs"], d["vvs"], d["uobs"], d["vobs"], nan, zero,
                                         d["icemaskobs"], None, 100.0, p)
    K.assim_low_speed(d["uvs"], d["vvs"], d["uobs"], d["vobs"], gu, gv, costs[0:1])
    key = f"{tag}_vel_thr{int(thr)}_low"
    tol = 1e-9 if tag == "f64" else 1e-4
    np.testing.assert_allclose(float(costs[0].item()), float(g[f"{key}_cost"]), rtol=tol)
    for a, k in ((gu, "g_u"), (gv, "g_v")):
        ref = g[f"{key}_{k}"]
        np.testing.assert_allclose(a.cpu().numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["iso", "aniso"])
def test_sole_mask_regularisations_match_reference(golden, tag, mode):
    """regu_thk (igm_assim_cost_grad), regu_slidingco and regu_arrhenius
    (igm_assim_field_regu) with sole_mask, against the reference source."""
    g = golden("assim_controls")
    dt = torch.float64 if tag == "f64" else torch.float32
    d = {k: dev(g[f"{tag}_{k}"], dt) for k in ("thk", "usurf", "slidingco", "arrhenius", "icemaskobs3")}
    dx = float(g[f"{tag}_dx"])
    key = f"{tag}_sole_{mode}"
    tol = 1e-9 if tag == "f64" else 1e-4
    flow = (dev(g[f"{tag}_slaniso_flowdirx"], dt), dev(g[f"{tag}_slaniso_flowdiry"], dt))

    def close(a, ref):
        ref = np.asarray(ref)
        np.testing.assert_allclose(np.asarray(a), ref, rtol=tol, atol=tol * max(np.abs(ref).max(), 1e-30))

    p = L.AssimParams()
    p.velsurfobs_std, p.velsurfobs_thr, p.thkobs_std, p.regu_thk = 1.0, 0.0, 3.0, 10.0
    area = float((g[f"{tag}_icemaskobs"] > 0.5).sum()) * dx ** 2
    p.gamma, p.n_vel, p.n_thk = 0.002 * area ** (1.3 - 2.0), 1.0, 1.0
    p.aniso_factor = 0.2 if mode == "aniso" else 1.0
    p.penalty, p.icemask_cost, p.regularize_thk, p.mask_velsurf, p.sole_mask = 0, 0, 0, 1, 1
    nan = torch.full_like(d["thk"], float("nan"))
    zero = torch.zeros_like(d["thk"])
    costs, gt, _, _ = K.assim_cost_grad(d["thk"], d["usurf"], zero, zero, nan, nan, nan, zero, d["icemaskobs3"],
                                        flow if mode == "aniso" else None, dx, p)
    close(costs.cpu().numpy()[4], g[f"{key}_regu_thk"])
    close(gt.cpu().numpy(), g[f"{key}_g_thk"])
    for field, w, an in (("slidingco", 7.0, 0.3 if mode == "aniso" else 1.0), ("arrhenius", 2.0, 1.0)):
        c, gr = K.assim_field_regu(d[field], dx, w, an, flow if an != 1.0 else None, penalty=False,
                                   sole_mask_icemaskobs=d["icemaskobs3"])
        close(c[4].item(), g[f"{key}_regu_{field}"])
        close(gr.cpu().numpy(), g[f"{key}_g_{field}"])
