"""The oracle against golden vectors produced by the reference's own source
(tests/golden/make_golden.py).  CPU only."""

import numpy as np
import pytest
import torch

from oracle import iceflow_oracle as O


def T(a):
    return torch.as_tensor(a)


@pytest.fixture(autouse=True)
def single_thread():
    """The golden vectors were generated with one CPU thread; torch's reduction
    order depends on the thread count, and the solver's early-stopping test
    (a threshold on the relative energy change) can flip on the last bits."""
    n = torch.get_num_threads()
    torch.set_num_threads(1)
    yield
    torch.set_num_threads(n)


def test_vert_disc(golden):
    g = golden("vert_disc")
    for nz in [2, 3, 5, 10, 16, 30]:
        for sp in [1.0, 2.0, 4.0]:
            k = f"nz{nz}_s{int(sp)}"
            lv = O.compute_levels(nz, sp)
            z, dz = O.compute_zeta_dzeta(lv)
            w = O.define_vertical_weight(nz, sp)[:, 0, 0]
            np.testing.assert_array_equal(lv.numpy(), g[k + "_levels"])
            np.testing.assert_array_equal(z.numpy(), g[k + "_zeta"])
            np.testing.assert_array_equal(dz.numpy(), g[k + "_dzeta"])
            np.testing.assert_array_equal(w.numpy(), g[k + "_weight"])


@pytest.mark.parametrize("case", ["small_f64", "small_f32", "nz2_f64", "mid_f32", "mid_f64", "nz16_f64"])
def test_energy_and_autodiff_gradient(golden, case):
    g = golden(f"energy_{case}")
    f64 = g["U"].dtype == np.float64
    rtol = 1e-12 if f64 else 2e-6
    args = [T(g[k]) for k in ["U", "V", "thk", "usurf", "arrhenius", "slidingco"]]
    dx = float(g["dx"])
    terms = O.energy_terms(*args, dx, T(g["dzeta"]))
    for name, t in zip(["shear", "sliding", "gravity"], terms):
        np.testing.assert_allclose(t[0].numpy(), g[name], rtol=rtol, atol=rtol * np.abs(g[name]).max())
    cost, means, gU, gV = O.energy_and_grad(*args, dx, T(g["dzeta"]))
    np.testing.assert_allclose(float(cost), float(g["cost"]), rtol=rtol)
    for a, b in [(gU, g["gradU"]), (gV, g["gradV"])]:
        np.testing.assert_allclose(a.numpy(), b, rtol=rtol * 10, atol=rtol * 10 * np.abs(b).max())


@pytest.mark.parametrize("case,nsolve", [("f64", 3), ("f32", 2)])
def test_solver_sequence(golden, case, nsolve):
    """solve_iceflow called repeatedly on one optimizer: the Adam iteration
    counter carries over between solves while the moment slots restart."""
    g = golden(f"solver_{case}")
    f64 = case == "f64"
    dt = torch.float64 if f64 else torch.float32
    thk, usurf, A, c = (T(g[k]) for k in ["thk", "usurf", "arrhenius", "slidingco"])
    nz = g["s0_U"].shape[0]
    dzeta = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).to(dt))[1]
    vw = O.define_vertical_weight(nz, 4.0).to(dt)
    opt = O.KerasLegacyAdam(lr=1.0)
    U = torch.zeros((nz,) + thk.shape, dtype=dt)
    V = torch.zeros_like(U)
    for s in range(nsolve):
        U, V, costs = O.solve_iceflow(U, V, thk, usurf, A, c, float(g["dx"]), dzeta, opt, nbitmax=int(g["nbitmax"]))
        assert len(costs) == len(g[f"s{s}_costs"])
        assert opt.iterations == int(g[f"s{s}_iterations_after"])
        tol = 1e-9 if f64 else 2e-3
        np.testing.assert_allclose(costs, g[f"s{s}_costs"], rtol=tol)
        scale = np.abs(g[f"s{s}_U"]).max()
        np.testing.assert_allclose(U.numpy(), g[f"s{s}_U"], rtol=tol, atol=tol * scale)
        np.testing.assert_allclose(V.numpy(), g[f"s{s}_V"], rtol=tol, atol=tol * scale)
        ub, vb = O.get_velbar(U, V, vw)
        np.testing.assert_allclose(ub.numpy(), g[f"s{s}_ubar"], rtol=tol, atol=tol * scale)


def test_divflux_all_limiters(golden):
    g = golden("transport")
    for tag in ["f32", "f64"]:
        h, u, v = T(g[f"{tag}_h"]), T(g[f"{tag}_u"]), T(g[f"{tag}_v"])
        for st in ["godunov", "minmod", "superbee"]:
            out = O.compute_divflux_slope_limiter(u, v, h, 50.0, 50.0, 0.7, st)
            np.testing.assert_array_equal(out.numpy(), g[f"{tag}_{st}"])


def test_thk_update(golden):
    g = golden("transport")
    lsurf, usurf = O.thk_surfaces(T(g["thk_h"]), T(g["thk_topg"]))
    np.testing.assert_array_equal(usurf.numpy(), g["thk_init_usurf"])
    thk, lsurf, usurf, div = O.thk_update(T(g["thk_h"]), T(g["thk_topg"]), T(g["f32_u"]), T(g["f32_v"]),
                                          T(g["thk_smb"]), 50.0, torch.tensor(0.7))
    for a, k in [(thk, "thk_new"), (lsurf, "thk_lsurf"), (usurf, "thk_usurf"), (div, "thk_divflux")]:
        np.testing.assert_array_equal(a.numpy(), g[k])


def test_clock(golden):
    g = golden("time")
    rng = np.random.default_rng(3)
    clk = O.Clock(start=0.0, end=3.0, save=1.0)
    ts, dts = [], []
    for k in range(12):
        sc = [80.0, 120.0, 15.0, 300.0][k % 4]
        ub = T(rng.normal(0, sc, (6, 5)).astype(np.float32))
        vb = T(rng.normal(0, sc, (6, 5)).astype(np.float32))
        clk.update(ub, vb, 100.0, k)
        ts.append(clk.t)
        dts.append(clk.dt)
        if not clk.continue_run:
            break
    np.testing.assert_allclose(ts, g["t"], rtol=1e-6)
    np.testing.assert_allclose(dts, g["dt"], rtol=1e-5)


def test_emulator_retrain_loop(golden):
    """Patch split, lr schedule, clipnorm and iteration gating of the
    emulator retraining (emulate.py:155-281), in float64."""
    g = golden("emulator")
    nz = g["U"].shape[0]
    thk, usurf, A, c = (T(g[k]) for k in ["thk", "usurf", "arrhenius", "slidingco"])
    X = O.fieldin_to_X([thk, usurf, A, c, torch.full_like(thk, float(g["dx"]))])
    params = [T(g[f"w0_{i}"]).clone() for i in range(6)]
    ws, bs = params[0::2], params[1::2]
    dzeta = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).to(torch.float64))[1]
    opt = O.KerasLegacyAdam(lr=1e-3, epsilon=1e-7, clipnorm=1.0)
    tr = O.EmulatorTraining(retrain_freq=2, lr=1e-3, lr_init=3e-3, warm_up_it=0, nbit_init=3, nbit=2, framesizemax=9)
    for step, it in enumerate([0, 1, 2]):
        O.emulator_retrain(ws, bs, opt, X, it, tr, nz, dzeta)
        for i, p in enumerate(params):
            np.testing.assert_allclose(p.numpy(), g[f"w{step + 1}_{i}"], rtol=1e-9, atol=1e-12)
    assert opt.iterations == int(g["opt_iterations"])
    Y = O.cnn_forward(X, ws, bs)
    U, V = O.Y_to_UV(Y, nz)
    mask = (thk > 0)[None]
    U = torch.where(mask, U[0], 0.0)
    np.testing.assert_allclose(U.numpy(), g["U"], rtol=1e-9, atol=1e-9 * np.abs(g["U"]).max())


@pytest.mark.parametrize("tag", ["f32", "f64", "nz5_f32", "nz2_f32"])
def test_vertical_velocity_kinematic(golden, tag):
    """vert_flow version 2, kinematic: bit-identical to the reference's
    compute_w_kinematic_tf (FP32 and FP64)."""
    g = golden("vert_flow")
    W = O.vertical_velocity_kinematic(T(g[f"{tag}_U"]), T(g[f"{tag}_V"]), T(g[f"{tag}_topg"]), T(g[f"{tag}_thk"]),
                                      T(g[f"{tag}_levels"]), T(g[f"{tag}_weight"])[:, None, None],
                                      float(g[f"{tag}_dx"]))
    np.testing.assert_array_equal(W.numpy(), g[f"{tag}_W"])


def test_vertical_velocity_analytic():
    """Plug flow (U, V the same on every level) over a bed of uniform slope
    with uniform thickness: no divergence, so W = U dz/dx + V dz/dy = the bed
    slope times the flow on every layer (away from nothing: the extrapolated
    border faces of a linear field are exact too)."""
    ny, nx, nz, dx = 12, 15, 6, 100.0
    y, x = np.meshgrid(np.arange(ny) * dx, np.arange(nx) * dx, indexing="ij")
    topg = T(2000.0 - 0.05 * x + 0.02 * y)
    thk = T(np.full((ny, nx), 120.0))
    U = T(np.full((nz, ny, nx), 30.0))
    V = T(np.full((nz, ny, nx), -12.0))
    lv = O.compute_levels(nz, 1.0, torch.float64)
    w = O.define_vertical_weight(nz, 1.0, torch.float64)
    W = O.vertical_velocity_kinematic(U, V, topg, thk, lv, w, dx)
    np.testing.assert_allclose(W.numpy(), 30.0 * -0.05 + -12.0 * 0.02, rtol=1e-12)


@pytest.mark.parametrize("tag", ["f32", "f64", "nz5_f32", "nz2_f32"])
def test_vertical_velocity_incompressibility(golden, tag):
    """vert_flow version 2, incompressibility: bit-identical to the
    reference's compute_vertical_velocity_incompressibility_v2 (uniform dX)."""
    g = golden("vert_flow")
    W = O.vertical_velocity_incompressibility(T(g[f"{tag}_U"]), T(g[f"{tag}_V"]), T(g[f"{tag}_topg"]),
                                              T(g[f"{tag}_thk"]), T(g[f"{tag}_levels"]),
                                              T(g[f"{tag}_weight"])[:, None, None], float(g[f"{tag}_dx"]))
    np.testing.assert_array_equal(W.numpy(), g[f"{tag}_Wi"])


@pytest.mark.parametrize("tag", ["f64", "f32", "iso_f64", "thk_f64"])
def test_assimilation_costs_and_gradients(golden, tag):
    """The data-assimilation cost terms and their gradients w.r.t. thk and the
    surface velocities, against the reference's cost_terms executed on the
    same inputs (FP64 to 1e-10: sums in another order; FP32 to 1e-5); the flow directions of the
    anisotropic regularisation against the reference's utils."""
    g = {k[len(tag) + 1:]: v for k, v in golden("assim").items() if k.startswith(tag + "_")}
    thk = T(g["thk"]).clone().requires_grad_(True)
    uvs, vvs = T(g["uvs"]).clone().requires_grad_(True), T(g["vvs"]).clone().requires_grad_(True)
    if bool(g["aniso"]):
        fx, fy = O.da_flow_direction(T(g["uvs"]), T(g["vvs"]))
        tol_f = 1e-6 if g["thk"].dtype == np.float64 else 1e-5
        np.testing.assert_allclose(fx.numpy(), g["flowdirx"], rtol=tol_f, atol=tol_f)
        np.testing.assert_allclose(fy.numpy(), g["flowdiry"], rtol=tol_f, atol=tol_f)
        flow = (T(g["flowdirx"]), T(g["flowdiry"]))
        f = 0.2
    else:
        flow, f = None, 1.0
    p = O.AssimParams(smooth_anisotropy_factor=f, to_regularize="thk" if bool(g["to_thk"]) else "topg")
    c = O.da_costs(thk, T(g["usurf"]), uvs, vvs, T(g["uobs"]), T(g["vobs"]), T(g["thkobs"]), T(g["dens"]),
                   T(g["icemaskobs"]), T(g["icemaskobs"]), flow, float(g["dx"]), p)
    tol = 1e-10 if g["thk"].dtype == np.float64 else 1e-5
    for k, ref in [("velsurf", "c_vel"), ("thk", "c_thk"), ("icemask", "c_ice"), ("thk_positive", "c_pos"),
                   ("thk_regu", "c_reg")]:
        np.testing.assert_allclose(c[k].item(), float(g[ref]), rtol=tol, atol=tol * abs(float(g[ref])) + 1e-30)
    gt, gu, gv = torch.autograd.grad(sum(c.values()), [thk, uvs, vvs])
    for a, ref in [(gt, "g_thk"), (gu, "g_u"), (gv, "g_v")]:
        np.testing.assert_allclose(a.numpy(), g[ref], rtol=tol, atol=tol * np.abs(g[ref]).max())


def test_divflux_upwind_conserves_mass():
    """compute_divflux, upwind: zero flux through the border for ice away from
    it, so the divergence sums to zero."""
    ny = nx = 40
    y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    h = T(np.maximum(0, 100 - ((y - 20) ** 2 + (x - 20) ** 2)).astype(np.float64))
    u = T(np.full((ny, nx), 7.0)); v = T(np.full((ny, nx), -3.0))
    d = O.divflux_upwind(u, v, h, 50.0)
    assert abs(float(d.sum())) < 1e-9 * float(h.sum())


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_compute_divflux_both_methods(golden, tag):
    """compute_divflux of the reference source, upwind and centered."""
    g = golden("divflux")
    u, v, h = (torch.as_tensor(g[f"{tag}_{k}"]) for k in ("u", "v", "thk"))
    for m in ("upwind", "centered"):
        out = O.compute_divflux(u, v, h, float(g[f"{tag}_dx"]), m).numpy()
        np.testing.assert_array_equal(out, g[f"{tag}_div_{m}"])


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("method", ["upwind", "centered"])
@pytest.mark.parametrize("kind", ["obs", "obs_zs", "fcz", "fcz_zs"])
def test_divflux_cost_terms(golden, tag, method, kind):
    """cost_divfluxobs / cost_divfluxfcz of the reference source, with their
    gradients w.r.t. ubar, vbar, thk; the fcz regression of the oracle against
    scipy's (run by the reference)."""
    g = golden("divflux")
    key = f"{tag}_{method}_{kind}"
    t = {k: torch.as_tensor(g[f"{tag}_{k}"]) for k in ("u", "v", "thk", "usurf", "icemaskobs", "divfluxobs")}
    u, v, h = (t[k].clone().requires_grad_(True) for k in ("u", "v", "thk"))
    dx = float(g[f"{tag}_dx"])
    kw = dict(std=0.7, regu=3.0, force_zero_sum=kind.endswith("_zs"), method=method)
    if kind.startswith("fcz"):
        act = t["icemaskobs"] > 0.5
        D = O.compute_divflux(t["u"], t["v"], t["thk"], dx, method)
        slope, intercept = O.linregress(t["usurf"][act].numpy(), D[act].numpy())
        tol_r = 1e-9 if tag == "f64" else 1e-4
        np.testing.assert_allclose([slope, intercept], [g[f"{key}_slope"], g[f"{key}_intercept"]], rtol=tol_r)
        c = O.da_cost_divflux("fcz", u, v, h, dx, t["icemaskobs"], usurf=t["usurf"],
                              slope=float(g[f"{key}_slope"]), intercept=float(g[f"{key}_intercept"]), **kw)
    else:
        c = O.da_cost_divflux("obs", u, v, h, dx, t["icemaskobs"], divfluxobs=t["divfluxobs"], **kw)
    gu, gv, gh = torch.autograd.grad(c, [u, v, h])
    tol = 1e-12 if tag == "f64" else 2e-5
    np.testing.assert_allclose(c.item(), float(g[f"{key}_cost"]), rtol=tol)
    for a, k in [(gu, "g_u"), (gv, "g_v"), (gh, "g_h")]:
        ref = g[f"{key}_{k}"]
        np.testing.assert_allclose(a.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_other_control_cost_terms(golden, tag):
    """regu_slidingco (isotropic and anisotropic), regu_arrhenius,
    misfit_usurf, the slidingco / arrhenius penalties and regu_thk's usurf
    gradient, against the reference source."""
    g = golden("assim_controls")
    t = {k: torch.as_tensor(g[f"{tag}_{k}"]) for k in ("thk", "usurf", "slidingco", "arrhenius", "usurfobs",
                                                       "icemaskobs")}
    dx = float(g[f"{tag}_dx"])
    tol = 1e-12 if tag == "f64" else 2e-5

    def check(c, gr, kc, kg, tol=tol):
        np.testing.assert_allclose(float(c.detach()), float(g[kc]), rtol=tol)
        ref = g[kg]
        np.testing.assert_allclose(gr.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())

    for mode, aniso in (("sliso", 1.0), ("slaniso", 0.3)):
        s = t["slidingco"].clone().requires_grad_(True)
        flow = (torch.as_tensor(g[f"{tag}_{mode}_flowdirx"]), torch.as_tensor(g[f"{tag}_{mode}_flowdiry"]))
        c = O.da_regu_field(s, dx, 7.0, aniso, flow)
        check(c, torch.autograd.grad(c, s)[0], f"{tag}_{mode}_regu_slidingco", f"{tag}_{mode}_g_slidingco")
    a = t["arrhenius"].clone().requires_grad_(True)
    c = O.da_regu_field(a, dx, 2.0)
    check(c, torch.autograd.grad(c, a)[0], f"{tag}_regu_arrhenius", f"{tag}_g_arrhenius")
    c = O.da_penalty(a, 1.0)
    check(c, torch.autograd.grad(c, a)[0], f"{tag}_pen_arrhenius", f"{tag}_g_pen_arrhenius")
    s = t["slidingco"].clone().requires_grad_(True)
    c = O.da_penalty(s, 0.0)
    check(c, torch.autograd.grad(c, s)[0], f"{tag}_pen_slidingco", f"{tag}_g_pen_slidingco")
    u = t["usurf"].clone().requires_grad_(True)
    c = O.da_misfit_usurf(u, t["usurfobs"], t["icemaskobs"], 1.5)
    check(c, torch.autograd.grad(c, u)[0], f"{tag}_misfit_usurf", f"{tag}_g_usurf")
    u = t["usurf"].clone().requires_grad_(True)
    p = O.AssimParams(regu_thk=10.0, smooth_anisotropy_factor=1.0, to_regularize="topg")
    c = O.da_costs(t["thk"], u, t["thk"] * 0, t["thk"] * 0, t["thk"] * 0, t["thk"] * 0,
                   torch.full_like(t["thk"], float("nan")), t["thk"] * 0, t["icemaskobs"], t["icemaskobs"], None, dx,
                   p)["thk_regu"]
    # the reference sums the ice-mask area in float32 (tf.where(..., 1.0, 0.0)): 1e-10 in FP64
    check(c, torch.autograd.grad(c, u)[0], f"{tag}_regu_thk_topg", f"{tag}_g_usurf_regu_thk",
          tol=max(tol, 1e-10))



@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["iso", "aniso"])
def test_normalised_regularisations(golden, tag, mode):
    """regu_thk, regu_slidingco, regu_arrhenius with
    fix_opti_normalization_issue, against the reference source."""
    g = golden("assim_controls")
    t = {k: torch.as_tensor(g[f"{tag}_{k}"]) for k in ("thk", "usurf", "slidingco", "arrhenius", "icemaskobs")}
    dx = float(g[f"{tag}_dx"])
    key = f"{tag}_norm_{mode}"
    tol = 1e-10 if tag == "f64" else 2e-5
    aniso = 0.2 if mode == "aniso" else 1.0
    flow = (torch.as_tensor(g[f"{tag}_slaniso_flowdirx"]), torch.as_tensor(g[f"{tag}_slaniso_flowdiry"]))
    th = t["thk"].clone().requires_grad_(True)
    p = O.AssimParams(regu_thk=10.0, smooth_anisotropy_factor=aniso, to_regularize="topg", fix_normalization=True)
    nan = torch.full_like(th, float("nan"))
    c = O.da_costs(th, t["usurf"], th * 0, th * 0, nan, nan, nan, th * 0, t["icemaskobs"], t["icemaskobs"], flow, dx,
                   p)["thk_regu"]
    gr = torch.autograd.grad(c, th)[0]
    np.testing.assert_allclose(float(c.detach()), float(g[f"{key}_regu_thk"]), rtol=tol)
    np.testing.assert_allclose(gr.numpy(), g[f"{key}_g_thk"], rtol=tol, atol=tol * np.abs(g[f"{key}_g_thk"]).max())
    for field, w, an in (("slidingco", 7.0, 0.3 if mode == "aniso" else 1.0), ("arrhenius", 2.0, 1.0)):
        x = t[field].clone().requires_grad_(True)
        c = O.da_regu_field(x, dx, w, an, flow, normalize=True)
        gr = torch.autograd.grad(c, x)[0]
        np.testing.assert_allclose(float(c.detach()), float(g[f"{key}_regu_{field}"]), rtol=tol)
        ref = g[f"{key}_g_{field}"]
        np.testing.assert_allclose(gr.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())



@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("case", ["thr0_plain", "thr0_low", "thr15_low"])
def test_velsurf_misfit_low_speed_term(golden, tag, case):
    """misfit_velsurf with and without include_low_speed_term and a speed
    threshold, against the reference source."""
    g = golden("assim_controls")
    u, v = (torch.as_tensor(g[f"{tag}_{k}"]).clone().requires_grad_(True) for k in ("uvs", "vvs"))
    uo, vo = torch.as_tensor(g[f"{tag}_uobs"]), torch.as_tensor(g[f"{tag}_vobs"])
    thr = 15.0 if case.startswith("thr15") else 0.0
    c = O.da_misfit_velsurf(u, v, uo, vo, 1.0, thr, case.endswith("low"))
    gu, gv = torch.autograd.grad(c, [u, v])
    key = f"{tag}_vel_{case}"
    tol = 1e-12 if tag == "f64" else 2e-5
    np.testing.assert_allclose(float(c.detach()), float(g[f"{key}_cost"]), rtol=tol)
    for a, k in ((gu, "g_u"), (gv, "g_v")):
        ref = g[f"{key}_{k}"]
        np.testing.assert_allclose(a.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())



@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("mode", ["iso", "aniso"])
def test_sole_mask_regularisations(golden, tag, mode):
    """regu_thk, regu_slidingco, regu_arrhenius with sole_mask (an ice mask
    with values 0, 1 and 2), against the reference source."""
    g = golden("assim_controls")
    t = {k: torch.as_tensor(g[f"{tag}_{k}"]) for k in ("thk", "usurf", "slidingco", "arrhenius", "icemaskobs",
                                                       "icemaskobs3")}
    dx = float(g[f"{tag}_dx"])
    key = f"{tag}_sole_{mode}"
    tol = 1e-10 if tag == "f64" else 2e-5
    aniso = 0.2 if mode == "aniso" else 1.0
    flow = (torch.as_tensor(g[f"{tag}_slaniso_flowdirx"]), torch.as_tensor(g[f"{tag}_slaniso_flowdiry"]))
    th = t["thk"].clone().requires_grad_(True)
    p = O.AssimParams(regu_thk=10.0, smooth_anisotropy_factor=aniso, to_regularize="topg", sole_mask=True)
    nan = torch.full_like(th, float("nan"))
    c = O.da_costs(th, t["usurf"], th * 0, th * 0, nan, nan, nan, th * 0, t["icemaskobs3"], t["icemaskobs"], flow,
                   dx, p)["thk_regu"]
    gr = torch.autograd.grad(c, th)[0]
    np.testing.assert_allclose(float(c.detach()), float(g[f"{key}_regu_thk"]), rtol=tol)
    np.testing.assert_allclose(gr.numpy(), g[f"{key}_g_thk"], rtol=tol, atol=tol * np.abs(g[f"{key}_g_thk"]).max())
    for field, w, an in (("slidingco", 7.0, 0.3 if mode == "aniso" else 1.0), ("arrhenius", 2.0, 1.0)):
        x = t[field].clone().requires_grad_(True)
        c = O.da_regu_field(x, dx, w, an, flow, icemaskobs=t["icemaskobs3"])
        gr = torch.autograd.grad(c, x)[0]
        np.testing.assert_allclose(float(c.detach()), float(g[f"{key}_regu_{field}"]), rtol=tol)
        ref = g[f"{key}_g_{field}"]
        np.testing.assert_allclose(gr.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())
