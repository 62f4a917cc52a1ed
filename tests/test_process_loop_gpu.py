"""The drop-in processes through initialize/update, several model time steps
of the reference's loop (smb_simple -> iceflow -> time -> thk, the order of
the reference's test experiment), against the oracle's restatement of each
step -- for iceflow methods "solved", "emulated" and "diagnostic" -- plus the
fallback decision and the emulator's save/load round trip.

Each step is replayed by the oracle from the device state at the start of
that step (thickness, surfaces, velocities, clock, optimizer counters), so a
difference is caught where it is made instead of accumulating:

* smb_simple (smb_simple.py:24-50) and the slope-limited transport with the
  surfaces (thk.py:27-54) are bit-identical, given the same inputs;
* the clock (time.py:28-65: CFL step, save-time snapping, t) is identical
  given the same depth-averaged velocities;
* the solve (solve.py:22-119: Adam on a persistent optimizer, early
  stopping, the thk == 0 mask) matches the FP32 oracle to 1e-4 relative L2
  and takes the same number of iterations;
* the emulator's forward (emulate.py:116-152) matches the oracle's
  bf16-operand network to 1e-2 and its retraining cost (emulate.py:155-281)
  to 2e-2 (the tolerances of the network tests);
* the diagnostic (diagnostic.py:34-84) writes the row of errors_diagno.txt
  that the oracle's solve from the emulated velocities gives.
"""

import os

import numpy as np
import pytest
import torch

from igm_b200 import emulator as E
from igm_b200.config import default_cfg
from igm_b200.processes import iceflow, smb_simple, thk
from igm_b200.processes import time as tproc
from igm_b200 import state as S
from igm_b200.state import State
from oracle import iceflow_oracle as O
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu

NZ = 4
DX = 100.0
SCALES = [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 100.0]
OUT = 50.0
TABLE = [["time", "gradabl", "gradacc", "ela", "accmax"], [0.0, 0.009, 0.009, 2900.0, 2.0],
         [100.0, 0.009, 0.005, 2950.0, 1.5]]


def make_cfg(method, retrain_freq=3, nbitmax=20, fallback_every=0, margin=0.02):
    return default_cfg({
        "iceflow": {"method": method, "numerics": {"Nz": NZ}, "solver": {"nbitmax": nbitmax},
                    "emulator": {"pretrained": False, "retrain_freq": retrain_freq, "lr": 1e-4,
                                 "framesizemax": 1000, "input_scales": SCALES, "output_scale": OUT, "seed": 3,
                                 "network": {"nb_layers": 3, "weight_initialization": "he_normal"}},
                    "fallback": {"every": fallback_every, "margin": margin, "nbitmax": nbitmax}},
        "time": {"start": 0.0, "end": 100.0, "save": 0.002, "cfl": 0.3, "step_max": 1.0},
        "smb_simple": {"array": TABLE, "update_freq": 0.0},
    })


def make_state(seed=2, ny=36, nx=44):
    g = O.valley_glacier(ny, nx, DX, seed=seed, varying_coeffs=True)
    st = State()
    for k in ("topg", "thk", "arrhenius", "slidingco"):
        setattr(st, k, torch.as_tensor(g[k]).cuda())
    st.dx = DX
    st.it = -1
    return st


def init(cfg, st):
    mods = [smb_simple, iceflow, tproc, thk]
    thk.initialize(cfg, st)  # usurf from topg + thk before iceflow reads it
    for m in mods:
        m.initialize(cfg, st)
    st.it = 0
    return mods


def cpu(t):
    return t.detach().cpu().clone()


def snapshot(st):
    s = {k: cpu(getattr(st, k)) for k in ("thk", "usurf", "topg", "arrhenius", "slidingco", "U", "V")}
    s.update(t=np.float32(st.t), itsave=int(st.itsave), it=int(st.it))
    if hasattr(st, "iceflow_solver"):
        s["solver_iterations"] = st.iceflow_solver.iterations
    if hasattr(st, "iceflow_model"):
        s["net"] = [torch.as_tensor(a.copy()) for a in st.iceflow_model.get_variables()]
        s["net_iterations"] = st.iceflow_model.opt_iterations
    return s


def oracle_smb(s):
    p = np.array(TABLE[1:], np.float32)
    par = [np.float32(O.interp1d(p[:, 0], p[:, j], float(s["t"]))) for j in range(1, 5)]
    return O.smb_simple(s["usurf"], *par)


def oracle_solve(s, U, V, n_iter_before, nbitmax):
    dz = torch.as_tensor(iceflow.compute_zeta_dzeta(iceflow.compute_levels(NZ, 4.0))[1])
    opt = O.KerasLegacyAdam(lr=1.0)
    opt.iterations = n_iter_before
    return O.solve_iceflow(U, V, s["thk"], s["usurf"], s["arrhenius"], s["slidingco"], DX, dz, opt, nbitmax=nbitmax)


def oracle_forward(weights, s):
    fl = [s[k] for k in ("thk", "usurf", "arrhenius", "slidingco")]
    X = O.fieldin_to_X(fl + [torch.full_like(fl[0], DX)]) * torch.tensor(SCALES, dtype=torch.float32)
    Y = O.cnn_forward(X, weights[0::2], weights[1::2], bf16=True, bf16_first=False, out_scale=OUT)
    U, V = O.Y_to_UV(Y, NZ)
    m = (s["thk"] > 0)[None]
    return torch.where(m, U[0], torch.zeros_like(U[0])), torch.where(m, V[0], torch.zeros_like(V[0]))


def oracle_retrain_cost(s):
    """Mean energy of the (unmasked) network output on the whole domain, the
    cost of one retraining step on one patch (emulate.py:207-252)."""
    fl = [s[k] for k in ("thk", "usurf", "arrhenius", "slidingco")]
    X = O.fieldin_to_X(fl + [torch.full_like(fl[0], DX)]) * torch.tensor(SCALES, dtype=torch.float32)
    Y = O.cnn_forward(X, s["net"][0::2], s["net"][1::2], bf16=True, bf16_first=False, out_scale=OUT)
    U, V = O.Y_to_UV(Y, NZ)
    dz = torch.as_tensor(iceflow.compute_zeta_dzeta(iceflow.compute_levels(NZ, 4.0))[1])
    cost, _ = O.energy(U, V, *[f[None] for f in fl], DX, dz)
    return float(cost)


def check_clock_and_transport(cfg, st, s, smb_used):
    w = torch.as_tensor(iceflow.define_vertical_weight(NZ, 4.0))
    ub, vb = O.get_velbar(cpu(st.U), cpu(st.V), w)
    assert rel_l2(cpu(st.ubar).numpy(), ub.numpy()) < 1e-6
    assert rel_l2(cpu(st.vbar).numpy(), vb.numpy()) < 1e-6
    c = cfg.processes.time
    clk = O.Clock(start=c.start, end=c.end, save=c.save, cfl=c.cfl, step_max=c.step_max)
    clk.t, clk.itsave = s["t"], s["itsave"]
    clk.update(cpu(st.ubar), cpu(st.vbar), DX, s["it"])
    assert np.float32(st.dt) == clk.dt and np.float32(st.t) == clk.t and st.saveresult == clk.saveresult
    th, ls, us, div = O.thk_update(s["thk"], s["topg"], cpu(st.ubar), cpu(st.vbar), smb_used, DX,
                                   torch.tensor(np.float32(st.dt)))
    for a, b in ((st.thk, th), (st.lsurf, ls), (st.usurf, us), (st.divflux, div)):
        np.testing.assert_array_equal(cpu(a).numpy(), b.numpy())


def test_solved_loop_matches_oracle():
    cfg = make_cfg("solved")
    st = make_state()
    mods = init(cfg, st)
    for k in range(8):
        s = snapshot(st)
        for m in mods:
            m.update(cfg, st)
        st.it += 1
        smb = oracle_smb(s)
        np.testing.assert_array_equal(cpu(st.smb).numpy(), smb.numpy())
        U, V, costs = oracle_solve(s, s["U"], s["V"], s["solver_iterations"], 20)
        assert st.iceflow_solver.iterations - s["solver_iterations"] == len(costs), k
        assert rel_l2(cpu(st.U).numpy(), U.numpy()) < 1e-4, k
        assert rel_l2(cpu(st.V).numpy(), V.numpy()) < 1e-4, k
        np.testing.assert_allclose(st.COST_Glen, costs[-1], rtol=1e-5)
        check_clock_and_transport(cfg, st, s, cpu(st.smb))
    assert st.it == 8 and float(st.t) > 0


def test_emulated_loop_matches_oracle():
    cfg = make_cfg("emulated", retrain_freq=3)
    st = make_state(seed=4)
    mods = init(cfg, st)
    retrained = 0
    for k in range(7):
        s = snapshot(st)
        n_costs = len(st.COST_EMULATOR)
        for m in mods:
            m.update(cfg, st)
        st.it += 1
        if s["it"] > 0 and s["it"] % 3 == 0:
            # one Adam step on the single patch: its cost is that of the weights before it
            cost = oracle_retrain_cost(s)
            np.testing.assert_allclose(st.COST_EMULATOR[-1], float(cost), rtol=2e-2)
            assert st.iceflow_model.opt_iterations == s["net_iterations"] + 1
            retrained += 1
        else:
            assert st.iceflow_model.opt_iterations == s["net_iterations"] and len(st.COST_EMULATOR) == n_costs
        # the forward of this step runs on the weights after the retraining
        w_now = [torch.as_tensor(a.copy()) for a in st.iceflow_model.get_variables()]
        Uo, Vo = oracle_forward(w_now, s)
        assert rel_l2(cpu(st.U).numpy(), Uo.numpy()) < 1e-2, k
        assert rel_l2(cpu(st.V).numpy(), Vo.numpy()) < 1e-2, k
        check_clock_and_transport(cfg, st, s, cpu(st.smb))
    assert retrained == 2


def test_diagnostic_row_matches_oracle(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    cfg = make_cfg("diagnostic", retrain_freq=0)
    st = make_state(seed=5)
    mods = init(cfg, st)
    s = snapshot(st)
    for m in mods:
        m.update(cfg, st)
    st.it += 1
    # the diagnostic solves from the emulated velocities and keeps them as the state's
    Ue, Ve = cpu(st.U), cpu(st.V)
    Us, Vs, costs = oracle_solve(s, Ue, Ve, s["solver_iterations"], 20)
    w = torch.as_tensor(iceflow.define_vertical_weight(NZ, 4.0)).double()
    ub, vb = O.get_velbar((Ue - Us).double(), (Ve - Vs).double(), w)
    ma = (s["thk"] > 1).double()
    l1 = float((ma * ub.abs()).sum() + (ma * vb.abs()).sum()) / float(2 * ma.sum())
    l2 = np.sqrt(float((ma * ub ** 2).sum() + (ma * vb ** 2).sum()) / float(2 * ma.sum()))
    row = np.loadtxt("errors_diagno.txt", delimiter=",", skiprows=1, ndmin=2)
    assert row.shape == (1, 8)
    t, rl1, rl2, cg, ce, nit, nem, vol = row[0]
    assert t == pytest.approx(float(s["t"]), abs=1e-3)
    assert rl1 == pytest.approx(l1, rel=1e-3, abs=2e-3) and rl2 == pytest.approx(l2, rel=1e-3, abs=2e-3)
    assert cg == pytest.approx(costs[-1], rel=1e-4, abs=2e-3)
    assert int(nit) == len(costs) and int(nem) == len(st.COST_EMULATOR)
    assert vol == pytest.approx(float(s["thk"].double().sum()) * DX ** 2 / 1e9, rel=1e-5, abs=2e-3)
    check_clock_and_transport(cfg, st, s, cpu(st.smb))


def device_emulated(st):
    """The emulator's (masked) velocities for the state as it is now, through
    the same device forward the iceflow process runs, copied out."""
    net = st.iceflow_model
    ny, nx = st.thk.shape
    buf = net.buffers(1, ny, nx, train=False)
    net.prepare_input([st.thk, st.usurf, st.arrhenius, st.slidingco], DX, [(0, 0)], ny, nx, buf)
    U, V = net.forward(buf, 1, ny, nx, thk_mask=st.thk)
    return U[0].clone(), V[0].clone()


@pytest.mark.parametrize("mode", ["step", "takeover"])
@pytest.mark.parametrize("margin,expect", [(-10.0, True), (1e9, False)])
def test_fallback_decision(margin, expect, mode):
    """margin -10 makes every check fall back (the emulated energy always
    exceeds the solved one minus ten times its magnitude); 1e9 never does.
    A check solves from the solver's last solution (the emulated velocities
    the first time) and is logged.  On fallback the state's velocities are
    that solve's (checked against the oracle's solve from the same start);
    mode "step" returns to the emulator at the next update, mode "takeover"
    keeps solving, warm-started from the previous solve, until the next check.
    Without fallback the velocities stay the emulated ones, bit for bit."""
    cfg = make_cfg("emulated", retrain_freq=0, fallback_every=2, margin=margin)
    cfg.processes.iceflow.fallback.mode = mode
    st = make_state(seed=6)
    mods = init(cfg, st)
    for k in range(4):
        s = snapshot(st)
        Ue, Ve = device_emulated(st)
        prev = st.__dict__.get("_igm_solved")
        prev = (cpu(prev[0]), cpu(prev[1])) if prev is not None else None
        for m in mods:
            m.update(cfg, st)
        st.it += 1
        log = st.fallback_log
        checked = len(log) > 0 and log[-1]["it"] == s["it"]
        assert checked == (k % 2 == 0)
        solving = expect and (checked or mode == "takeover")
        if solving:
            start = prev if (mode == "takeover" and prev is not None) else (cpu(Ue), cpu(Ve))
            Us, Vs, costs = oracle_solve(s, start[0], start[1], s["solver_iterations"], 20)
            if checked:
                assert log[-1]["fallback"] and log[-1]["solver_iterations"] == len(costs)
            assert st.iceflow_solver.iterations - s["solver_iterations"] == len(costs)
            assert rel_l2(cpu(st.U).numpy(), Us.numpy()) < 1e-4, k
            assert rel_l2(cpu(st.V).numpy(), Vs.numpy()) < 1e-4, k
            assert not torch.equal(st.U, Ue)
        else:
            assert not (checked and log[-1]["fallback"])
            assert torch.equal(st.U, Ue) and torch.equal(st.V, Ve)
        check_clock_and_transport(cfg, st, s, cpu(st.smb))
    assert len(st.fallback_log) == 2


def test_save_load_round_trip(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    cfg = make_cfg("emulated", retrain_freq=1)
    cfg.processes.iceflow.emulator.save_model = True
    st = make_state(seed=7)
    mods = init(cfg, st)
    for _ in range(2):
        for m in mods:
            m.update(cfg, st)
        st.it += 1
    iceflow.finalize(cfg, st)
    net = st.iceflow_model
    cfg2 = make_cfg("emulated", retrain_freq=1)
    cfg2.processes.iceflow.emulator.pretrained = True
    cfg2.processes.iceflow.emulator.name = "iceflow-model"
    st2 = make_state(seed=7)
    st2.original_cwd = str(tmp_path)
    thk.initialize(cfg2, st2)
    E.initialize_iceflow_emulator(cfg2, st2)
    net2 = st2.iceflow_model
    assert torch.equal(net.params, net2.params) and torch.equal(net.m, net2.m) and torch.equal(net.v, net2.v)
    assert net2.opt_iterations == net.opt_iterations and net2.out_scale == net.out_scale
    np.testing.assert_array_equal(net2.scales, net.scales)
    for f in ("fieldin.dat", "vert_grid.dat"):
        assert (tmp_path / "iceflow-model" / f).exists()
    # the same forward on both
    st.dzeta = st2.dzeta = iceflow.compute_zeta_dzeta(iceflow.compute_levels(NZ, 4.0))[1]
    st2.vert_weight = iceflow.define_vertical_weight(NZ, 4.0)
    for k in ("thk", "usurf"):
        setattr(st2, k, getattr(st, k).clone())
    E.update_iceflow_emulated(cfg, st)
    E.update_iceflow_emulated(cfg2, st2)
    assert torch.equal(st.U, st2.U) and torch.equal(st.V, st2.V)


def test_saved_keras_file_loads(tmp_path, monkeypatch):
    """The model.h5 that save_iceflow_model writes (the network on raw fields,
    its scales folded into the weights) loads through the reference's route
    -- a pretrained emulator directory holding model.h5 and fieldin.dat
    (emulate.py:64-93) -- and gives the saved network's velocities to the
    BF16 rounding of the refolded weights."""
    import shutil
    monkeypatch.chdir(tmp_path)
    cfg = make_cfg("emulated", retrain_freq=1)
    cfg.processes.iceflow.emulator.save_model = True
    st = make_state(seed=7)
    mods = init(cfg, st)
    for _ in range(2):
        for m in mods:
            m.update(cfg, st)
        st.it += 1
    iceflow.finalize(cfg, st)
    os.mkdir(tmp_path / "keras-only")
    for f in ("model.h5", "fieldin.dat", "vert_grid.dat"):
        shutil.copy(tmp_path / "iceflow-model" / f, tmp_path / "keras-only" / f)
    cfg2 = make_cfg("emulated", retrain_freq=1)
    cfg2.processes.iceflow.emulator.pretrained = True
    cfg2.processes.iceflow.emulator.name = "keras-only"
    st2 = make_state(seed=7)
    st2.original_cwd = str(tmp_path)
    thk.initialize(cfg2, st2)
    E.initialize_iceflow_emulator(cfg2, st2)
    net2 = st2.iceflow_model
    assert net2.out_scale == 1.0 and np.all(net2.scales == 1.0)
    st.dzeta = st2.dzeta = iceflow.compute_zeta_dzeta(iceflow.compute_levels(NZ, 4.0))[1]
    st2.vert_weight = iceflow.define_vertical_weight(NZ, 4.0)
    for k in ("thk", "usurf"):
        setattr(st2, k, getattr(st, k).clone())
    E.update_iceflow_emulated(cfg, st)
    E.update_iceflow_emulated(cfg2, st2)
    assert float(st.U.abs().max()) > 0
    assert rel_l2(cpu(st2.U).numpy(), cpu(st.U).numpy()) < 2e-2
    assert rel_l2(cpu(st2.V).numpy(), cpu(st.V).numpy()) < 2e-2


@pytest.mark.parametrize("method", ["emulated", "solved"])
def test_force_max_velbar_in_the_process(method):
    """With force_max_velbar > 0 the velocities the process leaves are capped
    (emulate.py:147-148, solve.py:178-179) before velbar, velbase and velsurf
    are derived from them."""
    cfg = make_cfg(method, retrain_freq=0)
    cfg.processes.iceflow.force_max_velbar = 5.0
    st = make_state(seed=8)
    mods = init(cfg, st)
    for m in mods:
        m.update(cfg, st)
    st.it += 1
    speed = torch.sqrt(st.U * st.U + st.V * st.V)
    assert float(speed.max()) <= 5.0 * (1 + 1e-6)
    w = torch.as_tensor(iceflow.define_vertical_weight(NZ, 4.0))
    ub, _ = O.get_velbar(cpu(st.U), cpu(st.V), w)
    assert rel_l2(cpu(st.ubar).numpy(), ub.numpy()) < 1e-6
    assert torch.equal(st.uvelsurf, st.U[-1]) and torch.equal(st.uvelbase, st.U[0])


def _host_and_device_states(cfg):
    """The same glacier as a device-resident state and as a host-resident
    one whose input fields are the caller's numpy arrays."""
    dev_st, host_st = make_state(seed=5), make_state(seed=5)
    orig = {}
    for k in ("topg", "thk", "arrhenius", "slidingco"):
        orig[k] = getattr(host_st, k).cpu().numpy().copy()
        setattr(host_st, k, orig[k].copy())
    host_st.device = "cuda"
    return dev_st, host_st, orig


def _steps(cfg, states, mods, n):
    for st, ms in zip(states, mods):
        for _ in range(n):
            for m in ms:
                m.update(cfg, st)
            st.it += 1


def _assert_same(dev_st, host_st, keys=("thk", "usurf", "ubar", "vbar", "smb")):
    S.sync_host(host_st)
    for k in keys:
        h = getattr(host_st, k)
        assert isinstance(h, np.ndarray), k
        assert torch.from_numpy(h).is_pinned(), k
        np.testing.assert_array_equal(h, cpu(getattr(dev_st, k)).numpy(), err_msg=k)
    assert float(host_st.t) == float(dev_st.t)


def test_host_resident_state_matches_device_resident():
    """The same three solved time steps with the state in host numpy arrays
    and on the device: identical fields once sync_host returned; the
    caller's input arrays are replaced by pinned arrays of the same values
    (so each copy is a DMA), the outputs come back as pinned numpy arrays,
    and a field the state holds on the device is not copied again."""
    cfg = make_cfg("solved", nbitmax=10)
    dev_st, host_st, orig = _host_and_device_states(cfg)
    mods = [init(cfg, st) for st in (dev_st, host_st)]
    for st in (dev_st, host_st):
        S.reset_transfer_counts(st)
    _steps(cfg, (dev_st, host_st), mods, 3)
    # each of the caller's four input fields goes to the device at most once over the run
    h2d, d2h = S.transfer_counts(host_st)
    field = orig["thk"].nbytes
    assert h2d <= 4 * field and h2d % field == 0, (h2d, field)
    assert d2h >= 3 * 10 * field and S.transfer_counts(dev_st) == (0, 0), d2h
    _assert_same(dev_st, host_st)
    for k in ("arrhenius", "slidingco", "topg"):
        h = getattr(host_st, k)
        assert isinstance(h, np.ndarray) and torch.from_numpy(h).is_pinned(), k
        np.testing.assert_array_equal(h, orig[k], err_msg=k)


def test_host_resident_state_sees_rebound_and_invalidated_fields():
    """A host field the caller rebinds to another array, or changes in place
    and declares with invalidate(), reaches the device on the next update
    (one copy each); results stay identical to a device-resident state given
    the same changes."""
    cfg = make_cfg("solved", nbitmax=10)
    dev_st, host_st, _ = _host_and_device_states(cfg)
    mods = [init(cfg, st) for st in (dev_st, host_st)]
    _steps(cfg, (dev_st, host_st), mods, 2)
    _assert_same(dev_st, host_st)
    field = np.asarray(host_st.thk).nbytes
    # rebinding: a new array
    host_st.slidingco = np.asarray(host_st.slidingco) * np.float32(1.5)
    dev_st.slidingco = dev_st.slidingco * 1.5
    S.reset_transfer_counts(host_st)
    _steps(cfg, (dev_st, host_st), mods, 1)
    assert S.transfer_counts(host_st)[0] == field
    _assert_same(dev_st, host_st)
    # in place: the state's own (pinned) arrays, declared changed
    host_st.thk[...] = np.maximum(host_st.thk - np.float32(5.0), np.float32(0.0))
    host_st.topg += np.float32(1.0)
    S.invalidate(host_st, "thk", "topg")
    dev_st.thk = torch.clamp(dev_st.thk - 5.0, min=0.0)
    dev_st.topg = dev_st.topg + 1.0
    S.reset_transfer_counts(host_st)
    _steps(cfg, (dev_st, host_st), mods, 1)
    assert S.transfer_counts(host_st)[0] == 2 * field
    _assert_same(dev_st, host_st)
