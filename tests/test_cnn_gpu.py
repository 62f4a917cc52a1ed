"""The emulator network end to end through the C ABI against the oracle
(torch-CPU float32 with the same bf16 rounding of conv inputs and weights):
forward (U, V), the physics-informed gradient (energy adjoint -> head ->
dgrad/wgrad chain) and one Adam step with per-variable clipnorm.

Tolerances: bf16 activations make single roundings differ where the two
sides accumulate in different orders, so fields are compared in relative L2:
forward <= 1e-2, parameter gradients <= 5e-2, one Adam update <= 5e-2."""

import numpy as np
import pytest
import torch

from igm_b200 import kernels as K
from igm_b200.cnn import CNN
from igm_b200.emulator import EmulatorOptimizer, train_step
from oracle import iceflow_oracle as O
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu

SCALES = [1 / 300.0, 1 / 3000.0, 1 / 100.0, 10.0, 1 / 100.0]


OUT = 50.0


def setup(nl=3, nz=4, ny=40, nx=70, seed=0):
    st = O.valley_glacier(ny, nx, 100.0, seed=seed, varying_coeffs=True)
    net = CNN(nb_layers=nl, cin=5, nout=2 * nz, init="he_normal", seed=seed, scales=SCALES, out_scale=OUT)
    # non-zero biases so that every bias path is exercised
    host = net.params.cpu().numpy()
    rng = np.random.default_rng(seed + 1)
    for i, s in enumerate(net.shapes):
        if len(s) == 1:
            host[net.offsets[i]:net.offsets[i + 1]] = rng.normal(0, 0.05, s)
    net.set_params(host)
    f = [torch.as_tensor(st[k]).cuda() for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    return st, net, f


def oracle_X(st, dx):
    fl = [torch.as_tensor(st[k]) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    fl.append(torch.full_like(fl[0], dx))
    X = O.fieldin_to_X(fl)
    return X * torch.tensor(SCALES, dtype=torch.float32)


def oracle_params(net):
    v = [torch.as_tensor(a.copy()) for a in net.get_variables()]
    return v[0::2], v[1::2]


@pytest.mark.parametrize("nl,nz,ny,nx", [(3, 4, 40, 70), (2, 10, 33, 129), (4, 5, 64, 64)])
def test_forward_matches_oracle(nl, nz, ny, nx):
    st, net, f = setup(nl, nz, ny, nx)
    buf = net.buffers(1, ny, nx, train=False)
    net.prepare_input(f, 100.0, [(0, 0)], ny, nx, buf)
    U, V = net.forward(buf, 1, ny, nx)
    ws, bs = oracle_params(net)
    Y = O.cnn_forward(oracle_X(st, 100.0), ws, bs, bf16=True, bf16_first=False, out_scale=OUT)
    Uo, Vo = O.Y_to_UV(Y, nz)
    assert rel_l2(U.cpu().numpy(), Uo.numpy()) < 1e-2
    assert rel_l2(V.cpu().numpy(), Vo.numpy()) < 1e-2
    net.check_errors()


def test_masked_inference():
    st, net, f = setup(2, 3, 30, 40)
    buf = net.buffers(1, 30, 40, train=False)
    net.prepare_input(f, 100.0, [(0, 0)], 30, 40, buf)
    U, V = net.forward(buf, 1, 30, 40, thk_mask=f[0])
    m = (st["thk"] > 0)[None]
    assert np.all(U.cpu().numpy()[0][np.broadcast_to(~m, U.shape[1:])] == 0)


def test_physics_gradient_and_adam_step_match_oracle():
    nl, nz, ny, nx, dx = 3, 4, 40, 70, 100.0
    st, net, f = setup(nl, nz, ny, nx, seed=3)
    ws, bs = oracle_params(net)
    params = []
    for w, b in zip(ws, bs):
        params += [w.clone().requires_grad_(True), b.clone().requires_grad_(True)]
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0))[1]
    X = oracle_X(st, dx)
    Y = O.cnn_forward(X, params[0::2], params[1::2], bf16=True, bf16_first=False, out_scale=OUT)
    Uo, Vo = O.Y_to_UV(Y, nz)
    fl = [torch.as_tensor(st[k])[None] for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    cost, _ = O.energy(Uo, Vo, *fl, dx, dz)
    grads = torch.autograd.grad(cost, params)
    # device: one physics-informed training step
    opt = EmulatorOptimizer(lr=1e-3, epsilon=1e-7, clipnorm=1.0)
    p0 = net.params.clone()
    terms = train_step(net, f, dx, [(0, 0)], ny, nx, dz.numpy(), None, 1e-3, opt)
    net.check_errors()
    np.testing.assert_allclose(float(terms.sum()) / ((ny - 1) * (nx - 1)), float(cost), rtol=2e-2)
    g = net.grads.cpu().numpy()
    for i, (s, gr) in enumerate(zip(net.shapes, grads)):
        gd = g[net.offsets[i]:net.offsets[i + 1]].reshape(s)
        e = rel_l2(gd, gr.numpy())
        assert e < 5e-2, (i, s, e)
    # the Adam update with per-variable clipnorm, against the oracle's Keras Adam
    opt_o = O.KerasLegacyAdam(lr=1e-3, epsilon=1e-7, clipnorm=1.0)
    xs = [p.detach().clone() for p in params]
    gs = [torch.as_tensor(g[net.offsets[i]:net.offsets[i + 1]].reshape(s)) for i, s in enumerate(net.shapes)]
    opt_o.apply_gradients(list(zip(gs, xs)))
    new = net.params.cpu().numpy()
    old = p0.cpu().numpy()
    for i, s in enumerate(net.shapes):
        dn = new[net.offsets[i]:net.offsets[i + 1]] - old[net.offsets[i]:net.offsets[i + 1]]
        do = (xs[i] - params[i].detach()).numpy().ravel()
        assert rel_l2(dn, do) < 1e-4, (i, rel_l2(dn, do))


def test_input_field_gradient_matches_oracle():
    """d(sum U RU + V RV)/d(fields) through the whole network (the gradient data
    assimilation takes to its control fields), against torch autograd of the
    oracle network; relative L2 per field <= 5e-2 (bf16 activations)."""
    nl, nz, ny, nx, dx = 3, 4, 40, 70, 100.0
    st, net, f = setup(nl, nz, ny, nx, seed=5)
    ws, bs = oracle_params(net)
    rng = np.random.default_rng(9)
    RU = rng.normal(0, 1, (1, nz, ny, nx)).astype(np.float32)
    RV = rng.normal(0, 1, (1, nz, ny, nx)).astype(np.float32)
    fl = [torch.as_tensor(st[k]).clone().requires_grad_(True) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    X = O.fieldin_to_X(fl + [torch.full_like(fl[0], dx)]) * torch.tensor(SCALES, dtype=torch.float32)
    Y = O.cnn_forward(X, ws, bs, bf16=True, bf16_first=False, out_scale=OUT)
    Uo, Vo = O.Y_to_UV(Y, nz)
    loss = (Uo * torch.as_tensor(RU)).sum() + (Vo * torch.as_tensor(RV)).sum()
    go = torch.autograd.grad(loss, fl)
    buf = net.buffers(1, ny, nx, train=True)
    net.prepare_input(f, dx, [(0, 0)], ny, nx, buf)
    net.forward(buf, 1, ny, nx, keep_acts=True)
    G = torch.zeros((1, 5, ny, nx), dtype=torch.float32, device="cuda")
    net.backward(buf, 1, ny, nx, torch.as_tensor(RU).cuda(), torch.as_tensor(RV).cuda(), field_grad=G)
    net.check_errors()
    # the data-assimilation path: the thk field only, no parameter gradients -- the same data chain
    G1 = torch.zeros((1, 1, ny, nx), dtype=torch.float32, device="cuda")
    grads = net.grads.clone()
    net.backward(buf, 1, ny, nx, torch.as_tensor(RU).cuda(), torch.as_tensor(RV).cuda(), field_grad=G1,
                 param_grads=False)
    assert torch.equal(net.grads, grads)
    G = G.cpu().numpy()[0]
    np.testing.assert_array_equal(G1.cpu().numpy()[0, 0], G[0])
    for c in range(4):
        e = rel_l2(G[c], go[c].numpy())
        assert e < 5e-2, (c, e)


@pytest.mark.parametrize("with_da", [False, True])
def test_perturbed_retraining_gradient_matches_oracle(with_da):
    """Retraining on pertubate_X's copies (emulate.py:310-328): thk and usurf
    scaled by 1.2 and 0.8 (without data assimilation), or the control fields
    (with it: control_list [thk, slidingco]); the batch's energy and its
    gradient against the oracle (relative L2 <= 5e-2, bf16 activations)."""
    from igm_b200 import emulator as E
    from igm_b200.config import default_cfg
    from igm_b200.state import State
    nl, nz, ny, nx, dx = 3, 4, 40, 70, 100.0
    st, net, f = setup(nl, nz, ny, nx, seed=6)
    ws, bs = oracle_params(net)
    params = []
    for w, b in zip(ws, bs):
        params += [w.clone().requires_grad_(True), b.clone().requires_grad_(True)]
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0))[1]
    over = {"iceflow": {"numerics": {"Nz": nz}, "emulator": {"retrain_freq": 1, "nbit": 1, "lr": 1e-3,
                                                             "framesizemax": 1000}}}
    if with_da:
        over["data_assimilation"] = {"control_list": ["thk", "slidingco"]}
    cfg = default_cfg(over)
    s = State()
    s.thk, s.usurf, s.arrhenius, s.slidingco = f
    s.dx, s.dzeta = dx, dz.numpy()
    s.iceflow_model = net
    s.opti_retrain = E.EmulatorOptimizer(lr=1e-3, epsilon=1e-7, clipnorm=1.0)
    E.update_iceflow_emulator(cfg, s, 1, pertubate=True)
    net.check_errors()
    chans = [0, 3] if with_da else [0, 1]
    fl = [torch.as_tensor(st[k]) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    Xr = O.pertubate_X(O.fieldin_to_X(fl + [torch.full_like(fl[0], dx)]), chans)
    assert Xr.shape[0] == 5
    Y = O.cnn_forward(Xr * torch.tensor(SCALES, dtype=torch.float32), params[0::2], params[1::2], bf16=True,
                      bf16_first=False, out_scale=OUT)
    Uo, Vo = O.Y_to_UV(Y, nz)
    cost, _ = O.energy(Uo, Vo, Xr[..., 0], Xr[..., 1], Xr[..., 2], Xr[..., 3], dx, dz)
    grads = torch.autograd.grad(cost, params)
    np.testing.assert_allclose(s.COST_EMULATOR[-1], float(cost), rtol=2e-2)
    g = net.grads.cpu().numpy()
    for i, (sh, gr) in enumerate(zip(net.shapes, grads)):
        e = rel_l2(g[net.offsets[i]:net.offsets[i + 1]].reshape(sh), gr.numpy())
        assert e < 5e-2, (i, sh, e)


def test_production_network_forward_and_gradient_match_oracle():
    """The network of the benchmark, 16 layers of 3x3 x 32 filters and the
    1x1 head to 2 Nz = 20 channels, at 128 x 128: forward and the physics
    gradient of every variable against the oracle (same bf16 operand
    rounding).  Over 16 layers an activation that lands on the other side of
    a bf16 rounding boundary (different FP32 accumulation orders) carries
    its one-ulp difference forward, so the bounds are 2e-2 (forward) and
    1e-1 (parameter gradients, relative L2 per variable)."""
    nl, nz, ny, nx, dx = 16, 10, 128, 128, 100.0
    st, net, f = setup(nl, nz, ny, nx, seed=11)
    ws, bs = oracle_params(net)
    params = []
    for w, b in zip(ws, bs):
        params += [w.clone().requires_grad_(True), b.clone().requires_grad_(True)]
    X = oracle_X(st, dx)
    Y = O.cnn_forward(X, params[0::2], params[1::2], bf16=True, bf16_first=False, out_scale=OUT)
    Uo, Vo = O.Y_to_UV(Y, nz)
    buf = net.buffers(1, ny, nx, train=False)
    net.prepare_input(f, dx, [(0, 0)], ny, nx, buf)
    U, V = net.forward(buf, 1, ny, nx)
    eu, ev = rel_l2(U.cpu().numpy(), Uo.detach().numpy()), rel_l2(V.cpu().numpy(), Vo.detach().numpy())
    print(f"16-layer forward: U {eu:.2e}, V {ev:.2e}")
    assert eu < 2e-2 and ev < 2e-2
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0))[1]
    fl = [torch.as_tensor(st[k])[None] for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    cost, _ = O.energy(Uo, Vo, *fl, dx, dz)
    grads = torch.autograd.grad(cost, params)
    opt = EmulatorOptimizer(lr=1e-3, epsilon=1e-7, clipnorm=1.0)
    terms = train_step(net, f, dx, [(0, 0)], ny, nx, dz.numpy(), None, 1e-3, opt)
    net.check_errors()
    np.testing.assert_allclose(float(terms.sum()) / ((ny - 1) * (nx - 1)), float(cost), rtol=2e-2)
    g = net.grads.cpu().numpy()
    worst = 0.0
    for i, (s, gr) in enumerate(zip(net.shapes, grads)):
        e = rel_l2(g[net.offsets[i]:net.offsets[i + 1]].reshape(s), gr.numpy())
        worst = max(worst, e)
        assert e < 1e-1, (i, s, e)
    print(f"16-layer parameter gradients: worst relative L2 {worst:.2e}")
