"""The stencil and transport kernels at the benchmark's full sizes, checked
through properties that do not need a CPU run of the whole grid: central
differences of the FP64 energy against the FP64 adjoint (1000 x 1000 x Nz 10,
1000 random nodes, eps = 1e-3 m/a, half of them on ice), FP32 against FP64
energy and adjoint
(4096 x 4096 x Nz 16) and the transport bit for bit against the oracle
(4096 x 4096)."""

import numpy as np
import pytest
import torch

from igm_b200 import kernels as K
from igm_b200.synthetic import ridge_glacier, valley_glacier
from oracle import iceflow_oracle as O
from tests.gpu_util import dev, rel_l2

pytestmark = pytest.mark.gpu


def _dzeta(nz):
    return O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).double())[1].numpy()


def test_adjoint_central_differences_1000x1000():
    """The full-size adjoint against central differences.  A node's value
    enters only the four staggered cells around it, and each cell's energy
    density depends only on its four corner columns, so the difference of the
    total energy equals the difference of the energy of a 7 x 7-node window
    around the node -- taken on the window, it is free of the cancellation of
    two totals over 10^6 cells."""
    n, nz, dx = 1000, 10, 50.0
    st = valley_glacier(n, n, dx, seed=0, varying_coeffs=True)
    dz = _dzeta(nz)
    rng = np.random.default_rng(1)
    g = torch.Generator("cuda").manual_seed(1)
    Ud = torch.randn((nz, n, n), dtype=torch.float64, device="cuda", generator=g) * 15 + 20
    Vd = torch.randn((nz, n, n), dtype=torch.float64, device="cuda", generator=g) * 15 - 5
    f = [dev(st[k], torch.float64) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    _, dU, dV = K.energy(Ud, Vd, *f, dx, dz, grad=True, grad_scale=1.0)
    eps = 1e-3
    errs = []
    ice = np.argwhere(st["thk"] > 0)
    for t in range(1000):
        k = int(rng.integers(0, nz))
        j, i = (ice[rng.integers(0, len(ice))] if t % 2 == 0 else (rng.integers(0, n), rng.integers(0, n)))
        j, i = int(j), int(i)
        j0, j1, i0, i1 = max(0, j - 3), min(n, j + 4), max(0, i - 3), min(n, i + 4)
        Uw = Ud[:, j0:j1, i0:i1].clone()
        Vw = Vd[:, j0:j1, i0:i1].clone()
        fw = [x[j0:j1, i0:i1].contiguous() for x in f]
        which = int(rng.integers(0, 2))
        base = Uw if which == 0 else Vw
        orig = float(base[k, j - j0, i - i0])
        base[k, j - j0, i - i0] = orig + eps
        ep = K.energy(Uw, Vw, *fw, dx, dz)[0].sum().item()
        base[k, j - j0, i - i0] = orig - eps
        em = K.energy(Uw, Vw, *fw, dx, dz)[0].sum().item()
        fd = (ep - em) / (2 * eps)
        ad = float((dU if which == 0 else dV)[k, j, i])
        errs.append(abs(fd - ad) / max(abs(ad), 1e-3))
    assert np.median(errs) < 1e-6 and np.max(errs) < 1e-3, (np.median(errs), np.max(errs))


def _ridge_state(n=4096, dx=25.0, nz=16):
    st = ridge_glacier(n, dx, seed=0)
    x = np.arange(n) * dx
    X, Y = np.meshgrid(x, x)
    thk = np.maximum(0.0, 250.0 * (1.0 + np.sin(X / 3000.0) * np.cos(Y / 4000.0)) - 60.0).astype(np.float32)
    usurf = (st["topg"] + thk).astype(np.float32)
    return thk, usurf, st["arrhenius"], st["slidingco"]


def test_fp32_matches_fp64_4096x4096_nz16():
    n, nz, dx = 4096, 16, 25.0
    thk, usurf, A, c = _ridge_state(n, dx, nz)
    dz = _dzeta(nz)
    g = torch.Generator("cuda").manual_seed(5)
    U64 = torch.randn((nz, n, n), dtype=torch.float64, device="cuda", generator=g) * 40 + 30
    V64 = torch.randn((nz, n, n), dtype=torch.float64, device="cuda", generator=g) * 40
    f64 = [dev(a, torch.float64) for a in (thk, usurf, A, c)]
    t64, dU64, dV64 = K.energy(U64, V64, *f64, dx, dz, grad=True, grad_scale=1.0 / (n - 1) ** 2)
    t64 = t64.cpu().numpy()
    dU64, dV64 = dU64.cpu().numpy(), dV64.cpu().numpy()
    U32, V32 = U64.float(), V64.float()
    del U64, V64, f64
    torch.cuda.empty_cache()
    f32 = [dev(a, torch.float32) for a in (thk, usurf, A, c)]
    t32, dU32, dV32 = K.energy(U32, V32, *f32, dx, dz, grad=True, grad_scale=1.0 / (n - 1) ** 2)
    np.testing.assert_allclose(t32.cpu().numpy(), t64, rtol=1e-5, atol=1e-5 * np.abs(t64).max())
    assert rel_l2(dU32.cpu().numpy(), dU64) < 1e-4
    assert rel_l2(dV32.cpu().numpy(), dV64) < 1e-4


def test_transport_bit_exact_4096x4096():
    n, dx = 4096, 25.0
    rng = np.random.default_rng(9)
    thk, usurf, _, _ = _ridge_state(n, dx)
    topg = (usurf - thk).astype(np.float32)
    u = rng.normal(0, 80, (n, n)).astype(np.float32)
    v = rng.normal(0, 80, (n, n)).astype(np.float32)
    smb = rng.normal(0, 1, (n, n)).astype(np.float32)
    dt = np.float32(0.07)
    ref = O.thk_update(*(torch.as_tensor(a) for a in (thk, topg, u, v, smb)), dx, torch.tensor(dt))
    out = K.transport_step(dev(u), dev(v), dev(thk), dev(topg), dev(smb), dx, float(dt))
    for a, b in zip([out[0], out[2], out[1], out[3]], ref):
        np.testing.assert_array_equal(a.cpu().numpy(), b.numpy())
