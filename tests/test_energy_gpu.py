"""Energy and hand-written adjoint kernels (through the C ABI) against the
golden vectors of the reference source and against the oracle.

Tolerances: FP64 kernels to 1e-11 relative; FP32 energy terms to 1e-5
relative; FP32 gradients to 1e-5 relative L2 over the field."""

import numpy as np
import pytest
import torch

from igm_b200 import kernels as K
from oracle import iceflow_oracle as O
from tests.gpu_util import dev, rel_l2

pytestmark = pytest.mark.gpu

CASES = ["small_f64", "small_f32", "nz2_f64", "mid_f32", "mid_f64", "nz16_f64"]


def run(g, grad=True, scale=None):
    f64 = g["U"].dtype == np.float64
    dt = torch.float64 if f64 else torch.float32
    args = [dev(g[k], dt) for k in ["U", "V", "thk", "usurf", "arrhenius", "slidingco"]]
    ns = (g["thk"].shape[0] - 1) * (g["thk"].shape[1] - 1)
    terms, dU, dV = K.energy(*args, float(g["dx"]), g["dzeta"], grad=grad, grad_scale=1.0 / ns if scale is None else scale)
    return terms.cpu().numpy(), dU, dV, ns


@pytest.mark.parametrize("case", CASES)
def test_energy_terms_match_reference(golden, case):
    g = golden(f"energy_{case}")
    terms, _, _, ns = run(g, grad=False)
    tol = 1e-11 if g["U"].dtype == np.float64 else 1e-5
    means = terms / ns
    np.testing.assert_allclose(means, g["means"], rtol=tol, atol=tol * np.abs(g["means"]).max())
    np.testing.assert_allclose(means.sum(), float(g["cost"]), rtol=tol)


@pytest.mark.parametrize("case", CASES)
def test_adjoint_matches_reference_autodiff(golden, case):
    g = golden(f"energy_{case}")
    terms, dU, dV, ns = run(g, grad=True)
    f64 = g["U"].dtype == np.float64
    tol = 1e-11 if f64 else 1e-5
    assert rel_l2(dU.cpu().numpy(), g["gradU"]) < tol
    assert rel_l2(dV.cpu().numpy(), g["gradV"]) < tol
    np.testing.assert_allclose(terms / ns, g["means"], rtol=tol, atol=tol * np.abs(g["means"]).max())


def test_adjoint_central_differences():
    """Central finite differences of the FP64 energy at random nodes
    (eps = 1e-3 m/a) against the FP64 adjoint."""
    st = O.valley_glacier(48, 40, 100.0, seed=3, varying_coeffs=True)
    nz = 10
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).double())[1].numpy()
    rng = np.random.default_rng(0)
    U = rng.normal(20, 15, (nz, 48, 40))
    V = rng.normal(-5, 15, (nz, 48, 40))
    f = [dev(st[k], torch.float64) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    Ud, Vd = dev(U, torch.float64), dev(V, torch.float64)
    _, dU, dV = K.energy(Ud, Vd, *f, 100.0, dz, grad=True, grad_scale=1.0)
    dU, dV = dU.cpu().numpy(), dV.cpu().numpy()
    eps = 1e-3
    errs = []
    for _ in range(200):
        k, j, i = rng.integers(0, nz), rng.integers(0, 48), rng.integers(0, 40)
        which = rng.integers(0, 2)
        base = (Ud if which == 0 else Vd)
        orig = float(base[k, j, i])
        base[k, j, i] = orig + eps
        ep = K.energy(Ud, Vd, *f, 100.0, dz)[0].sum().item()
        base[k, j, i] = orig - eps
        em = K.energy(Ud, Vd, *f, 100.0, dz)[0].sum().item()
        base[k, j, i] = orig
        fd = (ep - em) / (2 * eps)
        ad = (dU if which == 0 else dV)[k, j, i]
        errs.append(abs(fd - ad) / max(abs(ad), 1e-3))
    assert np.median(errs) < 1e-6 and np.max(errs) < 1e-3, (np.median(errs), np.max(errs))


@pytest.mark.parametrize("shape", [(2, 7, 5), (3, 33, 65), (1, 9, 12), (5, 40, 17), (10, 100, 100), (16, 23, 31)])
def test_odd_shapes_against_oracle(shape):
    nz, ny, nx = shape
    rng = np.random.default_rng(nz * 1000 + ny)
    st = O.valley_glacier(ny, nx, 100.0, seed=ny, varying_coeffs=True)
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).double())[1] if nz > 1 else torch.ones(1, dtype=torch.float64)
    U = rng.normal(30, 20, (nz, ny, nx))
    V = rng.normal(0, 20, (nz, ny, nx))
    fl = {k: torch.as_tensor(st[k]).double() for k in ["thk", "usurf", "arrhenius", "slidingco"]}
    cost, means, gU, gV = O.energy_and_grad(torch.as_tensor(U), torch.as_tensor(V), fl["thk"], fl["usurf"],
                                            fl["arrhenius"], fl["slidingco"], 100.0, dz)
    ns = (ny - 1) * (nx - 1)
    terms, dU, dV = K.energy(dev(U, torch.float64), dev(V, torch.float64), *[dev(fl[k]) for k in fl], 100.0,
                             dz.numpy(), grad=True, grad_scale=1.0 / ns)
    np.testing.assert_allclose(terms.cpu().numpy() / ns, torch.stack(means).numpy(), rtol=1e-11, atol=1e-9)
    assert rel_l2(dU.cpu().numpy(), gU.numpy()) < 1e-11
    assert rel_l2(dV.cpu().numpy(), gV.numpy()) < 1e-11
    # FP32 kernel against the FP64 oracle: the FP32 error is stated by this bound
    terms32, dU32, dV32 = K.energy(dev(U, torch.float32), dev(V, torch.float32),
                                   *[dev(fl[k], torch.float32) for k in fl], 100.0, dz.numpy(), grad=True,
                                   grad_scale=1.0 / ns)
    np.testing.assert_allclose(terms32.cpu().numpy() / ns, torch.stack(means).numpy(), rtol=1e-5,
                               atol=1e-5 * float(cost.abs()))
    assert rel_l2(dU32.cpu().numpy(), gU.numpy()) < 2e-5
    assert rel_l2(dV32.cpu().numpy(), gV.numpy()) < 2e-5


def test_batched_equals_separate():
    rng = np.random.default_rng(5)
    nz, ny, nx, B = 4, 21, 26, 3
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0))[1].numpy()
    sts = [O.valley_glacier(ny, nx, 100.0, seed=s, varying_coeffs=True) for s in range(B)]
    U = rng.normal(30, 20, (B, nz, ny, nx)).astype(np.float32)
    V = rng.normal(0, 20, (B, nz, ny, nx)).astype(np.float32)
    F = {k: np.stack([s[k] for s in sts]) for k in ["thk", "usurf", "arrhenius", "slidingco"]}
    tb, dUb, dVb = K.energy(dev(U), dev(V), *[dev(F[k]) for k in F], 100.0, dz, grad=True)
    tot = np.zeros(3)
    for b in range(B):
        t, dU, dV = K.energy(dev(U[b]), dev(V[b]), *[dev(F[k][b]) for k in F], 100.0, dz, grad=True)
        tot += t.cpu().numpy()
        np.testing.assert_array_equal(dU.cpu().numpy(), dUb[b].cpu().numpy())
    np.testing.assert_allclose(tb.cpu().numpy(), tot, rtol=1e-12)


def test_energy_reduction_is_deterministic():
    st = O.valley_glacier(300, 257, 50.0, seed=1, varying_coeffs=True)
    rng = np.random.default_rng(1)
    U = dev(rng.normal(30, 20, (10, 300, 257)).astype(np.float32))
    V = dev(rng.normal(0, 20, (10, 300, 257)).astype(np.float32))
    f = [dev(st[k]) for k in ["thk", "usurf", "arrhenius", "slidingco"]]
    dz = O.compute_zeta_dzeta(O.compute_levels(10, 4.0))[1].numpy()
    a = [K.energy(U, V, *f, 50.0, dz, grad=True) for _ in range(3)]
    for t, dU, dV in a[1:]:
        assert torch.equal(t, a[0][0]) and torch.equal(dU, a[0][1]) and torch.equal(dV, a[0][2])


@pytest.mark.parametrize("n,m,fnge", [(2.5, 2.0, False), (3.0, 3.0, True), (4.0, 1.5, True)])
def test_other_physics_against_oracle(n, m, fnge):
    """Glen and Weertman exponents other than 3 and the forced-negative
    gravitational energy take the kernel's general path (generic powers,
    per-layer gravity clamp); FP64 against the FP64 oracle."""
    nz, ny, nx = 6, 37, 45
    rng = np.random.default_rng(int(n * 10 + m))
    st = O.valley_glacier(ny, nx, 100.0, seed=7, varying_coeffs=True)
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).double())[1]
    U = rng.normal(30, 20, (nz, ny, nx))
    V = rng.normal(0, 20, (nz, ny, nx))
    fl = {k: torch.as_tensor(st[k]).double() for k in ["thk", "usurf", "arrhenius", "slidingco"]}
    ph = O.Physics(exp_glen=n, exp_weertman=m, force_negative_gravitational_energy=fnge)
    cost, means, gU, gV = O.energy_and_grad(torch.as_tensor(U), torch.as_tensor(V), fl["thk"], fl["usurf"],
                                            fl["arrhenius"], fl["slidingco"], 100.0, dz, ph)
    ns = (ny - 1) * (nx - 1)
    phys = dict(exp_glen=n, exp_weertman=m, force_negative_gravitational_energy=fnge)
    terms, dU, dV = K.energy(dev(U, torch.float64), dev(V, torch.float64), *[dev(fl[k]) for k in fl], 100.0,
                             dz.numpy(), phys, grad=True, grad_scale=1.0 / ns)
    np.testing.assert_allclose(terms.cpu().numpy() / ns, torch.stack(means).numpy(), rtol=1e-10,
                               atol=1e-10 * float(cost.abs()))
    assert rel_l2(dU.cpu().numpy(), gU.numpy()) < 1e-10
    assert rel_l2(dV.cpu().numpy(), gV.numpy()) < 1e-10
