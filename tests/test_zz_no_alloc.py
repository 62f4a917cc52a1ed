"""igm_energy_noalloc: the energy/adjoint entry point for callers that cannot
allocate device memory (a host model whose device memory is all in its own
pool, or code that must not call cudaMalloc because it may synchronise).  It
keeps its reduction scratch in a fixed array inside the library instead of a
caller workspace.  Checked through the C ABI against igm_energy, the
workspace version, on two calls in a row (the shared array keeps the previous
call's contents, so the second call checks that nothing stale leaks), and for
the clear rejection of a grid that needs more scratch than the array holds.

This file is collected last so that a failure here stops a run only after
every other test has run; it also passes on its own in a fresh process."""

import ctypes as C

import numpy as np
import pytest
import torch

from igm_b200 import _lib as L
from igm_b200 import kernels as K
from oracle import iceflow_oracle as O

pytestmark = pytest.mark.gpu


def _noalloc(U, V, f, dx, dz, grad, scale):
    B, nz, ny, nx = U.shape
    g = L.make_grid(B, nz, ny, nx, dx, dz)
    ph = L.make_physics()
    fs = K.fields_struct(*f)
    terms = torch.empty(3, dtype=torch.float64, device=U.device)
    dU = torch.empty_like(U) if grad else None
    dV = torch.empty_like(V) if grad else None
    rc = L.lib().igm_energy_noalloc(L.dtype_code(U.dtype), C.byref(g), C.byref(ph), C.byref(fs), L.ptr(U), L.ptr(V),
                                    L.ptr(dU), L.ptr(dV), float(scale), L.ptr(terms), L.stream_ptr())
    L.check(rc, "igm_energy_noalloc")
    return terms, dU, dV


def _case(ny, nx, nz, dtype, seed):
    st = O.valley_glacier(ny, nx, 100.0, seed=seed, varying_coeffs=True)
    rng = np.random.default_rng(seed)
    U = torch.as_tensor(rng.normal(30, 20, (1, nz, ny, nx))).to(dtype).cuda()
    V = torch.as_tensor(rng.normal(0, 20, (1, nz, ny, nx))).to(dtype).cuda()
    f = [torch.as_tensor(st[k])[None].to(dtype).cuda() for k in ("thk", "usurf", "arrhenius", "slidingco")]
    dz = O.compute_zeta_dzeta(O.compute_levels(nz, 4.0).double())[1].numpy()
    return U, V, f, dz


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_noalloc_matches_workspace_version_on_two_calls(dtype):
    tol = 1e-5 if dtype == torch.float32 else 1e-11  # the energy tests' tolerances
    for call, (ny, nx, nz, seed) in enumerate([(300, 257, 10, 1), (120, 95, 4, 2)]):
        U, V, f, dz = _case(ny, nx, nz, dtype, seed)
        scale = 1.0 / ((ny - 1) * (nx - 1))
        t_ref, dU_ref, dV_ref = K.energy(U, V, *f, 100.0, dz, grad=True, grad_scale=scale)
        t, dU, dV = _noalloc(U, V, f, 100.0, dz, grad=True, scale=scale)
        np.testing.assert_allclose(t.cpu().numpy(), t_ref.cpu().numpy(), rtol=tol, err_msg=f"call {call}")
        for a, b in ((dU, dU_ref), (dV, dV_ref)):
            e = float(torch.linalg.vector_norm((a - b).double()) / torch.linalg.vector_norm(b.double()))
            assert e <= tol, (call, e)
        # energy only, same array, immediately after
        t2, _, _ = _noalloc(U, V, f, 100.0, dz, grad=False, scale=1.0)
        np.testing.assert_allclose(t2.cpu().numpy(), t_ref.cpu().numpy(), rtol=tol, err_msg=f"call {call} (energy)")


def test_noalloc_rejects_grid_beyond_its_scratch():
    U, V, f, dz = _case(20, 20, 4, torch.float32, 3)
    g = L.make_grid(2, 4, 4096, 4096, 100.0, dz)  # needs more than the fixed array; nothing is launched
    # the buffers below are 20 x 20: the call is made only while this grid's scratch exceeds the
    # fixed array, so that the size check, not the launch, decides the outcome
    need = int(L.lib().igm_workspace_size(C.byref(g)))
    if need <= (2 << 20):
        pytest.fail(f"grid needs only {need} bytes of scratch: it would not be rejected, not calling")
    ph = L.make_physics()
    fs = K.fields_struct(*f)
    terms = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = L.lib().igm_energy_noalloc(0, C.byref(g), C.byref(ph), C.byref(fs), L.ptr(U), L.ptr(V), None, None, 1.0,
                                    L.ptr(terms), L.stream_ptr())
    assert rc == 7  # IGM_ERR_WORKSPACE
    msg = L.lib().igm_last_error().decode()
    assert "fixed" in msg and "igm_energy" in msg
    torch.cuda.synchronize()
    assert float(terms.abs().sum()) == 0.0
