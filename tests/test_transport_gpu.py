"""Transport, surfaces, smb and velocity-reduction kernels against the
golden vectors and the oracle: bit-identical (FP32 and FP64)."""

import numpy as np
import pytest
import torch

from igm_b200 import kernels as K
from oracle import iceflow_oracle as O
from tests.gpu_util import dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["f32", "f64"])
@pytest.mark.parametrize("st", ["godunov", "minmod", "superbee"])
def test_divflux_bit_exact(golden, tag, st):
    g = golden("transport")
    dt = torch.float32 if tag == "f32" else torch.float64
    h, u, v = dev(g[f"{tag}_h"], dt), dev(g[f"{tag}_u"], dt), dev(g[f"{tag}_v"], dt)
    topg = torch.zeros_like(h)
    _, _, _, div = K.transport_step(u, v, h, topg, None, 50.0, 0.7 if tag == "f64" else float(np.float32(0.7)),
                                    slope_type=st)
    np.testing.assert_array_equal(div.cpu().numpy(), g[f"{tag}_{st}"])


def test_thk_update_bit_exact(golden):
    g = golden("transport")
    h, topg, smb = dev(g["thk_h"]), dev(g["thk_topg"]), dev(g["thk_smb"])
    thk, usurf, lsurf, div = K.transport_step(dev(g["f32_u"]), dev(g["f32_v"]), h, topg, smb, 50.0,
                                              float(np.float32(0.7)))
    for a, k in [(thk, "thk_new"), (lsurf, "thk_lsurf"), (usurf, "thk_usurf"), (div, "thk_divflux")]:
        np.testing.assert_array_equal(a.cpu().numpy(), g[k])
    ls, us = K.surfaces(h, topg)
    np.testing.assert_array_equal(us.cpu().numpy(), g["thk_init_usurf"])


def test_transport_large_random_against_oracle():
    rng = np.random.default_rng(4)
    ny, nx = 257, 300
    h = np.maximum(0, rng.normal(80, 90, (ny, nx))).astype(np.float32)
    u = rng.normal(0, 50, (ny, nx)).astype(np.float32)
    v = rng.normal(0, 50, (ny, nx)).astype(np.float32)
    topg = rng.normal(0, 200, (ny, nx)).astype(np.float32)
    smb = rng.normal(0, 1, (ny, nx)).astype(np.float32)
    dt = np.float32(0.31)
    ref = O.thk_update(*(torch.as_tensor(a) for a in (h, topg, u, v, smb)), 50.0, torch.tensor(dt))
    out = K.transport_step(dev(u), dev(v), dev(h), dev(topg), dev(smb), 50.0, float(dt))
    for a, b in zip([out[0], out[2], out[1], out[3]], ref):
        np.testing.assert_array_equal(a.cpu().numpy(), b.numpy())


def test_transport_mass_conservation():
    """No smb, zero flux through the border: total thickness conserved to round-off."""
    ny = nx = 64
    y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    h = np.maximum(0, 100 - ((y - 32) ** 2 + (x - 32) ** 2)).astype(np.float64)
    u = np.full((ny, nx), 20.0)
    v = np.full((ny, nx), -10.0)
    thk, _, _, _ = K.transport_step(dev(u), dev(v), dev(h), dev(np.zeros_like(h)), None, 100.0, 0.5)
    np.testing.assert_allclose(thk.sum().item(), h.sum(), rtol=1e-13)


def test_dt_from_device_pointer():
    rng = np.random.default_rng(1)
    h = dev(np.maximum(0, rng.normal(50, 50, (30, 40))).astype(np.float32))
    u, v = dev(rng.normal(0, 30, (30, 40)).astype(np.float32)), dev(rng.normal(0, 30, (30, 40)).astype(np.float32))
    z = torch.zeros_like(h)
    a = K.transport_step(u, v, h, z, None, 50.0, 0.4)[0]
    b = K.transport_step(u, v, h, z, None, 50.0, 123.0, dt_device=torch.tensor([0.4], device="cuda"))[0]
    assert torch.equal(a, b)


def test_smb_simple_and_icemask():
    rng = np.random.default_rng(2)
    us = rng.uniform(2500, 3300, (50, 60)).astype(np.float32)
    mask = (rng.uniform(size=(50, 60)) > 0.3).astype(np.float32)
    out = K.smb_simple(dev(us), 0.009, 0.005, 2900.0, 2.0, icemask=dev(mask)).cpu().numpy()
    ref = O.smb_simple(torch.as_tensor(us), np.float32(0.009), np.float32(0.005), np.float32(2900.0), np.float32(2.0)).numpy()
    ref = np.where((ref < 0) | (mask > 0.5), ref, -10)
    np.testing.assert_array_equal(out, ref)


def test_velocity_reduce_and_mask():
    rng = np.random.default_rng(3)
    nz, ny, nx = 10, 33, 47
    U = rng.normal(0, 40, (nz, ny, nx)).astype(np.float32)
    V = rng.normal(0, 40, (nz, ny, nx)).astype(np.float32)
    thk = np.where(rng.uniform(size=(ny, nx)) > 0.3, 50.0, 0.0).astype(np.float32)
    w = O.define_vertical_weight(nz, 4.0)
    Ud, Vd = dev(U), dev(V)
    ub, vb, ub0, vb0, us0, vs0, vm = K.velocity_reduce(Ud, Vd, dev(thk), w.numpy(), mask=True)
    Um = np.where(thk > 0, U, 0)
    Vm = np.where(thk > 0, V, 0)
    np.testing.assert_array_equal(Ud.cpu().numpy(), Um)
    rb = O.get_velbar(torch.as_tensor(Um), torch.as_tensor(Vm), w)
    np.testing.assert_allclose(ub.cpu().numpy(), rb[0].numpy(), rtol=1e-6, atol=1e-4)
    np.testing.assert_array_equal(ub0.cpu().numpy(), Um[0])
    np.testing.assert_array_equal(vs0.cpu().numpy(), Vm[-1])
    expect = max(np.abs(ub.cpu().numpy()).max(), np.abs(vb.cpu().numpy()).max())
    assert vm.item() == expect
    assert K.absmax2(ub, vb).item() == expect


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_force_max_velbar_bit_identical(dtype):
    """force_max_velbar (utils.py:182-194) against the oracle, bit for bit:
    speeds above the cap scaled to it, the rest (and zero speeds) unchanged."""
    rng = np.random.default_rng(7)
    U = rng.normal(0, 300, (5, 37, 53))
    V = rng.normal(0, 300, (5, 37, 53))
    U[0, :3] = 0.0
    V[0, :3] = 0.0
    Ut, Vt = torch.as_tensor(U).to(dtype), torch.as_tensor(V).to(dtype)
    Uo, Vo = O.force_max_velbar(Ut, Vt, 250.0)
    Ud, Vd = Ut.cuda().contiguous(), Vt.cuda().contiguous()
    K.force_max_velbar(Ud, Vd, 250.0)
    np.testing.assert_array_equal(Ud.cpu().numpy(), Uo.numpy())
    np.testing.assert_array_equal(Vd.cpu().numpy(), Vo.numpy())
    assert float(torch.sqrt(Ud * Ud + Vd * Vd).max()) <= 250.0 * (1 + 1e-6)
    assert int((torch.sqrt(Ut * Ut + Vt * Vt) >= 250.0).sum()) > 100
