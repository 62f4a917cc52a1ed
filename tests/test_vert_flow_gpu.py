"""Vertical velocity (vert_flow version 2, kinematic and incompressibility) through the C ABI:
bit-identical to the golden vectors of the reference source and to the oracle
(FP32 and FP64), on ragged tiles and at 1000 x 1000 x 10; the process API on
device- and host-resident states."""

import numpy as np
import pytest
import torch

from igm_b200 import kernels as K
from igm_b200.config import default_cfg
from igm_b200.processes import vert_flow
from igm_b200.state import State, sync_host
from oracle import iceflow_oracle as O
from tests.gpu_util import dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["f32", "f64", "nz5_f32", "nz2_f32"])
def test_matches_reference_golden(golden, tag):
    g = golden("vert_flow")
    dt = torch.float64 if g[f"{tag}_U"].dtype == np.float64 else torch.float32
    W = K.vertical_velocity(dev(g[f"{tag}_U"], dt), dev(g[f"{tag}_V"], dt), dev(g[f"{tag}_topg"], dt),
                            dev(g[f"{tag}_thk"], dt), g[f"{tag}_levels"], g[f"{tag}_weight"], float(g[f"{tag}_dx"]))
    np.testing.assert_array_equal(W.cpu().numpy(), g[f"{tag}_W"])


@pytest.mark.parametrize("tag", ["f32", "f64", "nz5_f32", "nz2_f32"])
def test_incompressibility_matches_reference_golden(golden, tag):
    g = golden("vert_flow")
    dt = torch.float64 if g[f"{tag}_U"].dtype == np.float64 else torch.float32
    W = K.vertical_velocity(dev(g[f"{tag}_U"], dt), dev(g[f"{tag}_V"], dt), dev(g[f"{tag}_topg"], dt),
                            dev(g[f"{tag}_thk"], dt), g[f"{tag}_levels"], g[f"{tag}_weight"], float(g[f"{tag}_dx"]),
                            method="incompressibility")
    np.testing.assert_array_equal(W.cpu().numpy(), g[f"{tag}_Wi"])


def _case(nz, ny, nx, seed, dtype, spacing=4.0):
    rng = np.random.default_rng(seed)
    st = O.valley_glacier(ny, nx, 50.0, seed=seed, varying_coeffs=True)
    np_dt = np.float32 if dtype == torch.float32 else np.float64
    U = rng.normal(30, 40, (nz, ny, nx)).astype(np_dt)
    V = rng.normal(-5, 40, (nz, ny, nx)).astype(np_dt)
    topg = np.asarray(st["topg"], np_dt)
    thk = np.asarray(st["thk"], np_dt)
    lv = O.compute_levels(nz, spacing).to(dtype)
    w = O.define_vertical_weight(nz, spacing).to(dtype)
    return U, V, topg, thk, lv, w


@pytest.mark.parametrize("shape", [(2, 2, 2), (3, 2, 33), (10, 9, 2), (5, 33, 65), (10, 257, 300), (16, 23, 31)])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_ragged_shapes_against_oracle(shape, dtype):
    nz, ny, nx = shape
    U, V, topg, thk, lv, w = _case(nz, ny, nx, nz * 100 + ny, dtype)
    ref = O.vertical_velocity_kinematic(*(torch.as_tensor(a) for a in (U, V, topg, thk)), lv, w, 50.0)
    W = K.vertical_velocity(dev(U), dev(V), dev(topg), dev(thk), lv.numpy(), w.numpy()[:, 0, 0], 50.0)
    np.testing.assert_array_equal(W.cpu().numpy(), ref.numpy())


@pytest.mark.parametrize("shape", [(2, 2, 2), (3, 2, 33), (10, 9, 2), (5, 33, 65), (10, 257, 300), (16, 23, 31)])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_incompressibility_ragged_shapes_against_oracle(shape, dtype):
    nz, ny, nx = shape
    U, V, topg, thk, lv, w = _case(nz, ny, nx, nz * 100 + ny + 1, dtype)
    ref = O.vertical_velocity_incompressibility(*(torch.as_tensor(a) for a in (U, V, topg, thk)), lv, w, 50.0)
    W = K.vertical_velocity(dev(U), dev(V), dev(topg), dev(thk), lv.numpy(), w.numpy()[:, 0, 0], 50.0,
                            method="incompressibility")
    np.testing.assert_array_equal(W.cpu().numpy(), ref.numpy())


def test_full_size_against_oracle():
    """1000 x 1000 x 10, FP32: bit-identical to the oracle."""
    U, V, topg, thk, lv, w = _case(10, 1000, 1000, 11, torch.float32)
    ref = O.vertical_velocity_kinematic(*(torch.as_tensor(a) for a in (U, V, topg, thk)), lv, w, 50.0)
    W = K.vertical_velocity(dev(U), dev(V), dev(topg), dev(thk), lv.numpy(), w.numpy()[:, 0, 0], 50.0)
    np.testing.assert_array_equal(W.cpu().numpy(), ref.numpy())


@pytest.mark.parametrize("method", ["kinematic", "incompressibility"])
@pytest.mark.parametrize("host", [False, True])
def test_process_api(host, method):
    nz, ny, nx = 10, 40, 37
    U, V, topg, thk, lv, w = _case(nz, ny, nx, 3, torch.float32)
    cfg = default_cfg({"vert_flow": {"method": method}})
    st = State()
    st.dx = 50.0
    st.vert_weight = w.numpy()
    for k, a in [("U", U), ("V", V), ("topg", topg), ("thk", thk)]:
        setattr(st, k, a if host else dev(a))
    if host:
        st.device = "cuda"
    vert_flow.initialize(cfg, st)
    vert_flow.update(cfg, st)
    vert_flow.finalize(cfg, st)
    sync_host(st)  # a host-resident state holds the results once the copies have landed
    fn = O.vertical_velocity_kinematic if method == "kinematic" else O.vertical_velocity_incompressibility
    ref = fn(*(torch.as_tensor(a) for a in (U, V, topg, thk)), lv, w, 50.0).numpy()
    W = st.W if host else st.W.cpu().numpy()
    np.testing.assert_array_equal(np.asarray(W), ref)
    np.testing.assert_array_equal(np.asarray(st.wvelbase if host else st.wvelbase.cpu()), ref[0])
    np.testing.assert_array_equal(np.asarray(st.wvelsurf if host else st.wvelsurf.cpu()), ref[-1])


def test_unsupported_methods_raise():
    st = State()
    for over in [{"vert_flow": {"method": "twolayers"}}, {"vert_flow": {"version": 1}}]:
        with pytest.raises(NotImplementedError):
            vert_flow.update(default_cfg(over), st)
