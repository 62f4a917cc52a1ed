"""A pretrained emulator the reference ships, loaded through the drop-in
iceflow process and run on the device, against the oracle's network forward
on the same weights (read by igm_b200.keras_h5).

The shipped Keras files are not part of this repository: the test looks for
the reference's source tree in IGM_REFERENCE_ROOT (the directory holding
igm/), and for the installed igm package, and skips when neither holds
pinnbp_10_4_cnn_16_32_2_1_a/model.h5."""

import os

import pytest
import torch

from igm_b200.config import default_cfg
from igm_b200.emulator import emulator_dir_name, load_keras_h5, update_iceflow_emulated, initialize_iceflow_emulator
from igm_b200.keras_h5 import read_keras_weights
from igm_b200.processes import iceflow as P
from igm_b200.state import State
from oracle import iceflow_oracle as O
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu


def _shipped_dir(cfg):
    name = emulator_dir_name(cfg)
    roots = []
    if os.environ.get("IGM_REFERENCE_ROOT"):
        roots.append(os.path.join(os.environ["IGM_REFERENCE_ROOT"], "igm"))
    try:
        import importlib.util
        spec = importlib.util.find_spec("igm")
        if spec is not None and spec.submodule_search_locations:
            roots += list(spec.submodule_search_locations)
    except (ImportError, ValueError):
        pass
    for r in roots:
        d = os.path.join(r, "processes", "iceflow", "emulate", "emulators", name)
        if os.path.exists(os.path.join(d, "model.h5")):
            return d
    return None


def test_shipped_emulator_forward_matches_oracle():
    cfg = default_cfg({"iceflow": {"emulator": {"pretrained": False}}})
    d = _shipped_dir(cfg)
    if d is None:
        pytest.skip("the reference's shipped emulators are not available (set IGM_REFERENCE_ROOT)")
    g = O.valley_glacier(64, 80, 100.0, seed=3)
    st = State()
    for k in ("thk", "usurf", "arrhenius", "slidingco"):
        setattr(st, k, torch.as_tensor(g[k]).cuda())
    st.dx = 100.0
    P.initialize_iceflow_fields(cfg, st)
    initialize_iceflow_emulator(cfg, st)
    load_keras_h5(st, d, cfg)
    st.vert_weight = P.define_vertical_weight(10, 4.0)
    update_iceflow_emulated(cfg, st)
    layers = read_keras_weights(os.path.join(d, "model.h5"))
    ws = [torch.as_tensor(a) for _, wl in layers for n, a in wl if "kernel" in n]
    bs = [torch.as_tensor(a) for _, wl in layers for n, a in wl if "bias" in n]
    fl = [torch.as_tensor(g[k]) for k in ("thk", "usurf", "arrhenius", "slidingco")]
    X = O.fieldin_to_X(fl + [torch.full_like(fl[0], 100.0)])
    Y = O.cnn_forward(X, ws, bs, bf16=True, bf16_first=False)
    Uo, Vo = O.Y_to_UV(Y, 10)
    m = (fl[0] > 0)[None]
    Uo = torch.where(m, Uo[0], torch.zeros_like(Uo[0]))
    Vo = torch.where(m, Vo[0], torch.zeros_like(Vo[0]))
    assert rel_l2(st.U.cpu().numpy(), Uo.numpy()) < 2e-2
    assert rel_l2(st.V.cpu().numpy(), Vo.numpy()) < 2e-2
