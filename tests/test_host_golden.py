"""The product's host-side pieces of the path against the golden vectors made
by executing the reference's own source files (tests/golden/make_golden.py):
the vertical discretisation (igm_b200/vertical.py against
igm/processes/iceflow/vert_disc.py:10-47) and the time process
(igm_b200/processes/time.py against igm/processes/time/time.py:28-65,
including the save-time snapping and continue_run)."""

import numpy as np
import torch

from igm_b200 import vertical as Vd
from igm_b200.config import default_cfg
from igm_b200.processes import time as tproc
from igm_b200.state import State


def test_vertical_discretisation_matches_reference(golden):
    g = golden("vert_disc")
    for nz in [2, 3, 5, 10, 16, 30]:
        for sp in [1.0, 2.0, 4.0]:
            k = f"nz{nz}_s{int(sp)}"
            lv = Vd.compute_levels(nz, sp)
            z, dz = Vd.compute_zeta_dzeta(lv)
            w = Vd.define_vertical_weight(nz, sp)
            assert lv.dtype == np.float32 and w.shape == (nz, 1, 1)
            np.testing.assert_array_equal(lv, g[k + "_levels"], err_msg=k)
            np.testing.assert_array_equal(z, g[k + "_zeta"], err_msg=k)
            np.testing.assert_array_equal(dz, g[k + "_dzeta"], err_msg=k)
            np.testing.assert_array_equal(w[:, 0, 0], g[k + "_weight"], err_msg=k)


def test_time_process_matches_reference(golden):
    """The golden sequence: start 0, end 3, save 1, cfl 0.3, step_max 1, dx
    100 and twelve depth-averaged velocity fields of alternating scale.  The
    velocity maximum normally comes from the device's velocity reduction;
    here it is handed to the process through the same cache, as a CPU
    tensor, so that only the host logic runs."""
    g = golden("time")
    cfg = default_cfg({"time": {"start": 0.0, "end": 3.0, "save": 1.0, "cfl": 0.3, "step_max": 1.0}})
    st = State()
    st.dx = 100.0
    tproc.initialize(cfg, st)
    rng = np.random.default_rng(3)
    ts, dts, saves = [], [], []
    for k in range(12):
        sc = [80.0, 120.0, 15.0, 300.0][k % 4]
        ub = torch.as_tensor(rng.normal(0, sc, (6, 5)).astype(np.float32))
        vb = torch.as_tensor(rng.normal(0, sc, (6, 5)).astype(np.float32))
        st.ubar, st.vbar = ub, vb
        st._igm_velomax = (torch.maximum(ub.abs().max(), vb.abs().max()).reshape(1), st.ubar)
        st.it = k
        tproc.update(cfg, st)
        ts.append(float(st.t))
        dts.append(float(st.dt))
        saves.append(st.saveresult)
        if not st.continue_run:
            break
    assert len(ts) == len(g["t"])
    np.testing.assert_array_equal(np.float32(ts), g["t"])
    np.testing.assert_array_equal(np.float32(dts), g["dt"])
    # the steps that land on a save time (t = 0 first: dt 0) are the ones snapped to it
    for t, s in zip(ts, saves):
        assert s == (abs(t - round(t)) < 1e-6), (t, s)
    assert st.continue_run == (ts[-1] < 3.0)
