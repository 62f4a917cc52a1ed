"""smb_simple process (igm/processes/smb_simple/smb_simple.py:10-50):
ELA mass balance from a [time, gradabl, gradacc, ela, maxacc] table."""

from __future__ import annotations

import numpy as np

from .. import kernels as K
from .. import state as S


def _interp1d(xs, ys, x):
    """interp1d_tf (igm/utils/math/interp1d_tf.py): piecewise linear, constant
    outside the table."""
    x = np.clip(float(x), float(np.min(xs)), float(np.max(xs)))
    return np.float32(np.interp(x, np.asarray(xs, np.float64), np.asarray(ys, np.float64)))


def initialize(cfg, state):
    c = cfg.processes.smb_simple
    if len(c.array) == 0:
        state.smbpar = np.loadtxt(c.file, skiprows=1, dtype=np.float32)
    else:
        state.smbpar = np.array(c.array[1:]).astype(np.float32)
    state.smbpar = np.atleast_2d(state.smbpar)
    state.tlast_mb = -np.inf


def update(cfg, state):
    with S.update_scope(state):  # host-resident state: the results go back in one batch at the end
        _update(cfg, state)


def _update(cfg, state):
    c = cfg.processes.smb_simple
    t = float(state.t)
    if (t - float(state.tlast_mb)) >= c.update_freq:
        if hasattr(state, "logger"):
            state.logger.info("Construct mass balance at time : " + str(t))
        p = state.smbpar
        gradabl = _interp1d(p[:, 0], p[:, 1], t)
        gradacc = _interp1d(p[:, 0], p[:, 2], t)
        ela = _interp1d(p[:, 0], p[:, 3], t)
        maxacc = _interp1d(p[:, 0], p[:, 4], t)
        usurf = S.get(state, "usurf")
        icemask = S.get(state, "icemask") if hasattr(state, "icemask") else None
        smb = K.smb_simple(usurf, gradabl, gradacc, ela, maxacc, icemask=icemask)
        S.put(state, "smb", smb)
        state.tlast_mb = t


def finalize(cfg, state):
    pass
