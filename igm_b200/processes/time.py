"""time process (igm/processes/time/time.py:11-65): CFL-adaptive step snapped
to the save times.  The global max |ubar|, |vbar| comes from the velocity
reduction kernel (or igm_absmax2); the host reads that one float per step,
as the reference's Python branches on it do."""

from __future__ import annotations

import numpy as np

from .. import kernels as K
from .. import state as S


def initialize(cfg, state):
    c = cfg.processes.time
    state.t = np.float32(c.start)
    state.itsave = -1
    state.dt = np.float32(c.step_max)
    state.dt_target = np.float32(c.step_max)
    state.time_save = np.asarray(list(np.arange(c.start, c.end, c.save)) + [c.end], dtype=np.float32)


def velomax(state) -> np.float32:
    cached = state.__dict__.get("_igm_velomax")
    ub = getattr(state, "ubar")
    if cached is not None and cached[1] is ub:
        vm = cached[0]
    else:
        vm = K.absmax2(S.get(state, "ubar"), S.get(state, "vbar"))
    return np.float32(vm.item())


def update(cfg, state):
    with S.update_scope(state):  # host-resident state: the results go back in one batch at the end
        _update(cfg, state)


def _update(cfg, state):
    c = cfg.processes.time
    if hasattr(state, "logger"):
        state.logger.info("Update DT at time : " + str(float(state.t)))
    if c.cfl > 0:
        vm = velomax(state)
        if vm > 0:
            state.dt_target = np.float32(min(np.float32(c.cfl * state.dx) / vm, np.float32(c.step_max)))
        else:
            state.dt_target = np.float32(c.step_max)
    else:
        state.dt_target = np.float32(c.step_max)
    state.dt = state.dt_target
    if state.time_save[state.itsave + 1] <= state.t + state.dt:
        state.dt = np.float32(state.time_save[state.itsave + 1] - state.t)
        state.saveresult = True
        state.itsave += 1
    else:
        state.saveresult = False
    if state.it >= 0:
        state.t = np.float32(state.t + state.dt)
    state.continue_run = bool(state.t < c.end)


def finalize(cfg, state):
    pass
