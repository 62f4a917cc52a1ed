"""thk process (igm/processes/thk/thk.py:11-58): slope-limited upwind mass
conservation, flotation lower surface and upper surface, one kernel."""

from __future__ import annotations

import torch

from .. import kernels as K
from .. import state as S


def _sealevel(cfg, state):
    if hasattr(state, "sealevel"):
        sl = state.sealevel
        if hasattr(sl, "numel") and sl.numel() != 1:
            raise NotImplementedError("a sea-level field is not supported; give a scalar state.sealevel")
        return float(sl)
    return float(cfg.processes.thk.default_sealevel)


def initialize(cfg, state):
    if not hasattr(state, "topg"):
        raise ValueError("The 'thk' module requires an initial topography ('state.topg') to be defined. "
                         "Please define it through the preprocessing steps (not yet implemented)")
    thk = S.get(state, "thk")
    topg = S.get(state, "topg")
    lsurf, usurf = K.surfaces(thk, topg, cfg.processes.thk.ratio_density, _sealevel(cfg, state))
    S.put(state, "lsurf", lsurf)
    S.put(state, "usurf", usurf)
    S.sync_host(state)


def update(cfg, state):
    with S.update_scope(state):  # host-resident state: the results go back in one batch at the end
        _update(cfg, state)


def _update(cfg, state):
    if state.it >= 0:
        if hasattr(state, "logger"):
            state.logger.info("Ice thickness equation at time : " + str(float(state.t)))
        thk = S.get(state, "thk")
        if not hasattr(state, "smb"):
            S.put(state, "smb", torch.zeros_like(thk))
        thk_new, usurf, lsurf, divflux = K.transport_step(
            S.get(state, "ubar"), S.get(state, "vbar"), thk, S.get(state, "topg"), S.get(state, "smb"),
            float(state.dx), float(state.dt), slope_type=cfg.processes.thk.slope_type,
            ratio_density=cfg.processes.thk.ratio_density, sealevel=_sealevel(cfg, state))
        S.put(state, "divflux", divflux)
        S.put(state, "thk", thk_new)
        S.put(state, "lsurf", lsurf)
        S.put(state, "usurf", usurf)


def finalize(cfg, state):
    pass
