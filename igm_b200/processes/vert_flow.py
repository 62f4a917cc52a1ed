"""vert_flow process (igm/processes/vert_flow/vert_flow.py:18-59): the
vertical ice velocity W [Nz, Ny, Nx] from the horizontal velocities U, V the
iceflow process produced, plus its bed and surface values wvelbase, wvelsurf.

Supported: the Lagrange vertical basis with version 2 (the default of
igm/conf/processes/vert_flow.yaml) and both of its methods, kinematic (the
default; igm_vertical_velocity) and incompressibility
(igm_vertical_velocity_incompressibility, uniform dX), one kernel each.
Version 1 and the Legendre / SIA bases raise."""

from __future__ import annotations

import numpy as np

from .. import kernels as K
from .. import state as S
from ..vertical import compute_levels


def initialize(cfg, state):
    pass


def update(cfg, state):
    with S.update_scope(state):  # host-resident state: the results go back in one batch at the end
        _update(cfg, state)


def _update(cfg, state):
    vert_basis = cfg.processes.iceflow.numerics.vert_basis
    vf = cfg.processes.vert_flow
    if vert_basis not in ("Lagrange", "Legendre", "SIA"):
        raise ValueError(f"Unknown vertical basis: {vert_basis}")
    if vert_basis != "Lagrange" or int(vf.version) != 2 or vf.method not in ("kinematic", "incompressibility"):
        raise NotImplementedError("igm_b200 vert_flow: only vert_basis 'Lagrange', version 2, methods 'kinematic' "
                                  f"and 'incompressibility' (got {vert_basis!r}, {vf.version}, {vf.method!r})")
    num = cfg.processes.iceflow.numerics
    U, V = S.get(state, "U"), S.get(state, "V")
    levels = compute_levels(int(num.Nz), float(num.vert_spacing))
    if levels.shape[0] != U.shape[0]:
        raise ValueError(f"state.U has {U.shape[0]} levels, iceflow.numerics.Nz = {levels.shape[0]}")
    W = K.vertical_velocity(U, V, S.get(state, "topg"), S.get(state, "thk"), levels,
                            np.asarray(state.vert_weight, np.float64).reshape(-1), float(state.dx),
                            method=vf.method)
    S.put(state, "W", W)
    S.put(state, "wvelbase", W[0])
    S.put(state, "wvelsurf", W[-1])


def finalize(cfg, state):
    pass
