"""iceflow process (igm/processes/iceflow/iceflow.py:46-119).

Same dispatch as the reference: "solved" minimises the Blatter-Pattyn energy
over (U, V) with the device Adam solver; "emulated" evaluates the CNN
emulator and retrains it on the same energy every ``retrain_freq`` updates;
"diagnostic" additionally runs the solver from the emulated state every 10
model years and logs the misfit.  This implementation adds an optional
fallback (``cfg.processes.iceflow.fallback``): in emulated mode the solver
judges the emulator every ``every`` updates and replaces its velocities when
the emulated energy exceeds the solved one by more than ``margin`` -- until
the next check (``mode`` "takeover", the default) or for that update
alone (``mode`` "step").

Supported configuration: vert_basis "Lagrange", staggered_grid 1, the
default energy components, no sliding_law, dim_arrhenius 2, architecture
"cnn", exclude_borders 0, multiple_window_size 0.  Anything else raises.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import kernels as K
from .. import state as S
from ..solver import DeviceAdamSolver
from ..vertical import compute_levels, compute_zeta_dzeta, define_vertical_weight


def _check_supported(cfg):
    ic = cfg.processes.iceflow
    bad = []
    if ic.numerics.vert_basis != "Lagrange":
        bad.append(f"vert_basis={ic.numerics.vert_basis!r} (only 'Lagrange')")
    if int(ic.numerics.staggered_grid) != 1:
        bad.append(f"staggered_grid={ic.numerics.staggered_grid} (only 1)")
    if list(ic.physics.energy_components) != ["shear", "sliding_weertman", "gravity"]:
        bad.append(f"energy_components={list(ic.physics.energy_components)}")
    if len(ic.physics.sliding_law) > 0:
        bad.append(f"sliding_law={ic.physics.sliding_law!r}")
    if int(ic.physics.dim_arrhenius) != 2:
        bad.append(f"dim_arrhenius={ic.physics.dim_arrhenius} (only 2)")
    if ic.method not in ("emulated", "solved", "diagnostic"):
        bad.append(f"method={ic.method!r}")
    if ic.method != "solved":
        if ic.emulator.network.architecture != "cnn":
            bad.append(f"architecture={ic.emulator.network.architecture!r} (only 'cnn')")
        if ic.emulator.exclude_borders != 0 or ic.emulator.network.multiple_window_size != 0:
            bad.append("exclude_borders / multiple_window_size must be 0")
    if ic.solver.lbfgs:
        raise ValueError("solve_iceflow_lbfgs formely implemented, not working yet, will be updated.")
    if bad:
        raise NotImplementedError("igm_b200 iceflow: unsupported configuration: " + "; ".join(bad))


def physics(cfg):
    from .._lib import make_physics
    return make_physics(cfg.processes.iceflow.physics)


def initialize_iceflow_fields(cfg, state):
    """iceflow/utils.py:15-32."""
    ph = cfg.processes.iceflow.physics
    Nz = cfg.processes.iceflow.numerics.Nz
    thk = S.get(state, "thk")
    if not hasattr(state, "arrhenius"):
        S.put(state, "arrhenius", torch.full_like(thk, ph.init_arrhenius * ph.enhancement_factor))
    if not hasattr(state, "slidingco"):
        S.put(state, "slidingco", torch.full_like(thk, ph.init_slidingco))
    if not hasattr(state, "U"):
        state.U = torch.zeros((Nz,) + tuple(thk.shape), dtype=torch.float32, device=thk.device)
        state.V = torch.zeros_like(state.U)


def _fieldin(state):
    return [S.get(state, f) for f in ("thk", "usurf", "arrhenius", "slidingco")]


def _dx(state):
    if hasattr(state, "dx"):
        return float(state.dx)
    dX = getattr(state, "dX")
    return float(dX.reshape(-1)[0]) if hasattr(dX, "reshape") else float(dX)


def initialize_iceflow_solver(cfg, state):
    """solve.py:11-20: one optimizer object for the whole run."""
    state.iceflow_solver = DeviceAdamSolver(lr=cfg.processes.iceflow.solver.step_size)


def solve_iceflow(cfg, state, U, V):
    """solve.py:22-119 (Adam, EarlyStopping(2e-4, 10), mask thk == 0); the
    early stopping can be switched off (solver.early_stopping, an igm_b200
    key) to run nbitmax iterations per solve."""
    thk, usurf, A, c = _fieldin(state)
    sv = cfg.processes.iceflow.solver
    return state.iceflow_solver.solve(
        U, V, thk, usurf, A, c, _dx(state), state.dzeta, nbitmax=int(sv.nbitmax),
        phys=physics(cfg), relative_min_delta=0.0002, patience=10, early_stopping=bool(sv.get("early_stopping", True)))


def set_derived_velocities(cfg, state, mask):
    """velbase / velsurf / velbar (iceflow/utils.py:21-51) and the CFL max,
    one kernel; optionally masks U, V where thk == 0 first."""
    ub, vb, ub0, vb0, us0, vs0, vm = K.velocity_reduce(state.U, state.V, S.get(state, "thk"), state.vert_weight,
                                                       mask=mask)
    S.put(state, "uvelbase", ub0)
    S.put(state, "vvelbase", vb0)
    S.put(state, "uvelsurf", us0)
    S.put(state, "vvelsurf", vs0)
    S.put(state, "ubar", ub)
    S.put(state, "vbar", vb)
    state._igm_velomax = (vm, state.ubar)


def update_iceflow_solved(cfg, state):
    """solve.py:169-188."""
    state.U, state.V, costs = solve_iceflow(cfg, state, state.U, state.V)
    if cfg.processes.iceflow.force_max_velbar > 0:  # solve.py:178-179
        K.force_max_velbar(state.U, state.V, cfg.processes.iceflow.force_max_velbar)
    if len(cfg.processes.iceflow.solver.save_cost) > 0:
        np.savetxt(cfg.processes.iceflow.emulator.output_directory + cfg.processes.iceflow.solver.save_cost
                   + "-" + str(state.it) + ".dat", np.array(costs), fmt="%5.10f")
    state.COST_Glen = float(costs[-1]) if len(costs) else float("nan")
    set_derived_velocities(cfg, state, mask=False)


def initialize(cfg, state):
    if hasattr(state, "was_initialize_iceflow_already_called"):
        return
    _check_supported(cfg)
    ic = cfg.processes.iceflow
    initialize_iceflow_fields(cfg, state)
    from .. import emulator as E
    if ic.method == "emulated":
        E.initialize_iceflow_emulator(cfg, state)
    elif ic.method == "solved":
        initialize_iceflow_solver(cfg, state)
    elif ic.method == "diagnostic":
        E.initialize_iceflow_diagnostic(cfg, state)
    if ic.method == "emulated" and ic.fallback.every > 0:
        initialize_iceflow_solver(cfg, state)
    state.vert_weight = define_vertical_weight(ic.numerics.Nz, ic.numerics.vert_spacing)
    state.levels = compute_levels(ic.numerics.Nz, ic.numerics.vert_spacing)
    state.zeta, state.dzeta = compute_zeta_dzeta(state.levels)
    state.Leg_P, state.Leg_dPdz, state.Leg_I = None, None, None
    state.PAD = [[0, 0], [0, 0], [0, 0], [0, 0]]
    if ic.method != "solved":
        E.update_iceflow_emulator(cfg, state, 0)
        E.update_iceflow_emulated(cfg, state)
    state.was_initialize_iceflow_already_called = True


def update(cfg, state):
    with S.update_scope(state):  # host-resident state: the results go back in one batch at the end
        _update(cfg, state)


def _update(cfg, state):
    if hasattr(state, "logger"):
        state.logger.info("Update ICEFLOW at iteration : " + str(state.it))
    ic = cfg.processes.iceflow
    if ic.method in ("emulated", "diagnostic"):
        from .. import emulator as E
        if (ic.emulator.retrain_freq > 0) & (state.it > 0):
            E.update_iceflow_emulator(cfg, state, state.it, pertubate=ic.emulator.pertubate)
        if ic.method == "emulated" and ic.fallback.every > 0 and ic.fallback.get("mode", "takeover") == "takeover":
            E.update_iceflow_takeover(cfg, state)
            return
        E.update_iceflow_emulated(cfg, state)
        if ic.method == "diagnostic":
            E.update_iceflow_diagnostic(cfg, state)
        elif ic.fallback.every > 0:
            E.update_iceflow_fallback(cfg, state)
    elif ic.method == "solved":
        update_iceflow_solved(cfg, state)


def finalize(cfg, state):
    if cfg.processes.iceflow.emulator.save_model:
        from .. import emulator as E
        E.save_iceflow_model(cfg, state)
