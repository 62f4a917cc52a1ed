"""Emulator side of the iceflow process (igm/processes/iceflow/emulate/emulate.py
and diagnostic/diagnostic.py), on the device.

* ``update_iceflow_emulated``: one forward pass of the CNN over the whole
  domain, masked where thk == 0, then velbase / velsurf / velbar
  (emulate.py:116-152).
* ``update_iceflow_emulator``: physics-informed retraining by minimising the
  Blatter-Pattyn energy of the emulated velocities, one Adam step per patch
  (split_into_patches, emulate.py:155-308), gated by retrain_freq / warm_up_it,
  optionally on the perturbed copies of pertubate_X (emulate.py:310-328).
* ``update_iceflow_diagnostic``: every 10 model years the plain solver is run
  from the emulated velocities and the L1/L2 velbar misfit is logged
  (diagnostic.py:34-84).
* ``update_iceflow_fallback`` / ``update_iceflow_takeover`` (this
  implementation's addition): every ``fallback.every`` updates the solver
  judges the emulator; when the emulated energy exceeds the solved one by
  more than ``fallback.margin`` (relative) the solved velocities replace the
  emulated ones -- for that update alone (fallback.mode "step") or for the
  updates until the next check, each a warm-started solve (mode "takeover",
  the default).
* ``save_iceflow_model`` / ``load_iceflow_model``: the reference's Keras
  ``model.h5`` (written by igm_b200.keras_h5, no h5py needed) with its
  ``fieldin.dat`` and ``vert_grid.dat`` text files (emulate.py:331-359), and
  beside them weights, Adam moments and iteration count as ``model.npz``;
  ``load_keras_h5`` reads Keras ``model.h5`` files, so the emulators the
  reference ships run as pretrained networks and the reference loads the
  networks trained here.
"""

from __future__ import annotations

import os
import shutil

import numpy as np
import torch

from . import kernels as K
from . import state as S
from .cnn import CNN
from .processes import iceflow as P


def _patch_windows(ny, nx, nbmax):
    """split_into_patches (emulate.py:283-308): sy = ny//nbmax + 1 patches of
    int(ny/sy) rows, column-major patch order."""
    sy, sx = ny // nbmax + 1, nx // nbmax + 1
    ly, lx = int(ny / sy), int(nx / sx)
    wins = []
    for i in range(sx):
        for j in range(sy):
            wins.append((j * ly, i * lx))
    return wins, ly, lx


class EmulatorOptimizer:
    """State of ``state.opti_retrain``: the Keras legacy Adam hyper-parameters;
    the moments and the global iteration count live with the network."""

    def __init__(self, lr, epsilon, clipnorm):
        self.lr, self.epsilon, self.clipnorm = float(lr), float(epsilon), float(clipnorm)


def initialize_iceflow_emulator(cfg, state):
    """emulate.py:22-114."""
    ic = cfg.processes.iceflow
    e = ic.emulator
    state.opti_retrain = EmulatorOptimizer(e.lr, e.optimizer_epsilon, e.optimizer_clipnorm)
    net = e.network
    nb_inputs = len(e.fieldin)
    if nb_inputs != 5 or list(e.fieldin) != ["thk", "usurf", "arrhenius", "slidingco", "dX"]:
        raise NotImplementedError(f"emulator fieldin {list(e.fieldin)}: only the default five fields are supported")
    if net.activation != "LeakyReLU" or net.conv_ker_size != 3 or net.dropout_rate > 0 or net.cnn3d_for_vertical:
        raise NotImplementedError("only LeakyReLU 3x3 CNNs without dropout are supported")
    thk = S.get(state, "thk")
    state.iceflow_model = CNN(nb_layers=int(net.nb_layers), cin=nb_inputs, nout=2 * int(ic.numerics.Nz),
                              init=net.weight_initialization, seed=int(e.get("seed", 0)),
                              scales=list(e.get("input_scales", [1.0] * 5)), device=thk.device,
                              nb_out_filter=int(net.nb_out_filter), out_scale=float(e.get("output_scale", 1.0)))
    loaded = False
    if e.pretrained:
        if e.name:
            path = os.path.join(getattr(state, "original_cwd", os.getcwd()), e.name)
        else:
            path = _packaged_emulator_dir(cfg)
        if path and os.path.exists(os.path.join(path, "model.npz")):
            load_iceflow_model(state, path, cfg)
            loaded = True
        elif path and os.path.exists(os.path.join(path, "model.h5")):
            load_keras_h5(state, path, cfg)
            loaded = True
        if loaded:
            print("Found pretrained emulator: " + path)
    if not loaded:
        print("No pretrained emulator, start from scratch.")
    state.COST_EMULATOR = []
    state.GRAD_EMULATOR = []


def _fields(state):
    return [S.get(state, f) for f in ("thk", "usurf", "arrhenius", "slidingco")]


def update_iceflow_emulated(cfg, state):
    """emulate.py:116-152."""
    model: CNN = state.iceflow_model
    f = _fields(state)
    ny, nx = f[0].shape
    buf = model.buffers(1, ny, nx, train=False)
    model.prepare_input(f, P._dx(state), [(0, 0)], ny, nx, buf)
    U, V = model.forward(buf, 1, ny, nx, thk_mask=f[0])
    state.U, state.V = U[0], V[0]
    if cfg.processes.iceflow.force_max_velbar > 0:  # emulate.py:147-148
        K.force_max_velbar(state.U, state.V, cfg.processes.iceflow.force_max_velbar)
    P.set_derived_velocities(cfg, state, mask=False)


def train_step(model: CNN, fields_full, dx, windows, h, w, dzeta, phys, lr, opt: EmulatorOptimizer):
    """One physics-informed Adam step on a batch of windows: forward, energy
    and adjoint on the windowed fields, backward, Adam.  Returns the device
    energy sums [3] (divide by B (h-1)(w-1) for COST)."""
    B = len(windows)
    buf = model.buffers(B, h, w, train=True)
    model.prepare_input(fields_full, dx, windows, h, w, buf)
    U, V = model.forward(buf, B, h, w, keep_acts=True)
    count = B * (h - 1) * (w - 1)
    terms, dU, dV = K.energy(U, V, *buf["fields"], dx, dzeta, phys, grad=True, grad_scale=1.0 / count)
    model.backward(buf, B, h, w, dU, dV)
    model.adam_step(lr, epsilon=opt.epsilon, clipnorm=opt.clipnorm)
    return terms


def update_iceflow_emulator(cfg, state, it, pertubate=False):
    """emulate.py:155-281."""
    e = cfg.processes.iceflow.emulator
    run_it = e.retrain_freq > 0 and (it % e.retrain_freq == 0)
    warm_up = int(it <= e.warm_up_it)
    if not (warm_up or run_it):
        return
    model: CNN = state.iceflow_model
    f = _fields(state)
    ny, nx = f[0].shape
    wins, ly, lx = _patch_windows(ny, nx, int(e.framesizemax))
    copies = 1
    if pertubate:
        f, copies = _pertubate_fields(cfg, f)
    nbit, lr = (int(e.nbit_init), float(e.lr_init)) if warm_up else (int(e.nbit), float(e.lr))
    phys = P.physics(cfg)
    dx = P._dx(state)
    state.COST_EMULATOR = []
    state.GRAD_EMULATOR = []
    parallel = e.split_patch_method == "parrallel"
    # a patch's batch: its window in each (perturbed) copy, the copies stacked along y
    batch = lambda ws: [(k * ny + y0, x0) for (y0, x0) in ws for k in range(copies)]  # noqa: E731
    for _ in range(nbit):
        sums = []
        if parallel:
            sums.append(train_step(model, f, dx, batch(wins), ly, lx, state.dzeta, phys, lr, state.opti_retrain))
        else:
            for i, win in enumerate(wins):
                lr_i = lr * (e.lr_decay ** (i / 1000)) if e.lr_decay < 1 else lr
                sums.append(train_step(model, f, dx, batch([win]), ly, lx, state.dzeta, phys, lr_i,
                                       state.opti_retrain))
        count = (ly - 1) * (lx - 1) * copies * (len(wins) if parallel else 1)
        state.COST_EMULATOR.append(float(torch.stack(sums).sum(1).sum().item()) / count)
    model.check_errors()
    if len(e.save_cost) > 0:
        np.savetxt(e.save_cost + "-" + str(it) + ".dat", np.array(state.COST_EMULATOR), fmt="%5.10f")


def _pertubate_fields(cfg, f):
    """pertubate_X (emulate.py:310-328): the input and, for each perturbed
    field, copies with that field scaled by 1.2 and 0.8 -- the fields of
    data_assimilation's control_list when that process is configured, else
    thk and usurf -- stacked along y (each copy ny rows).  Returns (stacked
    [thk, usurf, arrhenius, slidingco], number of copies)."""
    names = ["thk", "usurf", "arrhenius", "slidingco"]
    if hasattr(cfg.processes, "data_assimilation"):
        which = [n for n in names if n in list(cfg.processes.data_assimilation.control_list)]
    else:
        which = ["thk", "usurf"]
    copies = [list(f)]
    for n in which:
        c = names.index(n)
        for s in (1.2, 0.8):
            g = list(f)
            g[c] = f[c] * s
            copies.append(g)
    stacked = [torch.cat([cp[c] for cp in copies], 0).contiguous() for c in range(4)]
    return stacked, len(copies)


def initialize_iceflow_diagnostic(cfg, state):
    """diagnostic.py:16-31."""
    initialize_iceflow_emulator(cfg, state)
    P.initialize_iceflow_solver(cfg, state)
    state.diagno = []
    state.tlast_diagno = -(10 ** 10)


def _velbar_misfit(state, dU, dV, thk):
    """computemisfit (diagnostic.py:74-84): L1 and L2 of the velbar difference where thk > 1."""
    w = np.asarray(state.vert_weight, np.float64)
    ub = (dU.double().cpu().numpy() * w).sum(0)
    vb = (dV.double().cpu().numpy() * w).sum(0)
    vel = np.stack([ub, vb])
    ma = np.broadcast_to((thk.cpu().numpy() > 1)[None], vel.shape).astype(np.float64)
    n = ma.sum()
    if n == 0:
        return 0.0, 0.0
    return float((ma * np.abs(vel)).sum() / n), float(np.sqrt((ma * vel ** 2).sum() / n))


def update_iceflow_diagnostic(cfg, state):
    """diagnostic.py:34-71."""
    t = float(state.t)
    if (t - state.tlast_diagno) >= 10:
        import time as _t
        t0 = _t.time()
        U, V, costs = P.solve_iceflow(cfg, state, state.U, state.V)
        l1, l2 = _velbar_misfit(state, state.U - U, state.V - V, S.get(state, "thk"))
        vol = float(S.get(state, "thk").double().sum().item()) * (P._dx(state) ** 2) / 1e9
        cost_em = state.COST_EMULATOR[-1] if state.COST_EMULATOR else float("nan")
        state.diagno.append([t, l1, l2, float(costs[-1]), cost_em, len(costs), len(state.COST_EMULATOR), vol])
        np.savetxt("errors_diagno.txt", np.stack(state.diagno), delimiter=",", fmt="%10.3f",
                   header="time,l1,l2,COST_Glen,COST_Emulator,nb_it_solve,nb_it_emul,vol", comments="")
        state.tlast_diagno = t
        state.diagno_time_solve = _t.time() - t0


def update_iceflow_fallback(cfg, state):
    """Solver as judge and fallback of the emulator (see module docstring)."""
    fb = cfg.processes.iceflow.fallback
    n = state.__dict__.setdefault("_igm_fallback_counter", 0)
    state._igm_fallback_counter = n + 1
    if n % int(fb.every) != 0:
        return
    f = _fields(state)
    dx = P._dx(state)
    phys = P.physics(cfg)
    e_em = float(K.energy(state.U, state.V, *f, dx, state.dzeta, phys)[0].sum().item())
    U, V, costs = state.iceflow_solver.solve(state.U, state.V, *f, dx, state.dzeta, nbitmax=int(fb.nbitmax),
                                             phys=phys, relative_min_delta=0.0002, patience=10)
    e_sv = float(K.energy(U, V, *f, dx, state.dzeta, phys)[0].sum().item())
    ny, nx = f[0].shape
    ns = (ny - 1) * (nx - 1)
    e_em, e_sv = e_em / ns, e_sv / ns
    du = torch.cat([(state.U - U).reshape(-1), (state.V - V).reshape(-1)])
    ref = torch.cat([U.reshape(-1), V.reshape(-1)])
    rel = float(torch.linalg.vector_norm(du.double()) / torch.linalg.vector_norm(ref.double()).clamp_min(1e-30))
    fallback = e_em > e_sv + float(fb.margin) * abs(e_sv)
    log = state.__dict__.setdefault("fallback_log", [])
    log.append(dict(t=float(state.t), it=int(state.it), e_emulated=e_em, e_solved=e_sv, vel_rel_l2=rel,
                    fallback=bool(fallback), solver_iterations=len(costs)))
    if fallback:
        state.U, state.V = U, V
        P.set_derived_velocities(cfg, state, mask=False)


def update_iceflow_takeover(cfg, state):
    """The emulator with the plain solver as its fallback, taking over
    (fallback.mode "takeover"): every ``fallback.every`` updates the solver
    judges the emulator -- it solves from its own last solution (the
    emulated velocities the first time), and the emulated energy is compared
    with the solved one -- and the outcome holds until the next check: while
    the emulator passes, each update is one network evaluation; after a
    failed check each update is a solve warm-started from the previous one,
    as the plain method runs, while the emulator keeps retraining on the
    states the run produces.  Every check is logged in state.fallback_log."""
    fb = cfg.processes.iceflow.fallback
    n = state.__dict__.setdefault("_igm_fallback_counter", 0)
    state._igm_fallback_counter = n + 1
    f = _fields(state)
    dx = P._dx(state)
    phys = P.physics(cfg)
    solved = state.__dict__.get("_igm_solved")
    if n % int(fb.every) == 0:
        update_iceflow_emulated(cfg, state)
        U0, V0 = solved if solved is not None else (state.U, state.V)
        U, V, costs = state.iceflow_solver.solve(U0, V0, *f, dx, state.dzeta, nbitmax=int(fb.nbitmax), phys=phys,
                                                 relative_min_delta=0.0002, patience=10)
        ny, nx = f[0].shape
        ns = (ny - 1) * (nx - 1)
        e_em = float(K.energy(state.U, state.V, *f, dx, state.dzeta, phys)[0].sum().item()) / ns
        e_sv = float(K.energy(U, V, *f, dx, state.dzeta, phys)[0].sum().item()) / ns
        du = torch.cat([(state.U - U).reshape(-1), (state.V - V).reshape(-1)])
        ref = torch.cat([U.reshape(-1), V.reshape(-1)])
        rel = float(torch.linalg.vector_norm(du.double()) / torch.linalg.vector_norm(ref.double()).clamp_min(1e-30))
        fallback = e_em > e_sv + float(fb.margin) * abs(e_sv)
        state.__dict__.setdefault("fallback_log", []).append(
            dict(t=float(state.t), it=int(state.it), e_emulated=e_em, e_solved=e_sv, vel_rel_l2=rel,
                 fallback=bool(fallback), solver_iterations=len(costs)))
        state._igm_solved = (U, V)
        state._igm_fallback_active = bool(fallback)
        if fallback:
            state.U, state.V = U, V
            P.set_derived_velocities(cfg, state, mask=False)
        return
    if state.__dict__.get("_igm_fallback_active", False):
        U, V, _ = state.iceflow_solver.solve(solved[0], solved[1], *f, dx, state.dzeta, nbitmax=int(fb.nbitmax),
                                             phys=phys, relative_min_delta=0.0002, patience=10)
        state._igm_solved = (U, V)
        state.U, state.V = U, V
        P.set_derived_velocities(cfg, state, mask=False)
    else:
        update_iceflow_emulated(cfg, state)


def keras_variables(m: CNN):
    """The network as the reference's Keras ``cnn`` computes it on the raw
    fields: the input scales folded into the first kernel (input channel c
    times scales[c]) and the output scale into the head's kernel and bias."""
    v = [np.array(a, dtype=np.float32) for a in m.get_variables()]
    v[0] = v[0] * m.scales[None, None, :v[0].shape[2], None]
    v[-2] = v[-2] * np.float32(m.out_scale)
    v[-1] = v[-1] * np.float32(m.out_scale)
    return v


def save_iceflow_model(cfg, state, directory="iceflow-model"):
    """emulate.py:331-359: model.h5 (a Keras HDF5 model file of the network on
    raw fields, which the reference's load_model reads), fieldin.dat and
    vert_grid.dat; beside them model.npz, the exact parameters with their
    input and output scales and the Adam state, which this package's loader
    prefers."""
    from .keras_h5 import write_keras_cnn
    if os.path.exists(directory):
        shutil.rmtree(directory)
    os.mkdir(directory)
    m: CNN = state.iceflow_model
    net = cfg.processes.iceflow.emulator.network
    write_keras_cnn(os.path.join(directory, "model.h5"), keras_variables(m), m.L, m.cin, m.nout, alpha=m.alpha,
                    init=str(net.weight_initialization))
    np.savez(os.path.join(directory, "model.npz"), params=m.params.cpu().numpy(), adam_m=m.m.cpu().numpy(),
             adam_v=m.v.cpu().numpy(), iterations=np.array(m.opt_iterations), nb_layers=np.array(m.L),
             nout=np.array(m.nout), cin=np.array(m.cin), scales=m.scales, out_scale=np.array(m.out_scale))
    with open(os.path.join(directory, "fieldin.dat"), "w") as fid:
        for key in cfg.processes.iceflow.emulator.fieldin:
            fid.write("%s \n" % key)
    with open(os.path.join(directory, "vert_grid.dat"), "w") as fid:
        fid.write("%4.0f  %s \n" % (cfg.processes.iceflow.numerics.Nz, "# number of vertical grid point (Nz)"))
        fid.write("%2.2f  %s \n" % (cfg.processes.iceflow.numerics.vert_spacing,
                                    "# param for vertical spacing (vert_spacing)"))


def emulator_dir_name(cfg) -> str:
    """The name under which the reference ships its pretrained emulators
    (emulate.py:37-62): pinnbp_<Nz>_<vert_spacing>_<architecture>_<nb_layers>_
    <nb_out_filter>_<dim_arrhenius>_1_<a (Lagrange) | e (Legendre)>."""
    ic = cfg.processes.iceflow
    net = ic.emulator.network
    basis = "e" if ic.numerics.vert_basis == "Legendre" else "a"
    return (f"pinnbp_{ic.numerics.Nz}_{int(ic.numerics.vert_spacing)}_{net.architecture}_{net.nb_layers}_"
            f"{net.nb_out_filter}_{ic.physics.dim_arrhenius}_1_{basis}")


def _packaged_emulator_dir(cfg):
    """The directory of the emulators the reference package ships
    (igm/processes/iceflow/emulate/emulators/<name>, emulate.py:64-77), found
    through the installed ``igm`` package without importing it; None when the
    reference is not installed or ships no emulator of that name."""
    import importlib.util
    try:
        spec = importlib.util.find_spec("igm")
    except (ImportError, ValueError):
        return None
    if spec is None or not spec.submodule_search_locations:
        return None
    for root in spec.submodule_search_locations:
        d = os.path.join(root, "processes", "iceflow", "emulate", "emulators", emulator_dir_name(cfg))
        if os.path.isdir(d):
            return d
    return None


def _check_fieldin(directory, cfg):
    """emulate.py:79-84: the emulator's input fields must be the configured ones."""
    fin = os.path.join(directory, "fieldin.dat")
    if cfg is not None and os.path.exists(fin):
        with open(fin) as f:
            names = [ln.split()[0] for ln in f if ln.strip()]
        if list(cfg.processes.iceflow.emulator.fieldin) != names:
            raise ValueError(f"{fin} lists {names}, the configuration {list(cfg.processes.iceflow.emulator.fieldin)}")


def load_keras_h5(state, directory, cfg=None):
    """Loads a Keras emulator saved by the reference (``model.h5``, the files it
    ships under igm/processes/iceflow/emulate/emulators and the ones
    ``save_iceflow_model`` writes) into the network: the weights of its
    nb_layers 3x3 convolutions and of the 1x1 head, in Keras order.  The
    inputs are the raw fields and the outputs the raw velocities, as in the
    reference, so the input scales and the output scale are reset to 1.
    Adam starts afresh, as the reference's ``opti_retrain`` does."""
    from .keras_h5 import cnn_params_from_keras, read_keras_weights
    _check_fieldin(directory, cfg)
    m: CNN = state.iceflow_model
    layers = read_keras_weights(os.path.join(directory, "model.h5"))
    m.set_params(cnn_params_from_keras(layers, m.L, m.cin, m.nout))
    m.scales = np.ones(5, np.float32)
    m.out_scale = 1.0
    m.m.zero_()
    m.v.zero_()
    m.opt_iterations = 0


def load_iceflow_model(state, directory, cfg=None):
    d = np.load(os.path.join(directory, "model.npz"))
    m: CNN = state.iceflow_model
    if int(d["nb_layers"]) != m.L or int(d["nout"]) != m.nout or int(d["cin"]) != m.cin:
        raise ValueError("saved emulator has a different architecture")
    m.set_params(d["params"])
    m.m.copy_(torch.as_tensor(d["adam_m"]))
    m.v.copy_(torch.as_tensor(d["adam_v"]))
    m.opt_iterations = int(d["iterations"])
    m.scales = np.asarray(d["scales"], np.float32)
    if "out_scale" in d.files:
        m.out_scale = float(d["out_scale"])
    _check_fieldin(directory, cfg)
