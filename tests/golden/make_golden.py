"""Generate the golden vectors in this directory by executing the reference's
own source files (IGM 3.0.0) for the iceflow + thk path.

TensorFlow is not installable here, so ``tf_shim`` stands in for it (every
``tf.*`` call maps to the torch op with the same semantics; GradientTape is
torch autograd).  The reference package's ``__init__`` files import Hydra,
xarray, OGGM and the rest of the model, so the packages on the path are
registered as bare namespace stubs and only the hot-path modules are loaded
from their files.

Run from the repository root:  python tests/golden/make_golden.py REF_ROOT [case ...]
(REF_ROOT: the root of the reference's source tree, the directory holding
``igm/``; or set IGM_REFERENCE_ROOT; the optional case names, functions of
this file, run those cases alone).  Writes ``*.npz`` / ``*.json`` next to this file.
The generated inputs are seeded; re-running reproduces the files bit for bit.
"""

from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np
import torch
import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import tf_shim  # noqa: E402

tf_shim.install()
import tensorflow as tf  # noqa: E402  (the shim)

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IGM_REFERENCE_ROOT", "")
if not REF or not os.path.isdir(os.path.join(REF, "igm")):
    sys.exit("usage: python tests/golden/make_golden.py REF_ROOT (the reference source tree, holding igm/), "
             "or set IGM_REFERENCE_ROOT")
IGM = os.path.join(REF, "igm")


def _stub(name, path):
    m = types.ModuleType(name)
    m.__path__ = [path]
    sys.modules[name] = m
    parent, _, child = name.rpartition(".")
    if parent:
        setattr(sys.modules[parent], child, m)
    return m


for pkg in ["", "processes", "processes/iceflow", "processes/iceflow/energy",
            "processes/iceflow/energy/sliding_laws", "processes/iceflow/emulate",
            "processes/iceflow/emulate/emulators", "processes/iceflow/solve",
            "processes/iceflow/diagnostic", "processes/thk", "processes/time", "processes/vert_flow",
            "utils", "utils/gradient", "utils/math", "processes/data_assimilation",
            "processes/data_assimilation/cost_terms"]:
    _stub("igm" + ("." + pkg.replace("/", ".") if pkg else ""), os.path.join(IGM, pkg))

energy_pkg = sys.modules["igm.processes.iceflow.energy"]
for comp in ["cost_shear", "cost_gravity", "cost_sliding_weertman"]:
    mod = importlib.import_module(f"igm.processes.iceflow.energy.{comp}")
    setattr(energy_pkg, comp, getattr(mod, comp))

vert_disc = importlib.import_module("igm.processes.iceflow.vert_disc")
ice_utils = importlib.import_module("igm.processes.iceflow.utils")
energy_mod = importlib.import_module("igm.processes.iceflow.energy.energy")
solve_mod = importlib.import_module("igm.processes.iceflow.solve.solve")
emulate_mod = importlib.import_module("igm.processes.iceflow.emulate.emulate")
divflux_mod = importlib.import_module("igm.utils.gradient.compute_divflux_slope_limiter")
thk_mod = importlib.import_module("igm.processes.thk.thk")
time_mod = importlib.import_module("igm.processes.time.time")
vflow_mod = importlib.import_module("igm.processes.vert_flow.vert_flow_v2")


def ns(d):
    if isinstance(d, dict):
        return types.SimpleNamespace(**{k: ns(v) for k, v in d.items()})
    return d


def load_cfg(**over):
    procs = {}
    for p in ["iceflow", "thk", "time"]:
        with open(os.path.join(IGM, "conf", "processes", f"{p}.yaml")) as f:
            procs.update(yaml.safe_load(f))
    for path, val in over.items():
        d = procs
        keys = path.split(".")
        for k in keys[:-1]:
            d = d[k]
        d[keys[-1]] = val
    return ns({"processes": procs})


def glacier(ny, nx, dx, seed, dtype, c_neg=False):
    """Seeded small valley-glacier state with varying A, c and some ice-free cells."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(ny) * dx, np.arange(nx) * dx, indexing="ij")
    Ly, Lx = ny * dx, nx * dx
    topg = 2500 - 0.08 * x + 4e-4 * (y - Ly / 2) ** 2 / (Ly / 2000) + rng.normal(0, 3, (ny, nx))
    thk = np.maximum(0, 150 * (1 - ((y - Ly / 2) / (0.4 * Ly)) ** 2) * (1 - x / (1.1 * Lx)))
    thk = thk + rng.uniform(0, 5, (ny, nx)) * (thk > 0)
    usurf = topg + thk
    A = np.exp(rng.uniform(np.log(20), np.log(150), (ny, nx)))
    c = np.exp(rng.uniform(np.log(0.01), np.log(0.1), (ny, nx)))
    if c_neg:
        c[rng.uniform(size=(ny, nx)) < 0.1] = 0.0
    f = lambda a: torch.as_tensor(a, dtype=dtype)
    return dict(topg=f(topg), thk=f(thk), usurf=f(usurf), arrhenius=f(A), slidingco=f(c),
                dX=f(np.full((ny, nx), dx)), dx=dx)


def vel(nz, ny, nx, seed, dtype, scale=40.0):
    rng = np.random.default_rng(seed + 1000)
    base = rng.normal(0, scale, (2, nz, ny, nx))
    prof = np.linspace(0.3, 1.0, nz)[:, None, None]
    return (torch.as_tensor(base[0] * prof + 30, dtype=dtype),
            torch.as_tensor(base[1] * prof - 5, dtype=dtype))


def energy_case(name, ny, nx, nz, dx, seed, dtype, spacing=4.0, c_neg=False):
    cfg = load_cfg(**{"iceflow.numerics.Nz": nz, "iceflow.numerics.vert_spacing": spacing})
    g = glacier(ny, nx, dx, seed, dtype, c_neg)
    U, V = vel(nz, ny, nx, seed, dtype)
    levels = vert_disc.compute_levels(nz, spacing).to(dtype)
    zeta, dzeta = vert_disc.compute_zeta_dzeta(levels)
    fieldin = [g[f][None] for f in cfg.processes.iceflow.emulator.fieldin]
    Uv = U.clone().requires_grad_(True)
    Vv = V.clone().requires_grad_(True)
    with tf.GradientTape(persistent=True) as t:
        terms = energy_mod.iceflow_energy(cfg, Uv[None], Vv[None], fieldin, [zeta, dzeta, None, None])
        means = [tf.reduce_mean(e) for e in terms]
        COST = tf.add_n(means)
    gU, gV = t.gradient(COST, [Uv, Vv])
    out = dict(U=U, V=V, thk=g["thk"], usurf=g["usurf"], arrhenius=g["arrhenius"], slidingco=g["slidingco"],
               dx=np.array(dx), levels=levels, dzeta=dzeta, cost=COST.detach(),
               shear=terms[0][0].detach(), sliding=terms[1][0].detach(), gravity=terms[2][0].detach(),
               means=torch.stack([m.detach() for m in means]), gradU=gU, gradV=gV)
    save(f"energy_{name}", out)


def vert_cases():
    out = {}
    for nz in [2, 3, 5, 10, 16, 30]:
        for sp in [1.0, 2.0, 4.0]:
            lv = vert_disc.compute_levels(nz, sp)
            z, dz = vert_disc.compute_zeta_dzeta(lv)
            w = vert_disc.define_vertical_weight(nz, sp)
            key = f"nz{nz}_s{int(sp)}"
            out[key + "_levels"] = lv
            out[key + "_zeta"] = z
            out[key + "_dzeta"] = dz
            out[key + "_weight"] = w[:, 0, 0]
    save("vert_disc", out)


def solver_case(name, ny, nx, nz, dx, seed, dtype, nbitmax, n_solves):
    cfg = load_cfg(**{"iceflow.numerics.Nz": nz, "iceflow.solver.nbitmax": nbitmax,
                      "iceflow.method": "solved"})
    g = glacier(ny, nx, dx, seed, dtype)
    state = types.SimpleNamespace(**{k: g[k] for k in ["thk", "usurf", "arrhenius", "slidingco", "dX", "topg"]})
    state.it = 5
    state.U = torch.zeros((nz, ny, nx), dtype=dtype)
    state.V = torch.zeros((nz, ny, nx), dtype=dtype)
    state.levels = vert_disc.compute_levels(nz, 4.0).to(dtype)
    state.zeta, state.dzeta = vert_disc.compute_zeta_dzeta(state.levels)
    state.Leg_P = state.Leg_dPdz = None
    state.vert_weight = vert_disc.define_vertical_weight(nz, 4.0).to(dtype)
    solve_mod.initialize_iceflow_solver(cfg, state)
    out = dict(thk=g["thk"], usurf=g["usurf"], arrhenius=g["arrhenius"], slidingco=g["slidingco"],
               dx=np.array(dx), nbitmax=np.array(nbitmax))
    for s in range(n_solves):
        U0 = state.U.detach().clone()
        Uf, Vf, costs = solve_mod.solve_iceflow(cfg, state, state.U, state.V)
        solve_mod.update_iceflow_solved(cfg, state) if False else None
        state.U, state.V = Uf.detach(), Vf.detach()
        state.COST_Glen = costs[-1].numpy()
        ub, vb = ice_utils.get_velbar(state.U, state.V, state.vert_weight, "Lagrange")
        out[f"s{s}_U"] = state.U
        out[f"s{s}_V"] = state.V
        out[f"s{s}_ubar"] = ub
        out[f"s{s}_vbar"] = vb
        out[f"s{s}_costs"] = torch.stack([c.detach() for c in costs])
        out[f"s{s}_iterations_after"] = np.array(state.optimizer.iterations)
    save(f"solver_{name}", out)


def transport_cases():
    rng = np.random.default_rng(7)
    out = {}
    ny, nx = 17, 13
    h = np.maximum(0, rng.normal(50, 60, (ny, nx)))
    h[:, :2] = 0
    u = rng.normal(5, 30, (ny, nx))
    v = rng.normal(-3, 30, (ny, nx))
    for dtype, tag in [(torch.float32, "f32"), (torch.float64, "f64")]:
        H, Uu, Vv = (torch.as_tensor(a, dtype=dtype) for a in (h, u, v))
        out[f"{tag}_h"], out[f"{tag}_u"], out[f"{tag}_v"] = H, Uu, Vv
        for st in ["godunov", "minmod", "superbee"]:
            out[f"{tag}_{st}"] = divflux_mod.compute_divflux_slope_limiter(Uu, Vv, H, 50.0, 50.0, 0.7, slope_type=st)
    # thk.update through the reference process (superbee, smb present)
    cfg = load_cfg()
    topg = torch.as_tensor(rng.normal(100, 150, (ny, nx)), dtype=torch.float32)
    smb = torch.as_tensor(rng.normal(0, 2, (ny, nx)), dtype=torch.float32)
    state = types.SimpleNamespace(topg=topg, thk=torch.as_tensor(h, dtype=torch.float32), it=3,
                                  ubar=torch.as_tensor(u, dtype=torch.float32),
                                  vbar=torch.as_tensor(v, dtype=torch.float32),
                                  dx=50.0, dt=torch.tensor(0.7), smb=smb)
    thk_mod.initialize(cfg, state)
    out["thk_init_usurf"] = state.usurf
    out["thk_topg"], out["thk_smb"], out["thk_h"] = topg, smb, state.thk
    thk_mod.update(cfg, state)
    out["thk_new"], out["thk_usurf"], out["thk_lsurf"], out["thk_divflux"] = state.thk, state.usurf, state.lsurf, state.divflux
    save("transport", out)


def time_case():
    cfg = load_cfg(**{"time.start": 0.0, "time.end": 3.0, "time.save": 1.0})
    state = types.SimpleNamespace(dx=100.0, it=0)
    time_mod.initialize(cfg, state)
    rng = np.random.default_rng(3)
    ts, dts = [], []
    for k in range(12):
        sc = [80.0, 120.0, 15.0, 300.0][k % 4]
        state.ubar = torch.as_tensor(rng.normal(0, sc, (6, 5)), dtype=torch.float32)
        state.vbar = torch.as_tensor(rng.normal(0, sc, (6, 5)), dtype=torch.float32)
        time_mod.update(cfg, state)
        ts.append(float(state.t))
        dts.append(float(state.dt))
        state.it += 1
        if not bool(state.continue_run):
            break
    save("time", dict(t=np.array(ts, np.float32), dt=np.array(dts, np.float32)))


class TinyCNN:
    """Stand-in for the Keras model object: callable on NHWC input, with
    ``trainable_variables`` ordered as Keras orders them (kernel, bias per layer)."""

    def __init__(self, cin, nfilt, nlayers, nout, seed, dtype):
        rng = np.random.default_rng(seed)
        self.w, self.b = [], []
        c = cin
        for _ in range(nlayers):
            self.w.append(torch.as_tensor(rng.normal(0, np.sqrt(2 / (9 * c)), (3, 3, c, nfilt)), dtype=dtype).requires_grad_(True))
            self.b.append(torch.as_tensor(rng.normal(0, 0.01, (nfilt,)), dtype=dtype).requires_grad_(True))
            c = nfilt
        self.w.append(torch.as_tensor(rng.normal(0, np.sqrt(1 / c), (1, 1, c, nout)) * 20, dtype=dtype).requires_grad_(True))
        self.b.append(torch.as_tensor(rng.normal(0, 0.01, (nout,)), dtype=dtype).requires_grad_(True))

    @property
    def trainable_variables(self):
        out = []
        for w, b in zip(self.w, self.b):
            out += [w, b]
        return out

    def __call__(self, X):
        x = X.permute(0, 3, 1, 2)
        for w, b in zip(self.w[:-1], self.b[:-1]):
            x = torch.nn.functional.leaky_relu(torch.nn.functional.conv2d(x, w.permute(3, 2, 0, 1), b, padding=1), 0.01)
        return torch.nn.functional.conv2d(x, self.w[-1].permute(3, 2, 0, 1), self.b[-1]).permute(0, 2, 3, 1)


def emulator_case():
    """update_iceflow_emulator (emulate.py:155-281) + update_iceflow_emulated (:116-152)."""
    nz, ny, nx, dx = 4, 22, 19, 100.0
    dtype = torch.float64
    cfg = load_cfg(**{"iceflow.numerics.Nz": nz, "iceflow.emulator.framesizemax": 9,
                      "iceflow.emulator.nbit": 2, "iceflow.emulator.nbit_init": 3,
                      "iceflow.emulator.lr": 1e-3, "iceflow.emulator.lr_init": 3e-3,
                      "iceflow.emulator.warm_up_it": 0, "iceflow.emulator.retrain_freq": 2})
    g = glacier(ny, nx, dx, 11, dtype)
    state = types.SimpleNamespace(**{k: g[k] for k in ["thk", "usurf", "arrhenius", "slidingco", "dX", "topg"]})
    state.levels = vert_disc.compute_levels(nz, 4.0).to(dtype)
    state.zeta, state.dzeta = vert_disc.compute_zeta_dzeta(state.levels)
    state.Leg_P = state.Leg_dPdz = None
    state.vert_weight = vert_disc.define_vertical_weight(nz, 4.0).to(dtype)
    state.iceflow_model = TinyCNN(5, 6, 2, 2 * nz, 5, dtype)
    state.opti_retrain = tf.keras.optimizers.legacy.Adam(
        learning_rate=cfg.processes.iceflow.emulator.lr,
        epsilon=cfg.processes.iceflow.emulator.optimizer_epsilon,
        clipnorm=cfg.processes.iceflow.emulator.optimizer_clipnorm)
    out = dict(thk=g["thk"], usurf=g["usurf"], arrhenius=g["arrhenius"], slidingco=g["slidingco"], dx=np.array(dx))
    for i, v in enumerate(state.iceflow_model.trainable_variables):
        out[f"w0_{i}"] = v.detach().clone()
    for step, it in enumerate([0, 1, 2]):
        emulate_mod.update_iceflow_emulator(cfg, state, it)
        for i, v in enumerate(state.iceflow_model.trainable_variables):
            out[f"w{step + 1}_{i}"] = v.detach().clone()
        if hasattr(state, "COST_EMULATOR"):
            out[f"cost{step + 1}"] = torch.stack([torch.as_tensor(c).detach() for c in state.COST_EMULATOR])
    emulate_mod.update_iceflow_emulated(cfg, state)
    out["U"], out["V"], out["ubar"], out["vbar"] = state.U, state.V, state.ubar, state.vbar
    out["opt_iterations"] = np.array(state.opti_retrain.iterations)
    save("emulator", out)


def vert_flow_cases():
    """compute_w_kinematic_tf (vert_flow_v2.py:30-37) on seeded glaciers, with
    dz from compute_dz and the weights of define_vertical_weight, as
    compute_vertical_velocity_kinematic_v2 (:17-27) calls it."""
    out = {}
    for tag, ny, nx, nz, sp, dx, seed, dtype in [("f32", 23, 31, 10, 4.0, 100.0, 7, torch.float32),
                                                 ("f64", 23, 31, 10, 4.0, 100.0, 7, torch.float64),
                                                 ("nz5_f32", 17, 12, 5, 1.0, 50.0, 8, torch.float32),
                                                 ("nz2_f32", 9, 14, 2, 2.0, 25.0, 9, torch.float32)]:
        g = glacier(ny, nx, dx, seed, dtype)
        U, V = vel(nz, ny, nx, seed, dtype)
        levels = vert_disc.compute_levels(nz, sp).to(dtype)
        w = vert_disc.define_vertical_weight(nz, sp).to(dtype)
        dz = vert_disc.compute_dz(g["thk"], levels)
        W = vflow_mod.compute_w_kinematic_tf(U, V, g["topg"], g["thk"], dz, torch.tensor(dx, dtype=dtype), w)
        # the incompressibility method (:40-57) reads cfg and state; dX is the uniform spacing field
        cfg = load_cfg(**{"iceflow.numerics.Nz": nz, "iceflow.numerics.vert_spacing": sp})
        st = types.SimpleNamespace(U=U, V=V, topg=g["topg"], thk=g["thk"], vert_weight=w,
                                   dX=torch.full_like(g["thk"], dx))
        orig = vflow_mod.compute_levels
        vflow_mod.compute_levels = lambda n, s_: orig(n, s_).to(dtype)  # FP64 cases: levels in the case's dtype
        Wi = vflow_mod.compute_vertical_velocity_incompressibility_v2(cfg, st)
        vflow_mod.compute_levels = orig
        out.update({f"{tag}_U": U, f"{tag}_V": V, f"{tag}_topg": g["topg"], f"{tag}_thk": g["thk"],
                    f"{tag}_levels": levels, f"{tag}_weight": w[:, 0, 0], f"{tag}_dx": np.asarray(dx),
                    f"{tag}_W": W, f"{tag}_Wi": Wi})
    save("vert_flow", out)


def keras_h5_cases():
    """The Keras emulators the reference ships (igm/processes/iceflow/emulate/
    emulators/*/model.h5) read by igm_b200.keras_h5: per file the weight names,
    shapes, float64 sums and first values, as a JSON summary (the weights
    themselves stay in the reference)."""
    import glob
    import json
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from igm_b200.keras_h5 import read_keras_weights
    root = os.path.join(IGM, "processes", "iceflow", "emulate", "emulators")
    out = {}
    for path in sorted(glob.glob(os.path.join(root, "**", "model.h5"), recursive=True)):
        rel = os.path.relpath(os.path.dirname(path), root)
        layers = read_keras_weights(path)
        out[rel] = [{"layer": ln, "weights": [{"name": wn, "shape": list(a.shape), "sum": float(a.astype(np.float64).sum()),
                                               "sumsq": float((a.astype(np.float64) ** 2).sum()),
                                               "first": [float(v) for v in a.reshape(-1)[:4]]} for wn, a in ws]}
                    for ln, ws in layers if ws]
    dst = os.path.join(HERE, "keras_h5.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {dst} ({os.path.getsize(dst)} B)")


def keras_h5_layout_case():
    """The file layout of the newest emulator the reference ships without
    dropout layers (pinnbp_5_4_cnn_16_32_2_1_e, written by tf.keras 2.15):
    the SHA-256 and length of its model_config, its layer and weight names,
    its root attribute names, and the raw bytes of the superblock's format
    fields and of the header messages of one kernel dataset -- what
    igm_b200.keras_h5's writer must reproduce for the reference's
    load_model to read the networks trained here."""
    import hashlib
    import json
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from igm_b200.keras_h5 import _File
    path = os.path.join(IGM, "processes", "iceflow", "emulate", "emulators", "pinnbp_5_4_cnn_16_32_2_1_e", "model.h5")
    f = _File(path)
    attrs = f.attributes(f.root)
    mc = str(attrs["model_config"].reshape(-1)[0]).encode()
    mw = f.lookup("model_weights")
    lnames = [str(x) for x in f.attributes(mw)["layer_names"].reshape(-1)]
    kids = f.children(mw)
    layer_weights = {n: [str(x) for x in np.asarray(f.attributes(kids[n])["weight_names"]).reshape(-1)] for n in lnames}
    conv = f.children(kids["conv2d"])["conv2d"]
    kern = f.children(conv)["kernel:0"]
    msgs = {"0x%02x" % t: f.b[p - 8:p + n].hex() for t, p, n in f.messages(kern) if t in (1, 3, 5)}
    layout = [f.b[p:p + 2].hex() for t, p, n in f.messages(kern) if t == 8]
    out = {"file": os.path.relpath(path, IGM), "model_config_sha256": hashlib.sha256(mc).hexdigest(),
           "model_config_len": len(mc), "root_attributes": sorted(attrs),
           "keras_version": str(attrs["keras_version"].reshape(-1)[0]),
           "model_weights_attributes": sorted(f.attributes(mw)), "layer_names": lnames,
           "weight_names": layer_weights, "superblock_format": f.b[8:24].hex(),
           "kernel_messages": msgs, "kernel_layout_version_class": layout[0]}
    dst = os.path.join(HERE, "keras_h5_layout.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {dst} ({os.path.getsize(dst)} B)")


def assim_cases():
    """The data-assimilation cost terms of the default configuration (control
    thk; costs velsurf, thk, icemask; penalty constraint; anisotropic and
    isotropic thickness regularisation), executed from the reference's files
    (cost_terms/misfit_velsurf.py, misfit_thk.py, regu_thk.py, the penalties of
    total_cost.py:36-46, utils.py create_density_matrix and
    compute_flow_direction_for_anisotropic_smoothing), with torch autograd
    gradients w.r.t. thk and the surface velocities."""
    dau = importlib.import_module("igm.processes.data_assimilation.utils")
    mv = importlib.import_module("igm.processes.data_assimilation.cost_terms.misfit_velsurf")
    mt = importlib.import_module("igm.processes.data_assimilation.cost_terms.misfit_thk")
    rt = importlib.import_module("igm.processes.data_assimilation.cost_terms.regu_thk")
    out = {}
    for tag, dtype, aniso, reg in [("f64", torch.float64, True, "topg"), ("f32", torch.float32, True, "topg"),
                                   ("iso_f64", torch.float64, False, "topg"), ("thk_f64", torch.float64, True, "thk")]:
        rng = np.random.default_rng(11)
        ny, nx, dx = 23, 31, 100.0
        g = glacier(ny, nx, dx, 12, dtype)
        f = lambda a: torch.as_tensor(np.asarray(a), dtype=dtype)  # noqa: E731
        thk = g["thk"] + f(rng.normal(0, 10, (ny, nx)))  # some negative values: the penalty is active
        usurf = g["usurf"]
        icemaskobs = f((g["thk"].numpy() > 0).astype(np.float64))
        uvs, vvs = f(rng.normal(20, 15, (ny, nx))), f(rng.normal(-5, 15, (ny, nx)))
        uo, vo = f(rng.normal(20, 15, (ny, nx))), f(rng.normal(-5, 15, (ny, nx)))
        uo[rng.uniform(size=(ny, nx)) < 0.2] = float("nan")
        vo[rng.uniform(size=(ny, nx)) < 0.1] = float("nan")
        thkobs = torch.full_like(thk, float("nan"))
        thkobs[:, 7] = g["thk"][:, 7] + 3.0
        thkobs[11, :] = g["thk"][11, :] - 2.0
        cfg = load_cfg()
        with open(os.path.join(IGM, "conf", "processes", "data_assimilation.yaml")) as fh:
            da = yaml.safe_load(fh)["data_assimilation"]
        da["regularization"]["smooth_anisotropy_factor"] = 0.2 if aniso else 1.0
        da["regularization"]["to_regularize"] = reg
        da.setdefault("cook", {"infer_params": False})
        cfg.processes.data_assimilation = ns(da)
        dens = dau.create_density_matrix(thkobs, kernel_size=5)
        dens = torch.where(dens > 0, 1.0 / dens, torch.zeros_like(dens))
        dens = torch.where(torch.isnan(thkobs), torch.zeros_like(dens), dens)
        dens = dens / torch.mean(dens[dens > 0])
        thk_v = thk.clone().requires_grad_(True)
        uvs_v, vvs_v = uvs.clone().requires_grad_(True), vvs.clone().requires_grad_(True)
        st = types.SimpleNamespace(thk=thk_v, usurf=usurf, uvelsurf=uvs_v, vvelsurf=vvs_v, uvelsurfobs=uo,
                                   vvelsurfobs=vo, thkobs=thkobs, dens_thkobs=dens, icemaskobs=icemaskobs,
                                   icemask=icemaskobs, dx=dx)
        if aniso:
            dau.compute_flow_direction_for_anisotropic_smoothing(st)
            fx, fy = f(np.asarray(st.flowdirx)), f(np.asarray(st.flowdiry))
            st.flowdirx, st.flowdiry = fx, fy
        else:
            fx = fy = torch.zeros((ny - 1, nx - 1), dtype=dtype)
        c_vel = mv.misfit_velsurf(cfg, st)
        c_thk = mt.misfit_thk(cfg, st)
        c_ice = 10 ** 10 * torch.mean(torch.where(icemaskobs > 0.5, torch.zeros_like(thk_v), thk_v ** 2))
        c_pos = 10 ** 10 * torch.mean(torch.where(thk_v >= 0, torch.zeros_like(thk_v), thk_v ** 2))
        c_reg = rt.regu_thk(cfg, st)
        total = c_vel + c_thk + c_ice + c_pos + c_reg
        gt, gu, gv = torch.autograd.grad(total, [thk_v, uvs_v, vvs_v])
        out.update({f"{tag}_{k}": v for k, v in dict(
            thk=thk, usurf=usurf, icemaskobs=icemaskobs, uvs=uvs, vvs=vvs, uobs=uo, vobs=vo, thkobs=thkobs,
            dens=dens, flowdirx=fx, flowdiry=fy, c_vel=c_vel, c_thk=c_thk, c_ice=c_ice, c_pos=c_pos, c_reg=c_reg,
            g_thk=gt, g_u=gu, g_v=gv, dx=np.asarray(dx), aniso=np.asarray(aniso), to_thk=np.asarray(reg == "thk")).items()})
    save("assim", out)


def divflux_cases():
    """compute_divflux (utils/gradient/compute_divflux.py:6-51), both methods,
    and the flux-divergence cost terms cost_divfluxobs (with and without
    force_zero_sum) and cost_divfluxfcz, executed from the reference's files,
    with torch autograd gradients w.r.t. ubar, vbar and thk.  cost_divfluxfcz
    is called twice, as in the reference's loop: at i = 0 on detached inputs
    (its scipy regression sets state.res), then at i = 1 with gradients."""
    cd = importlib.import_module("igm.utils.gradient.compute_divflux")
    co = importlib.import_module("igm.processes.data_assimilation.cost_terms.cost_divfluxobs")
    cf = importlib.import_module("igm.processes.data_assimilation.cost_terms.cost_divfluxfcz")
    out = {}
    for tag, dtype in [("f64", torch.float64), ("f32", torch.float32)]:
        rng = np.random.default_rng(17)
        ny, nx, dx = 19, 27, 100.0
        g = glacier(ny, nx, dx, 13, dtype)
        f = lambda a: torch.as_tensor(np.asarray(a), dtype=dtype)  # noqa: E731
        thk = g["thk"] + f(np.abs(rng.normal(0, 5, (ny, nx))))
        usurf = g["usurf"]
        u, v = f(rng.normal(15, 20, (ny, nx))), f(rng.normal(0, 20, (ny, nx)))
        for m in ("upwind", "centered"):
            out[f"{tag}_div_{m}"] = cd.compute_divflux(u, v, thk, dx, dx, method=m)
        icemaskobs = f((g["thk"].numpy() > 0).astype(np.float64))
        dobs = f(rng.normal(0, 2, (ny, nx)))
        dobs[rng.uniform(size=(ny, nx)) < 0.3] = float("nan")
        out.update({f"{tag}_{k}": x for k, x in dict(u=u, v=v, thk=thk, usurf=usurf, icemaskobs=icemaskobs,
                                                     divfluxobs=dobs, dx=np.asarray(dx)).items()})
        with open(os.path.join(IGM, "conf", "processes", "data_assimilation.yaml")) as fh:
            da = yaml.safe_load(fh)["data_assimilation"]
        for method in ("upwind", "centered"):
            for kind, fzs in (("obs", False), ("obs", True), ("fcz", False), ("fcz", True)):
                cfg = load_cfg()
                da["divflux"]["method"] = method
                da["divflux"]["force_zero_sum"] = fzs
                da["fitting"]["divfluxobs_std"] = 0.7
                da["regularization"]["divflux"] = 3.0
                cfg.processes.data_assimilation = ns(da)
                key = f"{tag}_{method}_{kind}{'_zs' if fzs else ''}"

                def state(grad):
                    w = (lambda t: t.clone().requires_grad_(True)) if grad else (lambda t: t.clone())
                    return types.SimpleNamespace(ubar=w(u), vbar=w(v), thk=w(thk), usurf=usurf, dx=dx,
                                                 divfluxobs=dobs, icemaskobs=icemaskobs)
                if kind == "obs":
                    st = state(True)
                    c = co.cost_divfluxobs(cfg, st, 0)
                else:
                    st0 = state(False)
                    cf.cost_divfluxfcz(cfg, st0, 0)
                    st = state(True)
                    st.res = st0.res
                    c = cf.cost_divfluxfcz(cfg, st, 1)
                    out[f"{key}_slope"] = np.asarray(st0.res.slope)
                    out[f"{key}_intercept"] = np.asarray(st0.res.intercept)
                gu, gv, gh = torch.autograd.grad(c, [st.ubar, st.vbar, st.thk])
                out.update({f"{key}_cost": c, f"{key}_g_u": gu, f"{key}_g_v": gv, f"{key}_g_h": gh})
    save("divflux", out)


def assim_control_cases():
    """The cost terms of the other controls, executed from the reference's
    files: regu_slidingco (isotropic, and anisotropic with
    smooth_anisotropy_factor_sl), regu_arrhenius, misfit_usurf, the
    slidingco / arrhenius positivity penalties of total_cost.py:45-54, and
    regu_thk's dependence on usurf (to_regularize "topg"), with torch
    autograd gradients w.r.t. the fields."""
    dau = importlib.import_module("igm.processes.data_assimilation.utils")
    rs = importlib.import_module("igm.processes.data_assimilation.cost_terms.regu_slidingco")
    ra = importlib.import_module("igm.processes.data_assimilation.cost_terms.regu_arrhenius")
    mu = importlib.import_module("igm.processes.data_assimilation.cost_terms.misfit_usurf")
    rt = importlib.import_module("igm.processes.data_assimilation.cost_terms.regu_thk")
    out = {}
    for tag, dtype in [("f64", torch.float64), ("f32", torch.float32)]:
        rng = np.random.default_rng(23)
        ny, nx, dx = 21, 29, 100.0
        g = glacier(ny, nx, dx, 14, dtype)
        f = lambda a: torch.as_tensor(np.asarray(a), dtype=dtype)  # noqa: E731
        thk = g["thk"] + f(np.abs(rng.normal(0, 5, (ny, nx))))
        usurf = g["usurf"] + f(rng.normal(0, 2, (ny, nx)))
        sl = f(np.abs(rng.normal(0.05, 0.03, (ny, nx))))
        sl[rng.uniform(size=(ny, nx)) < 0.05] *= -1.0  # a few negative values: the penalty is active
        ar = f(rng.normal(60, 30, (ny, nx)))
        ar[rng.uniform(size=(ny, nx)) < 0.05] = 0.5   # below 1: the arrhenius penalty is active
        usobs = usurf + f(rng.normal(0, 3, (ny, nx)))
        icemaskobs = f((g["thk"].numpy() > 0).astype(np.float64))
        uvs, vvs = f(rng.normal(20, 15, (ny, nx))), f(rng.normal(-5, 15, (ny, nx)))
        with open(os.path.join(IGM, "conf", "processes", "data_assimilation.yaml")) as fh:
            da = yaml.safe_load(fh)["data_assimilation"]
        da.setdefault("cook", {"infer_params": False})
        out.update({f"{tag}_{k}": x for k, x in dict(thk=thk, usurf=usurf, slidingco=sl, arrhenius=ar, usurfobs=usobs,
                                                     icemaskobs=icemaskobs, uvs=uvs, vvs=vvs,
                                                     dx=np.asarray(dx)).items()})
        for aniso_sl in (1.0, 0.3):
            cfg = load_cfg()
            da["regularization"]["smooth_anisotropy_factor_sl"] = aniso_sl
            da["regularization"]["slidingco"] = 7.0
            da["regularization"]["arrhenius"] = 2.0
            da["fitting"]["usurfobs_std"] = 1.5
            cfg.processes.data_assimilation = ns(da)
            st = types.SimpleNamespace(thk=thk, usurf=usurf.clone().requires_grad_(True),
                                       slidingco=sl.clone().requires_grad_(True),
                                       arrhenius=ar.clone().requires_grad_(True), usurfobs=usobs,
                                       icemaskobs=icemaskobs, icemask=icemaskobs, uvelsurf=uvs, vvelsurf=vvs, dx=dx)
            dau.compute_flow_direction_for_anisotropic_smoothing(st)
            st.flowdirx, st.flowdiry = f(np.asarray(st.flowdirx)), f(np.asarray(st.flowdiry))
            key = f"{tag}_sl{'aniso' if aniso_sl != 1.0 else 'iso'}"
            c = rs.regu_slidingco(cfg, st)
            (gs,) = torch.autograd.grad(c, [st.slidingco])
            out.update({f"{key}_regu_slidingco": c, f"{key}_g_slidingco": gs, f"{key}_flowdirx": st.flowdirx,
                        f"{key}_flowdiry": st.flowdiry})
        c = ra.regu_arrhenius(cfg, st)
        (ga,) = torch.autograd.grad(c, [st.arrhenius])
        cp_s = 10 ** 10 * torch.mean(torch.where(st.slidingco >= 0, torch.zeros_like(st.slidingco),
                                                 st.slidingco ** 2))
        cp_a = 10 ** 10 * torch.mean(torch.where(st.arrhenius >= 1, torch.zeros_like(st.arrhenius),
                                                 st.arrhenius ** 2))
        (gps,) = torch.autograd.grad(cp_s, [st.slidingco])
        (gpa,) = torch.autograd.grad(cp_a, [st.arrhenius])
        cu = mu.misfit_usurf(cfg, st)
        (gu,) = torch.autograd.grad(cu, [st.usurf])
        # regu_thk (topg, isotropic) depends on usurf through the bed usurf - thk
        da["regularization"]["smooth_anisotropy_factor"] = 1.0
        cfg.processes.data_assimilation = ns(da)
        crt = rt.regu_thk(cfg, st)
        (gru,) = torch.autograd.grad(crt, [st.usurf])
        out.update({f"{tag}_regu_arrhenius": c, f"{tag}_g_arrhenius": ga, f"{tag}_pen_slidingco": cp_s,
                    f"{tag}_g_pen_slidingco": gps, f"{tag}_pen_arrhenius": cp_a, f"{tag}_g_pen_arrhenius": gpa,
                    f"{tag}_misfit_usurf": cu, f"{tag}_g_usurf": gu, f"{tag}_regu_thk_topg": crt,
                    f"{tag}_g_usurf_regu_thk": gru})
        # include_low_speed_term of misfit_velsurf (a global-norm term)
        uo, vo = f(rng.normal(20, 15, (ny, nx))), f(rng.normal(-5, 15, (ny, nx)))
        uo[rng.uniform(size=(ny, nx)) < 0.2] = float("nan")
        vo[rng.uniform(size=(ny, nx)) < 0.1] = float("nan")
        mv = importlib.import_module("igm.processes.data_assimilation.cost_terms.misfit_velsurf")
        for thr, flag in ((0.0, False), (0.0, True), (15.0, True)):
            da["fitting"]["include_low_speed_term"] = flag
            da["fitting"]["velsurfobs_thr"] = thr
            cfg.processes.data_assimilation = ns(da)
            stv = types.SimpleNamespace(uvelsurf=uvs.clone().requires_grad_(True),
                                        vvelsurf=vvs.clone().requires_grad_(True), uvelsurfobs=uo, vvelsurfobs=vo)
            c = mv.misfit_velsurf(cfg, stv)
            gu_, gv_ = torch.autograd.grad(c, [stv.uvelsurf, stv.vvelsurf])
            key = f"{tag}_vel_thr{int(thr)}_{'low' if flag else 'plain'}"
            out.update({f"{key}_cost": c, f"{key}_g_u": gu_, f"{key}_g_v": gv_})
        out.update({f"{tag}_uobs": uo, f"{tag}_vobs": vo})
        da["fitting"]["include_low_speed_term"] = False
        da["fitting"]["velsurfobs_thr"] = 0.0
        # fix_opti_normalization_issue: the regularisations as means
        da["optimization"]["fix_opti_normalization_issue"] = True
        for aniso in (1.0, 0.2):
            da["regularization"]["smooth_anisotropy_factor"] = aniso
            da["regularization"]["smooth_anisotropy_factor_sl"] = 0.3 if aniso != 1.0 else 1.0
            cfg.processes.data_assimilation = ns(da)
            key = f"{tag}_norm_{'aniso' if aniso != 1.0 else 'iso'}"
            th = thk.clone().requires_grad_(True)
            st2 = types.SimpleNamespace(thk=th, usurf=usurf, slidingco=sl.clone().requires_grad_(True),
                                        arrhenius=ar.clone().requires_grad_(True), icemaskobs=icemaskobs,
                                        icemask=icemaskobs, dx=dx, flowdirx=st.flowdirx, flowdiry=st.flowdiry)
            c_t = rt.regu_thk(cfg, st2)
            (g_t,) = torch.autograd.grad(c_t, [th])
            c_s = rs.regu_slidingco(cfg, st2)
            (g_s,) = torch.autograd.grad(c_s, [st2.slidingco])
            c_a = ra.regu_arrhenius(cfg, st2)
            (g_a,) = torch.autograd.grad(c_a, [st2.arrhenius])
            out.update({f"{key}_regu_thk": c_t, f"{key}_g_thk": g_t, f"{key}_regu_slidingco": c_s,
                        f"{key}_g_slidingco": g_s, f"{key}_regu_arrhenius": c_a, f"{key}_g_arrhenius": g_a})
        da["optimization"]["fix_opti_normalization_issue"] = False
        # sole_mask: the regularisations restricted to the observed ice (a mask with values 0, 1, 2)
        im3 = icemaskobs.clone()
        im3[(rng.uniform(size=(ny, nx)) < 0.15) & (g["thk"].numpy() > 0)] = 2.0
        da["optimization"]["sole_mask"] = True
        for aniso in (1.0, 0.2):
            da["regularization"]["smooth_anisotropy_factor"] = aniso
            da["regularization"]["smooth_anisotropy_factor_sl"] = 0.3 if aniso != 1.0 else 1.0
            cfg.processes.data_assimilation = ns(da)
            key = f"{tag}_sole_{'aniso' if aniso != 1.0 else 'iso'}"
            th = thk.clone().requires_grad_(True)
            st3 = types.SimpleNamespace(thk=th, usurf=usurf, slidingco=sl.clone().requires_grad_(True),
                                        arrhenius=ar.clone().requires_grad_(True), icemaskobs=im3,
                                        icemask=icemaskobs, dx=dx, flowdirx=st.flowdirx, flowdiry=st.flowdiry)
            c_t = rt.regu_thk(cfg, st3)
            (g_t,) = torch.autograd.grad(c_t, [th])
            c_s = rs.regu_slidingco(cfg, st3)
            (g_s,) = torch.autograd.grad(c_s, [st3.slidingco])
            c_a = ra.regu_arrhenius(cfg, st3)
            (g_a,) = torch.autograd.grad(c_a, [st3.arrhenius])
            out.update({f"{key}_regu_thk": c_t, f"{key}_g_thk": g_t, f"{key}_regu_slidingco": c_s,
                        f"{key}_g_slidingco": g_s, f"{key}_regu_arrhenius": c_a, f"{key}_g_arrhenius": g_a})
        out[f"{tag}_icemaskobs3"] = im3
        da["optimization"]["sole_mask"] = False
        da["regularization"]["smooth_anisotropy_factor"] = 0.2
    save("assim_controls", out)


def save(name, d):
    arrs = {}
    for k, v in d.items():
        if isinstance(v, torch.Tensor):
            v = v.detach().cpu().numpy()
        arrs[k] = np.asarray(v)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **arrs)
    print(f"wrote {path} ({os.path.getsize(path)} B)")


if __name__ == "__main__" and len(sys.argv) > 2:  # only the named cases: make_golden.py REF_ROOT case ...
    torch.set_num_threads(1)
    for name in sys.argv[2:]:
        globals()[name]()
elif __name__ == "__main__":
    torch.set_num_threads(1)
    vert_cases()
    energy_case("small_f64", 13, 11, 4, 100.0, 1, torch.float64, c_neg=True)
    energy_case("small_f32", 13, 11, 4, 100.0, 1, torch.float32, c_neg=True)
    energy_case("nz2_f64", 9, 12, 2, 50.0, 2, torch.float64)
    energy_case("mid_f32", 40, 30, 10, 100.0, 3, torch.float32)
    energy_case("mid_f64", 40, 30, 10, 100.0, 3, torch.float64, spacing=1.0)
    energy_case("nz16_f64", 21, 35, 16, 25.0, 4, torch.float64)
    solver_case("f64", 20, 16, 5, 100.0, 5, torch.float64, nbitmax=40, n_solves=3)
    solver_case("f32", 20, 16, 5, 100.0, 5, torch.float32, nbitmax=40, n_solves=2)
    transport_cases()
    time_case()
    emulator_case()
    vert_flow_cases()
    divflux_cases()
    assim_control_cases()
    keras_h5_cases()
    assim_cases()
