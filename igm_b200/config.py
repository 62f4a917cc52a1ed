"""Default parameters under the reference's key names.

The processes read ``cfg.processes.<name>.<key>`` by attribute access, so an
OmegaConf DictConfig composed by the reference's Hydra setup works as is;
``default_cfg()`` builds an equivalent plain object for callers without
Hydra.  Keys and defaults follow igm/conf/processes/iceflow.yaml,
thk.yaml, time.yaml, smb_simple.yaml, vert_flow.yaml,
data_assimilation.yaml and pretraining.yaml.  Keys this implementation adds are
marked "(igm_b200)".
"""

from __future__ import annotations

import copy
from types import SimpleNamespace

DEFAULTS = {
    "iceflow": {
        "method": "emulated",
        "force_max_velbar": 0.0,
        "physics": {
            "energy_components": ["shear", "sliding_weertman", "gravity"],
            "sliding_law": "",
            "gravity_cst": 9.81,
            "ice_density": 910.0,
            "init_slidingco": 0.0464,
            "init_arrhenius": 78.0,
            "enhancement_factor": 1.0,
            "exp_glen": 3.0,
            "exp_weertman": 3.0,
            "regu_glen": 1.0e-5,
            "regu_weertman": 1.0e-10,
            "dim_arrhenius": 2,
            "thr_ice_thk": 0.1,
            "min_sr": 1.0e-20,
            "max_sr": 1.0e20,
            "force_negative_gravitational_energy": False,
            "cf_eswn": [],
        },
        "numerics": {"Nz": 10, "vert_spacing": 4.0, "staggered_grid": 1, "vert_basis": "Lagrange"},
        "solver": {"step_size": 1.0, "nbitmax": 100, "stop_if_no_decrease": True, "optimizer": "Adam",
                   "lbfgs": False, "save_cost": "", "plot_sol": False,
                   # (igm_b200) EarlyStopping(2e-4, 10) of solve.py:36,112; False runs nbitmax iterations
                   "early_stopping": True},
        "emulator": {
            "fieldin": ["thk", "usurf", "arrhenius", "slidingco", "dX"],
            "retrain_freq": 10,
            "lr": 2.0e-5,
            "lr_init": 1.0e-4,
            "lr_decay": 0.95,
            "warm_up_it": -10000000000.0,
            "nbit_init": 1,
            "nbit": 1,
            "framesizemax": 750,
            "split_patch_method": "sequential",
            "pretrained": True,
            "name": "",
            "save_model": False,
            "exclude_borders": 0,
            "optimizer": "Adam",
            "optimizer_clipnorm": 1.0,
            "optimizer_epsilon": 1.0e-7,
            "save_cost": "",
            "output_directory": "",
            "plot_sol": False,
            "pertubate": False,
            # (igm_b200) fixed input scales per fieldin channel (1.0 = raw, as the reference)
            "input_scales": [1.0, 1.0, 1.0, 1.0, 1.0],
            # (igm_b200) weight seed for networks built from scratch
            "seed": 0,
            # (igm_b200) fixed factor multiplying the head's output (m/a); 1.0 = raw, as the reference
            "output_scale": 1.0,
            "network": {
                "architecture": "cnn",
                "multiple_window_size": 0,
                "activation": "LeakyReLU",
                "nb_layers": 16,
                "nb_blocks": 4,
                "nb_out_filter": 32,
                "conv_ker_size": 3,
                "dropout_rate": 0,
                "weight_initialization": "glorot_uniform",
                "cnn3d_for_vertical": False,
            },
        },
        # (igm_b200) emulator fallback / judge: every `every` updates the plain
        # solver is run from the emulated velocities; when the emulated energy
        # exceeds the solved one by more than `margin` (relative), the solved
        # velocities replace the emulated ones: until the next check, each update
        # then a warm-started solve ("takeover"), or for that update alone
        # ("step").  every <= 0 disables it.
        "fallback": {"every": 0, "margin": 0.02, "nbitmax": 100, "mode": "takeover"},
    },
    "thk": {"slope_type": "superbee", "ratio_density": 0.910, "default_sealevel": 0.0},
    "vert_flow": {"version": 2, "method": "kinematic"},
    "time": {"start": 2000.0, "end": 2100.0, "save": 10.0, "cfl": 0.3, "step_max": 1.0},
    "smb_simple": {"update_freq": 1.0, "file": "param.txt", "array": []},
}

# Processes whose configuration is present only when a run uses them (the
# reference composes cfg.processes from the selected processes, and the
# emulator's pertubate option tests for data_assimilation's presence):
# default_cfg adds them when the overrides or ``with_processes`` name them.
OPTIONAL = {
    "data_assimilation": {
        "control_list": ["thk"],
        "cost_list": ["velsurf", "thk", "icemask"],
        "optimization": {"nbitmin": 50, "nbitmax": 500, "step_size": 1.0, "step_size_decay": 0.9,
                         "init_zero_thk": False, "sole_mask": False, "retrain_iceflow_model": True,
                         "fix_opti_normalization_issue": False, "method": "ADAM",
                         "obstacle_constraint": ["reproject", "penalty"], "optimizer_clipnorm": 1.0e7,
                         "optimizer_epsilon": 1.0e-7, "pertubate": False},
        "regularization": {"thk": 10.0, "slidingco": 1.0, "arrhenius": 10.0, "divflux": 1.0,
                           "smooth_anisotropy_factor": 0.2, "smooth_anisotropy_factor_sl": 1.0,
                           "convexity_weight": 0.002, "convexity_power": 1.3, "to_regularize": "topg"},
        "fitting": {"usurfobs_std": 2.0, "velsurfobs_std": 1.0, "thkobs_std": 3.0, "divfluxobs_std": 1.0,
                    "uniformize_thkobs": True, "include_low_speed_term": False, "velsurfobs_thr": 0.0,
                    "log_slidingco": False},
        "divflux": {"method": "upwind", "force_zero_sum": False},
        "scaling": {"thk": 2.0, "usurf": 0.5, "slidingco": 0.0001, "arrhenius": 0.1},
        "output": {"freq": 50, "plot2d_live": True, "plot2d": True, "save_result_in_ncdf": "geology-optimized.nc",
                   "save_iterat_in_ncdf": True, "editor_plot2d": "vs",
                   "vars_to_save": ["usurf", "thk", "slidingco", "velsurf_mag", "velsurfobs_mag", "divflux",
                                    "icemask"]},
        "cook": {"infer_params": False, "tidewater_glacier": False, "vol_std": 1000.0},
    },
    "pretraining": {
        "data_dir": "surflib3d_shape_100", "batch_size": 1, "freq_test": 20, "train_iceflow_emulator_restart_lr": 2500,
        "epochs": 5000, "min_arrhenius": 5.0, "max_arrhenius": 151.0, "min_slidingco": 0.0,
        "max_slidingco": 20000.0, "min_coarsen": 0, "max_coarsen": 2, "soft_begining": 500,
        # (igm_b200) seed of the sampling (the reference draws unseeded)
        "seed": 0,
    },
}


class Cfg(SimpleNamespace):
    """Attribute-access config node (the subset of OmegaConf's interface the
    processes use)."""

    def get(self, key, default=None):
        return getattr(self, key, default)

    def __contains__(self, key):
        return hasattr(self, key)


def to_cfg(d):
    if isinstance(d, dict):
        return Cfg(**{k: to_cfg(v) for k, v in d.items()})
    return d


def _merge(base: dict, over: dict):
    for k, v in over.items():
        if isinstance(v, dict) and isinstance(base.get(k), dict):
            _merge(base[k], v)
        else:
            base[k] = v


def default_cfg(overrides: dict | None = None, with_processes=(), **dotted):
    """``default_cfg({"iceflow": {"method": "solved"}}, **{"iceflow.numerics.Nz": 5})``;
    the optional processes (data_assimilation) are included when ``overrides``
    or ``with_processes`` name them."""
    d = copy.deepcopy(DEFAULTS)
    for name, block in OPTIONAL.items():
        if name in with_processes or (overrides and name in overrides) or any(
                k.split(".")[0] == name for k in dotted):
            d[name] = copy.deepcopy(block)
    if overrides:
        _merge(d, overrides)
    for path, val in dotted.items():
        node = d
        keys = path.split(".")
        for k in keys[:-1]:
            node = node[k]
        node[keys[-1]] = val
    return to_cfg({"processes": d})
