"""ctypes binding of libigmb200.so (the C ABI declared in include/igm_b200.h).

The library is the only compute path: if it cannot be loaded, every call
raises.  Torch tensors are passed as raw device pointers (``data_ptr()``)
together with the current CUDA stream.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libigmb200.so")

IGM_MAX_NZ = 64
IGM_F32, IGM_F64 = 0, 1
SLOPE = {"godunov": 0, "minmod": 1, "superbee": 2}

STATUS = {
    0: "IGM_OK", 1: "IGM_ERR_BAD_SHAPE", 2: "IGM_ERR_BAD_ARGUMENT", 3: "IGM_ERR_NAN_DETECTED",
    4: "IGM_ERR_NOT_CONVERGED", 5: "IGM_ERR_CUDA", 6: "IGM_ERR_UNSUPPORTED", 7: "IGM_ERR_WORKSPACE",
}


class IgmError(RuntimeError):
    def __init__(self, status: int, detail: str):
        super().__init__(f"{STATUS.get(status, status)}: {detail}")
        self.status = status


class Physics(C.Structure):
    _fields_ = [("exp_glen", C.c_double), ("exp_weertman", C.c_double), ("regu_glen", C.c_double),
                ("regu_weertman", C.c_double), ("thr_ice_thk", C.c_double), ("min_sr", C.c_double),
                ("max_sr", C.c_double), ("ice_density", C.c_double), ("gravity_cst", C.c_double),
                ("force_negative_gravitational_energy", C.c_int32), ("reserved", C.c_int32)]


class Grid(C.Structure):
    _fields_ = [("batch", C.c_int32), ("nz", C.c_int32), ("ny", C.c_int32), ("nx", C.c_int32),
                ("dx", C.c_double), ("dzeta", C.c_double * IGM_MAX_NZ)]


class Fields(C.Structure):
    _fields_ = [("thk", C.c_void_p), ("usurf", C.c_void_p), ("arrhenius", C.c_void_p), ("slidingco", C.c_void_p)]


class Adam(C.Structure):
    _fields_ = [("lr", C.c_double), ("beta_1", C.c_double), ("beta_2", C.c_double), ("epsilon", C.c_double)]


class DivfluxCostParams(C.Structure):
    """igm_divflux_cost_params."""
    _fields_ = [("kind", C.c_int32), ("method", C.c_int32), ("force_zero_sum", C.c_int32), ("reserved", C.c_int32),
                ("divfluxobs_std", C.c_double), ("regu_divflux", C.c_double), ("slope", C.c_double),
                ("intercept", C.c_double)]


class AssimParams(C.Structure):
    _fields_ = [("velsurfobs_std", C.c_double), ("velsurfobs_thr", C.c_double), ("thkobs_std", C.c_double),
                ("regu_thk", C.c_double), ("gamma", C.c_double), ("aniso_factor", C.c_double), ("n_vel", C.c_double),
                ("n_thk", C.c_double), ("penalty", C.c_int32), ("icemask_cost", C.c_int32),
                ("regularize_thk", C.c_int32), ("mask_velsurf", C.c_int32), ("usurfobs_std", C.c_double),
                ("n_usurf", C.c_double), ("usurf_cost", C.c_int32), ("no_thk_control", C.c_int32),
                ("fix_normalization", C.c_int32), ("sole_mask", C.c_int32)]


class AssimControlParams(C.Structure):
    """igm_assim_control_params."""
    _fields_ = [("mode", C.c_int32), ("transform", C.c_int32), ("mask", C.c_int32), ("reproject", C.c_int32),
                ("reproject_mask", C.c_int32), ("reserved", C.c_int32), ("scale", C.c_double),
                ("lower", C.c_double)]


class EarlyStop(C.Structure):
    _fields_ = [("relative_min_delta", C.c_double), ("patience", C.c_int32), ("enabled", C.c_int32)]


class SolverCtl(C.Structure):
    _fields_ = [("iter", C.c_int32), ("stopped", C.c_int32), ("status", C.c_int32), ("wait", C.c_int32),
                ("adam_t0", C.c_int64), ("best", C.c_double), ("last_cost", C.c_double),
                ("terms", C.c_double * 3)]


P = C.c_void_p
I = C.c_int
D = C.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "igm_status_string": (C.c_char_p, [I]),
    "igm_last_error": (C.c_char_p, []),
    "igm_version": (I, []),
    "igm_launch_count": (C.c_longlong, []),
    "igm_workspace_size": (C.c_size_t, [C.POINTER(Grid)]),
    "igm_energy": (I, [I, C.POINTER(Grid), C.POINTER(Physics), C.POINTER(Fields), P, P, P, P, D, P, P,
                       C.c_size_t, P]),
    "igm_energy_noalloc": (I, [I, C.POINTER(Grid), C.POINTER(Physics), C.POINTER(Fields), P, P, P, P, D, P, P]),
    "igm_solver_begin": (I, [P, C.c_int64, P]),
    "igm_solver_iterate": (I, [I, C.POINTER(Grid), C.POINTER(Physics), C.POINTER(Fields), P, P, P, P, P, P, P, P,
                               C.POINTER(Adam), C.POINTER(EarlyStop), I, I, P, P, P, C.c_size_t, P]),
    "igm_velocity_reduce": (I, [I, I, I, I, I, P, P, P, I, C.POINTER(C.c_double), P, P, P, P, P, P, P, P]),
    "igm_transport_step": (I, [I, I, I, D, P, P, P, P, P, P, P, P, P, D, P, I, D, D, P]),
    "igm_thk_surfaces": (I, [I, I, P, P, P, P, D, D, P]),
    "igm_vertical_velocity": (I, [I, I, I, I, D, P, P, P, P, P, P, P, P]),
    "igm_vertical_velocity_incompressibility": (I, [I, I, I, I, D, P, P, P, P, P, P, P, P]),
    "igm_smb_simple": (I, [I, I, P, P, P, D, D, D, D, P]),
    "igm_absmax2": (I, [I, I, P, P, P, P]),
    "igm_force_max_velbar": (I, [I, C.c_size_t, P, P, D, P]),
    "igm_cfl_dt": (I, [P, P, D, D, D, P]),
    "igm_conv3x3": (I, [I, I, I, I, I, P, P, P, P, P, P, I, C.c_float, P, P]),
    "igm_conv3x3_wgrad": (I, [I, I, I, I, P, P, P, I, P, P]),
    "igm_conv1x1_wgrad": (I, [I, I, I, P, P, P, I, P, P]),
    "igm_conv3x3_backward": (I, [I, I, I, P, P, P, P, P, P, I, C.c_float, P, P, P, P, P, P]),
    "igm_conv3x3_stack": (I, [I, I, I, I, P, P, P, P, P, I, C.c_float, P, P]),
    "igm_conv3x3_stack_flags_len": (C.c_size_t, [I, I, I, I]),
    "igm_conv_sm_count": (I, []),
    "igm_conv3x3_wgrad_partial_len": (C.c_size_t, [I]),
    "igm_cnn_param_count": (C.c_size_t, [I, I, I]),
    "igm_cnn_param_offset": (C.c_size_t, [I, I, I, I, I]),
    "igm_cnn_pack_weights": (I, [I, I, I, P, P, P, P]),
    "igm_cnn_input": (I, [I, I, I, I, I, P, P, P, P, D, P, P, P, P, P, P, P, P, P]),
    "igm_cnn_layer1_forward": (I, [I, I, I, I, P, P, P, P, D, P, P, P, C.c_float, P, P]),
    "igm_cnn_layer1_wgrad": (I, [I, I, I, I, P, P, P, P, D, P, P, P, I, P]),
    "igm_cnn_head_forward": (I, [I, I, I, I, P, P, P, C.c_float, P, P, P, P]),
    "igm_cnn_head_partial_len": (C.c_size_t, [I]),
    "igm_cnn_head_backward": (I, [I, I, I, I, P, P, P, P, C.c_float, C.c_float, P, P, I, P]),
    "igm_reduce_partials": (I, [P, I, I, I, P, I, P]),
    "igm_cnn_wgrad_finish": (I, [P, I, I, I, P, P]),
    "igm_cnn_wgrad_finish_split": (I, [P, I, I, P, P]),
    "igm_cnn_head_backward_tc": (I, [I, I, I, I, P, P, P, P, C.c_float, C.c_float, P, P, P, I, P]),
    "igm_cnn_head_wgrad_finish": (I, [P, I, I, P, P]),
    "igm_cnn_input_gradient": (I, [I, I, I, I, I, P, P, P, P, P]),
    "igm_assim_cost_grad": (I, [I, I, I, D] + [P] * 12 + [P, P, P, P, P, P, I, P, P]),
    "igm_assim_field_regu": (I, [I, I, I, D, P, P, P, D, D, I, D, I, P, I, P, P, I, P, P]),
    "igm_assim_low_speed": (I, [I, I, I, P, P, P, P, P, P, P, I, P, P]),
    "igm_assim_flow_direction": (I, [I, I, I, P, P, P, P, P, P]),
    "igm_divflux_upwind": (I, [I, I, I, D, P, P, P, P, P]),
    "igm_assim_control": (I, [I, C.c_size_t, P, P, P, P, P, P, P, P, P, P]),
    "igm_assim_stats": (I, [I, I, I, D] + [P] * 11 + [P, I, P, P]),
    "igm_divflux": (I, [I, I, I, I, D, P, P, P, P, P]),
    "igm_assim_divflux_cost_grad": (I, [I, I, I, D, I, P] + [P] * 8 + [P, P, P, P, P, P, I, P, P]),
    "igm_assim_divflux_partials_len": (C.c_size_t, [I]),
    "igm_adam_clipnorm": (I, [I, P, P, P, P, P, P, D, D, D, D, D, C.c_int64, P]),
    "igm_adam_norms_len": (C.c_size_t, [I, P]),
}

_lib = None


def lib():
    """Load (once) and return the library; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libigmb200.so not found at {LIB_PATH}: build it with `python -m igm_b200.build` "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = ""):
    if rc != 0:
        detail = lib().igm_last_error().decode()
        raise IgmError(rc, f"{what}: {detail}" if what else detail)


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None passes NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def stream_ptr(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def dtype_code(dt) -> int:
    import torch
    if dt == torch.float32:
        return IGM_F32
    if dt == torch.float64:
        return IGM_F64
    raise ValueError(f"unsupported dtype {dt} (float32 or float64)")


def make_grid(batch, nz, ny, nx, dx, dzeta) -> Grid:
    g = Grid()
    g.batch, g.nz, g.ny, g.nx, g.dx = int(batch), int(nz), int(ny), int(nx), float(dx)
    dz = np.asarray(dzeta, dtype=np.float64).reshape(-1)
    if nz > IGM_MAX_NZ:
        raise ValueError(f"nz={nz} > {IGM_MAX_NZ}")
    for i, v in enumerate(dz[:IGM_MAX_NZ]):
        g.dzeta[i] = float(v)
    return g


def make_physics(p=None, **over) -> Physics:
    """From a dict/namespace with the keys of cfg.processes.iceflow.physics."""
    d = dict(exp_glen=3.0, exp_weertman=3.0, regu_glen=1e-5, regu_weertman=1e-10, thr_ice_thk=0.1,
             min_sr=1e-20, max_sr=1e20, ice_density=910.0, gravity_cst=9.81,
             force_negative_gravitational_energy=False)
    if p is not None:
        src = p if isinstance(p, dict) else vars(p)
        for k in d:
            if k in src:
                d[k] = src[k]
    d.update(over)
    ph = Physics()
    for k, v in d.items():
        setattr(ph, k, int(bool(v)) if k == "force_negative_gravitational_energy" else float(v))
    return ph
