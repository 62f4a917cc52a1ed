"""The C ABI: the library loads on a CPU-only host and exports every entry
point include/igm_b200.h declares; argument validation runs without a GPU."""

import ctypes as C
import os
import re

import pytest

from igm_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "igm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(igm_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from igm_b200.build import build
    build()
    return L.lib()


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/igm_b200.h but not exported"


def test_bindings_cover_header():
    assert set(declared_symbols()) == set(L.SIGNATURES), "ctypes signatures out of sync with the header"


def test_status_strings(lib):
    assert lib.igm_status_string(0) == b"IGM_OK"
    assert lib.igm_status_string(3) == b"IGM_ERR_NAN_DETECTED"
    assert lib.igm_version() >= 100


def test_struct_sizes_match_c_layout():
    assert C.sizeof(L.SolverCtl) == 64
    assert C.sizeof(L.Grid) == 4 * 4 + 8 + 8 * L.IGM_MAX_NZ


def test_argument_validation_without_gpu(lib):
    g = L.make_grid(1, 0, 10, 10, 100.0, [])
    assert lib.igm_workspace_size(C.byref(g)) == 0
    g = L.make_grid(1, 5, 10, 10, 100.0, [0.25] * 4)
    assert lib.igm_workspace_size(C.byref(g)) > 0
    ph = L.make_physics()
    f = L.Fields()
    rc = lib.igm_energy(0, C.byref(g), C.byref(ph), C.byref(f), None, None, None, None, 1.0, None, None, 0, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    rc = lib.igm_transport_step(0, 5, 5, 100.0, 16, 32, 48, 64, 80, None, 96, None, None, 1.0, None, 9, 0.91, 0.0, None)
    assert rc == 2 and b"slope_type" in lib.igm_last_error()


def test_vertical_velocity_validation_without_gpu(lib):
    lv = (C.c_double * 2)(0.0, 1.0)
    rc = lib.igm_vertical_velocity(0, 1, 5, 5, 100.0, 16, 32, 48, 64, lv, lv, 80, None)
    assert rc == 1 and b"nz, ny, nx >= 2" in lib.igm_last_error()
    rc = lib.igm_vertical_velocity(0, 2, 5, 5, 100.0, 16, None, 48, 64, lv, lv, 80, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    rc = lib.igm_vertical_velocity(0, 2, 5, 5, 0.0, 16, 32, 48, 64, lv, lv, 80, None)
    assert rc == 2 and b"dx" in lib.igm_last_error()


def test_vertical_velocity_incompressibility_validation_without_gpu(lib):
    lv = (C.c_double * 2)(0.0, 1.0)
    rc = lib.igm_vertical_velocity_incompressibility(0, 1, 5, 5, 100.0, 16, 32, 48, 64, lv, lv, 80, None)
    assert rc == 1 and b"nz, ny, nx >= 2" in lib.igm_last_error()
    rc = lib.igm_vertical_velocity_incompressibility(7, 2, 5, 5, 100.0, 16, 32, 48, 64, lv, lv, 80, None)
    assert rc == 2 and b"dtype" in lib.igm_last_error()


def test_assimilation_entries_validate_without_gpu(lib):
    """The data-assimilation entry points reject bad arguments before any
    launch, with the status and message of the C ABI."""
    p = L.AssimParams()
    p.velsurfobs_std, p.thkobs_std, p.regu_thk, p.aniso_factor, p.n_vel, p.n_thk = 1.0, 3.0, 10.0, 1.0, 1.0, 1.0
    args = [16] * 11  # thk .. flowdiry: placeholders, never dereferenced on these paths
    rc = lib.igm_assim_cost_grad(0, 1, 5, 100.0, *args, None, C.byref(p), 16, 16, 16, None, 16, 4, 16, None)
    assert rc == 1 and b"bad shape" in lib.igm_last_error()
    rc = lib.igm_assim_cost_grad(0, 5, 5, 100.0, None, *args[1:], None, C.byref(p), 16, 16, 16, None, 16, 4, 16, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    p.aniso_factor = 0.2
    a2 = args[:9] + [None, None]
    rc = lib.igm_assim_cost_grad(0, 5, 5, 100.0, *a2, None, C.byref(p), 16, 16, 16, None, 16, 4, 16, None)
    assert rc == 2 and b"flowdirx" in lib.igm_last_error()
    p.aniso_factor, p.usurf_cost, p.usurfobs_std = 1.0, 1, 2.0
    rc = lib.igm_assim_cost_grad(0, 5, 5, 100.0, *args, None, C.byref(p), 16, 16, 16, None, 16, 4, 16, None)
    assert rc == 2 and b"misfit_usurf" in lib.igm_last_error()
    rc = lib.igm_assim_field_regu(0, 5, 5, 100.0, 16, None, None, 1.0, 1.0, 1, 0.0, 0, None, 1, 16, 16, 4, 16, None)
    assert rc == 2 and b"sole_mask" in lib.igm_last_error()
    rc = lib.igm_assim_field_regu(0, 5, 5, 100.0, 16, None, None, 1.0, 0.3, 1, 0.0, 0, None, 0, 16, 16, 4, 16, None)
    assert rc == 2 and b"flowdirx" in lib.igm_last_error()
    cp = L.AssimControlParams()
    cp.mode, cp.scale = 4, 1.0
    rc = lib.igm_assim_control(0, 25, C.byref(cp), 16, 16, None, 16, 16, 16, 16, 16, None)
    assert rc == 2 and b"bad mode" in lib.igm_last_error()
    cp.mode, cp.mask = 1, 1
    rc = lib.igm_assim_control(0, 25, C.byref(cp), 16, None, None, 16, 16, 16, 16, 16, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    rc = lib.igm_divflux(0, 5, 5, 5, 100.0, 16, 16, 16, 16, None)
    assert rc == 2 and b"unknown method" in lib.igm_last_error()
    dp = L.DivfluxCostParams()
    dp.kind, dp.divfluxobs_std = 0, 1.0
    w = (C.c_double * 1)(1.0)
    rc = lib.igm_assim_divflux_cost_grad(0, 5, 5, 100.0, 1, w, 16, 16, 16, 16, None, None, 16, None, C.byref(dp), 16,
                                         16, 16, 16, 16, 4, 16, None)
    assert rc == 2 and b"kind 0 needs divfluxobs" in lib.igm_last_error()
    rc = lib.igm_assim_stats(0, 5, 5, 100.0, None, None, None, None, None, None, 16, None, None, None, None, 16, 4,
                             16, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    rc = lib.igm_assim_low_speed(0, 5, 5, 16, 16, None, 16, 16, 16, 16, 4, 16, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()


def test_emulator_entries_validate_without_gpu(lib):
    sc = (C.c_double * 5)(*[1.0] * 5)
    rc = lib.igm_cnn_input_gradient(1, 8, 8, 5, 6, 16, 16, sc, 16, None)
    assert rc == 1 and b"bad shape" in lib.igm_last_error()
    rc = lib.igm_cnn_head_backward_tc(1, 8, 8, 10, 16, 16, 16, 16, 1.0, 0.01, 16, None, 16, 4, None)
    assert rc == 2 and b"NULL" in lib.igm_last_error()
    offs = (C.c_size_t * 3)(0, 5000, 5001)
    assert lib.igm_adam_norms_len(2, offs) == 2 + 2 + 1  # the norms, then 4096-element chunks per variable
    assert lib.igm_adam_norms_len(0, offs) == 0
    empty = (C.c_size_t * 3)(0, 10, 10)
    rc = lib.igm_adam_clipnorm(2, empty, 16, 16, 16, 16, 16, 1e-3, 0.9, 0.999, 1e-7, 1.0, 1, None)
    assert rc == 2 and b"empty variable" in lib.igm_last_error()
