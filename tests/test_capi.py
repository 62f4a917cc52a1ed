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
