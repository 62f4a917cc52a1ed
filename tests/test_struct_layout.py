"""The C ABI's parameter structs: include/igm_b200.h compiles as C99 and as
C++17, and each ctypes mirror in igm_b200._lib has the C struct's size and
field offsets (compiled with the host C compiler; no GPU needed)."""

import ctypes as C
import os
import shutil
import subprocess

import pytest

from igm_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")

PAIRS = [("igm_physics", L.Physics), ("igm_grid", L.Grid), ("igm_fields", L.Fields), ("igm_adam", L.Adam),
         ("igm_early_stop", L.EarlyStop), ("igm_solver_ctl", L.SolverCtl), ("igm_assim_params", L.AssimParams),
         ("igm_assim_control_params", L.AssimControlParams), ("igm_divflux_cost_params", L.DivfluxCostParams)]

pytestmark = pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")


@pytest.mark.parametrize("std,compiler", [("c99", "gcc"), ("c++17", "g++")])
def test_header_compiles(tmp_path, std, compiler):
    src = tmp_path / "h.c"
    src.write_text('#include "igm_b200.h"\nint main(void) { return 0; }\n')
    lang = ["-x", "c++"] if compiler == "g++" else []
    subprocess.run([compiler, *lang, f"-std={std}", "-Wall", "-Werror", "-pedantic", "-I", INC, "-c", str(src), "-o",
                    str(tmp_path / "h.o")], check=True)


def test_ctypes_mirrors_match_c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "igm_b200.h"', "int main(void) {"]
    for cname, py in PAIRS:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", INC, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        if ln:
            parts = ln.split()
            got[tuple(parts[:-1])] = int(parts[-1])
    for cname, py in PAIRS:
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
