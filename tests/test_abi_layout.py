"""The ctypes mirrors in plasticity_b200/capi.py have the layout of the C
structs in include/cp_gpu.h: every struct's size and every field's offset,
from a small C program compiled against the header (no GPU needed)."""
import ctypes as C
import os
import subprocess

import pytest

from plasticity_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OUT = os.path.join(ROOT, "tests", "kernel_emu", "_build")

STRUCTS = {"cp_material_t": capi.CpMaterial, "cp_options_t": capi.CpOptions, "cp_solver_t": capi.CpSolver,
           "cp_solve_info_t": capi.CpSolveInfo, "cp_tune_result_t": capi.CpTuneResult}


@pytest.fixture(scope="module")
def c_layout():
    os.makedirs(OUT, exist_ok=True)
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "cp_gpu.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        src.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            src.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src += ["  return 0;", "}"]
    cfile = os.path.join(OUT, "abi_layout.c")
    exe = os.path.join(OUT, "abi_layout")
    with open(cfile, "w") as fh:
        fh.write("\n".join(src) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), cfile, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    layout = {}
    for line in out:
        if line:
            s, f, v = line.split()
            layout[(s, f)] = int(v)
    return layout


@pytest.mark.parametrize("cname", list(STRUCTS))
def test_ctypes_mirror_matches_header(c_layout, cname):
    py = STRUCTS[cname]
    assert C.sizeof(py) == c_layout[(cname, "size")]
    for f, _ in py._fields_:
        assert getattr(py, f).offset == c_layout[(cname, f)], (cname, f)
