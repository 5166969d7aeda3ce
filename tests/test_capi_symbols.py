"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**\s*(cp_[A-Za-z0-9_]+)\s*\(", src,
                             flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_api():
    names = declared_functions()
    for must in ("cp_create", "cp_bind_qps", "cp_update", "cp_update_device", "cp_assemble", "cp_reorient",
                 "cp_commit", "cp_averages", "cp_get_state", "cp_set_state", "cp_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = ctypes.CDLL(os.path.join(ROOT, "plasticity_b200", "_build", "libcp_b200.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_calls_without_gpu(cuda_lib):
    """Calls that touch no device: option defaults and the dummy twin."""
    from plasticity_b200 import capi
    o = capi.CpOptions()
    assert cuda_lib.cp_options_default(ctypes.byref(o)) == 0
    assert o.stress_tolerance == 1e-9 and o.max_slip_search_iterations == 1
    m = capi.CpMaterial()
    m.n_slip = 12
    assert cuda_lib.cp_material_add_dummy_twin(ctypes.byref(m)) == 0
    assert m.n_twin == 1 and m.initial_slip_resistance[12] == 10e14 and m.saturation_stress[12] == 10e15
    assert m.slip_normal[36] == 1.0 and m.slip_direction[37] == 1.0
    assert cuda_lib.cp_create(None, 0, None, None) != 0


def test_product_never_imports_oracle():
    """The product package must not import, load or call the CPU oracle."""
    pat = re.compile(r"^\s*(from|import)\s+oracle\b|libcp_oracle|cp_oracle\.h|oracle_(update|assemble|reorient)",
                     re.M)
    for path in glob.glob(os.path.join(ROOT, "plasticity_b200", "**", "*.*"), recursive=True):
        if path.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
            assert not pat.search(open(path).read()), path
