"""Build the in-tree CUDA library plasticity_b200/_build/libcp_b200.so (sm_100a).

The product is a plain C-ABI shared library (include/cp_gpu.h); Python loads
it with ctypes.  Built with nvcc directly, so the .so lives in the source
tree and travels with it.  The large per-qp kernels are separate translation
units (one per lattice class, F source and launch shape of the sorted update;
one per lattice class of the plain and the batched kernels) compiled in
parallel and linked
into the one library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libcp_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-I" + os.path.join(ROOT, "include"),
]

U2_VARIANTS = 4  # thread-per-qp shapes (U2_THREAD_SHAPES in csrc/cp_launch.h)


def units():
    """(object name, source, extra defines) of every translation unit."""
    out = [("cp_api", "cp_api.cu", []), ("cp_tc", "cp_tc.cu", [])]
    for pmax in (16, 32, 48):
        for fsrc in ("FromArray", "FromMesh"):
            for v in range(U2_VARIANTS):
                out.append((f"u2_{pmax}_{fsrc}_{v}", "cp_update_tu.cu",
                            [f"-DCP_TU_PMAX={pmax}", f"-DCP_TU_FSRC={fsrc}", f"-DCP_TU_VARIANT={v}"]))
    for pmax in (16, 32, 48):
        for fsrc in ("FromArray", "FromMesh"):
            out.append((f"quad_{pmax}_{fsrc}", "cp_quad_tu.cu", [f"-DCP_TU_PMAX={pmax}", f"-DCP_TU_FSRC={fsrc}"]))
    for nt, pmax in ((16, 16), (32, 32), (64, 48)):
        out.append((f"plain_{nt}", "cp_plain_tu.cu", [f"-DCP_TU_NT={nt}", f"-DCP_TU_PMAX={pmax}"]))
    for pmax in (16, 32, 48):
        out.append((f"batch_{pmax}", "cp_batch_tu.cu", [f"-DCP_TU_PMAX={pmax}"]))
    # the reference-order update: no multiply-add contraction
    out.append(("ref", "cp_ref_tu.cu", ["-fmad=false"]))
    return [u for u in out if os.path.exists(os.path.join(CSRC, u[1]))]


def deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "cp_gpu.h")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _newest_dep() -> float:
    return max(os.path.getmtime(d) for d in deps() if os.path.exists(d))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    return _newest_dep() <= os.path.getmtime(LIB)


def _obj(name):
    return os.path.join(OBJ_DIR, name + ".o")


def build(force: bool = False, verbose: bool = False, extra=None, jobs: int | None = None) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest = _newest_dep()
    todo = [u for u in units()
            if force or extra or not os.path.exists(_obj(u[0])) or os.path.getmtime(_obj(u[0])) < newest]

    def compile_one(u):
        name, src, defs = u
        cmd = [nvcc()] + NVCC_FLAGS + (extra or []) + defs + ["-c", os.path.join(CSRC, src), "-o", _obj(name)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return name, cmd, r

    failed = []
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for name, cmd, r in ex.map(compile_one, todo):
            if verbose:
                print(" ".join(cmd))
                if r.stdout or r.stderr:
                    print(r.stdout + r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                failed.append(name)
    if failed:
        raise RuntimeError("nvcc failed: " + ", ".join(failed))
    link = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC"] + [_obj(u[0]) for u in units()] + ["-o", LIB]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
