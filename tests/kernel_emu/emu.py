"""The CUDA qp kernel source compiled for the host, behind the oracle
backend's interface (tests only)."""
import ctypes as C
import os
import subprocess

from oracle import oracle as O
from plasticity_b200.capi import CpMaterial, CpOptions

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "libcp_emu.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
        L = C.CDLL(LIB)
        D, I32 = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        L.emu_update.argtypes = [C.POINTER(CpMaterial), C.POINTER(CpOptions), C.POINTER(O.OrState), D, C.c_int32,
                                 C.c_double, C.c_double, D, D, D, I32, I32, C.c_int32]
        L.emu_lu_compare.argtypes = [D, D, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.emu_ref_pow.argtypes = [C.c_double, C.c_double]
        L.emu_ref_pow.restype = C.c_double
        _lib = L
    return _lib


class _EmuLib:
    """Routes oracle_update to the host build of the kernel."""

    def __init__(self, base):
        self.base = base

    def __getattr__(self, name):
        if name == "oracle_update":
            return lib().emu_update
        return getattr(self.base, name)


class EmuBackend(O.OracleBackend):
    def update(self, *a, **k):
        real = O.lib
        O.lib = lambda: _EmuLib(real())
        try:
            return super().update(*a, **k)
        finally:
            O.lib = real
