"""ctypes wrapper around the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product path (plasticity_b200/) never imports it.

``OracleBackend`` exposes the same methods as plasticity_b200.capi.CpHandle
(bind_qps / update / bind_mesh / assemble / averages / reorient / commit /
get_state / set_state) so the Newton harness and the parity tests can drive
either one.  State is held per lattice in the qp-major layout of
cp_oracle.h; qps keep the caller's order across lattices.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from plasticity_b200.capi import CP_MAX_SYSTEMS, CpMaterial, CpOptions, default_options

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "libcp_oracle.so")

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)


class OrState(C.Structure):
    _fields_ = [("n_qp", C.c_int64)] + [
        (name, D) for name in ("Fp_conv", "Fe_conv", "s_conv", "W_conv", "rot_conv", "rotnew_conv",
                               "twinfrac_conv", "slipfrac_conv")
    ] + [("twin_conv", I32)] + [
        (name, D) for name in ("Fp_iter", "Fe_iter", "s_iter", "W_iter", "rot_iter", "rotnew_iter",
                               "twinfrac_iter", "slipfrac_iter")
    ] + [("twin_iter", I32)]


def _stale(path) -> bool:
    if not os.path.exists(path):
        return True
    t = os.path.getmtime(path)
    srcs = [os.path.join(_HERE, f) for f in ("cp_oracle.cpp", "cp_oracle.h", "Makefile")]
    srcs.append(os.path.join(os.path.dirname(_HERE), "include", "cp_gpu.h"))
    return any(os.path.exists(f) and os.path.getmtime(f) > t for f in srcs)


def build(force: bool = False) -> str:
    if force or _stale(LIB):
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    return LIB


_lib = None


def build_fma() -> str:
    """The oracle compiled with fused multiply-adds allowed (make fma)."""
    path = os.path.join(_HERE, "_build", "libcp_oracle_fma.so")
    if _stale(path):
        subprocess.run(["make", "-C", _HERE, "fma"], check=True, capture_output=True)
    return path


def build_parity() -> str:
    """The parity build (make parity): pow, the Gateaux factorials and the
    twin rotation from correctly rounded operations only, the CPU counterpart
    of the library's reference-order update (cp_options_t.reference_order)."""
    path = os.path.join(_HERE, "_build", "libcp_oracle_parity.so")
    if _stale(path):
        subprocess.run(["make", "-C", _HERE, "parity"], check=True, capture_output=True)
    return path


def use_library(path: str | None):
    """Route the module's calls to the oracle library at 'path' (None: the
    default build); returns the previous library so a caller can restore it."""
    global _lib
    prev = _lib
    _lib = None
    if path is not None:
        _lib = _load(path)
    return prev


def restore_library(prev):
    global _lib
    _lib = prev


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _load(build())
    return _lib


def _load(path) -> C.CDLL:
    L = C.CDLL(path)
    M, O, S = C.POINTER(CpMaterial), C.POINTER(CpOptions), C.POINTER(OrState)
    L.oracle_update.argtypes = [M, O, S, D, C.c_int32, C.c_double, C.c_double, D, D, D, I32, I32, C.c_int32]
    L.oracle_assemble.argtypes = [M, O, S, C.c_int64, D, D, D, C.c_int32, C.c_double, C.c_double,
                                  D, D, I32, I32, C.c_int32]
    L.oracle_reorient.argtypes = [S, C.c_int32]
    L.oracle_odfpoint.argtypes = [D, D]
    L.oracle_elasticmoduli.argtypes = [D, D, D]
    L.oracle_matrix_exponential.argtypes = [D, D]
    L.oracle_pinv_svd.argtypes = [D, C.c_int, D]
    L.oracle_invert.argtypes = [D, C.c_int, D]
    L.oracle_eig_sym3.argtypes = [D, D, D]
    L.oracle_parity_pow.argtypes = [C.c_double, C.c_double]
    L.oracle_parity_pow.restype = C.c_double
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(D)


def _pi(a):
    return None if a is None else a.ctypes.data_as(I32)


# ---------------------------------------------------------------- small helpers
def odfpoint(r):
    r = np.ascontiguousarray(r, float)
    out = np.empty(9)
    lib().oracle_odfpoint(_p(r), _p(out))
    return out.reshape(3, 3)


def elasticmoduli(R, C6):
    R = np.ascontiguousarray(R, float)
    C6 = np.ascontiguousarray(C6, float)
    out = np.empty(36)
    lib().oracle_elasticmoduli(_p(R), _p(C6), _p(out))
    return out.reshape(6, 6)


def matrix_exponential(A):
    A = np.ascontiguousarray(A, float)
    out = np.empty(9)
    terms = lib().oracle_matrix_exponential(_p(A), _p(out))
    return out.reshape(3, 3), terms


def pinv_svd(A):
    A = np.ascontiguousarray(A, float)
    n = A.shape[0]
    out = np.empty((n, n))
    sing = lib().oracle_pinv_svd(_p(A), n, _p(out))
    return out, sing


def invert(A):
    A = np.ascontiguousarray(A, float)
    n = A.shape[0]
    out = np.empty((n, n))
    sing = lib().oracle_invert(_p(A), n, _p(out))
    return out, sing


def eig_sym3(Cm):
    Cm = np.ascontiguousarray(Cm, float)
    ev = np.empty(3)
    V = np.empty(9)
    lib().oracle_eig_sym3(_p(Cm), _p(ev), _p(V))
    return ev, V.reshape(3, 3)


# ---------------------------------------------------------------- state groups
class _Group:
    """Per-lattice state arrays (qp-major)."""

    def __init__(self, mat: CpMaterial, idx: np.ndarray, rod: np.ndarray):
        self.mat = mat
        self.idx = idx
        m = len(idx)
        n, ns, nw = mat.n_total, mat.n_slip, mat.n_twin
        s0 = np.ctypeslib.as_array(mat.initial_slip_resistance)[:n]
        eye = np.tile(np.eye(3).ravel(), (m, 1))
        self.a = {}
        for suf in ("conv", "iter"):
            self.a["Fp_" + suf] = eye.copy()
            self.a["Fe_" + suf] = eye.copy()
            self.a["s_" + suf] = np.tile(s0, (m, 1)).copy()
            self.a["W_" + suf] = np.zeros((m, n))
            self.a["rot_" + suf] = rod.copy()
            self.a["rotnew_" + suf] = rod.copy()
            self.a["twinfrac_" + suf] = np.zeros((m, nw))
            self.a["slipfrac_" + suf] = np.zeros((m, ns))
            self.a["twin_" + suf] = np.zeros(m, dtype=np.int32)
        self.st = OrState()
        self.st.n_qp = m
        for k, v in self.a.items():
            setattr(self.st, k, _pi(v) if v.dtype == np.int32 else _p(v))


class OracleBackend:
    """CPU oracle with the CpHandle method set (single process, OpenMP)."""

    def __init__(self, lattices, options: CpOptions | None = None, nthreads: int = 0):
        self.lattices = list(lattices)
        self.options = options or default_options()
        self.nthreads = nthreads
        self.groups: list[_Group] = []
        self.n_qp = 0
        self.n_cells = 0
        self.last_F = None
        self.last_T = None
        self.last_stats = None

    def bind_qps(self, lattice_id, rodrigues):
        lid = np.asarray(lattice_id, dtype=np.int32)
        rod = np.ascontiguousarray(rodrigues, float).reshape(-1, 3)
        self.n_qp = len(lid)
        self.lattice_id = lid
        self.groups = []
        for L, mat in enumerate(self.lattices):
            idx = np.nonzero(lid == L)[0]
            if len(idx):
                g = _Group(mat, idx, rod[idx])
                g.lattice = L
                self.groups.append(g)

    def update(self, F, flag, F_e=0.0, F_r=0.0, want_T=True):
        F = np.ascontiguousarray(F, float).reshape(self.n_qp, 9)
        P = np.empty((self.n_qp, 9))
        T = np.empty((self.n_qp, 9))
        dPdF = np.empty((self.n_qp, 81)) if flag == 1 else None
        stats = np.zeros((self.n_qp, 8), dtype=np.int32)
        status = np.zeros(self.n_qp, dtype=np.int32)
        for L, g in self._lattice_groups():
            m = len(g.idx)
            Fg = np.ascontiguousarray(F[g.idx])
            Pg, Tg = np.empty((m, 9)), np.empty((m, 9))
            dg = np.empty((m, 81)) if flag == 1 else None
            sg = np.zeros((m, 8), dtype=np.int32)
            qs = np.zeros(m, dtype=np.int32)
            lib().oracle_update(C.byref(g.mat), C.byref(self.options), C.byref(g.st), _p(Fg), flag,
                                F_e, F_r, _p(Pg), _p(Tg), _p(dg), _pi(sg), _pi(qs), self.nthreads)
            P[g.idx], T[g.idx] = Pg, Tg
            if flag == 1:
                dPdF[g.idx] = dg
            sg[:, 6] = L
            stats[g.idx] = sg
            status[g.idx] = qs
        self.last_F, self.last_T, self.last_stats = F, T, stats
        return P, T, dPdF, status

    def _lattice_groups(self):
        return [(g.lattice, g) for g in self.groups]

    def stats(self):
        return self.last_stats

    def bind_mesh(self, n_cells, grad_N, JxW, uniform):
        self.n_cells = int(n_cells)
        self.grad_N = np.ascontiguousarray(grad_N, float)
        self.JxW = np.ascontiguousarray(JxW, float)
        self.uniform = bool(uniform)
        assert self.n_qp == 8 * self.n_cells

    def _cell_groups(self):
        """cells of one lattice (all 8 qps of a cell share the lattice)."""
        lid = self.lattice_id.reshape(self.n_cells, 8)
        assert np.all(lid == lid[:, :1]), "mixed-lattice cell"
        return lid[:, 0]

    def assemble(self, U_local, F_e=0.0, F_r=0.0):
        U = np.ascontiguousarray(U_local, float).reshape(self.n_cells, 24)
        Ke = np.empty((self.n_cells, 24, 24))
        Re = np.empty((self.n_cells, 24))
        cl = self._cell_groups()
        stats = np.zeros((self.n_qp, 8), dtype=np.int32)
        status = np.zeros(self.n_qp, dtype=np.int32)
        for L, g in self._lattice_groups():
            cells = np.nonzero(cl == L)[0]
            # group qps are ordered like the caller's qps, so cell-major order holds
            assert np.array_equal(g.idx, (8 * cells[:, None] + np.arange(8)).ravel())
            Ug = np.ascontiguousarray(U[cells])
            gN = self.grad_N if self.uniform else np.ascontiguousarray(
                self.grad_N.reshape(self.n_cells, -1)[cells])
            w = self.JxW if self.uniform else np.ascontiguousarray(self.JxW.reshape(self.n_cells, -1)[cells])
            Kg = np.empty((len(cells), 24, 24))
            Rg = np.empty((len(cells), 24))
            sg = np.zeros((len(g.idx), 8), dtype=np.int32)
            qs = np.zeros(len(g.idx), dtype=np.int32)
            lib().oracle_assemble(C.byref(g.mat), C.byref(self.options), C.byref(g.st), len(cells),
                                  _p(Ug), _p(gN), _p(w), 1 if self.uniform else 0, F_e, F_r,
                                  _p(Kg), _p(Rg), _pi(sg), _pi(qs), self.nthreads)
            Ke[cells], Re[cells] = Kg, Rg
            sg[:, 6] = L
            stats[g.idx] = sg
            status[g.idx] = qs
        self.last_stats = stats
        return Ke, Re, status

    def averages(self):
        """updateAfterIncrement.cc:119-126,218-235,710-722 over the last update."""
        F = self.last_F.reshape(-1, 3, 3)
        T = self.last_T.reshape(-1, 3, 3)
        w = np.broadcast_to(self.JxW.reshape(-1, 8), (self.n_cells, 8)).reshape(-1)
        E = 0.5 * (np.einsum("kji,kjl->kil", F, F) - np.eye(3))
        vol = w.sum()
        out = np.zeros(22)
        out[0:9] = (E * w[:, None, None]).sum(0).ravel() / vol
        out[9:18] = (T * w[:, None, None]).sum(0).ravel() / vol
        Fr = Fe = Fs = 0.0
        for g in self.groups:
            wg = w[g.idx]
            n_tw = g.mat.n_twin
            Fr += (g.a["twinfrac_iter"][:, :n_tw].sum(1) * wg).sum()
            Fe += (g.a["twin_iter"] * wg).sum()
            Fs += (g.a["slipfrac_iter"].sum(1) * wg).sum()
        out[18], out[19], out[20], out[21] = Fr / vol, Fe / vol, Fs / vol, vol
        return out

    def reorient(self):
        for g in self.groups:
            lib().oracle_reorient(C.byref(g.st), self.nthreads)

    def commit(self):
        for g in self.groups:
            for k in list(g.a):
                if k.endswith("_iter"):
                    g.a[k.replace("_iter", "_conv")][...] = g.a[k]

    def get_state(self, name):
        parts = [(g, g.a[name]) for g in self.groups]
        w = max(a.shape[1] if a.ndim == 2 else 1 for _, a in parts)
        out = np.zeros((self.n_qp, w))
        for g, a in parts:
            if a.ndim == 1:
                out[g.idx, 0] = a
            else:
                out[g.idx, : a.shape[1]] = a
        return out

    def set_state(self, name, values):
        values = np.asarray(values, float)
        for g in self.groups:
            a = g.a[name]
            if a.ndim == 1:
                a[...] = values[g.idx, 0]
            else:
                a[...] = values[g.idx, : a.shape[1]]
