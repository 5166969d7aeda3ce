"""ctypes mirror of include/cp_gpu.h and the handle wrapper around libcp_b200.so.

The handle mirrors the reference's crystalPlasticity<dim> per-qp interface
(include/crystalPlasticity.h:77-78):

* ``update``      == calculatePlasticity(cellID, q, StiffnessCalFlag) over every qp
                     (src/materialModels/crystalPlasticity/calculatePlasticity.cc:13)
* ``assemble``    == getElementalValues over every cell (getElementalValues.cc:5)
* ``averages``    == the volume averages of updateAfterIncrement.cc:119-126,710-722
* ``reorient``    == reorient() (reorient.cc:4) plus the rotnew copies around it
* ``commit``      == the *_iter -> *_conv copy (updateAfterIncrement.cc:298-305)

There is no CPU fallback: if the shared library is missing the constructor
raises, and a CUDA failure inside a call raises ``CpError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

CP_MAX_SYSTEMS = 64
CP_MAX_LATTICES = 8

CP_OK = 0
CP_E_ARG = -1
CP_E_STATE = -2
CP_E_CUDA = -3
CP_E_NOMEM = -4
CP_E_UNSUPPORTED = -5
CP_QP_NONFINITE = 1
CP_QP_SINGULAR = 2
CP_QP_ACTIVE_OVERFLOW = 4
CP_QP_SERIES_CAP = 8
CP_QP_SLIP_SEARCH_CAP = 16
CP_QP_ILL_CONDITIONED = 32
CP_QP_ERROR_MASK = CP_QP_NONFINITE | CP_QP_SINGULAR | CP_QP_ACTIVE_OVERFLOW | CP_QP_SERIES_CAP

FIELDS = {
    "Fp_conv": 0, "Fe_conv": 1, "s_conv": 2, "W_conv": 3, "rot_conv": 4,
    "rotnew_conv": 5, "twinfrac_conv": 6, "slipfrac_conv": 7, "twin_conv": 8,
}
ITER_OFFSET = 16
for _k, _v in list(FIELDS.items()):
    FIELDS[_k.replace("_conv", "_iter")] = _v + ITER_OFFSET

_NM = CP_MAX_SYSTEMS


class CpMaterial(C.Structure):
    """cp_material_t: one lattice (phase); field names follow userInputParameters."""

    _fields_ = [
        ("n_slip", C.c_int32),
        ("n_twin", C.c_int32),
        ("twinning_enabled", C.c_int32),
        ("reserved", C.c_int32),
        ("elastic_stiffness", C.c_double * 36),
        ("slip_normal", C.c_double * (_NM * 3)),
        ("slip_direction", C.c_double * (_NM * 3)),
        ("latent_hardening", C.c_double * (_NM * _NM)),
        ("initial_slip_resistance", C.c_double * _NM),
        ("initial_hardening_modulus", C.c_double * _NM),
        ("saturation_stress", C.c_double * _NM),
        ("power_law_exponent", C.c_double * _NM),
        ("kinematic_c1", C.c_double * _NM),
        ("kinematic_c2", C.c_double * _NM),
        ("twin_threshold_fraction", C.c_double),
        ("twin_saturation_factor", C.c_double),
        ("twin_shear", C.c_double),
    ]

    @property
    def n_total(self) -> int:
        return int(self.n_slip + self.n_twin)


class CpOptions(C.Structure):
    _fields_ = [
        ("stress_tolerance", C.c_double),
        ("max_slip_search_iterations", C.c_int32),
        ("max_solver_iterations", C.c_int32),
        ("enable_multiphase", C.c_int32),
        ("device", C.c_int32),
        ("update_variant", C.c_int32),
        ("use_graphs", C.c_int32),
        ("plain_kernel", C.c_int32),
        ("reference_order", C.c_int32),
    ]


class CpSolver(C.Structure):
    """cp_solver_t: the Newton step's Krylov solve (solveLinearSystem.cc:10-36)."""

    _fields_ = [
        ("kind", C.c_int32),
        ("max_iterations", C.c_int32),
        ("rel_tolerance", C.c_double),
        ("precond_norm", C.c_int32),
        ("check_every", C.c_int32),
        ("precond", C.c_int32),
        ("kernel_mode", C.c_int32),
        ("precision", C.c_int32),
        ("max_refinements", C.c_int32),
        ("inner_tolerance", C.c_double),
    ]


class CpSolveInfo(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("breakdown", C.c_int32),
        ("refinements", C.c_int32),
        ("rhs_norm", C.c_double),
        ("residual_norm", C.c_double),
        ("fp64_iterations", C.c_int32),
        ("reserved", C.c_int32),
    ]


CP_UPDATE_VARIANTS = 5
CP_TUNE_UPDATE = 0
CP_TUNE_ASSEMBLE = 1
# launch shapes of the sorted update: (threads per block, registers per thread)
UPDATE_SHAPES = [(256, 255), (256, 128), (64, 255), (64, 128)]


class CpTuneResult(C.Structure):
    """cp_tune_result_t: one lattice group's autotuning outcome."""

    _fields_ = [
        ("lattice", C.c_int32),
        ("chosen", C.c_int32),
        ("default_variant", C.c_int32),
        ("reserved", C.c_int32),
        ("n_qp", C.c_int64),
        ("median_ms", C.c_double * CP_UPDATE_VARIANTS),
    ]


CP_SOLVER_BICG = 0
CP_SOLVER_BICGSTAB = 1
CP_PRECOND_JACOBI = 0
CP_PRECOND_NODE_BLOCK = 1
CP_PRECISION_FP64 = 0
CP_PRECISION_MIXED = 1


def default_solver(**kw) -> CpSolver:
    """The reference decks' settings: BiCG, 50000 iterations, 1e-10 x ||b||."""
    s = CpSolver()
    s.kind, s.max_iterations, s.rel_tolerance, s.precond_norm, s.check_every = CP_SOLVER_BICG, 50000, 1e-10, 0, 8
    s.precond = CP_PRECOND_JACOBI
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def default_options(**kw) -> CpOptions:
    """The reference's shipped values: Stress Tolerance 1e-9, caps 1/1."""
    o = CpOptions()
    o.stress_tolerance = 1.0e-9
    o.max_slip_search_iterations = 1
    o.max_solver_iterations = 1
    o.enable_multiphase = 0
    o.device = 0
    o.update_variant = 0
    o.use_graphs = 1
    o.plain_kernel = 0
    o.reference_order = 0
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def as_f64(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class CpError(RuntimeError):
    pass


_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "_build", "libcp_b200.so")
_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise CpError(f"CUDA library not built: {p} (run __graft_entry__.build())")
    lib = C.CDLL(p)
    D, I32, I64 = C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int64
    H = C.c_void_p
    sig = {
        "cp_options_default": (C.c_int, [C.POINTER(CpOptions)]),
        "cp_bind_dofs": (C.c_int, [H, I64, C.POINTER(C.c_int64), I64, C.POINTER(C.c_int64)]),
        "cp_set_displacement": (C.c_int, [H, D]),
        "cp_get_displacement": (C.c_int, [H, D]),
        "cp_solver_default": (C.c_int, [C.POINTER(CpSolver)]),
        "cp_newton_iteration": (C.c_int, [H, D, C.c_double, C.c_double, C.POINTER(CpSolver),
                                          C.POINTER(CpSolveInfo)]),
        "cp_update_from_displacement": (C.c_int, [H, C.c_double, C.c_double]),
        "cp_material_add_dummy_twin": (C.c_int, [C.POINTER(CpMaterial)]),
        "cp_create": (C.c_int, [C.POINTER(CpMaterial), C.c_int32, C.POINTER(CpOptions), C.POINTER(H)]),
        "cp_destroy": (None, [H]),
        "cp_last_error": (C.c_char_p, [H]),
        "cp_bind_qps": (C.c_int, [H, I64, I32, D]),
        "cp_num_qps": (C.c_int64, [H]),
        "cp_update": (C.c_int, [H, D, C.c_int32, C.c_double, C.c_double, D, D, D, I32]),
        "cp_update_device": (C.c_int, [H, C.c_void_p, C.c_int32, C.c_double, C.c_double,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "cp_get_stats": (C.c_int, [H, I32]),
        "cp_bind_mesh": (C.c_int, [H, I64, D, D, C.c_int32]),
        "cp_assemble": (C.c_int, [H, D, C.c_double, C.c_double, D, D, I32]),
        "cp_assemble_device": (C.c_int, [H, C.c_void_p, C.c_double, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
        "cp_assemble_mixed": (C.c_int, [H, D, C.c_double, C.c_double, C.POINTER(C.c_float), D, I32]),
        "cp_assemble_mixed_device": (C.c_int, [H, C.c_void_p, C.c_double, C.c_double,
                                               C.c_void_p, C.c_void_p, C.c_void_p]),
        "cp_averages": (C.c_int, [H, D]),
        "cp_averages_noalloc": (C.c_int, [H, D]),
        "cp_reorient": (C.c_int, [H]),
        "cp_commit": (C.c_int, [H]),
        "cp_field_width": (C.c_int32, [H, C.c_int32]),
        "cp_get_state": (C.c_int, [H, C.c_int32, D]),
        "cp_set_state": (C.c_int, [H, C.c_int32, D]),
        "cp_synchronize": (C.c_int, [H]),
        "cp_stream": (C.c_void_p, [H]),
        "cp_measure_fp64_peak": (C.c_int, [C.c_int32, D]),
        "cp_set_timing": (C.c_int, [H, C.c_int32]),
        "cp_get_timing": (C.c_int, [H, C.c_int32, I32, C.POINTER(C.c_int64), C.POINTER(C.c_int64), D]),
        "cp_get_contract_timing": (C.c_int, [H, C.c_int32, C.POINTER(C.c_int64), D]),
        "cp_autotune": (C.c_int, [H, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.POINTER(CpTuneResult),
                                  C.c_int32]),
        "cp_tune_select": (C.c_int32, [C.c_int32, C.c_int32, D, C.c_int32, C.c_double]),
        "cp_debug_barrier_test": (C.c_int, [H, C.c_int32, C.c_double]),
        "cp_newton_solve": (C.c_int, [H, D, C.POINTER(CpSolver), C.POINTER(CpSolveInfo)]),
        "cp_batch_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
        "cp_batch_destroy": (None, [C.c_void_p]),
        "cp_batch_last_error": (C.c_char_p, [C.c_void_p]),
        "cp_batch_launches": (C.c_int64, [C.c_void_p]),
        "cp_batch_assemble": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, D, D]),
        "cp_batch_post": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.c_int32, D, D]),
        "cp_graph_stats": (C.c_int, [H, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def measure_fp64_peak(device: int = 0) -> float:
    lib = load_library()
    out = C.c_double()
    rc = lib.cp_measure_fp64_peak(device, C.byref(out))
    if rc != CP_OK:
        raise CpError(f"cp_measure_fp64_peak failed ({rc})")
    return float(out.value)


class CpHandle:
    """One resident batch of quadrature points on one GPU (owns a cp_handle*)."""

    def __init__(self, lattices, options: CpOptions | None = None, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.lattices = list(lattices)
        n = len(self.lattices)
        arr = (CpMaterial * n)(*self.lattices)
        self.options = options or default_options()
        h = C.c_void_p()
        rc = self.lib.cp_create(arr, n, C.byref(self.options), C.byref(h))
        if rc != CP_OK:
            raise CpError(f"cp_create failed ({rc})")
        self.h = h
        self.n_qp = 0
        self.n_cells = 0

    # -- helpers --------------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc != CP_OK:
            msg = self.lib.cp_last_error(self.h)
            raise CpError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.cp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- API ------------------------------------------------------------------
    def bind_qps(self, lattice_id, rodrigues):
        lid = np.ascontiguousarray(lattice_id, dtype=np.int32)
        rod = as_f64(rodrigues, (-1, 3))
        assert rod.shape[0] == lid.shape[0]
        self._check(self.lib.cp_bind_qps(self.h, lid.shape[0], iptr(lid), dptr(rod)), "cp_bind_qps")
        self.n_qp = int(lid.shape[0])

    def update(self, F, flag: int, F_e: float = 0.0, F_r: float = 0.0, want_T=True):
        F = as_f64(F, (self.n_qp, 9))
        P = np.empty((self.n_qp, 9))
        T = np.empty((self.n_qp, 9)) if want_T else None
        dPdF = np.empty((self.n_qp, 81)) if flag == 1 else None
        st = np.empty(self.n_qp, dtype=np.int32)
        self._check(self.lib.cp_update(self.h, dptr(F), flag, F_e, F_r, dptr(P), dptr(T),
                                       dptr(dPdF), iptr(st)), "cp_update")
        return P, T, dPdF, st

    def update_device(self, F_ptr: int, flag: int, F_e, F_r, P_ptr: int, T_ptr: int | None,
                      dPdF_ptr: int | None, status_ptr: int | None):
        self._check(self.lib.cp_update_device(self.h, C.c_void_p(F_ptr), flag, F_e, F_r,
                                              C.c_void_p(P_ptr), C.c_void_p(T_ptr or 0) if T_ptr else None,
                                              C.c_void_p(dPdF_ptr) if dPdF_ptr else None,
                                              C.c_void_p(status_ptr) if status_ptr else None),
                    "cp_update_device")

    def stats(self):
        s = np.empty((self.n_qp, 8), dtype=np.int32)
        self._check(self.lib.cp_get_stats(self.h, iptr(s)), "cp_get_stats")
        return s

    def bind_mesh(self, n_cells, grad_N, JxW, uniform: bool):
        g = as_f64(grad_N)
        w = as_f64(JxW)
        self._check(self.lib.cp_bind_mesh(self.h, n_cells, dptr(g), dptr(w), 1 if uniform else 0),
                    "cp_bind_mesh")
        self.n_cells = int(n_cells)

    def assemble(self, U_local, F_e: float = 0.0, F_r: float = 0.0):
        U = as_f64(U_local, (self.n_cells, 24))
        Ke = np.empty((self.n_cells, 24, 24))
        Re = np.empty((self.n_cells, 24))
        st = np.empty(self.n_qp, dtype=np.int32)
        self._check(self.lib.cp_assemble(self.h, dptr(U), F_e, F_r, dptr(Ke), dptr(Re), iptr(st)),
                    "cp_assemble")
        return Ke, Re, st

    def assemble_mixed(self, U_local, F_e: float = 0.0, F_r: float = 0.0):
        """cp_assemble_mixed: FP32 Ke from the split-BF16 tensor-core contraction, FP64 Re."""
        U = as_f64(U_local, (self.n_cells, 24))
        Ke = np.empty((self.n_cells, 24, 24), dtype=np.float32)
        Re = np.empty((self.n_cells, 24))
        st = np.empty(self.n_qp, dtype=np.int32)
        self._check(self.lib.cp_assemble_mixed(self.h, dptr(U), F_e, F_r, Ke.ctypes.data_as(C.POINTER(C.c_float)),
                                               dptr(Re), iptr(st)), "cp_assemble_mixed")
        return Ke, Re, st

    def assemble_mixed_device(self, U_ptr, F_e, F_r, Ke_ptr, Re_ptr, status_ptr=None):
        self._check(self.lib.cp_assemble_mixed_device(self.h, C.c_void_p(U_ptr), F_e, F_r, C.c_void_p(Ke_ptr),
                                                      C.c_void_p(Re_ptr),
                                                      C.c_void_p(status_ptr) if status_ptr else None),
                    "cp_assemble_mixed_device")

    def assemble_device(self, U_ptr, F_e, F_r, Ke_ptr, Re_ptr, status_ptr=None):
        self._check(self.lib.cp_assemble_device(self.h, C.c_void_p(U_ptr), F_e, F_r, C.c_void_p(Ke_ptr),
                                                C.c_void_p(Re_ptr),
                                                C.c_void_p(status_ptr) if status_ptr else None),
                    "cp_assemble_device")

    def averages(self):
        out = np.empty(22)
        self._check(self.lib.cp_averages(self.h, dptr(out)), "cp_averages")
        return out

    # ---- the Newton step's global system on the device
    def bind_dofs(self, n_dofs: int, cell_dofs, constrained):
        cd = np.ascontiguousarray(cell_dofs, dtype=np.int64).reshape(-1)
        con = np.ascontiguousarray(constrained, dtype=np.int64).reshape(-1)
        p64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
        self._check(self.lib.cp_bind_dofs(self.h, int(n_dofs), p64(cd), len(con), p64(con) if len(con) else None),
                    "cp_bind_dofs")
        self.n_dofs = int(n_dofs)

    def set_displacement(self, u):
        u = as_f64(u, (self.n_dofs,))
        self._check(self.lib.cp_set_displacement(self.h, dptr(u)), "cp_set_displacement")

    def get_displacement(self):
        u = np.empty(self.n_dofs)
        self._check(self.lib.cp_get_displacement(self.h, dptr(u)), "cp_get_displacement")
        return u

    def newton_iteration(self, du_constrained=None, F_e: float = 0.0, F_r: float = 0.0, solver: CpSolver | None = None):
        """One device Newton pass (assemble, scatter, condense, solve, u += du); returns the solve info."""
        duc = None if du_constrained is None else as_f64(du_constrained)
        info = CpSolveInfo()
        self._check(self.lib.cp_newton_iteration(self.h, dptr(duc), F_e, F_r,
                                                 C.byref(solver) if solver is not None else None,
                                                 C.byref(info)), "cp_newton_iteration")
        return {"iterations": info.iterations, "converged": bool(info.converged), "breakdown": bool(info.breakdown),
                "refinements": info.refinements, "fp64_iterations": info.fp64_iterations,
                "rhs_norm": info.rhs_norm, "residual_norm": info.residual_norm}

    def newton_solve(self, du_constrained=None, solver: CpSolver | None = None):
        """cp_newton_solve: the solve half of a Newton pass whose Ke/Re a cp_batch_assemble wrote."""
        duc = None if du_constrained is None else as_f64(du_constrained)
        info = CpSolveInfo()
        self._check(self.lib.cp_newton_solve(self.h, dptr(duc), C.byref(solver) if solver is not None else None,
                                             C.byref(info)), "cp_newton_solve")
        return {"iterations": info.iterations, "converged": bool(info.converged), "breakdown": bool(info.breakdown),
                "refinements": info.refinements, "fp64_iterations": info.fp64_iterations,
                "rhs_norm": info.rhs_norm, "residual_norm": info.residual_norm}

    def update_from_displacement(self, F_e: float = 0.0, F_r: float = 0.0):
        self._check(self.lib.cp_update_from_displacement(self.h, F_e, F_r), "cp_update_from_displacement")

    def reorient(self):
        self._check(self.lib.cp_reorient(self.h), "cp_reorient")

    def commit(self):
        self._check(self.lib.cp_commit(self.h), "cp_commit")

    def field_width(self, name: str) -> int:
        return int(self.lib.cp_field_width(self.h, FIELDS[name]))

    def get_state(self, name: str) -> np.ndarray:
        w = self.field_width(name)
        buf = np.empty((self.n_qp, w))
        self._check(self.lib.cp_get_state(self.h, FIELDS[name], dptr(buf)), "cp_get_state")
        return buf

    def set_state(self, name: str, values):
        w = self.field_width(name)
        buf = as_f64(values, (self.n_qp, w))
        self._check(self.lib.cp_set_state(self.h, FIELDS[name], dptr(buf)), "cp_set_state")

    def synchronize(self):
        self._check(self.lib.cp_synchronize(self.h), "cp_synchronize")

    def stream(self) -> int:
        return int(self.lib.cp_stream(self.h) or 0)

    def set_timing(self, enable: bool):
        self._check(self.lib.cp_set_timing(self.h, 1 if enable else 0), "cp_set_timing")

    def autotune(self, in_ptr: int, path: int = CP_TUNE_UPDATE, reps: int = 3, min_gain: float = 0.02):
        """cp_autotune on device input (F for CP_TUNE_UPDATE, U_local for CP_TUNE_ASSEMBLE): one dict per
        lattice group with the shape chosen, the untuned default and the median ms of every shape."""
        res = (CpTuneResult * CP_MAX_LATTICES)()
        ng = self.lib.cp_autotune(self.h, C.c_void_p(in_ptr), path, reps, min_gain, res, CP_MAX_LATTICES)
        if ng < 0:
            self._check(ng, "cp_autotune")
        return [{"lattice": res[g].lattice, "n_qp": res[g].n_qp, "chosen": res[g].chosen,
                 "default": res[g].default_variant, "median_ms": list(res[g].median_ms)} for g in range(ng)]

    def contract_timing(self, kind: int):
        """(launches, total ms) of the timed element contractions: kind 0 FP64, 1 tensor-core."""
        a, b = C.c_int64(), C.c_double()
        self._check(self.lib.cp_get_contract_timing(self.h, kind, C.byref(a), C.byref(b)), "cp_get_contract_timing")
        return int(a.value), float(b.value)

    def graph_stats(self):
        """(graphs captured, graph launches) since the handle was created."""
        a, b = C.c_int64(), C.c_int64()
        self._check(self.lib.cp_graph_stats(self.h, C.byref(a), C.byref(b)), "cp_graph_stats")
        return int(a.value), int(b.value)

    def get_timing(self):
        """[(lattice, qp count, launches, total ms)] per internal group."""
        m = CP_MAX_LATTICES
        lat = np.zeros(m, np.int32)
        cnt = np.zeros(m, np.int64)
        lau = np.zeros(m, np.int64)
        ms = np.zeros(m)
        ng = self.lib.cp_get_timing(self.h, m, iptr(lat), cnt.ctypes.data_as(C.POINTER(C.c_int64)),
                                    lau.ctypes.data_as(C.POINTER(C.c_int64)), dptr(ms))
        if ng < 0:
            self._check(ng, "cp_get_timing")
        return [(int(lat[g]), int(cnt[g]), int(lau[g]), float(ms[g])) for g in range(ng)]


class CpBatch:
    """A cp_batch queue: the sorted updates of several handles on one device
    as shared launches (continuous batching of served requests)."""

    def __init__(self, device: int = 0, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        b = C.c_void_p()
        rc = self.lib.cp_batch_create(device, C.byref(b))
        if rc != CP_OK:
            raise CpError(f"cp_batch_create failed ({rc})")
        self.b = b

    def _run(self, fn, handles, F_e, F_r, what):
        n = len(handles)
        hs = (C.c_void_p * n)(*[h.h for h in handles])
        fe = np.ascontiguousarray(F_e, dtype=np.float64)
        fr = np.ascontiguousarray(F_r, dtype=np.float64)
        rc = fn(self.b, hs, n, dptr(fe), dptr(fr))
        if rc != CP_OK:
            msg = self.lib.cp_batch_last_error(self.b)
            raise CpError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def assemble(self, handles, F_e, F_r):
        self._run(self.lib.cp_batch_assemble, handles, F_e, F_r, "cp_batch_assemble")

    def post(self, handles, F_e, F_r):
        self._run(self.lib.cp_batch_post, handles, F_e, F_r, "cp_batch_post")

    def launches(self) -> int:
        return int(self.lib.cp_batch_launches(self.b))

    def close(self):
        if getattr(self, "b", None):
            self.lib.cp_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
