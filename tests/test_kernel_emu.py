"""The CUDA qp kernel source compiled for the host and run against the
oracle: the optimised update (plasticity_b200/csrc/cp_qp2.cuh, qp_update2)
and the plain form (cp_qp.cuh, qp_update; cp_options_t.plain_kernel).  Checks
the device code path's logic in the CPU suite (the GPU tests check the
compiled sm_100a build)."""
import numpy as np
import pytest

from plasticity_b200 import materials as M
from tests._parity import TOL, copy_state, evolve, random_increment, rel_err, well_posed


@pytest.fixture(scope="module")
def emu():
    from tests.kernel_emu import emu as E
    E.lib()
    return E


@pytest.mark.parametrize("variant", [0, 1], ids=["qp_update2", "qp_update_plain"])
@pytest.mark.parametrize("lat", ["fcc", "bcc", "hcp"])
def test_kernel_source_matches_oracle(oracle_lib, emu, lat, variant):
    emu.lib().emu_set_variant(variant)
    mat = {"fcc": M.fcc_cu, "bcc": M.bcc_48, "hcp": M.hcp_mg}[lat]()
    rng = np.random.default_rng(5)
    n = 400
    rod = M.random_rodrigues(rng, n)
    ob = oracle_lib.OracleBackend([mat])
    ob.bind_qps(np.zeros(n, np.int32), rod)
    F = evolve(ob, np.tile(np.eye(3).ravel(), (n, 1)), rng, 8)
    eb = emu.EmuBackend([mat])
    eb.bind_qps(np.zeros(n, np.int32), rod)
    copy_state(ob, eb)
    F1 = random_increment(rng, F)
    Po, To, Do, so = ob.update(F1, 1)
    Pe, Te, De, se = eb.update(F1, 1)
    ok = well_posed(ob.stats(), eb.stats())
    assert ok.mean() > 0.95
    assert np.array_equal(ob.stats()[:, 0], eb.stats()[:, 0])
    assert np.array_equal(ob.stats()[ok, :3], eb.stats()[ok, :3])
    assert rel_err(Pe[ok], Po[ok]) < TOL and rel_err(De[ok], Do[ok]) < TOL
    for f in ("Fp_iter", "s_iter"):
        assert rel_err(eb.get_state(f)[ok], ob.get_state(f)[ok]) < TOL
    emu.lib().emu_set_variant(0)


def test_kernel_source_general_caps(oracle_lib, emu):
    from plasticity_b200.capi import default_options
    opts = default_options(max_slip_search_iterations=3, max_solver_iterations=2)
    mat = M.hcp_mg()
    rng = np.random.default_rng(6)
    n = 300
    rod = M.random_rodrigues(rng, n)
    ob = oracle_lib.OracleBackend([mat], opts)
    ob.bind_qps(np.zeros(n, np.int32), rod)
    F = evolve(ob, np.tile(np.eye(3).ravel(), (n, 1)), rng, 6)
    eb = emu.EmuBackend([mat], opts)
    eb.bind_qps(np.zeros(n, np.int32), rod)
    copy_state(ob, eb)
    F1 = random_increment(rng, F)
    Po, _, Do, _ = ob.update(F1, 1)
    Pe, _, De, _ = eb.update(F1, 1)
    ok = well_posed(ob.stats(), eb.stats())
    assert ok.mean() > 0.95
    assert (ob.stats()[:, 5] > 2).any()  # more than one slip-search pass happened
    assert rel_err(Pe[ok], Po[ok]) < TOL and rel_err(De[ok], Do[ok]) < TOL


def _lu_cases(rng):
    """Dense, graded, rank-deficient, zero-column and zero-row matrices of the
    sizes the removal solves and the tangent solve see (1..48)."""
    for m in list(range(1, 13)) + [15, 16, 23, 31, 32, 47, 48]:
        yield m, rng.standard_normal((m, m))
        yield m, rng.standard_normal((m, m)) * np.logspace(0, 12, m)[None, :]
        if m > 1:
            A = rng.standard_normal((m, m))
            A[:, rng.integers(m)] = 0.0  # zero column: flagged singular, step skipped
            yield m, A
            A = rng.standard_normal((m, m))
            A[rng.integers(m)] = 0.0
            yield m, A
            A = rng.standard_normal((m, m))
            A[:, -1] = A[:, 0]  # rank deficient: exact cancellation in the last pivot
            yield m, A
            A = rng.standard_normal((m, m))
            A[:, 1] = 0.0  # the second step of a pair is the zero column
            yield m, A
        A = np.where(rng.random((m, m)) < 0.6, 0.0, rng.standard_normal((m, m)))  # sparse: zero multipliers
        yield m, A


@pytest.mark.parametrize("pair", [0, 1], ids=["one_step", "paired_steps"])
@pytest.mark.parametrize("nrhs", [1, 9])
def test_batched_lu_bit_identical_to_plain(emu, nrhs, pair):
    import ctypes as C
    rng = np.random.default_rng(11)
    D = C.POINTER(C.c_double)
    n = 0
    for m, A in _lu_cases(rng):
        ld = 48
        Ap = np.zeros((m, ld))
        Ap[:, :m] = A
        Ap = np.ascontiguousarray(Ap)
        B = np.ascontiguousarray(rng.standard_normal((m, nrhs)))
        ok = emu.lib().emu_lu_compare(Ap.ctypes.data_as(D), B.ctypes.data_as(D), m, ld, nrhs, pair)
        assert ok == 1, (m, nrhs, n)
        n += 1
    assert n > 100
