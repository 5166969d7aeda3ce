"""The reference-order update (cp_options_t.reference_order,
plasticity_b200/csrc/cp_qpref.cuh) against the oracle's parity build on the
CPU: the kernel source compiled for the host computes, at every qp, the same
bits as the oracle -- P, T, dP/dF, the whole _iter history, the statistics
and the status -- ill-conditioned qps (active-set solves with condition
> 1e12, where the optimised updates and the oracle part ways) included.

The parity build differs from the default oracle only in pow, the Gateaux
factorials and the twin rotation's cos(atan(.)), which it takes from
correctly rounded operations (oracle/cp_oracle.cpp, CP_ORACLE_PARITY); the
GPU test (tests/test_gpu_reference_order.py) checks the sm_100a build the same
way."""
import math

import numpy as np
import pytest

from plasticity_b200 import materials as M
from tests._parity import copy_state, evolve, random_increment


def same_bits(a, b):
    """Elementwise: identical bit patterns, or both NaN."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return (a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))


@pytest.fixture(scope="module")
def parity_oracle(oracle_lib):
    prev = oracle_lib.use_library(oracle_lib.build_parity())
    yield oracle_lib
    oracle_lib.restore_library(prev)


@pytest.fixture(scope="module")
def emu():
    from tests.kernel_emu import emu as E
    E.lib()
    return E


def test_ref_pow_same_bits_as_oracle_parity_pow(parity_oracle, emu):
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.random(20000), rng.random(5000) * 1e-3, 1 - rng.random(5000) * 1e-6,
                        rng.random(2000) * 50, [0.0, 1.0, 0.5, 2.0, -0.5, -2.0, np.inf, np.nan, 1e-300]])
    y = np.concatenate([rng.random(12000) * 4 - 2, rng.integers(-3, 4, 10000).astype(float),
                        rng.random(10000) * 0.3, [0.0, 1.0, -1.0, 2.0, 0.5, 3.0, -0.5, np.nan, 1.0]])
    L, E = parity_oracle.lib(), emu.lib()
    bad = 0
    worst = 0.0
    for xi, yi in zip(x, y):
        a = L.oracle_parity_pow(float(xi), float(yi))
        b = E.emu_ref_pow(float(xi), float(yi))
        if not same_bits(np.array([a]), np.array([b]))[0]:
            bad += 1
        if xi > 0 and np.isfinite(xi) and np.isfinite(yi):
            ref = math.pow(xi, yi)
            if ref != 0.0 and np.isfinite(ref) and abs(yi * math.log(xi)) < 5:
                worst = max(worst, abs(a - ref) / abs(ref))
    assert bad == 0
    assert worst < 2e-15  # a few ulp of math.pow where |y ln x| < 5


@pytest.mark.parametrize("lat, steps, amp", [("fcc", 10, 4e-4), ("bcc", 8, 3e-4), ("hcp", 8, 3e-4)])
def test_reference_order_source_same_bits_as_oracle_parity_build(parity_oracle, emu, lat, steps, amp):
    mat = {"fcc": M.fcc_cu(), "bcc": M.bcc_48(), "hcp": M.hcp_mg()}[lat]
    rng = np.random.default_rng(21)
    n = 240 if lat == "bcc" else 320
    rod = M.random_rodrigues(rng, n)
    ob = parity_oracle.OracleBackend([mat])
    ob.bind_qps(np.zeros(n, np.int32), rod)
    F = evolve(ob, np.tile(np.eye(3).ravel(), (n, 1)), rng, steps, amp)
    eb = emu.EmuBackend([mat])
    eb.bind_qps(np.zeros(n, np.int32), rod)
    copy_state(ob, eb)
    F1 = random_increment(rng, F, amp)
    emu.lib().emu_set_variant(2)
    try:
        Po, To, Do, so = ob.update(F1, 1)
        Pe, Te, De, se = eb.update(F1, 1)
    finally:
        emu.lib().emu_set_variant(0)
    st_o, st_e = ob.stats(), eb.stats()
    assert (st_o[:, 1] > 0).mean() > 0.5  # mostly plastic
    if lat != "hcp":  # the FCC and BCC samples hold ill-conditioned active-set solves
        assert (st_o[:, 7] > 12).sum() >= 5
    for name, a, b in (("P", Pe, Po), ("T", Te, To), ("dPdF", De, Do)):
        assert same_bits(a, b).all(), name
    assert np.array_equal(se, so)
    assert np.array_equal(st_e[:, :6], st_o[:, :6])
    assert np.abs(st_e[:, 7] - st_o[:, 7]).max() <= 1
    for f in ("Fp_iter", "Fe_iter", "s_iter", "W_iter", "rot_iter", "rotnew_iter", "twinfrac_iter",
              "slipfrac_iter", "twin_iter"):
        assert same_bits(eb.get_state(f), ob.get_state(f)).all(), f
