"""The reference-order update on the GPU (cp_options_t.reference_order = 1,
the sm_100a build of plasticity_b200/csrc/cp_qpref.cuh compiled with
-fmad=false) against the oracle's parity build: the same bits at every qp --
P, T, dP/dF, the whole _iter history, the statistics and the status --
including the qps whose active-set solves have condition > 1e12, where the
optimised updates are compared to the oracle only in distribution.

Two states: a mixed FCC/BCC/HCP sample under random loading histories, and
the 8x8x8 FCC RVE driven to 2 % strain by the device Newton loop."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import CpHandle, default_options
from tests._parity import STATE_FIELDS, evolve, random_increment
from tests.test_reference_order import same_bits

pytestmark = pytest.mark.gpu

OUT_FIELDS = ("Fp_iter", "Fe_iter", "s_iter", "W_iter", "rot_iter", "rotnew_iter", "twinfrac_iter", "slipfrac_iter",
              "twin_iter")


@pytest.fixture(scope="module")
def parity_oracle(oracle_lib):
    prev = oracle_lib.use_library(oracle_lib.build_parity())
    yield oracle_lib
    oracle_lib.restore_library(prev)


def _set_state(dst, src_get):
    for f in STATE_FIELDS:
        for suf in ("_conv", "_iter"):
            dst.set_state(f + suf, src_get(f + suf))


def _mismatching_qps(gh, ob, F1, flag):
    """One update on both sides; the qps at which any output differs in a bit."""
    Pg, Tg, Dg, sg = gh.update(F1, flag)
    Po, To, Do, so = ob.update(F1, flag)
    bad = ~same_bits(Pg, Po).all(axis=1)
    bad |= ~same_bits(Tg, To).all(axis=1)
    if flag == 1:
        bad |= ~same_bits(Dg, Do).all(axis=1)
    bad |= sg != so
    stg, sto = gh.stats(), ob.stats()
    bad |= (stg[:, :6] != sto[:, :6]).any(axis=1)
    for f in OUT_FIELDS:
        a, b = gh.get_state(f), ob.get_state(f)
        bad |= ~same_bits(a.reshape(len(a), -1), b.reshape(len(b), -1)).all(axis=1)
    return bad, sto


def test_reference_order_same_bits_as_oracle_parity_mixed_lattices(cuda_lib, parity_oracle):
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    rng = np.random.default_rng(3)
    n = 12288
    lid = rng.permutation(np.repeat(np.arange(3, dtype=np.int32), [n // 2, 3 * n // 10, n - n // 2 - 3 * n // 10]))
    rod = M.random_rodrigues(rng, n)
    ob = parity_oracle.OracleBackend(mats, nthreads=0)
    ob.bind_qps(lid, rod)
    F = evolve(ob, np.tile(np.eye(3).ravel(), (n, 1)), rng, 10)
    gh = CpHandle(mats, default_options(reference_order=1))
    gh.bind_qps(lid, rod)
    _set_state(gh, ob.get_state)
    ill = 0
    for step in range(3):  # a short trajectory: each increment from the previous one's committed state
        F1 = random_increment(rng, F)
        bad, st = _mismatching_qps(gh, ob, F1, 1 if step != 1 else 0)
        assert not bad.any(), (step, np.flatnonzero(bad)[:10])
        ill += int((st[:, 7] > 12).sum())
        gh.commit()
        ob.commit()
        F = F1
    assert ill >= 20  # the comparison covers ill-conditioned active-set solves
    gh.close()


def test_reference_order_same_bits_at_rve_state(cuda_lib, parity_oracle):
    """The config-0 RVE (8x8x8 FCC Cu, one grain per element) pulled to 2 %
    by the device Newton loop (the sorted update), then one more increment of
    x-stretch evaluated in reference order on the GPU and by the oracle."""
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(0), mesh.n_cells), 8, axis=0)
    bc = np.array([[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.02]])
    lid = np.zeros(mesh.n_cells * 8, np.int32)
    loop = CpHandle([M.fcc_cu()], default_options())
    loop.bind_qps(lid, rod)
    H.NewtonHarness(loop, mesh, bc, 20, 4, device_system=True).run()
    gh = CpHandle([M.fcc_cu()], default_options(reference_order=1))
    gh.bind_qps(lid, rod)
    ob = parity_oracle.OracleBackend([M.fcc_cu()], nthreads=0)
    ob.bind_qps(lid, rod)
    _set_state(gh, loop.get_state)
    _set_state(ob, loop.get_state)
    Fe = loop.get_state("Fe_conv").reshape(-1, 3, 3)
    Fp = loop.get_state("Fp_conv").reshape(-1, 3, 3)
    loop.close()
    stretch = np.eye(3)
    stretch[0, 0] += 1e-3
    F1 = (stretch @ (Fe @ Fp)).reshape(-1, 9)
    bad, st = _mismatching_qps(gh, ob, F1, 1)
    assert not bad.any(), np.flatnonzero(bad)[:10]
    assert (st[:, 1] > 0).mean() > 0.5
    assert (st[:, 7] > 12).sum() >= 100  # hundreds of ill-conditioned qps at 2 % strain
    gh.close()
