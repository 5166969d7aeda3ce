"""FP64 parity of the CUDA path (through the C ABI) with the CPU oracle:
identical potentially-active and active slip sets at every qp, and P, T,
dP/dF and the history within 1e-10 relative per qp."""
import numpy as np
import pytest

from plasticity_b200 import materials as M
from plasticity_b200.capi import CP_QP_ERROR_MASK, CpHandle, default_options
from tests._parity import TOL, STATE_FIELDS, copy_state, evolve, make_pair, random_increment, rel_err, well_posed

pytestmark = pytest.mark.gpu

LATTICES = {"fcc": M.fcc_cu, "bcc": M.bcc_48, "hcp": M.hcp_mg}


def _compare_update(gh, ob, F, flag, F_e=0.0, F_r=0.0, min_well_posed=0.97):
    Pg, Tg, Dg, sg = gh.update(F, flag, F_e, F_r)
    Po, To, Do, so = ob.update(F, flag, F_e, F_r)
    stg, sto = gh.stats(), ob.stats()
    assert np.all((sg & CP_QP_ERROR_MASK) == 0), np.unique(sg)
    ok = well_posed(stg, sto)
    assert ok.mean() >= min_well_posed, ok.mean()
    # the potentially active set is formed before any solve: identical everywhere
    assert np.array_equal(stg[:, 0], sto[:, 0]), "potentially active set sizes differ"
    assert np.array_equal(stg[ok, 1], sto[ok, 1]), "active set sizes differ"
    assert np.array_equal(stg[ok, 2], sto[ok, 2]), "removal rounds differ"
    assert rel_err(Pg[ok], Po[ok]) < TOL
    assert rel_err(Tg[ok], To[ok]) < TOL
    if flag == 1:
        assert rel_err(Dg[ok], Do[ok]) < TOL
    for f in ("Fp_iter", "Fe_iter", "s_iter", "W_iter", "twinfrac_iter", "slipfrac_iter"):
        a, b = gh.get_state(f)[ok], ob.get_state(f)[ok]
        if np.abs(b).max() == 0:
            assert np.abs(a).max() == 0, f
        else:
            assert rel_err(a + 1.0, b + 1.0) < TOL, f  # fractions start at 0: compare on a shifted scale
    # the flag is raised exactly where the condition estimate says so
    assert np.array_equal((sg & 32) != 0, stg[:, 7] > 12)
    return stg


@pytest.mark.parametrize("lat", ["fcc", "bcc", "hcp"])
@pytest.mark.parametrize("flag", [0, 1])
def test_update_parity_single_lattice(oracle_lib, cuda_lib, lat, flag):
    n = 2048 if lat != "bcc" else 1024
    gh, ob, F, rng = make_pair(oracle_lib, [LATTICES[lat]()], np.zeros(n, np.int32), seed=11, steps=10)
    F1 = random_increment(rng, F)
    st = _compare_update(gh, ob, F1, flag)
    assert (st[:, 1] > 0).mean() > 0.3  # a real plastic workload
    gh.close()


def test_update_parity_mixed_lattices(oracle_lib, cuda_lib):
    """One handle, shuffled FCC/BCC/HCP qps (50/30/20) in the caller's order."""
    rng = np.random.default_rng(5)
    n = 3000
    lid = rng.choice(3, size=n, p=[0.5, 0.3, 0.2]).astype(np.int32)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    gh, ob, F, rng = make_pair(oracle_lib, mats, lid, seed=12, steps=10)
    _compare_update(gh, ob, random_increment(rng, F), 1)
    # stats carry the lattice id in caller order
    assert np.array_equal(gh.stats()[:, 6], lid)
    gh.close()


def test_trajectory_parity(oracle_lib, cuda_lib):
    """GPU and oracle evolve independently for 8 committed increments."""
    rng = np.random.default_rng(21)
    n = 1024
    lid = rng.choice(3, size=n).astype(np.int32)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    rod = M.random_rodrigues(rng, n)
    gh = CpHandle(mats)
    gh.bind_qps(lid, rod)
    ob = __import__("oracle.oracle", fromlist=["x"]).OracleBackend(mats, default_options())
    ob.bind_qps(lid, rod)
    F = np.tile(np.eye(3).ravel(), (n, 1))
    ok = np.ones(n, dtype=bool)  # qps whose every solve so far was well posed
    for step in range(8):
        F = random_increment(rng, F, 2e-4)
        Pg, _, Dg, _ = gh.update(F, 1)
        Po, _, Do, _ = ob.update(F, 1)
        ok &= well_posed(gh.stats(), ob.stats())
        assert np.array_equal(gh.stats()[ok, 1], ob.stats()[ok, 1]), step
        assert rel_err(Pg[ok], Po[ok]) < TOL and rel_err(Dg[ok], Do[ok]) < TOL, step
        gh.update(F, 0)
        ob.update(F, 0)
        ok &= well_posed(gh.stats(), ob.stats())
        gh.commit()
        ob.commit()
    assert ok.mean() > 0.95
    for f in ("Fp_conv", "s_conv"):
        assert rel_err(gh.get_state(f)[ok], ob.get_state(f)[ok]) < TOL
    gh.close()


@pytest.mark.parametrize("caps", [(2, 1), (1, 3), (3, 2)])
def test_general_caps_parity(oracle_lib, cuda_lib, caps):
    """Max Slip Search / Max Solver Iterations above the shipped value of 1."""
    opts = default_options(max_slip_search_iterations=caps[0], max_solver_iterations=caps[1])
    rng = np.random.default_rng(31)
    lid = rng.choice(2, size=1024).astype(np.int32)
    gh, ob, F, rng = make_pair(oracle_lib, [M.fcc_cu(), M.hcp_mg()], lid, seed=31, steps=6, opts=opts)
    _compare_update(gh, ob, random_increment(rng, F), 1)
    gh.close()


def test_twin_reorientation_parity(oracle_lib, cuda_lib):
    """HCP qps pushed past the twin threshold reorient identically."""
    mats = [M.hcp_mg(twin_threshold=0.05)]
    n = 512
    gh, ob, F, rng = make_pair(oracle_lib, mats, np.zeros(n, np.int32), seed=41, steps=4)
    tw = ob.get_state("twinfrac_conv")
    tw[: n // 2, 2] += 0.2  # half the qps above the threshold on twin system 2
    for be in (gh, ob):
        be.set_state("twinfrac_conv", tw)
        be.set_state("twinfrac_iter", tw)
    F1 = random_increment(rng, F)
    st = _compare_update(gh, ob, F1, 1, F_e=0.01, F_r=0.05)
    ok = well_posed(st, ob.stats())
    tg, to = gh.get_state("twin_iter"), ob.get_state("twin_iter")
    assert np.array_equal(tg[ok], to[ok]) and tg.sum() > 0
    assert rel_err(gh.get_state("rot_iter")[ok], ob.get_state("rot_iter")[ok]) < TOL
    assert rel_err(gh.get_state("rotnew_iter")[ok], ob.get_state("rotnew_iter")[ok]) < TOL
    gh.close()


def test_reorient_and_commit_parity(oracle_lib, cuda_lib):
    rng = np.random.default_rng(51)
    lid = rng.choice(3, size=777).astype(np.int32)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    gh, ob, F, rng = make_pair(oracle_lib, mats, lid, seed=51, steps=5)
    F1 = random_increment(rng, F)
    gh.update(F1, 0)
    ob.update(F1, 0)
    ok = well_posed(gh.stats(), ob.stats())
    gh.reorient()
    ob.reorient()
    assert rel_err(gh.get_state("rotnew_conv")[ok], ob.get_state("rotnew_conv")[ok]) < TOL
    gh.commit()
    ob.commit()
    for f in STATE_FIELDS:
        a, b = gh.get_state(f + "_conv")[ok], ob.get_state(f + "_conv")[ok]
        assert rel_err(a + 1.0, b + 1.0) < TOL, f
        assert np.array_equal(gh.get_state(f + "_conv"), gh.get_state(f + "_iter")), f
    gh.close()


def test_elastic_identity_and_edge_sizes(oracle_lib, cuda_lib):
    """F = I from the initial state: zero stress, elastic tangent; qp counts
    that are not multiples of the block size; a single qp."""
    for n in (1, 7, 129):
        mats = [M.fcc_cu()]
        gh = CpHandle(mats)
        rod = M.random_rodrigues(np.random.default_rng(n), n)
        gh.bind_qps(np.zeros(n, np.int32), rod)
        ob = __import__("oracle.oracle", fromlist=["x"]).OracleBackend(mats)
        ob.bind_qps(np.zeros(n, np.int32), rod)
        F = np.tile(np.eye(3).ravel(), (n, 1))
        Pg, Tg, Dg, sg = gh.update(F, 1)
        Po, To, Do, so = ob.update(F, 1)
        assert np.abs(Pg).max() < 1e-9
        assert rel_err(Dg, Do) < TOL
        assert np.all(gh.stats()[:, 1] == 0)
        gh.close()


def test_nonfinite_input_is_flagged(cuda_lib):
    gh = CpHandle([M.fcc_cu()])
    gh.bind_qps(np.zeros(4, np.int32), np.zeros((4, 3)))
    F = np.tile(np.eye(3).ravel(), (4, 1))
    F[2, 0] = np.nan
    _, _, _, st = gh.update(F, 1)
    assert st[2] & 1 and np.all(st[[0, 1, 3]] & 1 == 0)
    gh.close()


def test_determinism(oracle_lib, cuda_lib):
    gh, ob, F, rng = make_pair(oracle_lib, [M.bcc_48()], np.zeros(512, np.int32), seed=61, steps=6)
    F1 = random_increment(rng, F)
    s0 = {f: gh.get_state(f) for f in ("Fp_conv", "s_conv")}
    a = gh.update(F1, 1)
    b = gh.update(F1, 1)  # conv state unchanged by update: same inputs, same bytes
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    for f, v in s0.items():
        assert np.array_equal(gh.get_state(f), v)
    gh.close()


def test_api_errors(cuda_lib):
    from plasticity_b200.capi import CpError
    gh = CpHandle([M.fcc_cu()])
    with pytest.raises(CpError):
        gh.n_qp = 3
        gh.update(np.zeros((3, 9)), 1)  # nothing bound yet
    with pytest.raises(CpError):
        gh.bind_qps(np.array([0, 5], np.int32), np.zeros((2, 3)))  # lattice id out of range
    gh.close()


def test_ill_conditioned_blocks_are_flagged(oracle_lib, cuda_lib):
    """A large first increment from the annealed state makes many FCC A_PA
    blocks numerically singular: both sides flag them (condition > 1e12),
    and every unflagged qp still matches."""
    mats = [M.fcc_cu()]
    n = 512
    rng = np.random.default_rng(71)
    rod = M.random_rodrigues(rng, n)
    gh = CpHandle(mats)
    gh.bind_qps(np.zeros(n, np.int32), rod)
    ob = __import__("oracle.oracle", fromlist=["x"]).OracleBackend(mats)
    ob.bind_qps(np.zeros(n, np.int32), rod)
    F = (np.eye(3) + 3e-3 * rng.standard_normal((n, 3, 3))).reshape(n, 9)
    st = _compare_update(gh, ob, F, 1, min_well_posed=0.0)
    flagged = ~well_posed(st, ob.stats())
    assert flagged.sum() > n // 4
    # the two condition estimates agree on which blocks are singular (SVD on
    # the oracle side, LU pivots on the GPU): at least 95 % agreement
    agree = np.mean((st[:, 7] > 12) == (ob.stats()[:, 7] > 12))
    assert agree > 0.95, agree
    gh.close()


def test_ill_conditioned_qps_agree_in_distribution(oracle_lib, cuda_lib):
    """At qps whose active-set solves are ill conditioned the reference's own
    result is set by rounding: the oracle compiled with fused multiply-adds
    (another valid rounding of the same arithmetic) ends some of them with
    other active sets and about a tenth of them with stresses apart by 1e-6
    to tens of percent (2^15 qps: 253 ill conditioned, 16 other active sets,
    25 such stresses).  The GPU's shipped update must stay inside that spread: on a
    mixed-lattice sample, at the ill-conditioned qps, no more active-set
    mismatches against the oracle, no more stress outliers and no larger
    difference in the histogram of final active-set sizes than about twice the
    oracle's against itself, and the sample's summed stress as close."""
    n = 1 << 15
    rng = np.random.default_rng(23)
    lid = rng.choice(3, size=n, p=[0.5, 0.3, 0.2]).astype(np.int32)
    gh, ob, F, rng = make_pair(oracle_lib, [M.fcc_cu(), M.bcc_48(), M.hcp_mg()], lid, seed=23, steps=10)
    F1 = random_increment(rng, F)
    state = {f + s: ob.get_state(f + s) for f in STATE_FIELDS for s in ("_conv", "_iter")}
    Pg, _, _, sg = gh.update(F1, 1)
    stg = gh.stats()
    Po, _, _, _ = ob.update(F1, 1)
    sto = ob.stats().copy()
    prev = oracle_lib.use_library(oracle_lib.build_fma())
    try:
        for k, v in state.items():
            ob.set_state(k, v)
        Pf, _, _, _ = ob.update(F1, 1)
        stf = ob.stats().copy()
    finally:
        oracle_lib.restore_library(prev)
    assert np.all((sg & CP_QP_ERROR_MASK) == 0)
    ill = ~well_posed(stg, sto, stf)
    assert ill.sum() >= 100, ill.sum()

    def spread(P, st):
        per_qp = np.abs(P - Po).max(axis=1) / np.maximum(np.abs(Po).max(axis=1), 1e-300)
        return {"mismatches": int((~np.all(st[:, :3] == sto[:, :3], axis=1))[ill].sum()),
                "outliers": int((per_qp[ill] > 1e-6).sum()),
                "histogram": int(np.abs(np.bincount(st[ill, 1], minlength=64)[:64]
                                        - np.bincount(sto[ill, 1], minlength=64)[:64]).sum()),
                "summed": float(np.abs(P - Po).sum() / np.abs(Po).sum())}

    g, f = spread(Pg, stg), spread(Pf, stf)
    print(f"ill-conditioned qps {int(ill.sum())} of {n}: GPU vs oracle {g}; oracle FMA build vs oracle {f}")
    for k in ("mismatches", "outliers", "histogram"):
        assert g[k] <= 2 * f[k] + 10, (k, g, f)
    assert g["summed"] <= 3 * f["summed"] + 1e-4, (g, f)
    # and the well-posed qps of the same sample meet the parity bar
    ok = ~ill
    assert np.array_equal(stg[ok, :3], sto[ok, :3]) and rel_err(Pg[ok], Po[ok]) < TOL
    gh.close()


@pytest.mark.parametrize("n", [(1 << 18) + 777, (1 << 20) + 123])
def test_chunked_host_update_matches_device_update(cuda_lib, n):
    """cp_update with host buffers runs in caller-order chunks (2 above 2^18
    qps, 4 above 2^20) whose copies overlap the other chunks' kernels; each
    qp's update is independent, so its outputs must equal the unchunked
    device-pointer call's bit for bit."""
    import torch
    rng = np.random.default_rng(71)
    lid = rng.choice(3, size=n, p=[0.5, 0.3, 0.2]).astype(np.int32)
    gh = CpHandle([M.fcc_cu(), M.bcc_48(), M.hcp_mg()])
    gh.bind_qps(lid, M.random_rodrigues(rng, n))
    F = np.tile(np.eye(3).ravel(), (n, 1))
    F = evolve(gh, F, rng, 3)
    F1 = random_increment(rng, F)
    P, T, D, st = gh.update(F1, 1)
    s_host = gh.stats()
    dev = torch.device("cuda", 0)
    Fd = torch.from_numpy(F1).to(dev)
    Pd = torch.empty(n, 9, dtype=torch.float64, device=dev)
    Td = torch.empty(n, 9, dtype=torch.float64, device=dev)
    Dd = torch.empty(n, 81, dtype=torch.float64, device=dev)
    Sd = torch.empty(n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    gh.update_device(Fd.data_ptr(), 1, 0.0, 0.0, Pd.data_ptr(), Td.data_ptr(), Dd.data_ptr(), Sd.data_ptr())
    gh.synchronize()
    assert np.array_equal(P, Pd.cpu().numpy())
    assert np.array_equal(T, Td.cpu().numpy())
    assert np.array_equal(D, Dd.cpu().numpy())
    assert np.array_equal(st, Sd.cpu().numpy())
    assert np.array_equal(s_host, gh.stats())
    assert (s_host[:, 1] > 0).mean() > 0.3  # a plastic workload
    gh.close()
