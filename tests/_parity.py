"""Helpers shared by the GPU parity tests: seeded random loading histories
driven through the CPU oracle, state transfer oracle -> GPU, and the
per-qp relative error used for the FP64 parity bar (1e-10)."""
import numpy as np

from plasticity_b200 import materials as M

TOL = 1e-10  # FP64 parity bar for stresses, tangents and history (relative, per qp)
COND_MAX_EXP = 12  # active-set solves with condition > 1e12 are ill-posed (see well_posed)

STATE_FIELDS = ["Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac", "slipfrac", "twin"]


def rel_err(a, b, floor=1e-300):
    """max over qps of |a_k - b_k|_inf / |b_k|_inf."""
    a = np.asarray(a, float).reshape(len(a), -1)
    b = np.asarray(b, float).reshape(len(b), -1)
    num = np.abs(a - b).max(axis=1)
    den = np.maximum(np.abs(b).max(axis=1), floor)
    return float((num / den).max()) if len(a) else 0.0


def random_increment(rng, F, amp=2e-4):
    G = rng.standard_normal((len(F), 3, 3))
    return (F.reshape(-1, 3, 3) @ (np.eye(3) + amp * G)).reshape(-1, 9)


def evolve(be, F, rng, steps, amp=2e-4, flag=0, F_e=0.0, F_r=0.0):
    """'steps' increments of F_new = F (I + amp G), each committed."""
    for _ in range(steps):
        F = random_increment(rng, F, amp)
        be.update(F, flag, F_e, F_r)
        be.commit()
    return F


def copy_state(src, dst):
    for f in STATE_FIELDS:
        for suf in ("_conv", "_iter"):
            dst.set_state(f + suf, src.get_state(f + suf))


def make_pair(oracle_lib, mats, lattice_id, seed, steps, opts=None, amp=2e-4):
    """A GPU handle and an oracle backend holding the same evolved state."""
    from plasticity_b200.capi import CpHandle, default_options
    opts = opts or default_options()
    rng = np.random.default_rng(seed)
    lattice_id = np.asarray(lattice_id, np.int32)
    rod = M.random_rodrigues(rng, len(lattice_id))
    ob = oracle_lib.OracleBackend(mats, opts, nthreads=0)
    ob.bind_qps(lattice_id, rod)
    F = np.tile(np.eye(3).ravel(), (len(lattice_id), 1))
    F = evolve(ob, F, rng, steps, amp)
    gh = CpHandle(mats, opts)
    gh.bind_qps(lattice_id, rod)
    copy_state(ob, gh)
    return gh, ob, F, rng


def well_posed(*stats):
    """qps whose active-set solves were well conditioned (condition <= 1e12)
    on every side compared.  Above that, the reference's
    compute_inverse_svd(0.0) solution is set by rounding noise (A_PA is
    numerically singular: for FCC both the latent-hardening part and the
    Schmid part of A have rank <= 5), so no two implementations agree; those
    qps are flagged CP_QP_ILL_CONDITIONED and counted instead."""
    m = np.ones(len(stats[0]), dtype=bool)
    for s in stats:
        m &= np.asarray(s)[:, 7] <= COND_MAX_EXP
    return m
