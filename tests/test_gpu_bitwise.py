"""The plain FP64 drop-in kernel (cp_options_t.plain_kernel = 1: one thread
per qp in bind order) and the shipped sorted pipeline give the same bits:
P, T, dP/dF, status, work statistics and every history field, on a sample of
the batched mixed-lattice workload, ill-conditioned active-set solves
included; the same for the fused assembly's Ke/Re and for the whole device
Newton loop of the 8x8x8 FCC RVE.  Also: graph replay, every launch shape and
the autotuner change no bit."""
import numpy as np
import pytest

from plasticity_b200 import harness as H
from plasticity_b200 import materials as M
from plasticity_b200.capi import (CP_TUNE_ASSEMBLE, CP_TUNE_UPDATE, CP_UPDATE_VARIANTS, CpHandle, default_options)
from tests._parity import STATE_FIELDS

pytestmark = pytest.mark.gpu

ITER_FIELDS = [f + "_iter" for f in STATE_FIELDS]


def _mixed_workload(n, seed=1, steps=10, amp=2e-4):
    """n shuffled qps 50/30/20 FCC/BCC/HCP with a history of 'steps' committed
    increments F <- F (I + amp G) built on the GPU (sorted pipeline)."""
    rng = np.random.default_rng(seed)
    lid = rng.choice(3, size=n, p=[0.5, 0.3, 0.2]).astype(np.int32)
    rod = M.random_rodrigues(rng, n)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    h = CpHandle(mats, default_options())
    h.bind_qps(lid, rod)
    F = np.tile(np.eye(3).ravel(), (n, 1))
    for _ in range(steps):
        F = (F.reshape(-1, 3, 3) @ (np.eye(3) + amp * rng.standard_normal((n, 3, 3)))).reshape(-1, 9)
        h.update(F, 0)
        h.commit()
    F = (F.reshape(-1, 3, 3) @ (np.eye(3) + amp * rng.standard_normal((n, 3, 3)))).reshape(-1, 9)
    return h, mats, lid, rod, F


def _clone(src, mats, lid, rod, **opts):
    h = CpHandle(mats, default_options(**opts))
    h.bind_qps(lid, rod)
    for f in STATE_FIELDS:
        for suf in ("_conv", "_iter"):
            h.set_state(f + suf, src.get_state(f + suf))
    return h


def _same(a, b, what):
    assert np.array_equal(a, b), f"{what}: {np.count_nonzero(a != b)} entries differ"


def _assert_same_update(ha, hb, F, flag):
    ra, rb = ha.update(F, flag), hb.update(F, flag)
    for name, x, y in zip(("P", "T", "dPdF", "status"), ra, rb):
        if x is not None:
            _same(x, y, name)
    _same(ha.stats(), hb.stats(), "stats")
    for f in ITER_FIELDS:
        _same(ha.get_state(f), hb.get_state(f), f)
    return ha.stats()


@pytest.mark.parametrize("flag", [1, 0])
def test_plain_and_sorted_update_bit_identical(cuda_lib, flag):
    hs, mats, lid, rod, F = _mixed_workload(1 << 15)
    hp = _clone(hs, mats, lid, rod, plain_kernel=1)
    st = _assert_same_update(hp, hs, F, flag)
    assert (st[:, 1] > 0).mean() > 0.5  # mostly plastic
    if flag == 1:
        assert (st[:, 7] > 12).sum() > 20  # ill-conditioned active-set solves are in the sample and agree too
    hs.close()
    hp.close()


def test_plain_and_sorted_assembly_bit_identical(cuda_lib):
    mesh = H.StructuredMesh((6, 6, 6))
    rng = np.random.default_rng(3)
    lid = np.repeat(rng.choice(3, size=mesh.n_cells, p=[0.5, 0.3, 0.2]), 8).astype(np.int32)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    hs = CpHandle(mats, default_options())
    hs.bind_qps(lid, rod)
    hp = CpHandle(mats, default_options(plain_kernel=1))
    hp.bind_qps(lid, rod)
    u = np.zeros(mesh.n_dofs)
    for be in (hs, hp):
        be.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    for _ in range(6):  # a few committed increments of macroscopic stretch with noise
        u = u + (mesh.node_xyz @ (1e-3 * np.diag([1.0, -0.3, -0.3]) + 2e-4 * rng.standard_normal((3, 3))).T).ravel()
        for be in (hs, hp):
            be.assemble(u[mesh.cell_dofs])
            be.commit()
    Ks, Rs, ss = hs.assemble(u[mesh.cell_dofs])
    Kp, Rp, sp = hp.assemble(u[mesh.cell_dofs])
    _same(Ks, Kp, "Ke")
    _same(Rs, Rp, "Re")
    _same(ss, sp, "status")
    assert (hs.stats()[:, 1] > 0).mean() > 0.5
    hs.close()
    hp.close()


def test_rve_device_loop_plain_and_sorted_bit_identical(cuda_lib):
    """The 8x8x8 FCC RVE of the RVE measurement, first 6 increments, device
    Newton loop (the same BiCG) with the plain kernel and with the sorted one:
    the stress-strain rows and the final displacement are the same bits,
    although the run crosses yield and creates ill-conditioned solves."""
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(0), mesh.n_cells), 8, axis=0)
    bc = np.array([[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.02]])
    out = []
    for plain in (1, 0):
        be = CpHandle([M.fcc_cu()], default_options(plain_kernel=plain))
        be.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), rod)
        h = H.NewtonHarness(be, mesh, bc, 20, 4, device_system=True)
        rows = h.run(6)
        out.append((rows, h.u.copy(), be.stats()))
        be.close()
    (rp, up, sp), (rs, us, ss) = out
    _same(rp, rs, "stress-strain rows")
    _same(up, us, "displacement")
    assert np.abs(rs[:, 6]).max() > 20.0  # MPa: past yield


def test_graphs_shapes_and_tuning_change_no_bit(cuda_lib):
    import torch
    hs, mats, lid, rod, F = _mixed_workload(1 << 14, seed=4)
    ref = _clone(hs, mats, lid, rod, use_graphs=0)
    Pr, Tr, Dr, sr = ref.update(F, 1)
    n = len(lid)
    dev = torch.device("cuda", 0)
    dF = torch.from_numpy(F).to(dev)
    dP = torch.empty(n, 9, dtype=torch.float64, device=dev)
    dD = torch.empty(n, 81, dtype=torch.float64, device=dev)
    dS = torch.empty(n, dtype=torch.int32, device=dev)
    g = _clone(hs, mats, lid, rod, use_graphs=1)
    c0, l0 = g.graph_stats()
    for _ in range(3):
        g.update_device(dF.data_ptr(), 1, 0.0, 0.0, dP.data_ptr(), None, dD.data_ptr(), dS.data_ptr())
    g.synchronize()
    c1, l1 = g.graph_stats()
    assert c1 - c0 == 1 and l1 - l0 == 3  # captured once, replayed
    _same(dP.cpu().numpy(), Pr, "P (graph)")
    _same(dD.cpu().numpy(), Dr, "dPdF (graph)")
    res = g.autotune(dF.data_ptr(), CP_TUNE_UPDATE, reps=2)
    assert len(res) == 3 and all(0 <= r["chosen"] < CP_UPDATE_VARIANTS for r in res)
    assert all(min(r["median_ms"]) > 0 for r in res)
    g.update_device(dF.data_ptr(), 1, 0.0, 0.0, dP.data_ptr(), None, dD.data_ptr(), dS.data_ptr())
    g.synchronize()
    assert g.graph_stats()[0] == c1 + 1  # re-captured with the tuned shapes
    _same(dP.cpu().numpy(), Pr, "P (tuned)")
    _same(dD.cpu().numpy(), Dr, "dPdF (tuned)")
    for v in range(1, CP_UPDATE_VARIANTS + 1):
        hv = _clone(hs, mats, lid, rod, update_variant=v)
        P, T, D, s = hv.update(F, 1)
        _same(P, Pr, f"P (shape {v - 1})")
        _same(D, Dr, f"dPdF (shape {v - 1})")
        hv.close()
    for x in (hs, ref, g):
        x.close()


def test_autotune_assembly_path(cuda_lib):
    import torch
    mesh = H.StructuredMesh((4, 4, 4))
    rng = np.random.default_rng(8)
    rod = np.repeat(M.random_rodrigues(rng, mesh.n_cells), 8, axis=0)
    be = CpHandle([M.fcc_cu()], default_options())
    be.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), rod)
    be.bind_mesh(mesh.n_cells, mesh.grad_N, mesh.JxW, True)
    u = (mesh.node_xyz @ (3e-3 * rng.standard_normal((3, 3))).T).ravel()
    Ul = u[mesh.cell_dofs]
    K0, R0, _ = be.assemble(Ul)
    dU = torch.from_numpy(np.ascontiguousarray(Ul)).cuda()
    res = be.autotune(dU.data_ptr(), CP_TUNE_ASSEMBLE, reps=2)
    assert len(res) == 1 and res[0]["n_qp"] == mesh.n_cells * 8
    K1, R1, _ = be.assemble(Ul)
    _same(K1, K0, "Ke after tuning")
    _same(R1, R0, "Re after tuning")
    be.close()


def test_reordered_history_gives_the_same_bits(cuda_lib):
    """cp_commit permutes a sorted handle's history into the order of its last
    sort (the plain handle keeps bind order).  Over several committed
    increments of the host call, which at this size runs in two caller-order
    chunks (of qps and, for the mesh-bound calls, of cells: the reorder keeps
    within the segments they bound), P, dP/dF, status, statistics, every
    history field in caller order and the volume averages stay the plain
    drop-in's bits."""
    n = (1 << 18) + 4096
    rng = np.random.default_rng(23)
    lid = np.repeat(rng.choice(3, size=n // 8, p=[0.5, 0.3, 0.2]), 8).astype(np.int32)  # one lattice per cell
    rod = M.random_rodrigues(rng, n)
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    hs = CpHandle(mats, default_options())
    hp = CpHandle(mats, default_options(plain_kernel=1))
    cell = H.StructuredMesh((1, 1, 1))  # every cell the unit cube's (the averages weigh by JxW)
    for h in (hs, hp):
        h.bind_qps(lid, rod)
        h.bind_mesh(n // 8, cell.grad_N, cell.JxW, True)
    F = np.tile(np.eye(3).ravel(), (n, 1))
    for inc in range(4):
        F = (F.reshape(-1, 3, 3) @ (np.eye(3) + 3e-4 * rng.standard_normal((n, 3, 3)))).reshape(-1, 9)
        _assert_same_update(hs, hp, F, 1)
        _assert_same_update(hs, hp, F, 0)
        _same(hs.averages(), hp.averages(), f"averages (increment {inc})")
        for h in (hs, hp):
            h.commit()
        for f in STATE_FIELDS:
            _same(hs.get_state(f + "_conv"), hp.get_state(f + "_conv"), f + "_conv")
    for h in (hs, hp):
        h.close()
