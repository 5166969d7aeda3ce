"""The served RVE stream on the GPU: requests of different sizes and
lattices solved concurrently (one handle and stream each) give the same
stress-strain rows as each solved alone."""
import numpy as np
import pytest

from plasticity_b200 import materials as M
from plasticity_b200 import serving as S

pytestmark = pytest.mark.gpu


def test_results_identical_alone_and_in_the_mix(cuda_lib):
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    reqs = S.request_stream(5, rate=0.0, seed=9, edges=(4, 5, 6), grains=(4, 12), increments=(3, 4),
                            norm=2e-3)
    assert len({r.lattice for r in reqs}) > 1 and len({r.edge for r in reqs}) > 1
    alone = S.RveServer(mats, budget_bytes=1 << 36, max_slots=1).run(reqs)
    srv = S.RveServer(mats, budget_bytes=1 << 36, max_slots=5)
    mixed = srv.run(reqs)
    assert srv.max_in_flight > 1
    for a, b in zip(alone, mixed):
        assert a.error is None and b.error is None, (a.error, b.error)
        assert a.converged and b.converged
        assert a.rows.shape == (reqs[a.rid].n_increments, 15)
        assert np.array_equal(a.rows, b.rows)
    assert any(np.abs(r.rows[-1, 14]) > 0 for r in mixed)  # plastic slip in the mix


def test_batched_serving_same_bits_as_one_at_a_time(cuda_lib):
    """Continuous batching (BatchedRveServer: the qp updates of every request
    in flight share launches) against the same requests solved one at a time
    without batching: the same stress-strain rows, bit for bit."""
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    reqs = S.request_stream(6, rate=0.0, seed=11, edges=(4, 5, 6), grains=(4, 12), increments=(3, 5),
                            norm=2e-3)
    assert len({r.lattice for r in reqs}) > 1 and len({r.edge for r in reqs}) > 1
    alone = S.RveServer(mats, budget_bytes=1 << 36, max_slots=1).run(reqs)
    srv = S.BatchedRveServer(mats, budget_bytes=1 << 36, max_slots=6)
    batched = srv.run(reqs)
    assert srv.max_in_flight > 1 and srv.batched_launches >= srv.ticks
    for a, b in zip(alone, batched):
        assert a.error is None and b.error is None, (a.error, b.error)
        assert a.converged and b.converged
        assert np.array_equal(a.rows, b.rows), a.rid
    assert any(np.abs(r.rows[-1, 14]) > 0 for r in batched)  # plastic slip in the mix


def test_admission_estimate_bounds_actual_device_memory(cuda_lib):
    """serving.device_bytes (the admission estimate) against the drop in the
    device's free memory that a request's set-up and first increment cause,
    after a warm-up request of the same lattice has loaded the kernels and
    the local-memory reservation."""
    import torch
    from plasticity_b200.capi import CpHandle, default_options, default_solver
    from plasticity_b200 import harness as H
    mats = [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]
    srv = S.RveServer(mats, budget_bytes=1 << 36, max_slots=1)
    warm = S.request_stream(1, rate=0.0, seed=3, edges=(4,), grains=(4, 5), increments=(2, 3))[0]
    warm.lattice = 1
    rows, conv = srv._device_solve(warm)
    assert conv
    for edge in (8, 12):
        req = S.request_stream(1, rate=0.0, seed=edge, edges=(edge,), grains=(8, 9), increments=(2, 3))[0]
        req.lattice = 1
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        mesh = H.StructuredMesh((edge, edge, edge))
        lid, rod = req.microstructure(mesh)
        be = CpHandle(mats, default_options())
        try:
            be.bind_qps(lid, rod)
            h = H.NewtonHarness(be, mesh, None, req.n_increments, 4, device_system=True,
                                solver=default_solver(), vel_grad=req.vel_grad, delT=req.delT)
            h.run(1)
            torch.cuda.synchronize()
            free1, _ = torch.cuda.mem_get_info(0)
        finally:
            be.close()
        used = free0 - free1
        est = srv.bytes_of(req)
        assert 0 < used <= est, (edge, used, est)
