"""The RVE server's host logic (admission by device-memory budget and slot
count, oldest first, rejection of oversize requests, latency accounting)
with a stand-in solve; the device solve alone and in a mix is in
tests/test_gpu_serving.py."""
import time

import numpy as np

from plasticity_b200 import materials as M
from plasticity_b200 import serving as S


def _mats():
    return [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]


class _FakeSolve:
    def __init__(self, seconds=0.05):
        self.seconds = seconds
        self.active = 0
        self.max_active = 0
        self.order = []

    def __call__(self, req):
        self.active += 1
        self.max_active = max(self.max_active, self.active)
        self.order.append(req.rid)
        time.sleep(self.seconds)
        self.active -= 1
        return np.full((req.n_increments, 15), float(req.rid)), True


def test_stream_generator_matches_the_request_distribution():
    reqs = S.request_stream(200, rate=16.0, seed=6)
    assert [r.rid for r in reqs] == list(range(200))
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and abs(arr[-1] / 200 - 1 / 16) < 0.03
    assert {r.edge for r in reqs} <= {8, 12, 16, 24, 32} and {r.lattice for r in reqs} == {0, 1, 2}
    assert all(8 <= r.n_grains <= 64 and 10 <= r.n_increments <= 50 for r in reqs)
    for r in reqs[:20]:
        assert abs(np.trace(r.vel_grad)) < 1e-15 and abs(np.linalg.norm(r.vel_grad) - 1e-3) < 1e-15
    # the same requests at every rate, only the arrivals differ
    other = S.request_stream(200, rate=0.0, seed=6)
    for a, b in zip(reqs, other):
        assert (a.edge, a.lattice, a.n_grains, a.n_increments, a.seed) == (b.edge, b.lattice, b.n_grains,
                                                                           b.n_increments, b.seed)
        assert np.array_equal(a.vel_grad, b.vel_grad) and b.arrival == 0.0


def test_admission_respects_slots_and_budget():
    mats = _mats()
    reqs = S.request_stream(12, rate=0.0, seed=1, edges=(8,), increments=(2, 3))
    fake = _FakeSolve(0.05)
    one = max(S.device_bytes(r, mats[r.lattice].n_slip + mats[r.lattice].n_twin) for r in reqs)
    srv = S.RveServer(mats, budget_bytes=int(2.5 * one), max_slots=4, solve_fn=fake)
    res = srv.run(reqs)
    assert [r.rid for r in res] == list(range(12))
    assert all(r.rows is not None and r.converged for r in res)
    assert srv.max_in_flight <= 2 and srv.max_bytes_in_flight <= srv.budget  # memory binds before slots
    assert fake.max_active <= 2
    srv2 = S.RveServer(mats, budget_bytes=100 * one, max_slots=3, solve_fn=_FakeSolve(0.05))
    srv2.run(reqs)
    assert srv2.max_in_flight == 3


def test_oldest_first_and_latency_accounting():
    mats = _mats()
    reqs = S.request_stream(6, rate=0.0, seed=2, edges=(8,), increments=(2, 2))
    for k, r in enumerate(reqs):
        r.arrival = 0.02 * k
    fake = _FakeSolve(0.03)
    res = S.RveServer(mats, budget_bytes=1 << 40, max_slots=1, solve_fn=fake).run(reqs)
    assert fake.order == list(range(6))
    for r in res:
        assert r.start >= r.arrival - 1e-6 and r.end - r.start >= 0.03 - 1e-3 and r.latency >= r.end - r.start
    summ = S.summarize(res)
    assert summ["completed"] == 6 and summ["latency_s"]["p50"] <= summ["latency_s"]["p99"]


def test_oversize_request_is_rejected_and_the_rest_served():
    mats = _mats()
    reqs = S.request_stream(4, rate=0.0, seed=3, edges=(8,), increments=(2, 2))
    reqs[1].edge = 32
    small = S.device_bytes(reqs[0], mats[reqs[0].lattice].n_slip + mats[reqs[0].lattice].n_twin)
    res = S.RveServer(mats, budget_bytes=2 * small, max_slots=2, solve_fn=_FakeSolve(0.01)).run(reqs)
    assert res[1].rows is None and "budget" in res[1].error
    assert all(res[k].rows is not None for k in (0, 2, 3))


def test_failed_solve_is_reported_not_raised():
    mats = _mats()
    reqs = S.request_stream(3, rate=0.0, seed=4, edges=(8,), increments=(2, 2))

    def solve(req):
        if req.rid == 1:
            raise RuntimeError("solver broke down")
        return np.zeros((2, 15)), True

    res = S.RveServer(mats, budget_bytes=1 << 40, max_slots=2, solve_fn=solve).run(reqs)
    assert res[1].rows is None and "broke down" in res[1].error
    assert res[0].rows is not None and res[2].rows is not None
