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


class _FakeHarness:
    """Stands in for NewtonHarness in the batched server: records its phases."""

    def __init__(self, req, log):
        self.req, self.log = req, log
        self.rows, self.solve_info, self.solver = [], [], None
        self.F_e = self.F_r = 0.0

    def begin_increment(self):
        self.log.append(("begin", self.req.rid, len(self.rows)))

    def constrained_increment(self, it):
        return np.ones(3) if it == 0 else None

    def finish_increment(self):
        self.log.append(("finish", self.req.rid, len(self.rows)))
        self.rows.append([float(self.req.rid)] * 15)
        self.F_e = self.F_r = float(len(self.rows))


class _FakeHandle:
    def __init__(self, req, log, fail_at=None):
        self.req, self.log, self.fail_at, self.solves, self.closed = req, log, fail_at, 0, False

    def newton_solve(self, duc, solver):
        self.solves += 1
        if self.fail_at is not None and self.solves == self.fail_at:
            raise RuntimeError("solver failed")
        self.log.append(("solve", self.req.rid, duc is not None))
        return {"converged": True, "iterations": 1}

    def close(self):
        self.closed = True


class _FakeBatch:
    def __init__(self, log):
        self.log, self.calls, self.sizes = log, [], []

    def assemble(self, handles, F_e, F_r):
        assert len(handles) == len(F_e) == len(F_r)
        self.calls.append("assemble")
        self.sizes.append(len(handles))
        self.log.append(("assemble", tuple(h.req.rid for h in handles)))

    def post(self, handles, F_e, F_r):
        self.calls.append("post")
        self.log.append(("post", tuple(h.req.rid for h in handles)))

    def launches(self):
        return len(self.calls)

    def close(self):
        pass


def _batched(reqs, max_slots=8, budget=1 << 40, fail=None):
    log, handles = [], {}

    def setup(req):
        be = _FakeHandle(req, log, fail_at=fail.get(req.rid) if fail else None)
        handles[req.rid] = be
        return be, _FakeHarness(req, log)

    fb = _FakeBatch(log)
    srv = S.BatchedRveServer(_mats(), budget, max_slots, setup_fn=setup, batch_fn=lambda: fb)
    return srv, srv.run(reqs), log, fb, handles


def test_batched_server_steps_requests_together():
    """Every tick is one shared assembly over all requests in their Newton
    passes, a solve per request (the increment prescribed on the first pass
    only), then one shared post-pass for those that finished their passes;
    each request runs its own increments, in order, and its handle is
    released when it completes."""
    reqs = S.request_stream(6, rate=0.0, seed=3, increments=(2, 5), edges=(8,))
    srv, res, log, fb, handles = _batched(reqs, max_slots=4)
    assert [r.rid for r in res] == list(range(6))
    for r in res:
        assert r.error is None and r.converged and r.rows.shape == (reqs[r.rid].n_increments, 15)
    assert max(fb.sizes) == 4 and srv.max_in_flight == 4  # four in flight share each launch
    for rid, be in handles.items():
        assert be.closed and be.solves == 4 * reqs[rid].n_increments
        solves = [e[2] for e in log if e[0] == "solve" and e[1] == rid]
        assert solves == [True, False, False, False] * reqs[rid].n_increments
        inc = [e[2] for e in log if e[0] == "finish" and e[1] == rid]
        assert inc == list(range(reqs[rid].n_increments))
    # posts follow every fourth assembly of a request
    for rid in handles:
        seq = [e[0] for e in log if (e[0] in ("assemble", "post") and rid in e[1])]
        assert seq == ["assemble"] * 4 + ["post"] + (["assemble"] * 4 + ["post"]) * (reqs[rid].n_increments - 1)


def test_batched_server_admission_and_failures():
    reqs = S.request_stream(5, rate=0.0, seed=4, increments=(2, 3), edges=(8, 12))
    big = max(reqs, key=lambda r: r.edge)
    budget = S.device_bytes(big, 13) * 2 + 1
    srv, res, log, fb, handles = _batched(reqs, max_slots=8, budget=budget, fail={2: 3})
    assert srv.max_bytes_in_flight <= budget
    assert res[2].error is not None and res[2].rows is None and handles[2].closed
    assert all(r.error is None for r in res if r.rid != 2)
    # an oversize request is rejected at once
    srv2, res2, _, _, _ = _batched(reqs, budget=S.device_bytes(min(reqs, key=lambda r: r.edge), 13) - 1)
    assert all(r.error and "budget" in r.error for r in res2)
