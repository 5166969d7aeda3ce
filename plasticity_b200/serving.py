"""Served RVE stream: independent RVE solves admitted as device memory and
slots free up, each on its own handle (its own CUDA stream and device
state), so that the work of requests in flight overlaps on the GPU.

A request is a Q1 unit cube of edge^3 elements, a Voronoi polycrystal of one
lattice, and a macroscopic velocity gradient applied in n_increments steps of
dt (the velocity-gradient boundary condition of the reference,
updateBeforeIncrement.cc:10-30, boundaryConditions.cc:269-274).  The server
admits waiting requests oldest first whenever the slots in use are fewer than
``max_slots`` and the request's device-memory estimate fits in what is left of
``budget_bytes``; a request whose estimate exceeds the whole budget is
rejected.  Each admitted request runs the device Newton loop (cp_bind_dofs /
cp_newton_iteration / cp_update_from_displacement) on a worker thread; the C
calls release the interpreter lock, so requests in flight overlap on the
device.  Latency is completion time minus arrival time.

``BatchedRveServer`` is the continuous-batching form: the requests in
flight advance in lockstep, one Newton pass (or the post-pass) per tick, and
at every tick the calculatePlasticity work of all of them runs as shared
launches (cp_batch_assemble / cp_batch_post: one update launch per lattice
class over the qps of every request in flight); each request's global system
is then solved on its own stream (cp_newton_solve, solves of different
requests overlapping).  Requests join at the next tick after admission (their
set-up runs meanwhile on a worker) and leave when their last increment is
committed.

This is host code over the C ABI (plasticity_b200.capi); the solve of a
request does not depend on what else is in flight (every kernel of a handle
runs on its own stream over its own buffers, and a shared launch runs each
qp with its own request's data and the same arithmetic), which the GPU tests
check bit for bit.
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait

import numpy as np

from . import harness as H
from . import materials as M


@dataclasses.dataclass
class RveRequest:
    rid: int
    edge: int                 # elements per cube edge
    lattice: int              # index into the server's materials
    n_grains: int             # Voronoi grains (nearest of n_grains seeded points)
    n_increments: int
    vel_grad: np.ndarray      # 3x3 macroscopic velocity gradient (1/s)
    seed: int
    arrival: float = 0.0      # seconds after the start of the stream
    delT: float = 1.0

    @property
    def n_cells(self):
        return self.edge ** 3

    @property
    def n_dofs(self):
        return 3 * (self.edge + 1) ** 3

    def microstructure(self, mesh: H.StructuredMesh):
        """Per-qp lattice ids and Rodrigues vectors of the seeded polycrystal."""
        rng = np.random.default_rng(self.seed)
        pts = rng.random((self.n_grains, 3))
        rod_g = M.random_rodrigues(rng, self.n_grains)
        cc = mesh.cell_centres()
        g = ((pts ** 2).sum(1)[None, :] - 2.0 * cc @ pts.T).argmin(axis=1)
        lid = np.full(mesh.n_cells * 8, self.lattice, dtype=np.int32)
        return lid, np.repeat(rod_g[g], 8, axis=0)


def device_bytes(req: RveRequest, n_systems: int) -> int:
    """An upper estimate of one request's device memory: per qp the history
    (3x3 state and per-system CRSS, backstress and fractions, converged and
    current), the stage of JxW P and JxW dP/dF and the sort keys; per cell Ke,
    Re and the dof map; per dof the CSR matrix (about 81 entries a row, the
    values twice) and the Krylov vectors; plus a fixed allowance."""
    qps = 8 * req.n_cells
    per_qp = 8 * (60 + 6 * n_systems + 90) + 16
    per_cell = 8 * 624 + 4 * 24
    per_dof = 81 * 20 + 8 * 16
    return int(qps * per_qp + req.n_cells * per_cell + req.n_dofs * per_dof + (64 << 20))


def random_traceless(rng, norm):
    L = rng.standard_normal((3, 3))
    L -= np.eye(3) * np.trace(L) / 3.0
    return L * (norm / np.linalg.norm(L))


def request_stream(n, rate, seed, edges=(8, 12, 16, 24, 32), n_lattices=3, grains=(8, 64),
                   increments=(10, 50), norm=1e-3):
    """n requests with Poisson arrivals at ``rate`` per second (all at 0 for
    rate 0): edge, lattice, grain count and increment count drawn uniformly, a
    random traceless velocity gradient of Frobenius norm ``norm`` (dt = 1 s).
    The arrivals come from their own generator, so one seed gives the same
    requests at every rate."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(np.random.default_rng([seed, 1]).exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    out = []
    for k in range(n):
        out.append(RveRequest(rid=k, edge=int(rng.choice(edges)), lattice=int(rng.integers(n_lattices)),
                              n_grains=int(rng.integers(grains[0], grains[1] + 1)),
                              n_increments=int(rng.integers(increments[0], increments[1] + 1)),
                              vel_grad=random_traceless(rng, norm), seed=int(rng.integers(1 << 31)),
                              arrival=float(t[k])))
    return out


@dataclasses.dataclass
class RveResult:
    rid: int
    rows: np.ndarray | None
    arrival: float
    start: float
    end: float
    converged: bool = True
    error: str | None = None

    @property
    def latency(self):
        return self.end - self.arrival


class RveServer:
    """Admission by device-memory budget and slot count; one worker thread
    per slot.  ``solve_fn(request) -> (rows, converged)`` replaces the device
    solve (the default builds a handle and runs the device Newton loop)."""

    def __init__(self, materials, budget_bytes: int, max_slots: int = 8, options_fn=None, solver=None,
                 solve_fn=None):
        self.materials = materials
        self.budget = int(budget_bytes)
        self.max_slots = int(max_slots)
        self.options_fn = options_fn
        self.solver = solver
        self.solve_fn = solve_fn or self._device_solve
        self.n_systems = [int(m.n_slip + m.n_twin) for m in materials]
        self.max_in_flight = 0
        self.max_bytes_in_flight = 0

    def bytes_of(self, req: RveRequest) -> int:
        return device_bytes(req, self.n_systems[req.lattice])

    def _device_solve(self, req: RveRequest):
        from .capi import CpHandle, default_options, default_solver
        mesh = H.StructuredMesh((req.edge, req.edge, req.edge))
        lid, rod = req.microstructure(mesh)
        be = CpHandle(self.materials, self.options_fn() if self.options_fn else default_options())
        try:
            be.bind_qps(lid, rod)
            h = H.NewtonHarness(be, mesh, None, req.n_increments, 4, device_system=True,
                                solver=self.solver or default_solver(), vel_grad=req.vel_grad, delT=req.delT)
            rows = h.run(req.n_increments)
            return rows, all(i["converged"] for i in h.solve_info)
        finally:
            be.close()

    def _run_one(self, req: RveRequest, t0: float):
        start = time.perf_counter() - t0
        try:
            rows, conv = self.solve_fn(req)
            return RveResult(req.rid, rows, req.arrival, start, time.perf_counter() - t0, conv)
        except Exception as e:  # the request fails, the server goes on
            return RveResult(req.rid, None, req.arrival, start, time.perf_counter() - t0, False, repr(e))

    def run(self, requests):
        """Serve a stream (arrival times relative to now); returns the results
        in request-id order."""
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting: deque = deque()
        running = {}
        results = {}
        used = 0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.max_slots) as ex:
            while pending or waiting or running:
                now = time.perf_counter() - t0
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # admit oldest first; a request that fits goes ahead of an
                # older one that must wait for memory
                for req in list(waiting):
                    b = self.bytes_of(req)
                    if b > self.budget:
                        waiting.remove(req)
                        results[req.rid] = RveResult(req.rid, None, req.arrival, now, now, False,
                                                     f"needs {b} bytes, budget {self.budget}")
                        continue
                    if len(running) < self.max_slots and used + b <= self.budget:
                        waiting.remove(req)
                        used += b
                        running[ex.submit(self._run_one, req, t0)] = (req, b)
                self.max_in_flight = max(self.max_in_flight, len(running))
                self.max_bytes_in_flight = max(self.max_bytes_in_flight, used)
                timeout = max(0.0, pending[0].arrival - (time.perf_counter() - t0)) if pending else None
                if running:
                    done, _ = wait(list(running), timeout=timeout, return_when=FIRST_COMPLETED)
                    for fut in done:
                        req, b = running.pop(fut)
                        used -= b
                        results[req.rid] = fut.result()
                elif timeout is not None:
                    time.sleep(timeout)
                elif waiting:  # nothing runs and nothing fits: cannot happen (oversize is rejected)
                    raise RuntimeError("server stalled")
        return [results[k] for k in sorted(results)]


@dataclasses.dataclass
class _Live:
    """A request in flight on the batched server."""
    req: RveRequest
    be: object
    h: object
    b: int            # its device-memory estimate
    start: float
    inc: int = 0      # committed increments
    it: int = 0       # Newton passes done in the current increment


class BatchedRveServer(RveServer):
    """Continuous batching: admission as in RveServer (device-memory budget,
    at most ``max_slots`` in flight, oldest first); the requests in flight
    step together, their qp updates sharing launches (cp_batch_*), their
    solves running concurrently on their own streams."""

    def __init__(self, materials, budget_bytes: int, max_slots: int = 8, options_fn=None, solver=None,
                 device: int = 0, max_newton: int = 4, setup_fn=None, batch_fn=None):
        """setup_fn(request) -> (handle, harness) and batch_fn() -> batch queue
        replace the device objects (the defaults build a CpHandle with its
        NewtonHarness and a CpBatch)."""
        super().__init__(materials, budget_bytes, max_slots, options_fn, solver)
        self.device = device
        self.max_newton = max_newton
        self.setup_fn = setup_fn
        self.batch_fn = batch_fn
        self.ticks = 0
        self.batched_launches = 0

    def _prepare(self, req: RveRequest, t0: float, b: int) -> _Live:
        if self.setup_fn is not None:
            be, h = self.setup_fn(req)
            return _Live(req, be, h, b, time.perf_counter() - t0)
        from .capi import CpHandle, default_options, default_solver
        mesh = H.StructuredMesh((req.edge, req.edge, req.edge))
        lid, rod = req.microstructure(mesh)
        be = CpHandle(self.materials, self.options_fn() if self.options_fn else default_options(device=self.device))
        try:
            be.bind_qps(lid, rod)
            h = H.NewtonHarness(be, mesh, None, req.n_increments, self.max_newton, device_system=True,
                                solver=self.solver or default_solver(), vel_grad=req.vel_grad, delT=req.delT)
        except Exception:
            be.close()
            raise
        return _Live(req, be, h, b, time.perf_counter() - t0)

    def _solve_pass(self, lv: _Live):
        lv.h.solve_info.append(lv.be.newton_solve(lv.h.constrained_increment(lv.it), lv.h.solver))

    def run(self, requests):
        if self.batch_fn is not None:
            batch = self.batch_fn()
        else:
            from .capi import CpBatch
            batch = CpBatch(self.device)
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        waiting: deque = deque()
        setting_up = {}
        live: list[_Live] = []
        results = {}
        used = 0
        t0 = time.perf_counter()

        def finish(lv, error=None):
            nonlocal used
            end = time.perf_counter() - t0
            rows = np.array(lv.h.rows) if error is None else None
            conv = error is None and all(i["converged"] for i in lv.h.solve_info)
            results[lv.req.rid] = RveResult(lv.req.rid, rows, lv.req.arrival, lv.start, end, conv, error)
            used -= lv.b
            lv.be.close()

        try:
            with ThreadPoolExecutor(max_workers=2) as setup_pool, \
                    ThreadPoolExecutor(max_workers=self.max_slots) as solve_pool:
                while pending or waiting or setting_up or live:
                    now = time.perf_counter() - t0
                    while pending and pending[0].arrival <= now:
                        waiting.append(pending.popleft())
                    for req in list(waiting):
                        b = self.bytes_of(req)
                        if b > self.budget:
                            waiting.remove(req)
                            results[req.rid] = RveResult(req.rid, None, req.arrival, now, now, False,
                                                         f"needs {b} bytes, budget {self.budget}")
                            continue
                        if len(live) + len(setting_up) < self.max_slots and used + b <= self.budget:
                            waiting.remove(req)
                            used += b
                            setting_up[setup_pool.submit(self._prepare, req, t0, b)] = (req, b)
                    # requests whose set-up finished join the next tick
                    block = not live and setting_up
                    for fut in list(setting_up):
                        if block or fut.done():
                            req, b = setting_up.pop(fut)
                            try:
                                live.append(fut.result())
                            except Exception as e:
                                used -= b
                                t = time.perf_counter() - t0
                                results[req.rid] = RveResult(req.rid, None, req.arrival, t, t, False, repr(e))
                            block = False
                    self.max_in_flight = max(self.max_in_flight, len(live))
                    self.max_bytes_in_flight = max(self.max_bytes_in_flight, used)
                    if not live:
                        if not setting_up and pending:
                            time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))
                        continue
                    # one tick: a Newton pass of every request still in its Newton passes ...
                    self.ticks += 1
                    for lv in live:
                        if lv.it == 0:
                            lv.h.begin_increment()
                    newton = [lv for lv in live if lv.it < self.max_newton]
                    failed = []
                    if newton:
                        batch.assemble([lv.be for lv in newton], [lv.h.F_e for lv in newton],
                                       [lv.h.F_r for lv in newton])
                        futs = {solve_pool.submit(self._solve_pass, lv): lv for lv in newton}
                        for fut, lv in futs.items():
                            try:
                                fut.result()
                                lv.it += 1
                            except Exception as e:
                                failed.append((lv, repr(e)))
                    for lv, err in failed:
                        live.remove(lv)
                        finish(lv, err)
                    # ... then the post-pass and commit of those that finished them
                    post = [lv for lv in live if lv.it == self.max_newton]
                    if post:
                        batch.post([lv.be for lv in post], [lv.h.F_e for lv in post], [lv.h.F_r for lv in post])
                        for lv in post:
                            lv.h.finish_increment()
                            lv.inc += 1
                            lv.it = 0
                            if lv.inc == lv.req.n_increments:
                                live.remove(lv)
                                finish(lv)
            self.batched_launches = batch.launches()
        finally:
            for lv in live:
                lv.be.close()
            batch.close()
        return [results[k] for k in sorted(results)]


def summarize(results, wall_s=None):
    """Throughput and latency percentiles of a served stream."""
    ok = [r for r in results if r.rows is not None]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    span = wall_s if wall_s is not None else (max(r.end for r in ok) - min(r.arrival for r in ok) if ok else 0.0)
    return {"requests": len(results), "completed": len(ok), "failed": len(results) - len(ok),
            "converged": int(sum(r.converged for r in ok)),
            "solves_per_s": len(ok) / span if span > 0 else 0.0,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
                          "p99": float(np.percentile(lat, 99)), "max": float(lat.max())}}
