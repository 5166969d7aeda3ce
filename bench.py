#!/usr/bin/env python
"""Benchmark of the B200 crystal-plasticity qp hot path.

Workload (one step): one batched calculatePlasticity with the algorithmic
tangent (StiffnessCalFlag = 1, dP/dF written out) over 2^21 quadrature points
shuffled 50 % FCC (12+1 systems), 30 % BCC (48+1), 20 % HCP (24 slip + 6
twins), each with a seeded random orientation and a history built by 10 prior
committed increments of random loading F <- F (I + 2e-4 G), G ~ N(0,1)^{3x3}
iid per qp; the timed increment is the next such F.  Synthetic data.

Metric: qp-updates/s (whole job).  ``value`` is timed on device-resident
inputs (CUDA events on the library's stream); ``e2e`` is the same step through
the public host-pointer call cp_update with page-locked host buffers (F in;
P, dP/dF, status out).  Inputs, outputs and state (~3 GB) are far larger than
the 126 MB L2, so no flush is needed between steps.

``--impl reference`` times the reference algorithm on the host cores instead:
the reference cannot be built here (deal.II/PETSc/p4est/MPI absent), so its
CPU implementation is the FP64 restatement under oracle/ (OpenMP over qps) on
a bounded sample of the same workload.

Run:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
      torchrun --nproc-per-node N bench.py --gpus N ...   (N independent replicas)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_QP = 1 << 21
MIX = (0.5, 0.3, 0.2)
SEED_LATTICE, SEED_ORIENT, SEED_LOAD = 1, 0, 2
PRIOR_STEPS = 10
AMP = 2e-4
METRIC = "qp-updates/s (calculatePlasticity + dP/dF, FP64)"
# DRAM bytes (read + write) per qp of the sorted update, per lattice class,
# from ncu --set full --clock-control none -k regex:update2 -s 30 -c 3 on the
# 2^18-qp case (python bench.py --n-qp 262144 --steps 1 --warmup 1 --no-tune
# with every leg off), the untuned default shape
NCU_DRAM_BYTES_PER_QP = {"fcc": 8957.8, "bcc": 32006.4, "hcp": 5758.1}


# --------------------------------------------------------------------- workload
def lattice_ids(n, rank=0):
    rng = np.random.default_rng(SEED_LATTICE + 1000 * rank)
    n_fcc = int(round(MIX[0] * n))
    n_bcc = int(round(MIX[1] * n))
    lid = np.concatenate([np.zeros(n_fcc), np.ones(n_bcc), np.full(n - n_fcc - n_bcc, 2)]).astype(np.int32)
    rng.shuffle(lid)
    return lid


def orientations(n, rank=0):
    from plasticity_b200 import materials as M
    return M.random_rodrigues(np.random.default_rng(SEED_ORIENT + 1000 * rank), n)


def materials():
    from plasticity_b200 import materials as M
    return [M.fcc_cu(), M.bcc_48(), M.hcp_mg()]


def flops_per_qp(n, p, rounds, e, c, flag):
    """FP64 flops of one qp-update: 2 [U + flag T] with
    U = 892 + 171n + 11n^2 + (2/3 p^3 + p^2) rounds + 27e and
    T = 4374 + 27c + p (420 + 18c^3 + 27e) + 18p^2 + p^3  (FMA-equivalents)."""
    p = p.astype(np.float64)
    U = 892 + 171 * n + 11 * n * n + (2.0 / 3.0 * p ** 3 + p ** 2) * np.maximum(rounds, 1) * (p > 0) + 27 * e
    T = 4374 + 27 * c + p * (420 + 18 * c ** 3 + 27 * e) + 18 * p ** 2 + p ** 3
    return 2.0 * (U + flag * T)


def bytes_per_qp(n, ns, nw, flag):
    """Minimal HBM bytes of one qp-update as the bench calls it: reads F, Fp,
    s, W, rotation, twin/slip fractions, twin flag; writes Fp, Fe, s, W,
    fractions, P, status and (flag 1) dP/dF."""
    rd = 8 * (9 + 9 + 2 * n + 3 + nw + ns) + 4
    wr = 8 * (9 + 9 + 2 * n + nw + ns + 9) + 4 + (648 if flag else 0)
    return rd + wr


# --------------------------------------------------------------------- replicas
def max_over_ranks(x: float, device) -> float:
    """The largest x over all ranks (a no-op without a process group): the
    job's time is its slowest replica's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def percentiles(ms):
    """p50 / p95 / p99 / max of per-step times (ms)."""
    a = np.asarray(ms, dtype=np.float64)
    return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
            "p99": float(np.percentile(a, 99)), "max": float(a.max()), "steps": int(len(a))}


def aggregate_value(world: int, n_qp_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job qp-updates/s: every rank's qps over the slowest rank's time."""
    return world * n_qp_per_rank * steps / seconds


# --------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (read-only queries)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def wait_first(self, timeout=3.0):
        """Until nvidia-smi has printed its first sample (bounded)."""
        t0 = time.perf_counter()
        while self.proc and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def stop(self, window=None):
        """Summary of the samples read inside window = (t0, t1) (perf_counter
        seconds; one sampling interval of slack at the end), or all."""
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for t, ln in self.lines if window is None or window[0] <= t <= window[1] + 0.15]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------- CPU legs
def cpu_sample_inputs(n_sample, rank=0):
    """A bounded sample of the workload for the host runs: the first n_sample
    qps (same lattice mix, orientations), history from 10 prior increments
    drawn with a host RNG."""
    lid = lattice_ids(N_QP, rank)[:n_sample]
    rod = orientations(N_QP, rank)[:n_sample]
    return lid, rod


def run_oracle_sample(lid, rod, steps_prior, rng, threads):
    from oracle import oracle as O
    from plasticity_b200.capi import default_options
    be = O.OracleBackend(materials(), default_options(), nthreads=threads)
    be.bind_qps(lid, rod)
    F = np.tile(np.eye(3).ravel(), (len(lid), 1))
    for _ in range(steps_prior):
        F = (F.reshape(-1, 3, 3) @ (np.eye(3) + AMP * rng.standard_normal((len(lid), 3, 3)))).reshape(-1, 9)
        be.update(F, 0)
        be.commit()
    Fn = (F.reshape(-1, 3, 3) @ (np.eye(3) + AMP * rng.standard_normal((len(lid), 3, 3)))).reshape(-1, 9)
    return be, Fn


def reference_arm(args):
    """The reference algorithm on the host cores (the oracle port; the
    reference itself cannot be built without deal.II/PETSc/p4est/MPI)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n_s = args.cpu_sample
    lid, rod = cpu_sample_inputs(n_s)
    be, Fn = run_oracle_sample(lid, rod, PRIOR_STEPS, np.random.default_rng(SEED_LOAD), threads)
    for _ in range(args.warmup):
        be.update(Fn, 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        be.update(Fn, 1)
    dt = time.perf_counter() - t0
    v = n_s * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "qp-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"mixed FCC/BCC/HCP qps 50/30/20, flag 1, sample {n_s} of {N_QP}",
                   "n_qp": n_s, "stiffness_flag": 1, "prior_increments": PRIOR_STEPS},
        "cpu_baseline": {"value": v, "unit": "qp-updates/s", "cores": threads, "kind": "port",
                         "sample": f"first {n_s} qps of the {N_QP}-qp workload, one flag-1 update per step"},
        "e2e": {"value": v, "unit": "qp-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (deal.II/PETSc/p4est/MPI) not buildable here; timed its FP64 CPU restatement (oracle/)",
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------- GPU arm
def ours(args):
    import torch
    import torch.distributed as dist
    from plasticity_b200 import capi
    from plasticity_b200.capi import CpHandle, default_options

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = args.n_qp
    lid = lattice_ids(n, rank)
    rod = orientations(n, rank)
    mats = materials()
    opts = default_options(device=local)
    opts.update_variant = args.update_variant
    h = CpHandle(mats, opts)
    h.bind_qps(lid, rod)
    stream = torch.cuda.ExternalStream(h.stream(), device=dev)

    # history: PRIOR_STEPS committed increments of random loading (untimed)
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED_LOAD + 1000 * rank)
    eye = torch.eye(3, dtype=torch.float64, device=dev)
    F = eye.expand(n, 3, 3).contiguous()
    P = torch.empty(n, 9, dtype=torch.float64, device=dev)
    dPdF = torch.empty(n, 81, dtype=torch.float64, device=dev)
    status = torch.empty(n, dtype=torch.int32, device=dev)
    for _ in range(PRIOR_STEPS):
        G = torch.randn(n, 3, 3, dtype=torch.float64, device=dev, generator=gen)
        F = F @ (eye + AMP * G)
        torch.cuda.synchronize()
        h.update_device(F.data_ptr(), 0, 0.0, 0.0, P.data_ptr(), None, None, status.data_ptr())
        h.commit()
        h.synchronize()
    G = torch.randn(n, 3, 3, dtype=torch.float64, device=dev, generator=gen)
    Fn = (F @ (eye + AMP * G)).contiguous()
    torch.cuda.synchronize()

    def step():
        h.update_device(Fn.data_ptr(), 1, 0.0, 0.0, P.data_ptr(), None, dPdF.data_ptr(), status.data_ptr())

    # launch shapes tuned on the live workload (cp_autotune), then every step
    # is one replay of the call's captured CUDA graph
    tune = None
    if not args.no_tune:
        tune = h.autotune(Fn.data_ptr(), capi.CP_TUNE_UPDATE, reps=3)
        h.synchronize()

    # the clock sampler starts before the warm-up (nvidia-smi needs a moment
    # to start) and keeps only the samples read during the timed steps
    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first()
    for _ in range(args.warmup):
        step()
    h.synchronize()
    st = status.cpu().numpy()
    bad = int(np.count_nonzero(st & capi.CP_QP_ERROR_MASK))

    if world > 1:
        dist.barrier()
    h.synchronize()
    g0 = h.graph_stats()
    t_begin = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k in range(args.steps):
            step()
            marks[k].record(stream)  # per-step latency (no synchronisation between steps)
        e1.record(stream)
    e1.synchronize()
    clk = clocks.stop((t_begin, time.perf_counter()))
    g1 = h.graph_stats()
    elapsed_ms = e0.elapsed_time(e1)
    step_ms = [e0.elapsed_time(marks[0])] + [marks[k - 1].elapsed_time(marks[k]) for k in range(1, args.steps)]
    elapsed_ms = max_over_ranks(elapsed_ms, dev)
    ms_per_step = elapsed_ms / args.steps
    value = aggregate_value(world, n, args.steps, elapsed_ms * 1e-3)
    graph_launches = (g1[1] - g0[1]) / args.steps

    # per-lattice-group kernel times for the roofline: the same steps with
    # every update launch bracketed by events (stream launches, no graph)
    h.set_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            step()
    timing = h.get_timing()
    h.set_timing(False)

    # StiffnessCalFlag = 0 (the post-pass form: no tangent), same inputs
    step0 = lambda: h.update_device(Fn.data_ptr(), 0, 0.0, 0.0, P.data_ptr(), None, None, status.data_ptr())
    for _ in range(args.warmup):
        step0()
    h.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        f0.record(stream)
        for _ in range(args.steps):
            step0()
        f1.record(stream)
    f1.synchronize()
    ms0 = max_over_ranks(f0.elapsed_time(f1), dev) / args.steps
    flag0 = {"value": aggregate_value(world, n, 1, ms0 * 1e-3), "unit": "qp-updates/s", "ms_per_step": ms0,
             "stiffness_flag": 0}
    step()  # the flag-1 outputs and stats again (the roofline and the parity leg read them)
    h.synchronize()

    # the plain thread-per-qp drop-in (cp_options_t.plain_kernel) on the same
    # inputs and history, for the speed-up of the optimised pipeline over it
    plain = None
    if not args.no_plain:
        hp = CpHandle(mats, default_options(device=local, plain_kernel=1))
        hp.bind_qps(lid, rod)
        for f in ("Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac", "slipfrac", "twin"):
            for suf in ("_conv", "_iter"):
                hp.set_state(f + suf, h.get_state(f + suf))
        stp = torch.cuda.ExternalStream(hp.stream(), device=dev)
        Pp = torch.empty_like(P)
        Dp = torch.empty_like(dPdF)
        Sp = torch.empty_like(status)
        stepp = lambda: hp.update_device(Fn.data_ptr(), 1, 0.0, 0.0, Pp.data_ptr(), None, Dp.data_ptr(),
                                         Sp.data_ptr())
        for _ in range(args.warmup):
            stepp()
        hp.synchronize()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stp):
            q0.record(stp)
            for _ in range(args.steps):
                stepp()
            q1.record(stp)
        q1.synchronize()
        pms = q0.elapsed_time(q1) / args.steps
        # the optimised handle's outputs for the same F: the two kernels give the same bits
        step()
        h.synchronize()
        hp.synchronize()
        same = bool(torch.equal(Pp, P) and torch.equal(Dp, dPdF) and torch.equal(Sp, status))
        plain = {"value": n / (pms * 1e-3), "unit": "qp-updates/s", "ms_per_step": pms,
                 "speedup_of_value": (n / (ms_per_step * 1e-3)) / (n / (pms * 1e-3)),
                 "outputs_bit_identical": same}
        hp.close()
        del Pp, Dp, Sp

    # roofline of the dominant kernel (the group with the largest time)
    stats = h.stats()
    dom = max(timing, key=lambda g: g[3])
    dom_lat = dom[0]
    lat_n = {i: (m.n_total, m.n_slip, m.n_twin) for i, m in enumerate(mats)}
    sel = stats[:, 6] == dom_lat
    nT, ns, nw = lat_n[dom_lat]
    fl = flops_per_qp(nT, stats[sel, 1], stats[sel, 2], stats[sel, 3], stats[sel, 4], 1).sum()
    by = bytes_per_qp(nT, ns, nw, 1) * int(sel.sum())
    dom_ms = dom[3] / max(dom[2], 1)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    if "hbm_gbs" in peaks:
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    else:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s (an earlier copy measurement on this pool; MEASURED_PEAKS.json absent)"
    fp64_peak = capi.measure_fp64_peak(local)
    lat_name = ["fcc", "bcc", "hcp"][dom_lat]
    # DRAM bytes per qp of the sorted update from an ncu capture of the 2^18-qp
    # case (a separately labelled, profile-derived figure, scaled to this
    # launch's qps; the full-size workload is too large for a multi-pass capture)
    traffic = NCU_DRAM_BYTES_PER_QP[lat_name] * int(sel.sum()) if lat_name in NCU_DRAM_BYTES_PER_QP else None
    all_fl = sum(flops_per_qp(lat_n[L][0], stats[stats[:, 6] == L, 1], stats[stats[:, 6] == L, 2],
                              stats[stats[:, 6] == L, 3], stats[stats[:, 6] == L, 4], 1).sum() for L in range(3))

    # e2e through the public host-pointer call with page-locked buffers
    e2e = None
    if not args.no_e2e:
        hF = torch.empty(n, 9, dtype=torch.float64, pin_memory=True)
        hF.copy_(Fn.reshape(n, 9).cpu())
        hP = torch.empty(n, 9, dtype=torch.float64, pin_memory=True)
        hD = torch.empty(n, 81, dtype=torch.float64, pin_memory=True)
        hS = torch.empty(n, dtype=torch.int32, pin_memory=True)
        import ctypes as C
        dp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
        ip = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int32))
        call = lambda: h.lib.cp_update(h.h, dp(hF), 1, 0.0, 0.0, dp(hP), None, dp(hD), ip(hS))
        for _ in range(max(1, args.warmup)):
            assert call() == 0
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        call_ms = []
        for _ in range(args.steps):
            tc = time.perf_counter()
            assert call() == 0
            call_ms.append(1e3 * (time.perf_counter() - tc))
        dt = max_over_ranks(time.perf_counter() - t0, dev)
        e2e = {"value": aggregate_value(world, n, args.steps, dt), "unit": "qp-updates/s",
               "h2d_bytes_per_step": 9 * 8 * n, "d2h_bytes_per_step": (9 + 81) * 8 * n + 4 * n,
               "ms_per_step": 1e3 * dt / args.steps, "latency_ms": percentiles(call_ms)}

    # CPU baseline and a live parity check on a bounded sample (rank 0, N=1)
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = cpu_leg(args, h, Fn, P, dPdF, lid, rod, local)
    asm = assembly_leg(args, local) if (world == 1 and not args.no_assembly) else None
    rve = rve_leg(args, local) if (world == 1 and not args.no_rve) else None
    rve_large = rve_large_leg(args, local, args.rve_large_increments) if (world == 1 and not args.no_rve_large) \
        else None
    dual = rve_dualphase_leg(args, local, args.rve_increments) if (world == 1 and not args.no_dualphase) else None
    serve = serve_leg(args, local, args.serve_requests, tuple(float(x) for x in args.serve_rates.split(","))) \
        if (world == 1 and not args.no_serve) else None

    line = {
        "metric": METRIC, "value": value, "unit": "qp-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "2^21 shuffled qps 50% FCC(12+1) / 30% BCC(48+1) / 20% HCP(24+6), "
                               "history of 10 random increments F<-F(I+2e-4 G), one flag-1 update per step",
                   "n_qp_per_gpu": n, "stiffness_flag": 1, "parallelism": f"replicas x{world}",
                   "l2": "inputs+outputs+state ~3 GB >> 126 MB L2 (no flush needed)"},
        "clocks": clk,
        "latency_ms": percentiles(step_ms),
        "e2e": e2e,
        # per lattice group: classify, scan, scatter, update (and a histogram memset), all in one graph
        "gpu_launches": args.steps * len(timing) * 4,
        "graph_launches_per_step": graph_launches,
        "autotune": tune,
        "roofline": {"bound": "hbm", "kernel": f"update_kernel[{lat_name}]", "achieved": by / (dom_ms * 1e-3) / 1e9,
                     "peak": hbm_peak, "unit": "GB/s", "frac": by / (dom_ms * 1e-3) / 1e9 / hbm_peak,
                     "traffic": traffic, "traffic_source": "ncu capture, 2^18-qp case, scaled per qp",
                     "algorithmic_bytes": by, "peak_source": hbm_src},
        "roofline_fp64": {"bound": "fp64", "kernel": f"update_kernel[{lat_name}]",
                          "achieved": fl / (dom_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                          "frac": fl / (dom_ms * 1e-3) / 1e12 / fp64_peak,
                          "peak_source": "measured FP64 FMA probe (cp_measure_fp64_peak), live",
                          "all_kernels_achieved": all_fl / (ms_per_step * 1e-3) / 1e12},
        "kernels": [{"lattice": ["fcc", "bcc", "hcp"][g[0]], "n_qp": g[1], "ms_per_launch": g[3] / max(g[2], 1)}
                    for g in timing],
        "flag0": flag0,
        "plain_drop_in": plain,
        "qp_error_flags": bad,
        "cpu_baseline": cpu,
        "parity": parity,
        "assembly": asm,
        "rve": rve,
        "rve_large": rve_large,
        "rve_dualphase": dual,
        "serve": serve,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    h.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_leg(args, h, Fn, P, dPdF, lid, rod, device=0):
    """Oracle on the first qps of this exact workload: the GPU's conv state of
    those qps and the same F; times one flag-1 update on all host cores and
    compares it with the GPU's P and dP/dF for those qps."""
    from oracle import oracle as O
    from plasticity_b200.capi import default_options
    n_s = args.cpu_sample
    threads = os.cpu_count() or 1
    be = O.OracleBackend(materials(), default_options(), nthreads=threads)
    be.bind_qps(lid[:n_s], rod[:n_s])
    for f in ("Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac", "slipfrac", "twin"):
        for suf in ("_conv", "_iter"):
            be.set_state(f + suf, h.get_state(f + suf)[:n_s])
    Fh = Fn.reshape(-1, 9)[:n_s].cpu().numpy()
    t0 = time.perf_counter()
    Po, _, Do, so = be.update(Fh, 1)
    dt = time.perf_counter() - t0
    Pg = P[:n_s].cpu().numpy()
    Dg = dPdF[:n_s].cpu().numpy()
    sg = h.stats()[:n_s]
    so_ = be.stats()

    def rel(a, b):
        return float((np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)).max())

    ok = (sg[:, 7] <= 12) & (so_[:, 7] <= 12)  # well-posed active-set solves on both sides
    same = np.all(sg[:, :3] == so_[:, :3], axis=1)
    # the oracle against itself compiled with fused multiply-adds (another
    # valid rounding of the same arithmetic): where the active-set solves are
    # ill conditioned, the reference's own result is set by rounding
    prev = O.use_library(O.build_fma())
    try:
        for f in ("Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac", "slipfrac", "twin"):
            for suf in ("_conv", "_iter"):
                be.set_state(f + suf, h.get_state(f + suf)[:n_s])
        be.update(Fh, 1)
        sf = be.stats()
    finally:
        O.restore_library(prev)
    okf = (sf[:, 7] <= 12) & (so_[:, 7] <= 12)
    samef = np.all(sf[:, :3] == so_[:, :3], axis=1)
    ref_order = reference_order_parity(h, Fh, lid[:n_s], rod[:n_s], n_s, threads, device)
    parity = {"sample_qps": n_s, "well_posed_qps": int(ok.sum()),
              "max_rel_err_P": rel(Pg[ok], Po[ok]), "max_rel_err_dPdF": rel(Dg[ok], Do[ok]),
              "active_sets_identical": bool(same[ok].all()), "tolerance": 1e-10,
              "ill_conditioned_qps": int((~ok).sum()),
              "ill_conditioned_active_set_mismatches": int((~same[~ok]).sum()),
              "oracle_fma_build_vs_oracle": {"ill_conditioned_qps": int((~okf).sum()),
                                             "ill_conditioned_active_set_mismatches": int((~samef[~okf]).sum()),
                                             "well_posed_active_sets_identical": bool(samef[okf].all())},
              "reference_order": ref_order,
              "criterion": "identical active sets and <=1e-10 on qps whose active-set solves have condition <= 1e12"}
    cpu = {"value": n_s / dt, "unit": "qp-updates/s", "cores": threads, "kind": "port",
           "sample": f"first {n_s} qps of the workload (GPU's history, same F), one flag-1 update"}
    return cpu, parity


def reference_order_parity(h, Fh, lid, rod, n_s, threads, device=0):
    """The library's reference-order update (cp_options_t.reference_order)
    on the GPU against the oracle's parity build on the CPU, both from the
    GPU's history of the sample's qps with the same F: qps whose outputs (P,
    dP/dF, status, statistics, the whole _iter history) differ in any bit."""
    from oracle import oracle as O
    from plasticity_b200.capi import CpHandle, default_options
    fields = ("Fp", "Fe", "s", "W", "rot", "rotnew", "twinfrac", "slipfrac", "twin")
    out_fields = [f + "_iter" for f in fields]
    g = CpHandle(materials(), default_options(device=device, reference_order=1))
    g.bind_qps(lid, rod)
    prev = O.use_library(O.build_parity())
    try:
        be = O.OracleBackend(materials(), default_options(), nthreads=threads)
        be.bind_qps(lid, rod)
        for f in fields:
            for suf in ("_conv", "_iter"):
                v = h.get_state(f + suf)[:n_s]
                be.set_state(f + suf, v)
                g.set_state(f + suf, v)
        t0 = time.perf_counter()
        Pg, _, Dg, sgs = g.update(Fh, 1)
        t_gpu = time.perf_counter() - t0
        Po, _, Do, sos = be.update(Fh, 1)
        stg, sto = g.stats(), be.stats()

        def same(a, b):
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(len(a), -1)
            b = np.ascontiguousarray(b, dtype=np.float64).reshape(len(b), -1)
            return ((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))).all(axis=1)

        ok = same(Pg, Po) & same(Dg, Do) & (sgs == sos) & (stg[:, :6] == sto[:, :6]).all(axis=1)
        for f in out_fields:
            ok &= same(g.get_state(f), be.get_state(f))
    finally:
        O.restore_library(prev)
        g.close()
    ill = sto[:, 7] > 12
    return {"sample_qps": n_s, "ill_conditioned_qps": int(ill.sum()),
            "mismatching_qps": int((~ok).sum()), "ill_conditioned_mismatching_qps": int((~ok & ill).sum()),
            "gpu_seconds": t_gpu,
            "criterion": "cp_options_t.reference_order on the GPU vs the oracle's parity build: every output "
                         "bit (P, dP/dF, status, stats, _iter history) at every qp"}


# --------------------------------------------------------------------- assembly
ASM_N = 64  # 64^3 cells = 2^21 qps


def assembly_leg(args, device):
    """Batched getElementalValues (cp_assemble) on a 64^3 Q1 cube whose cells
    are FCC/BCC/HCP grains shuffled 50/30/20 (seed SEED_LATTICE) with seeded
    orientations: 10 committed increments of macroscopic loading
    F <- F (I + 2e-4 G) plus per-node noise, then the next increment's
    assembly (update with dP/dF, contraction into Ke/Re) timed device-resident
    (CUDA events) and end to end through cp_assemble with page-locked host
    U_local / Ke / Re."""
    import torch
    from plasticity_b200 import harness as Hm
    from plasticity_b200.capi import CpHandle, default_options
    n = args.asm_n
    nc = n ** 3
    rng = np.random.default_rng(SEED_LOAD + 7)
    lid = lattice_ids(nc)
    rod = orientations(nc)
    h = CpHandle(materials(), default_options(device=device))
    h.bind_qps(np.repeat(lid, 8), np.repeat(rod, 8, axis=0))
    grad = Hm.q1_reference_gradients() * n  # [q][a][3], cell size 1/n
    jxw = np.full(8, 1.0 / (8 * nc))
    h.bind_mesh(nc, grad, jxw, True)
    # cell c = i + n (j + n k) (x fastest); its node a at (i, j, k) + (a&1, a>>1&1, a>>2&1)
    ijk = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1).reshape(-1, 3)
    ijk = ijk[np.lexsort((ijk[:, 0], ijk[:, 1], ijk[:, 2]))]
    off = np.array([[a & 1, (a >> 1) & 1, (a >> 2) & 1] for a in range(8)])
    cn = ijk[:, None, :] + off[None, :, :]
    node = cn[..., 0] + (n + 1) * (cn[..., 1] + (n + 1) * cn[..., 2])
    xyz = np.zeros(((n + 1) ** 3, 3))
    ii, jj, kk = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    xyz[(ii + (n + 1) * (jj + (n + 1) * kk)).ravel()] = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], -1) / n
    Fm = np.eye(3)
    noise = np.zeros_like(xyz)

    def u_local():
        u = xyz @ (Fm - np.eye(3)).T + noise
        return np.ascontiguousarray(u[node].reshape(nc, 24))

    for _ in range(PRIOR_STEPS):
        Fm = Fm @ (np.eye(3) + AMP * rng.standard_normal((3, 3)))
        noise += 2e-5 / n * rng.standard_normal(noise.shape)
        U = u_local().reshape(nc, 8, 3)
        F = (np.einsum("cai,qaj->cqij", U, grad) + np.eye(3)).reshape(-1, 9)
        h.update(F, 0)
        h.commit()
    Fm = Fm @ (np.eye(3) + AMP * rng.standard_normal((3, 3)))
    noise += 2e-5 / n * rng.standard_normal(noise.shape)
    U = u_local()
    dev = torch.device("cuda", device)
    Ud = torch.from_numpy(U).to(dev)
    Ked = torch.empty(nc, 576, dtype=torch.float64, device=dev)
    Red = torch.empty(nc, 24, dtype=torch.float64, device=dev)
    Sd = torch.empty(nc * 8, dtype=torch.int32, device=dev)
    stream = torch.cuda.ExternalStream(h.stream(), device=dev)
    step = lambda: h.assemble_device(Ud.data_ptr(), 0.0, 0.0, Ked.data_ptr(), Red.data_ptr(), Sd.data_ptr())
    for _ in range(args.warmup):
        step()
    h.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    plastic = float((h.stats()[:, 1] > 0).mean())
    hU = torch.empty(nc, 24, dtype=torch.float64, pin_memory=True)
    hU.copy_(torch.from_numpy(U))
    hK = torch.empty(nc, 576, dtype=torch.float64, pin_memory=True)
    hR = torch.empty(nc, 24, dtype=torch.float64, pin_memory=True)
    hS = torch.empty(nc * 8, dtype=torch.int32, pin_memory=True)
    import ctypes as C
    dp = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))
    ip = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_int32))
    call = lambda: h.lib.cp_assemble(h.h, dp(hU), 0.0, 0.0, dp(hK), dp(hR), ip(hS))
    for _ in range(args.warmup):
        assert call() == 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        assert call() == 0
    e2e_ms = 1e3 * (time.perf_counter() - t0) / args.steps
    same = bool(torch.equal(hK, Ked.cpu()) and torch.equal(hR, Red.cpu()))
    # the mixed-precision assembly: the same update, the contraction on the
    # tensor cores (split-BF16, FP32 accumulation; FP32 Ke, FP64 Re)
    Kmd = torch.empty(nc, 576, dtype=torch.float32, device=dev)
    Rmd = torch.empty(nc, 24, dtype=torch.float64, device=dev)
    stepm = lambda: h.assemble_mixed_device(Ud.data_ptr(), 0.0, 0.0, Kmd.data_ptr(), Rmd.data_ptr(), Sd.data_ptr())
    for _ in range(args.warmup):
        stepm()
    h.synchronize()
    m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        m0.record(stream)
        for _ in range(args.steps):
            stepm()
        m1.record(stream)
    m1.synchronize()
    ms_mixed = m0.elapsed_time(m1) / args.steps
    step()
    h.synchronize()
    kd = Ked.double()
    ke_err = float(((Kmd.double() - kd).abs().amax(dim=1) / kd.abs().amax(dim=1)).max())
    re_same = bool(torch.equal(Rmd, Red))
    # the contraction kernels alone (event-bracketed launches)
    h.set_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            step()
            stepm()
    h.synchronize()
    c64 = h.contract_timing(0)
    ctc = h.contract_timing(1)
    h.set_timing(False)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    bf16 = float(peaks.get("bf16_tflops", 1590.0))
    by64 = nc * (720 * 8 + 600 * 8)  # staged JxW P, JxW dP/dF in; Ke, Re (FP64) out
    bytc = nc * (720 * 8 + 576 * 4 + 24 * 8)  # the same in; Ke FP32, Re FP64 out
    tiles = -(-nc // 14)
    tc_flops = tiles * 6 * 5 * 2 * 128 * 64 * 16  # six split products, five K=16 steps of 128x64 per tile
    t64 = c64[1] / max(c64[0], 1)
    ttc = ctc[1] / max(ctc[0], 1)
    contraction = {
        "fp64": {"kernel": "contract_kernel", "ms_per_launch": t64, "bytes": by64,
                 "achieved_gbs": by64 / (t64 * 1e-3) / 1e9, "frac_hbm": by64 / (t64 * 1e-3) / 1e9 / hbm},
        "tensor_core": {"kernel": "ke_tc_kernel (tcgen05.mma kind::f16, split-BF16, FP32 accumulate in TMEM)",
                        "ms_per_launch": ttc, "bytes": bytc, "achieved_gbs": bytc / (ttc * 1e-3) / 1e9,
                        "frac_hbm": bytc / (ttc * 1e-3) / 1e9 / hbm, "tensor_flops": tc_flops,
                        "achieved_tflops": tc_flops / (ttc * 1e-3) / 1e12,
                        "frac_bf16": tc_flops / (ttc * 1e-3) / 1e12 / bf16, "bound": "hbm"},
        "peaks": {"hbm_gbs": hbm, "bf16_tflops": bf16}}
    h.close()
    return {"workload": "64^3 Q1 cells (2^21 qps), FCC/BCC/HCP grains 50/30/20, 10 prior increments, flag-1 "
                        "update + Ke/Re contraction per step",
            "cells": nc, "ms_per_step": ms, "elements_per_s": nc / (ms * 1e-3),
            "qp_updates_per_s": 8 * nc / (ms * 1e-3), "plastic_qp_fraction": plastic,
            "e2e": {"ms_per_step": e2e_ms, "elements_per_s": nc / (e2e_ms * 1e-3),
                    "h2d_bytes_per_step": 8 * 24 * nc, "d2h_bytes_per_step": 8 * 600 * nc + 4 * 8 * nc,
                    "matches_device_call": same},
            "mixed": {"ms_per_step": ms_mixed, "elements_per_s": nc / (ms_mixed * 1e-3),
                      "ke_rel_err_vs_fp64": ke_err, "re_bit_identical": re_same},
            "contraction": contraction}


# --------------------------------------------------------------------- RVE solve
RVE_INC, RVE_NEWTON = 20, 4


def rve_case():
    """The 8x8x8 FCC Cu cube: one grain per element (Rodrigues of a normalised
    N(0, I4) quaternion, seed SEED_ORIENT), faces x=0 held in x/y/z, face x=1
    pulled to u_x = 0.02 in 20 equal increments, 4 Newton iterations each."""
    from plasticity_b200 import harness as H
    from plasticity_b200 import materials as M
    mesh = H.StructuredMesh((8, 8, 8))
    rod = np.repeat(M.random_rodrigues(np.random.default_rng(SEED_ORIENT), mesh.n_cells), 8, axis=0)
    bc = np.array([[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.02]])
    return mesh, rod, bc


def rve_run(backend, device_system, solver=None):
    from plasticity_b200 import harness as H
    mesh, rod, bc = rve_case()
    backend.bind_qps(np.zeros(mesh.n_cells * 8, np.int32), rod)
    h = H.NewtonHarness(backend, mesh, bc, RVE_INC, RVE_NEWTON, device_system=device_system, solver=solver)
    t0 = time.perf_counter()
    rows = h.run()
    return rows, time.perf_counter() - t0, h


def rve_leg(args, device):
    """RVE solves/s on the 4,096-qp FCC cube, whole Newton loop on the device
    (sorted update, device scatter, condensation and BiCG), against:
    the plain FP64 GPU kernel in the same device loop (same solver; the two
    update kernels give the same bits, so the stress error is exactly 0);
    the plain GPU drop-in inside a host Newton loop with a direct sparse
    solve (the reference's own loop shape: GPU update/assembly, host solve);
    the mixed-precision device loop; and the oracle with the host solve on the
    host cores.  The stress rows of differently rounded solves drift apart:
    at 2 % strain most FCC qps have numerically singular active-set blocks
    whose pseudo-inverse solution is set by rounding (a 1e-12 change of each
    Newton update moves the oracle's own final stress by ~1 %), so only arms
    with the same arithmetic can meet a 1e-6 bar."""
    from plasticity_b200 import materials as M
    from plasticity_b200.capi import CP_PRECISION_MIXED, CpHandle, default_options, default_solver
    mats = [M.fcc_cu()]
    hw = CpHandle(mats, default_options(device=device))
    rve_run(hw, True)  # warm-up: first launches, allocations
    hw.close()
    hd = CpHandle(mats, default_options(device=device))
    rows_d, t_d, harness = rve_run(hd, True)
    iters = [i["iterations"] for i in harness.solve_info]
    ill = int((hd.stats()[:, 7] > 12).sum())
    hd.close()
    hp = CpHandle(mats, default_options(device=device, plain_kernel=1))
    rows_p, t_p, _ = rve_run(hp, True)
    hp.close()
    hh = CpHandle(mats, default_options(device=device, plain_kernel=1))
    rows_h, t_h, _ = rve_run(hh, False)
    hh.close()
    hm = CpHandle(mats, default_options(device=device))
    rows_m, t_m, hmh = rve_run(hm, True, default_solver(precision=CP_PRECISION_MIXED))
    hm.close()
    serr = lambda r, ref: float(np.abs(r[:, 6:12] - ref[:, 6:12]).max() / np.abs(ref[:, 6:12]).max())
    out = {"workload": "8x8x8 Q1 FCC Cu cube, 512 grains, x-tension to 2% in 20 increments x (4 Newton + post-pass)",
           "qp_updates": RVE_INC * (RVE_NEWTON + 1) * 4096,
           "rve_solves_per_s": 1.0 / t_d, "seconds": t_d, "linear_iterations_mean": float(np.mean(iters)),
           "plain_gpu_same_solver": {"seconds": t_p, "rve_solves_per_s": 1.0 / t_p,
                                     "rows_bit_identical": bool(np.array_equal(rows_d, rows_p))},
           "stress_rel_err_vs_plain_gpu": serr(rows_d, rows_p),
           "speedup_vs_plain_gpu_same_solver": t_p / t_d,
           "plain_drop_in_host_solve": {"seconds": t_h, "rve_solves_per_s": 1.0 / t_h,
                                        "stress_rel_err_vs_device_loop": serr(rows_h, rows_d),
                                        "speedup_of_device_loop": t_h / t_d},
           "mixed_precision": {"seconds": t_m, "rve_solves_per_s": 1.0 / t_m,
                               "stress_rel_err_vs_fp64_device_loop": serr(rows_m, rows_d),
                               "inner_iterations_mean": float(np.mean([i["iterations"] for i in hmh.solve_info])),
                               "fp64_iterations_mean": float(np.mean([i["fp64_iterations"]
                                                                      for i in hmh.solve_info])),
                               "all_converged": all(i["converged"] for i in hmh.solve_info)},
           "ill_conditioned_qps_at_end": ill,
           "final_stress_xx_mpa": float(rows_d[-1, 6])}
    if not args.no_cpu_baseline:
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        ob = O.OracleBackend(mats, default_options(), nthreads=threads)
        rows_c, t_c, _ = rve_run(ob, False)
        out["cpu_baseline"] = {"seconds": t_c, "rve_solves_per_s": 1.0 / t_c, "cores": threads, "kind": "port",
                               "stress_rel_err_vs_device_loop": serr(rows_c, rows_d)}
    return out


def _final_state_ke_error(be, mesh, u, device):
    """FP64 and tensor-core element matrices of the handle's current state at
    displacement u: max over cells of max|Ke_mixed - Ke_fp64| / max|Ke_fp64|."""
    import torch
    nc = mesh.n_cells
    dev = torch.device("cuda", device)
    Ul = torch.from_numpy(np.ascontiguousarray(u[mesh.cell_dofs])).to(dev)
    K64 = torch.empty(nc, 576, dtype=torch.float64, device=dev)
    K32 = torch.empty(nc, 576, dtype=torch.float32, device=dev)
    R = torch.empty(nc, 24, dtype=torch.float64, device=dev)
    be.assemble_device(Ul.data_ptr(), 0.0, 0.0, K64.data_ptr(), R.data_ptr())
    be.assemble_mixed_device(Ul.data_ptr(), 0.0, 0.0, K32.data_ptr(), R.data_ptr())
    be.synchronize()
    err = float(((K32.double() - K64).abs().amax(dim=1) / K64.abs().amax(dim=1)).max())
    del K64, K32, R, Ul
    return err


def _rve_arms(mesh, mats, lid, rod, increments, device, **harness_kw):
    """The same RVE solved by the FP64 device loop and by the mixed-precision
    one (tensor-core Ke, FP32 BiCG in FP64 refinement): times, solver
    statistics and the mixed run's errors against the FP64 run."""
    from plasticity_b200 import harness as Hm
    from plasticity_b200.capi import CP_PRECISION_MIXED, CpHandle, default_options, default_solver
    runs = {}
    for name, prec in (("fp64", 0), ("mixed", CP_PRECISION_MIXED)):
        t0 = time.perf_counter()
        be = CpHandle(mats, default_options(device=device))
        be.bind_qps(lid, rod)
        h = Hm.NewtonHarness(be, mesh, harness_kw.get("bc"), increments, 4, device_system=True,
                             solver=default_solver(precision=prec),
                             **{k: v for k, v in harness_kw.items() if k != "bc"})
        t_setup = time.perf_counter() - t0
        per_inc = []
        for _ in range(increments):
            t1 = time.perf_counter()
            h.step()
            per_inc.append(time.perf_counter() - t1)
        info = h.solve_info
        r = {"setup_s": t_setup, "seconds": float(np.sum(per_inc)),
             "seconds_per_increment": {"mean": float(np.mean(per_inc)), "max": float(np.max(per_inc))},
             "rve_solves_per_s": 1.0 / float(np.sum(per_inc)),
             "qp_updates_per_s": 5 * mesh.n_cells * 8 * increments / float(np.sum(per_inc)),
             "linear_iterations_mean": float(np.mean([i["iterations"] for i in info])),
             "fp64_iterations_mean": float(np.mean([i["fp64_iterations"] for i in info])),
             "all_converged": all(i["converged"] for i in info)}
        if prec:
            r["refinements_mean"] = float(np.mean([i["refinements"] for i in info]))
        rows = np.array(h.rows)
        u = h.u.copy()
        if name == "fp64":
            r["ke_rel_err_mixed_vs_fp64_at_final_state"] = _final_state_ke_error(be, mesh, u, device)
            r["max_potentially_active"] = int(be.stats()[:, 0].max())
            r["ill_conditioned_qps_at_end"] = int((be.stats()[:, 7] > 12).sum())
        be.close()
        runs[name] = (r, rows, u)
    (r64, rows64, u64), (rmx, rowsmx, umx) = runs["fp64"], runs["mixed"]
    srow = np.abs(rows64[:, 6:12]).max(axis=1)
    rmx["errors_vs_fp64"] = {
        "ke_rel_err_at_final_state": r64.pop("ke_rel_err_mixed_vs_fp64_at_final_state"),
        "stress_rel_err_first_increment": float(np.abs(rowsmx[0, 6:12] - rows64[0, 6:12]).max() / srow[0]),
        "stress_rel_err_max_over_run": float((np.abs(rowsmx[:, 6:12] - rows64[:, 6:12]).max(axis=1) / srow).max()),
        "u_rel_err_at_end": float(np.abs(umx - u64).max() / np.abs(u64).max())}
    r64["final_stress_mpa"] = [float(x) for x in rows64[-1, 6:9]]
    rmx["final_stress_mpa"] = [float(x) for x in rowsmx[-1, 6:9]]
    return {"fp64": r64, "mixed": rmx, "mixed_speedup": r64["seconds"] / rmx["seconds"]}


def rve_large_leg(args, device, increments=50):
    """The 48^3 FCC polycrystal (110,592 cells, 884,736 qps, 352,947 dofs;
    200 Voronoi grains: nearest of 200 seeded points, seeded orientations;
    x-tension to 5 % in 50 increments of 4 Newton iterations and the
    post-pass), solved whole by the FP64 device loop and by the mixed-precision
    one, with the mixed run's errors in Ke, stress and u against the FP64 run."""
    from plasticity_b200 import harness as Hm
    from plasticity_b200 import materials as M
    mesh = Hm.StructuredMesh((48, 48, 48))
    pts = np.random.default_rng(3).random((200, 3))
    grain_rod = M.random_rodrigues(np.random.default_rng(4), 200)
    cc = mesh.cell_centres()
    d2 = (pts ** 2).sum(1)[None, :] - 2.0 * cc @ pts.T  # |c - p|^2 up to the per-cell constant
    rod = np.repeat(grain_rod[d2.argmin(axis=1)], 8, axis=0)
    bc = np.array([[1, 1, 0.0], [1, 2, 0.0], [1, 3, 0.0], [2, 1, 0.05]])
    out = {"workload": f"48^3 Q1 FCC cube, 200 Voronoi grains, x-tension 5 % / 50 increments ({increments} run)",
           "cells": mesh.n_cells, "dofs": mesh.n_dofs, "increments": increments}
    out.update(_rve_arms(mesh, [M.fcc_cu()], np.zeros(mesh.n_cells * 8, np.int32), rod, increments, device, bc=bc))
    return out


def rve_dualphase_leg(args, device, increments=40):
    """The dual-phase RVE: a 32^3 Q1 cube (32,768 cells, 262,144 qps, 107,811
    dofs) of 100 Voronoi grains (nearest of 100 seeded points), each BCC or
    HCP with probability 1/2 (the batched workload's lattices; HCP twins
    reorient at twin fraction 0.9), under the velocity gradient of uniaxial
    z-compression, L = diag(5e-4, 5e-4, -1e-3)/s with dt = 1 s (4 % in 40
    increments), every boundary dof prescribed; the whole solve by the FP64
    device loop and by the mixed-precision one."""
    from plasticity_b200 import harness as Hm
    from plasticity_b200 import materials as M
    mesh = Hm.StructuredMesh((32, 32, 32))
    rng = np.random.default_rng(5)
    pts = rng.random((100, 3))
    grain_lat = (rng.random(100) < 0.5).astype(np.int32)  # 0 BCC, 1 HCP
    grain_rod = M.random_rodrigues(rng, 100)
    cc = mesh.cell_centres()
    d2 = (pts ** 2).sum(1)[None, :] - 2.0 * cc @ pts.T
    g = d2.argmin(axis=1)
    lid = np.repeat(grain_lat[g], 8).astype(np.int32)
    rod = np.repeat(grain_rod[g], 8, axis=0)
    L = np.diag([5e-4, 5e-4, -1e-3])
    out = {"workload": "32^3 Q1 BCC/HCP dual-phase cube, 100 Voronoi grains, velocity-gradient z-compression "
                       f"4 % / 40 increments ({increments} run)",
           "cells": mesh.n_cells, "dofs": mesh.n_dofs, "qps_hcp": int((lid == 1).sum()), "increments": increments}
    out.update(_rve_arms(mesh, [M.bcc_48(), M.hcp_mg(twin_threshold=0.9)], lid, rod, increments, device,
                         bc=None, vel_grad=L, delT=1.0))
    return out


def serve_leg(args, device, n_requests=16, rates=(4.0, 64.0), slots=8, edges=(8, 12, 16, 24, 32),
              increments=(10, 50)):
    """The served RVE stream: n_requests independent RVE solves per arrival
    rate (Poisson), each a Q1 cube of edge^3 elements (edge drawn from
    {8, 12, 16, 24, 32}), a lattice drawn from FCC/BCC/HCP (the batched
    workload's), 8-64 Voronoi grains and 10-50 increments of a random
    traceless velocity gradient of norm 1e-3/s (dt = 1 s); admitted by a
    device-memory budget (80 % of the free memory) with up to ``slots`` in
    flight.  Three servers: the same requests one at a time with the plain
    FP64 kernel (the baseline), concurrent requests each on its own handle
    and stream, and continuous batching (the qp updates of all requests in
    flight in shared launches).  Reports solves/s and p50/p95/p99 latency
    (completion minus arrival) and checks that every batched result equals
    its one-at-a-time result bit for bit."""
    import torch
    from plasticity_b200 import serving as S
    from plasticity_b200.capi import default_options
    mats = materials()
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(0.8 * free)
    out = {"workload": f"{n_requests} RVE requests per rate: edge {edges}, FCC/BCC/HCP, 8-64 grains, "
                       f"{increments[0]}-{increments[1]} increments of a random traceless velocity gradient "
                       "(norm 1e-3/s, dt 1 s)",
           "slots": slots, "budget_gb": budget / 1e9, "rates_per_s": list(rates)}
    warm = S.request_stream(2, 0.0, 99, edges=(8,), increments=(2, 2))
    S.RveServer(mats, budget, 1).run(warm)
    S.BatchedRveServer(mats, budget, 2, device=device).run(warm)
    base = S.request_stream(n_requests, 0.0, 6, edges=edges, increments=increments)
    t0 = time.perf_counter()
    plain = S.RveServer(mats, budget, 1, options_fn=lambda: default_options(device=device, plain_kernel=1)).run(base)
    out["sequential_plain_fp64"] = S.summarize(plain, time.perf_counter() - t0)
    t0 = time.perf_counter()
    seq = S.RveServer(mats, budget, 1).run(base)
    out["sequential"] = S.summarize(seq, time.perf_counter() - t0)
    for rate in rates:
        reqs = S.request_stream(n_requests, rate, 6, edges=edges, increments=increments)
        row = {}
        for name, srv in (("concurrent", S.RveServer(mats, budget, slots)),
                          ("batched", S.BatchedRveServer(mats, budget, slots, device=device))):
            t0 = time.perf_counter()
            res = srv.run(reqs)
            summ = S.summarize(res, time.perf_counter() - t0)
            summ["max_in_flight"] = srv.max_in_flight
            summ["same_rows_as_sequential"] = bool(all(np.array_equal(a.rows, b.rows) for a, b in zip(seq, res)
                                                       if a.rows is not None and b.rows is not None))
            if name == "batched":
                summ["ticks"] = srv.ticks
                summ["shared_update_launches"] = srv.batched_launches
            summ["solves_per_s_vs_sequential_plain_fp64"] = (summ["solves_per_s"]
                                                             / out["sequential_plain_fp64"]["solves_per_s"])
            row[name] = summ
        out[f"rate_{rate:g}"] = row
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-qp", type=int, default=N_QP)
    ap.add_argument("--cpu-sample", type=int, default=1 << 16)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain thread-per-qp kernel")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuning before the timing")
    ap.add_argument("--update-variant", type=int, default=0,
                    help="cp_options_t.update_variant: 0 = tuned/default shapes, k forces launch shape k-1")
    ap.add_argument("--no-rve", action="store_true", help="skip the RVE-solve leg")
    ap.add_argument("--no-assembly", action="store_true", help="skip the element-assembly leg")
    ap.add_argument("--asm-n", type=int, default=ASM_N, help="cells per edge of the element-assembly leg's cube")
    ap.add_argument("--assembly-only", action="store_true", help="only run the element-assembly leg")
    ap.add_argument("--rve-large", action="store_true", help="only run the 48^3 RVE leg")
    ap.add_argument("--rve-large-increments", type=int, default=50,
                    help="increments the 48^3 RVE leg runs (of its 50)")
    ap.add_argument("--no-rve-large", action="store_true", help="skip the 48^3 RVE leg")
    ap.add_argument("--no-dualphase", action="store_true", help="skip the 32^3 dual-phase RVE leg")
    ap.add_argument("--serve", action="store_true", help="only time the served RVE stream")
    ap.add_argument("--serve-requests", type=int, default=16, help="requests per arrival rate of the serve leg")
    ap.add_argument("--serve-rates", default="4,64", help="arrival rates (per s) of the serve leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the served RVE stream leg")
    ap.add_argument("--rve-only", action="store_true", help="only time the 8^3 RVE solve on the device")
    ap.add_argument("--rve-increments", type=int, default=40,
                    help="increments the dual-phase RVE leg times (of its 40)")
    ap.add_argument("--rve-dualphase", action="store_true",
                    help="only run the 32^3 BCC/HCP velocity-gradient RVE leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return reference_arm(args)
    if args.rve_large:
        print(json.dumps({"rve_large": rve_large_leg(args, int(os.environ.get("LOCAL_RANK", "0")),
                                                     args.rve_large_increments)}), flush=True)
        return 0
    if args.assembly_only:
        print(json.dumps({"assembly": assembly_leg(args, int(os.environ.get("LOCAL_RANK", "0")))}), flush=True)
        return 0
    if args.rve_only:
        from plasticity_b200.capi import CpHandle, default_options
        from plasticity_b200 import materials as M
        be = CpHandle([M.fcc_cu()], default_options(device=int(os.environ.get("LOCAL_RANK", "0"))))
        rows, t, h = rve_run(be, True)
        print(json.dumps({"rve_device": {"seconds": t, "rve_solves_per_s": 1.0 / t,
                                         "final_stress_xx_mpa": float(rows[-1][6]),
                                         "linear_iterations_mean": float(np.mean([i["iterations"]
                                                                                  for i in h.solve_info]))}}),
              flush=True)
        be.close()
        return 0
    if args.serve:
        print(json.dumps({"serve": serve_leg(args, int(os.environ.get("LOCAL_RANK", "0")), args.serve_requests,
                                             tuple(float(x) for x in args.serve_rates.split(",")))}), flush=True)
        return 0
    if args.rve_dualphase:
        print(json.dumps({"rve_dualphase": rve_dualphase_leg(args, int(os.environ.get("LOCAL_RANK", "0")),
                                                             args.rve_increments)}), flush=True)
        return 0
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
