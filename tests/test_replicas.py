"""The multi-GPU path is replicas only: every rank runs its own batch with
rank-offset seeds and no exchange on the data path; the job time is the
slowest rank's (max over ranks) and the value aggregates all ranks' qps.
Exercised here with two gloo processes on the CPU."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    n = 20000
    lid = bench.lattice_ids(n, rank)
    rod = bench.orientations(n, rank)
    local_s = 0.010 + 0.005 * rank  # this replica's time
    t = bench.max_over_ranks(local_s, torch.device("cpu"))
    v = bench.aggregate_value(world, n, 4, t)
    q.put((rank, t, v, np.bincount(lid, minlength=3).tolist(), lid[:64].tolist(), rod[:4].tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, c0, l0, o0), (r1, t1, v1, c1, l1, o1) = res
    assert t0 == t1 == pytest.approx(0.015)  # the slowest replica sets the job time
    assert v0 == v1 == pytest.approx(2 * 20000 * 4 / 0.015)
    assert l0 != l1 and o0 != o1  # rank-offset seeds: independent replicas
    for c in (c0, c1):  # each replica keeps the 50/30/20 FCC/BCC/HCP mix
        assert np.allclose(np.array(c) / 20000, [0.5, 0.3, 0.2], atol=1e-4)
