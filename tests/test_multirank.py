"""The N > 1 path of bench.py on CPU: two gloo ranks, each with its own replica (seeded by
its rank, no data exchanged), meet at the barrier, take the slowest rank's time by an
all-reduce and report the whole job's cell-steps/s; the reference arm runs on rank 0 only.
The GPU replicas use the same helpers with NCCL and a CUDA tensor."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys
    import time
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import dmplex_b200 as d
        from dmplex_b200 import workloads as w
        from oracle.oracle import Oracle
        g, y = bench.build_workload(seed=rank, level=3)
        o = Oracle(d.model_tables(g, pv_flux=bench.PV, kinetic_energy=bench.KE, **w.si_parameters()))
        bench.rank_barrier(world, cuda=False)
        t0 = time.perf_counter()
        o.rk4_step(y, bench.DT, 3)
        ms = (time.perf_counter() - t0) * 1e3 + 5.0 * rank  # ranks finish at different times
        slowest = bench.max_over_ranks_of(ms, world)
        times = [None] * world
        dist.all_gather_object(times, ms)
        states = [None] * world
        dist.all_gather_object(states, float(np.sum(y)))
        value = bench.whole_job_value(world, g.nc, 3, slowest)
        # the reference arm: rank 0 alone runs it, the others return at once
        if rank != 0:
            t1 = time.perf_counter()
            bench.run_reference(None, rank, world)
            ref_s = time.perf_counter() - t1
        else:
            ref_s = 0.0
        out.put((rank, slowest, max(times), value, g.nc, states, ref_s))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = [out.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    slowest = [r[1] for r in res]
    assert slowest[0] == slowest[1] == res[0][2]  # every rank holds the max over ranks
    nc = res[0][4]
    assert res[0][3] == pytest.approx(world * nc * 3 / (slowest[0] * 1e-3))
    sums = res[0][5]
    assert sums[0] != sums[1]  # each rank advanced its own replica
    assert res[1][6] < 1.0     # the reference arm does no work off rank 0
