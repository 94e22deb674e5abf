"""Domain decomposition with a halo exchange per tendency (the reference's TRiSKDistribution):
the equal-area partition, the owned/ghost sets, and the reference's 1-vs-n property
(test/finite_volumes.jl:245-261; "1, 3, 4 ranks bitwise identical", docs/STATUS.md:15-18):
owned values after RK4 steps on 2, 3 or 4 ranks equal the undivided run bit for bit. On CPU
the local tendency is the oracle's on the local tables (gloo ranks); on the GPU, two ranks
share one GPU and exchange through host memory (gloo), each running the library's kernels on
its local tables."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import trisk_grid


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_equal_area_partition():
    from dmplex_b200.distribution import balanced_counts, equal_area_partition, equal_area_zones
    for n in (1, 2, 3, 4, 6, 8, 13):
        assert sum(equal_area_zones(n)) == n
    g = trisk_grid(3, True)
    for n in (1, 2, 5):
        part = equal_area_partition(g.centers, n)
        counts = np.bincount(part, minlength=n + 1)[1:]
        assert sorted(counts.tolist()) == sorted(balanced_counts(g.nc, n))
    assert np.all(equal_area_partition(g.centers, 2)[g.centers[:, 2] > 0.5] == 1)  # north first


def test_distribution_sets():
    from dmplex_b200.distribution import TRiSKDistribution, equal_area_partition
    g = trisk_grid(3, True)
    part = equal_area_partition(g.centers, 3)
    ds = [TRiSKDistribution(g, part, 3, r) for r in range(3)]
    owned_cells = np.concatenate([d.cells.global_ids[:d.cells.n_owned] for d in ds])
    owned_edges = np.concatenate([d.edges.global_ids[:d.edges.n_owned] for d in ds])
    assert np.array_equal(np.sort(owned_cells), np.arange(g.nc))
    assert np.array_equal(np.sort(owned_edges), np.arange(g.ne))
    for r, d in enumerate(ds):  # what I send to q is what q receives from me
        for q, send in zip(d.state_neighbors, d.state_send):
            dq = ds[q]
            recv = dq.state_recv[dq.state_neighbors.index(r)]
            ne_r, ne_q = len(d.edges), len(dq.edges)

            def glob(dd, idx, ne):
                return [("e", int(dd.edges.global_ids[i])) if i < ne else ("c", int(dd.cells.global_ids[i - ne]))
                        for i in idx]
            assert glob(d, send, ne_r) == glob(dq, recv, ne_q)


def _rank_cpu(rank, world, port, pv, ke, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import dmplex_b200 as d
        from dmplex_b200 import workloads as w
        from dmplex_b200.distribution import DistributedShallowWater
        from oracle.oracle import Oracle
        from conftest import trisk_grid as tg
        g = tg(3, True)
        si = w.si_parameters()

        class _Engine:
            def __init__(self, coeffs):
                self.o = Oracle(coeffs)

            def tendency(self, y):
                return self.o.tendency(y)

        m = DistributedShallowWater(g, pv_flux=pv, kinetic_energy=ke, engine=_Engine, **si)
        y = w.synthetic_state(g, seed=5)
        yl = m.local_state(y)
        m.rk4_step(yl, 300.0, 3)
        out.put((rank, m.gather_state(yl)))
    finally:
        dist.destroy_process_group()


def _spawn(target, world, *args):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, *args, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return [r for _, r in sorted(res, key=lambda t: t[0])]


@pytest.mark.parametrize("world,pv,ke", [(2, "trisk", "cell"), (3, "gassmann", "vertex"),
                                         (2, "gassmann_mean", "mixed"), (4, "trisk", "mixed")])
def test_one_vs_n_bitwise_cpu(world, pv, ke):
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    g = trisk_grid(3, True)
    si = w.si_parameters()
    ref = w.synthetic_state(g, seed=5)
    Oracle(d.model_tables(g, pv_flux=pv, kinetic_energy=ke, **si)).rk4_step(ref, 300.0, 3)
    for got in _spawn(_rank_cpu, world, pv, ke):
        assert np.array_equal(got, ref)


def _rank_gpu(rank, world, port, out):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from dmplex_b200 import workloads as w
        from dmplex_b200.distribution import DistributedShallowWater
        from conftest import trisk_grid as tg
        g = tg(4, True)
        m = DistributedShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", device=0, **w.si_parameters())
        yl = torch.from_numpy(m.local_state(w.synthetic_state(g, seed=6))).cuda()
        m.rk4_step(yl, 300.0, 3)
        torch.cuda.synchronize()
        out.put((rank, m.gather_state(yl)))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_one_vs_n_bitwise_gpu(require_gpu):
    """Two ranks on one GPU (host-staged gloo exchange; their kernels never wait on each
    other) against the undivided GPU model."""
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **w.si_parameters())
    ref = w.synthetic_state(g, seed=6)
    d.rk4_step(ref, 300.0, d.tendency, d.RK4Cache(ref), m, nsteps=3)
    del m
    for got in _spawn(_rank_gpu, 2):
        assert np.array_equal(got, ref)
