"""Domain decomposition with a halo exchange per tendency (the reference's TRiSKDistribution):
the equal-area partition, the owned/ghost sets, the halo lists handed to the library, and the
reference's 1-vs-n property (test/finite_volumes.jl:245-261; "1, 3, 4 ranks bitwise
identical", docs/STATUS.md:15-18): owned values after RK4 steps on 2, 3 or 4 ranks equal the
undivided run bit for bit. On CPU the local tendency is the oracle's on the local tables and
the exchange is the library's HaloExchange over gloo ranks; on the GPU, two or three ranks
share one GPU, each running its part in the library (trisk_dist_*: RK4 stages fused, ghost
tendencies zeroed in the tendency kernel, halo packed and unpacked by kernels) and
exchanging through host memory (gloo), so their kernels never wait on each other."""
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


def test_halo_lists_for_the_library():
    """The halo as the library takes it: CSR offsets and 1-based local state indices in the
    neighbour order; sent entries owned, received entries ghosts."""
    from dmplex_b200.distribution import TRiSKDistribution, equal_area_partition, halo_lists
    g = trisk_grid(3, True)
    part = equal_area_partition(g.centers, 3)
    for r in range(3):
        d = TRiSKDistribution(g, part, 3, r)
        so, si, ro, ri = halo_lists(d)
        assert len(so) == len(d.state_neighbors) + 1 and so[0] == 0 and so[-1] == len(si)
        for k in range(len(d.state_neighbors)):
            assert np.array_equal(si[so[k]:so[k + 1]] - 1, d.state_send[k])
            assert np.array_equal(ri[ro[k]:ro[k + 1]] - 1, d.state_recv[k])
        ne = len(d.edges)
        owned = lambda x: (x < d.edges.n_owned) | ((x >= ne) & (x < ne + d.cells.n_owned))  # noqa: E731
        assert owned(si - 1).all() and not owned(ri - 1).any()


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


def _rank_gpu(rank, world, port, pv, ke, out):
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
        m = DistributedShallowWater(g, pv_flux=pv, kinetic_energy=ke, device=0, **w.si_parameters())
        yl = torch.from_numpy(m.local_state(w.synthetic_state(g, seed=6))).cuda()
        m.rk4_step(yl, 300.0, 3)
        torch.cuda.synchronize()
        dy = torch.empty_like(yl)
        m.tendency(dy, yl)
        d = m.dist
        ghosts_zero = bool((dy[d.edges.n_owned:m.ne] == 0).all() and (dy[m.ne + d.cells.n_owned:] == 0).all())
        out.put((rank, (m.gather_state(yl), ghosts_zero)))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("world,pv,ke", [(2, "gassmann", "vertex"), (3, "gassmann_mean", "mixed")])
def test_one_vs_n_bitwise_gpu(require_gpu, world, pv, ke):
    """Two or three ranks on one GPU, each part in the library (host-staged gloo exchange;
    their kernels never wait on each other), against the undivided GPU model; ghost
    tendencies are zero."""
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **w.si_parameters())
    ref = w.synthetic_state(g, seed=6)
    d.rk4_step(ref, 300.0, d.tendency, d.RK4Cache(ref), m, nsteps=3)
    del m
    for got, ghosts_zero in _spawn(_rank_gpu, world, pv, ke):
        assert np.array_equal(got, ref)
        assert ghosts_zero


@pytest.mark.gpu
def test_single_part_in_the_library(require_gpu):
    """One rank: the library's part (no neighbours, no exchange) is the model bit for bit, and
    its RK4 step is the model's 12 launches."""
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from dmplex_b200.distribution import DistributedShallowWater
    g = trisk_grid(4, True)
    si = w.si_parameters()
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    y = w.synthetic_state(g, seed=2)
    ref = y.copy()
    d.rk4_step(ref, 300.0, d.tendency, d.RK4Cache(ref), m, nsteps=2)
    part = DistributedShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    assert part.dist.state_neighbors == []
    yl = part.local_state(y)
    before = part.engine.launch_count()
    part.rk4_step(yl, 300.0, 2)
    assert part.engine.launch_count() - before == 2 * 12 + 2  # + the state's numbering in and out
    assert np.array_equal(part.gather_state(yl), ref)


@pytest.mark.gpu
def test_dist_rejects_bad_halos(require_gpu):
    """trisk_dist_create checks the halo on the host: a sent ghost or a received owned entry,
    and an index outside the local state, are TRISK_ERR_TABLE; decreasing offsets and owned
    counts beyond the local sizes are TRISK_ERR_ARGUMENT."""
    import ctypes as C
    import dmplex_b200 as d
    from dmplex_b200 import _lib
    from dmplex_b200.model import _coefficients_struct
    g = trisk_grid(3, True)
    t = d.model_tables(g)
    cs, keep = _coefficients_struct(t, 0, 1.0, 1.0)
    cfg = _lib.TriskConfig()
    cfg.alpha, cfg.gravity, cfg.omega, cfg.use_graph, cfg.use_pdl = 1.0, 1.0, 1.0, 1, 1

    def create(ne_owned, nc_owned, send, recv, so=None, ro=None):
        so = np.array(so if so is not None else [0, len(send)], dtype=np.int64)
        ro = np.array(ro if ro is not None else [0, len(recv)], dtype=np.int64)
        si, ri = np.array(send, dtype=np.int64), np.array(recv, dtype=np.int64)
        h = _lib.TriskHalo()
        h.ne_owned, h.nc_owned, h.nneighbors = ne_owned, nc_owned, len(so) - 1
        h.send_offsets, h.send_index, h.recv_offsets, h.recv_index = (a.ctypes.data for a in (so, si, ro, ri))
        out = C.c_void_p()
        status = _lib.lib.trisk_dist_create(C.byref(cs), C.byref(cfg), C.byref(h), C.byref(out))
        if status == 0:
            _lib.lib.trisk_dist_destroy(out)
        return status
    ne, nc = g.ne, g.nc
    assert create(ne - 10, nc - 5, [1, 2], [ne - 1, ne + nc]) == 0
    assert create(ne - 10, nc - 5, [ne - 1], [ne]) == 2          # a sent ghost edge
    assert create(ne - 10, nc - 5, [1], [3]) == 2                # a received owned edge
    assert create(ne - 10, nc - 5, [1], [ne + nc + 1]) == 2      # outside the local state
    assert create(ne - 10, nc - 5, [1, 2], [ne], so=[0, 2, 1], ro=[0, 1, 1]) == 1  # offsets go down
    assert create(ne + 1, nc, [], []) == 1
