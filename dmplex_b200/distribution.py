"""Domain decomposition of one TRiSK model over ranks with a halo exchange per tendency.

Mirrors the reference's distributed shallow-water path:

    equal_area_partition(dm, nparts)          src/Parallel/Partition.jl:47-106
    TRiSKDistribution(grid, part, n, rank)    src/FiniteVolumes/TRiSKDistribution.jl:70-106
    local_table / local_numbers               TRiSKDistribution.jl:108-125
    the local model of TRiSKShallowWater      src/FiniteVolumes/TRiSKShallowWater.jl:121-168
    tendency! with exchange_state!            TRiSKShallowWater.jl:379-394

Cells are split into parts of equal count along the zonal equal-area regions of the sphere;
each rank holds its owned cells plus `rings` vertex rings of ghost cells (two for the TRiSK
and Gassmann PV fluxes, three for the averaged Gassmann PV), and every edge and vertex of
them. Edges and vertices belong to the smallest part among their cells. Local numbering puts
the owned entities first; the state [u; h] is exchanged once per tendency (one message per
neighbour: its edges, then its cells) and the tendencies of ghosts are zeroed, so the owned
values are those of the undivided model bit for bit.

The rank's part runs in the library (trisk_dist_*: its tendency and RK4 steps with the stage
updates fused, the ghost tendencies zeroed in the tendency kernel, the halo packed and unpacked
by gather kernels), which calls back into HaloExchange once per tendency for the exchange
itself: torch.distributed point-to-point messages, on the library's stream with NCCL between
GPUs, or through host memory with gloo.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, lib
from .model import _alpha, _coefficients_struct, _pv_code, _state, model_tables

# ------------------------------------------------------------------ partition (Partition.jl)


def _area_of_cap(s_cap):
    return 4 * math.pi * math.sin(s_cap / 2) ** 2


def _sradius_of_cap(area):
    return 2 * math.asin(math.sqrt(area / math.pi) / 2)


def equal_area_zones(n: int) -> list:
    """Regions per zone (north cap, collars, south cap) of the zonal equal-area partition of
    the sphere into n regions (Partition.jl:15-33)."""
    if n < 1:
        raise ValueError("need at least one region")
    if n == 1:
        return [1]
    ideal_area = 4 * math.pi / n
    c_polar = math.pi / 2 if n == 2 else _sradius_of_cap(ideal_area)
    a_ideal = math.sqrt(ideal_area)
    n_collars = max(1, _round_half_even((math.pi - 2 * c_polar) / a_ideal)) if n > 2 else 1
    a_fitting = (math.pi - 2 * c_polar) / n_collars
    ideal = [1.0] + [(_area_of_cap(c_polar + k * a_fitting) - _area_of_cap(c_polar + (k - 1) * a_fitting))
                     / ideal_area for k in range(1, n_collars + 1)] + [1.0]
    regions, discrepancy = [], 0.0
    for r in ideal:  # round to naturals, carrying the discrepancy
        z = _round_half_even(r + discrepancy)
        regions.append(z)
        discrepancy += r - z
    return [r for r in regions if r > 0]


def _round_half_even(x: float) -> int:
    return int(round(x))  # Python's round ties to even, as Julia's round


def balanced_counts(n: int, parts: int) -> list:
    """n items in `parts` counts that differ by at most one (Partition.jl:36)."""
    return [n // parts + (1 if p <= n % parts else 0) for p in range(1, parts + 1)]


def equal_area_partition(centers: np.ndarray, nparts: int) -> np.ndarray:
    """Part (1-based) of every cell: cells sorted north to south and handed out zone by zone,
    each collar sorted west to east (Partition.jl:47-106, the sphere case)."""
    x = np.asarray(centers, dtype=np.float64)
    nc = len(x)
    if nparts > nc:
        raise ValueError("more parts than cells")
    north_south = np.arcsin(np.clip(x[:, 2] / np.linalg.norm(x, axis=1), -1, 1))
    west_east = np.mod(np.arctan2(x[:, 1], x[:, 0]), 2 * math.pi)
    zones = equal_area_zones(nparts)
    counts = balanced_counts(nc, nparts)
    order = np.lexsort((west_east, -north_south))  # latitude descending, then longitude
    part = np.zeros(nc, dtype=np.int64)
    region, start = 0, 0
    for nzone in zones:
        zone_count = sum(counts[region:region + nzone])
        cells = order[start:start + zone_count]
        cells = cells[np.lexsort((-north_south[cells], west_east[cells]))]
        offset = 0
        for r in range(nzone):
            part[cells[offset:offset + counts[region + r]]] = region + r + 1
            offset += counts[region + r]
        region += nzone
        start += zone_count
    return part


# ------------------------------------------------------------------ distribution


class DofDistribution:
    """Local numbering of one entity kind on one rank (Parallel/Distribution.jl:136-154):
    global_ids (0-based) with the owned ones first, and the halo lists per neighbour rank
    (local indices of my ghosts it owns, and of my owned entities it holds as ghosts)."""

    def __init__(self, locals_: list, owner: np.ndarray, rank: int):
        me = rank + 1
        mine = locals_[rank]
        owned = mine[owner[mine] == me]
        ghost = mine[owner[mine] != me]
        self.global_ids = np.concatenate([owned, ghost])
        self.n_owned = len(owned)
        to_local = {int(g): i for i, g in enumerate(self.global_ids)}
        self.neighbors, self.send, self.recv = [], [], []
        for q, theirs in enumerate(locals_):
            if q == rank:
                continue
            from_q = [to_local[int(dd)] for dd in mine if owner[dd] == q + 1]
            to_q = [to_local[int(dd)] for dd in theirs if owner[dd] == me]
            if not from_q and not to_q:
                continue
            self.neighbors.append(q)
            self.recv.append(np.array(from_q, dtype=np.int64))
            self.send.append(np.array(to_q, dtype=np.int64))

    def __len__(self):
        return len(self.global_ids)


class TRiSKDistribution:
    """Owned and ghost cells, edges and vertices of `rank` (0-based) for the cell partition
    `part` (1-based parts), with `rings` vertex rings of ghost cells (TRiSKDistribution.jl)."""

    def __init__(self, grid, part: np.ndarray, nranks: int, rank: int, rings: int = 2):
        g = grid
        nc, ne, nv = g.nc, g.ne, g.nv
        part = np.asarray(part, dtype=np.int64)
        self.part, self.nranks, self.rank = part, int(nranks), int(rank)
        cv = g.cell_vertices - 1
        corner = g.cell_kites > 0
        ce = g.cell_edges - 1
        side = g.cell_signs != 0
        cells_of_vertex = [[] for _ in range(nv)]
        for i in range(nc):
            for v in cv[i][corner[i]]:
                cells_of_vertex[v].append(i)

        def ring(cells):
            out = set(cells)
            for i in cells:
                for v in cv[i][corner[i]]:
                    out.update(cells_of_vertex[v])
            return out

        local_cells = []
        for p in range(1, nranks + 1):
            cells = set(np.nonzero(part == p)[0].tolist())
            for _ in range(rings):
                cells = ring(cells)
            local_cells.append(np.array(sorted(cells), dtype=np.int64))
        local_edges = [np.unique(np.concatenate([ce[i][side[i]] for i in cells])) for cells in local_cells]
        ec = g.edge_cells - 1
        edge_owner = np.minimum(part[ec[:, 0]], part[ec[:, 1]])
        vertex_owner = np.array([min(part[c] for c in cells_of_vertex[v]) for v in range(nv)], dtype=np.int64)
        me = rank + 1
        verts = []
        seen = set()
        for i in local_cells[rank]:
            for v in cv[i][corner[i]]:
                if v not in seen:
                    seen.add(v)
                    verts.append(v)
        verts = np.array(verts, dtype=np.int64)
        self.vertex_ids = np.concatenate([verts[vertex_owner[verts] == me], verts[vertex_owner[verts] != me]])
        self.n_owned_vertices = int((vertex_owner[verts] == me).sum())
        self.cells = DofDistribution(local_cells, part, rank)
        self.edges = DofDistribution(local_edges, edge_owner, rank)
        # the state [u; h]: one message per neighbour, its edges then its cells
        nle = len(self.edges)
        nbrs = sorted(set(self.edges.neighbors) | set(self.cells.neighbors))

        def lists(d, q, which):
            return getattr(d, which)[d.neighbors.index(q)] if q in d.neighbors else np.zeros(0, np.int64)

        self.state_neighbors = nbrs
        self.state_send = [np.concatenate([lists(self.edges, q, "send"), lists(self.cells, q, "send") + nle])
                           for q in nbrs]
        self.state_recv = [np.concatenate([lists(self.edges, q, "recv"), lists(self.cells, q, "recv") + nle])
                           for q in nbrs]


def local_numbers(global_ids: np.ndarray, n: int) -> np.ndarray:
    """Global -> local map, 1-based, 0 if not local (TRiSKDistribution.jl:121-125)."""
    to_local = np.zeros(n, dtype=np.int64)
    to_local[global_ids] = np.arange(1, len(global_ids) + 1)
    return to_local


def local_table(indices, weights, rows, to_local):
    """Rows `rows` of a 1-based (entity, k) neighbour table with its indices mapped to local
    numbers; neighbours that are not local get index 1 and weight 0 (TRiSKDistribution.jl:
    108-119: they only occur at the outer edge of the halo, whose values no owned tendency
    uses)."""
    I = to_local[indices[rows] - 1]
    missing = I == 0
    I[missing] = 1
    W = None
    if weights is not None:
        W = np.array(weights[rows], dtype=np.float64)
        W[missing] = 0.0
    return np.ascontiguousarray(I), (None if W is None else np.ascontiguousarray(W))


def local_coefficients(coeffs: dict, dist: TRiSKDistribution) -> dict:
    """The model tables of `model_tables` restricted to the rank's local entities, in local
    numbering (TRiSKShallowWater.jl:121-168)."""
    cells, edges, verts = dist.cells.global_ids, dist.edges.global_ids, dist.vertex_ids
    lc = local_numbers(cells, coeffs["nc"])
    le = local_numbers(edges, coeffs["ne"])
    lv = local_numbers(verts, coeffs["nv"])
    out = {k: coeffs[k] for k in ("cw", "vw", "tw", "pv_flux", "alpha", "gravity")}
    out.update(nc=len(cells), ne=len(edges), nv=len(verts))
    pairs = [  # index table, entity rows, target map, weights riding on it
        ("cell_edges", cells, le, ("divergence", "kinetic")),
        ("edge_cells", edges, lc, ("edge_height",)),
        ("edge_vertices", edges, lv, ("rhombus", "vk_height")),
        ("vertex_edges", verts, le, ("curl", "vk_weights")),
        ("vertex_cells", verts, lc, ("vertex_height",)),
        ("trisk_edges", edges, le, ("trisk",)),
        ("g_edges", edges, le, ("g_weights",)),
        ("g_pv_edges", edges, le, ()),
        ("vk_cell_vertices", cells, lv, ("vk_kites",)),
    ]
    for name, rows, target, wnames in pairs:
        if coeffs.get(name) is None:
            out[name] = None
            for wn in wnames:
                out[wn] = None
            continue
        I, _ = local_table(coeffs[name], None, rows, target)
        out[name] = I
        for wn in wnames:
            if coeffs.get(wn) is None:
                out[wn] = None
            else:
                _, W = local_table(coeffs[name], coeffs[wn], rows, target)
                out[wn] = W
    for name, rows in (("inverse_dual", edges), ("coriolis", verts), ("g_coriolis", edges),
                       ("cell_areas", cells), ("vertex_areas", verts)):
        out[name] = None if coeffs.get(name) is None else np.ascontiguousarray(coeffs[name][rows])
    return out


def halo_lists(dist: TRiSKDistribution):
    """The state halo of `dist` as the library's TriskHalo arrays: CSR offsets and 1-based
    local state indices, neighbour after neighbour in dist.state_neighbors' order."""
    def csr(lists):
        offsets = np.zeros(len(lists) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([len(x) for x in lists])
        index = np.concatenate(lists).astype(np.int64) + 1 if lists else np.zeros(0, np.int64)
        return offsets, np.ascontiguousarray(index)
    so, si = csr(dist.state_send)
    ro, ri = csr(dist.state_recv)
    return so, si, ro, ri


class HaloExchange:
    """The exchange the library calls once per tendency (exchange!, Halo.jl:80-99): `send`
    holds the packed owned values for every neighbour in turn, `recv` gets the neighbours'
    values of my ghosts in the same order. One message pair per neighbour through
    torch.distributed; host arrays (gloo), or device tensors on `stream` (NCCL)."""

    def __init__(self, dist: TRiSKDistribution, group=None):
        self.group = group
        self.peers = list(dist.state_neighbors)
        self.send_counts = [len(x) for x in dist.state_send]
        self.recv_counts = [len(x) for x in dist.state_recv]

    def __call__(self, send, recv, stream=None) -> None:
        import torch
        import torch.distributed as tdist
        ops = []
        a = b = 0
        ctx = torch.cuda.stream(torch.cuda.ExternalStream(stream)) if stream else _nullcontext()
        with ctx:
            for q, ns, nr in zip(self.peers, self.send_counts, self.recv_counts):
                peer = tdist.get_global_rank(self.group, q) if self.group is not None else q
                if ns:
                    ops.append(tdist.P2POp(tdist.isend, send[a:a + ns], peer, self.group))
                if nr:
                    ops.append(tdist.P2POp(tdist.irecv, recv[b:b + nr], peer, self.group))
                a, b = a + ns, b + nr
            if ops:
                for req in tdist.batch_isend_irecv(ops):
                    req.wait()


class _nullcontext:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class _CudaBuffer:
    """A device buffer given by the library as a torch tensor (no copy)."""

    def __init__(self, address: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (address, False), "version": 3}


class _DistModel:
    """The library's part of a distributed model (trisk_dist_*) with its exchange callback."""

    def __init__(self, coefficients, dist, centers, exchange: HaloExchange, device_exchange: bool, *, gravity,
                 omega, pv_flux, kinetic_energy, device):
        pv, alpha = _pv_code(pv_flux), _alpha(kinetic_energy)
        cs, self._keep = _coefficients_struct(coefficients, pv, alpha, gravity)
        cfg = _lib.TriskConfig()
        cfg.pv_flux, cfg.reorder, cfg.alpha, cfg.gravity, cfg.omega = pv, 1, alpha, gravity, omega
        cfg.device, cfg.use_graph, cfg.use_pdl, cfg.block = device, 1, 1, 0
        pos = np.ascontiguousarray(centers, dtype=np.float64)
        self._keep.append(pos)
        cfg.cell_positions = pos.ctypes.data
        so, si, ro, ri = halo_lists(dist)
        self._keep += [so, si, ro, ri]
        halo = _lib.TriskHalo()
        halo.ne_owned, halo.nc_owned = dist.edges.n_owned, dist.cells.n_owned
        halo.nneighbors = len(dist.state_neighbors)
        halo.send_offsets, halo.send_index = so.ctypes.data, si.ctypes.data
        halo.recv_offsets, halo.recv_index = ro.ctypes.data, ri.ctypes.data
        h = C.c_void_p()
        check(lib.trisk_dist_create(C.byref(cs), C.byref(cfg), C.byref(halo), C.byref(h)))
        self._h = h
        self.exchange = exchange
        self._error = None
        self._callback = _lib.EXCHANGE_FN(self._exchange)  # kept alive with the model
        mode = _lib.EXCHANGE_DEVICE if device_exchange else _lib.EXCHANGE_HOST
        check(lib.trisk_dist_set_exchange(h, self._callback, None, mode))
        self.state_size = len(dist.edges) + len(dist.cells)

    def _exchange(self, user, send, nsend, recv, nrecv, stream):
        try:
            if stream:
                import torch
                s = torch.as_tensor(_CudaBuffer(send, nsend), device="cuda") if nsend else None
                r = torch.as_tensor(_CudaBuffer(recv, nrecv), device="cuda") if nrecv else None
            else:
                import torch
                s = torch.from_numpy(np.ctypeslib.as_array((C.c_double * max(nsend, 1)).from_address(send)))[:nsend]
                r = torch.from_numpy(np.ctypeslib.as_array((C.c_double * max(nrecv, 1)).from_address(recv)))[:nrecv]
            self.exchange(s, r, stream)
            return 0
        except Exception as exc:  # noqa: BLE001 - re-raised by _call once the library returns
            self._error = exc
            return 1

    def _call(self, fn, *args):
        status = fn(self._h, *args)
        if self._error is not None:
            err, self._error = self._error, None
            raise err
        check(status)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_dist_destroy(self._h)
            self._h = None

    def tendency(self, dy, y):
        self._call(lib.trisk_dist_tendency, _state(y, self), _state(dy, self))

    def rk4_step(self, y, dt: float, nsteps: int):
        self._call(lib.trisk_dist_rk4_step, _state(y, self), float(dt), int(nsteps))

    def launch_count(self) -> int:
        return int(lib.trisk_dist_launch_count(self._h))


class DistributedShallowWater:
    """One rank's part of a TRiSK shallow-water model (TRiSKShallowWater(grid; comm, part)).

    group: a torch.distributed process group (None: the default group); part: the cell
    partition (default: equal_area_partition). The rank's part runs in the library on GPU
    `device`; its halo exchange is HaloExchange over the group (on the GPU with NCCL, through
    host memory with gloo). `engine`, if given, is called with the local tables and returns
    the object whose tendency(y) -> dy (numpy) replaces the library's part (the tests pass the
    CPU oracle); the RK4 steps and the exchange are then done here, with the same HaloExchange
    on numpy buffers. States are local [u; h] vectors, owned entities first: numpy arrays, or
    CUDA float64 tensors.
    """

    def __init__(self, grid, *, gravity=1.0, omega=1.0, pv_flux="trisk", kinetic_energy="cell", part=None,
                 group=None, device: int = 0, engine=None):
        import torch.distributed as tdist
        self.group = group
        self.nranks = tdist.get_world_size(group) if tdist.is_initialized() else 1
        self.rank = tdist.get_rank(group) if tdist.is_initialized() else 0
        self.grid = grid
        if part is None:
            part = equal_area_partition(grid.centers, self.nranks)
        rings = 3 if str(pv_flux).lstrip(":") == "gassmann_mean" else 2
        self.dist = TRiSKDistribution(grid, part, self.nranks, self.rank, rings)
        self.global_coefficients = model_tables(grid, gravity=gravity, omega=omega, pv_flux=pv_flux,
                                                kinetic_energy=kinetic_energy)
        self.coefficients = local_coefficients(self.global_coefficients, self.dist)
        self.ne, self.nc = len(self.dist.edges), len(self.dist.cells)
        self.state_size = self.ne + self.nc
        self.exchange = HaloExchange(self.dist, group)
        if engine is None:
            backend = tdist.get_backend(group) if tdist.is_initialized() else "gloo"
            self.engine = _DistModel(self.coefficients, self.dist, grid.centers[self.dist.cells.global_ids],
                                     self.exchange, backend == "nccl", gravity=gravity, omega=omega,
                                     pv_flux=pv_flux, kinetic_energy=kinetic_energy, device=device)
        else:
            self.engine = engine(self.coefficients)

    # ---------------------------------------------------------------- state helpers
    def local_state(self, y_global: np.ndarray) -> np.ndarray:
        """The rank's local [u; h] (owned and ghost values) from a global state."""
        d = self.dist
        ne = self.grid.ne
        return np.concatenate([y_global[d.edges.global_ids], y_global[ne + d.cells.global_ids]])

    def owned(self, y_local):
        """(global edge ids, owned u), (global cell ids, owned h)."""
        d = self.dist
        yl = _to_numpy(y_local)
        return ((d.edges.global_ids[:d.edges.n_owned], yl[:d.edges.n_owned]),
                (d.cells.global_ids[:d.cells.n_owned], yl[self.ne:self.ne + d.cells.n_owned]))

    def gather_state(self, y_local) -> np.ndarray:
        """Global [u; h] with the owned values of all ranks, on every rank (gather_state)."""
        import torch.distributed as tdist
        (ei, eu), (ci, ch) = self.owned(y_local)
        parts = [None] * self.nranks
        if self.nranks > 1:
            tdist.all_gather_object(parts, (ei, eu, ci, ch), group=self.group)
        else:
            parts = [(ei, eu, ci, ch)]
        out = np.zeros(self.grid.ne + self.grid.nc)
        for ei_, eu_, ci_, ch_ in parts:
            out[ei_] = eu_
            out[self.grid.ne + ci_] = ch_
        return out

    # ---------------------------------------------------------------- halo exchange
    def exchange_state(self, y: np.ndarray) -> None:
        """Ghost values of a numpy local state from their owners (exchange_state!,
        TRiSKShallowWater.jl:201): the library's pack, exchange and unpack, restated on the
        host for an injected engine."""
        import torch
        send = np.concatenate(self.dist.state_send) if self.dist.state_send else np.zeros(0, np.int64)
        recv = np.concatenate(self.dist.state_recv) if self.dist.state_recv else np.zeros(0, np.int64)
        if len(send) == 0 and len(recv) == 0:
            return
        buf = torch.from_numpy(np.ascontiguousarray(y[send]))
        out = torch.empty(len(recv), dtype=torch.float64)
        self.exchange(buf, out)
        y[recv] = out.numpy()

    # ---------------------------------------------------------------- tendency, RK4
    def tendency(self, dy, y):
        """tendency!(dy, y, m) of the local state (TRiSKShallowWater.jl:379-394): exchange,
        local tendency, ghost tendencies zero."""
        if isinstance(self.engine, _DistModel):
            self.engine.tendency(dy, y)
            return dy
        self.exchange_state(y)
        dy[:] = self.engine.tendency(_to_numpy(y))
        d = self.dist
        dy[d.edges.n_owned:self.ne] = 0.0
        dy[self.ne + d.cells.n_owned:] = 0.0
        return dy

    def rk4_step(self, y, dt: float, nsteps: int = 1):
        """rk4_step! (RungeKutta.jl:18-29) with a distributed tendency: in the library (stage
        updates fused, graph-free because of the exchange), or here for an injected engine with
        the stage sums in the reference's association; owned values match the undivided model
        bit for bit."""
        if isinstance(self.engine, _DistModel):
            self.engine.rk4_step(y, dt, nsteps)
            return y
        half, sixth = dt / 2, dt / 6
        k1, k2, k3, k4, st = (y.copy() for _ in range(5))
        for _ in range(nsteps):
            self.tendency(k1, y)
            st[:] = y + half * k1
            self.tendency(k2, st)
            st[:] = y + half * k2
            self.tendency(k3, st)
            st[:] = y + dt * k3
            self.tendency(k4, st)
            y += sixth * (k1 + 2 * k2 + 2 * k3 + k4)
        return y


def _to_numpy(y):
    return y.detach().cpu().numpy() if hasattr(y, "detach") else y
