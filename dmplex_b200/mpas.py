"""The horizontal operators of dmplex.jl's 3-D MPAS-Gassmann dycore on the GPU:

    slow_tendencies!(m, ys, pressure)      src/Nonhydrostatic/MPAS/Gassmann/Stepping.jl:22-56
      (flat ground: the kernels of src/Nonhydrostatic/MPAS/Operators.jl and
       vn_tendency_kernel!, Tendencies.jl:38-75)
    MPASGassmannNonhydrostatic(grid, vgrid; ...) tables, flat ground
                                           MPASGassmannNonhydrostatic.jl:152-307
    VerticalGrid(nlev, z_top; stretch)     src/Nonhydrostatic/Common/VerticalGrid.jl:36-53
    trisk_pv_edges(g)                      src/FiniteVolumes/TRiSKGrid.jl:331-372
    iap_trisk_weights(g)                   TRiSKGrid.jl:380-410

Fields live on the device in the reference's layout: a Julia (n, nlev) array is an
(nlev, n) C-ordered tensor (level slabs, the horizontal index fastest); ``vn`` (nlev, ne),
``w`` (nlev + 1, nc), ``rho``, ``rhotheta`` (nlev, nc). ``MPASOperators.slow_tendencies``
fills the work arrays slow_tendencies! fills (theta, exner, K, qv, zetav, rhov, Kv, qe,
rhoe, Fs, eta) and the tendencies tvn and tw, in five launches of the library's
``trisk_mpas_*`` kernels (the w and vn tendencies side by side on two streams).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .mesh import TRiSKGrid


def vertical_grid(nlev: int, z_top: float, stretch: float = 1.0) -> dict:
    """VerticalGrid(nlev, z_top; stretch) (VerticalGrid.jl:36-53): interfaces from the ground,
    layer centres, thicknesses dz, centre distances dzh (0 at ground and top) and the
    interpolation weight wlow of the layer below at each interface."""
    r = float(stretch) ** (1 / max(nlev - 1, 1))
    dz = np.array([r ** (k - 1) for k in range(1, nlev + 1)])
    total = 0.0
    for x in dz:
        total += x
    return vertical_grid_from_levels(np.concatenate([[0.0], np.cumsum(dz) * (z_top / total)]))


def vertical_grid_from_levels(z_half) -> dict:
    """VerticalGrid(z_half) (VerticalGrid.jl:36-46)."""
    z = np.asarray(z_half, dtype=np.float64)
    nlev = len(z) - 1
    if nlev < 1 or not np.all(np.diff(z) > 0):
        raise ValueError("z_half must increase")
    zf = (z[:nlev] + z[1:]) / 2
    dz = np.diff(z)
    dzh, wlow = np.zeros(nlev + 1), np.zeros(nlev + 1)
    dzh[1:nlev] = zf[1:] - zf[:-1]
    wlow[1:nlev] = (zf[1:] - z[1:nlev]) / dzh[1:nlev]
    return {"z_half": z, "z_full": zf, "dz": dz, "dzh": dzh, "wlow": wlow}


def _cell_walk(g: TRiSKGrid):
    """The walk around every cell that orders the TRiSK tables (TRiSKGrid.jl): for cell i,
    edge slot k and step s = 1..n-1, the edge e = edges[k], its TRiSK neighbour
    e' = edges[(k + s) mod n] and the slot of e' in e's TRiSK row. Returns flat arrays over
    all (i, k, s) in the walk's order plus the per-cell sizes."""
    n = (g.cell_signs != 0).sum(axis=1)
    cw = g.cell_edges.shape[1]
    i_idx, k_idx, s_idx = [], [], []
    for size in np.unique(n):
        cells = np.flatnonzero(n == size)
        k, s = np.meshgrid(np.arange(size), np.arange(1, size), indexing="ij")
        i_idx.append(np.repeat(cells, k.size))
        k_idx.append(np.tile(k.ravel(), len(cells)))
        s_idx.append(np.tile(s.ravel(), len(cells)))
    i, k, s = (np.concatenate(a) for a in (i_idx, k_idx, s_idx))
    order = np.lexsort((s, k, i))
    i, k, s = i[order], k[order], s[order]
    ni = n[i]
    e = g.cell_edges[i, k] - 1
    kp = (k + s) % ni
    ep = g.cell_edges[i, kp] - 1
    # e's TRiSK row: first the walk in the first of its cells (in cell order), then the other
    l, r = g.edge_cells[e, 0] - 1, g.edge_cells[e, 1] - 1
    other = np.where(l == i, r, l)
    first = i <= other
    slot = (s - 1) + np.where(first, 0, n[other] - 1)
    if not np.array_equal(g.trisk_edges[e, slot] - 1, ep):
        raise ValueError("TRiSK edge table out of order")
    assert cw >= n.max()
    return i, k, s, kp, e, ep, slot, ni


def trisk_pv_edges(g: TRiSKGrid) -> np.ndarray:
    """The PV edge of every TRiSK pair in ICON-IAP's i_cori_method = 4 (TRiSKGrid.jl:331-372):
    one step around the common cell the third edge of the shared vertex, two steps the edge in
    between, 0 (the mean of both edges' PV) for the opposite edge of a hexagon and where no
    such edge exists. (ne, tw), 1-based."""
    i, k, s, kp, e, ep, slot, n = _cell_walk(g)
    edges = g.cell_edges - 1
    corners = g.cell_vertices - 1

    def third_edge(v, a, b):
        ve = g.vertex_edges[v] - 1
        keep = (g.vertex_signs[v] != 0) & (ve != a[:, None]) & (ve != b[:, None])
        one = keep.sum(axis=1) == 1
        pick = ve[np.arange(len(v)), np.argmax(keep, axis=1)]
        return np.where(one, pick + 1, 0)

    out = np.zeros(g.trisk_edges.shape, dtype=np.int64)
    val = np.zeros(len(e), dtype=np.int64)
    c1 = 2 * s == n
    c2 = ~c1 & (s == 1)
    c3 = ~c1 & ~c2 & (s == n - 1)
    c4 = ~c1 & ~c2 & ~c3 & (s == 2)
    c5 = ~c1 & ~c2 & ~c3 & ~c4 & (s == n - 2)
    val[c2] = third_edge(corners[i[c2], (k[c2] + 1) % n[c2]], e[c2], ep[c2])
    val[c3] = third_edge(corners[i[c3], k[c3]], e[c3], ep[c3])
    val[c4] = edges[i[c4], (k[c4] + 1) % n[c4]] + 1
    val[c5] = edges[i[c5], (k[c5] - 1) % n[c5]] + 1
    out[e, slot] = val
    return out


def _arc(a, b):
    c = np.cross(a, b)
    return np.arctan2(np.sqrt(c[:, 0] * c[:, 0] + c[:, 1] * c[:, 1] + c[:, 2] * c[:, 2]),
                      a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2])


def iap_trisk_weights(g: TRiSKGrid) -> np.ndarray:
    """TRiSK weights of ICON-IAP (TRiSKGrid.jl:380-410): the walk of the TRiSK weights with the
    planar kite fractions R_{i,v} = sum over the two edges of cell i at v of
    d_{e,i} l_{e,v} / 2A_i. (ne, tw)."""
    i, k, s, kp, e, ep, slot, n = _cell_walk(g)
    nc, cw = g.cell_edges.shape
    ncell = (g.cell_signs != 0).sum(axis=1)
    R = np.zeros((nc, cw))
    for kk in range(cw):
        has = kk < ncell
        ci = np.flatnonzero(has)
        nn = ncell[ci]
        corner = g.cell_vertices[ci, kk] - 1

        def triangle(slot_k):
            ee = g.cell_edges[ci, slot_k] - 1
            side = np.where(g.edge_cells[ee, 0] - 1 == ci, 0, 1)
            return g.cell_distances[ee, side] * _arc(g.edge_points[ee], g.vertices[corner]) / 2
        R[ci, kk] = (triangle((kk - 1) % nn) + triangle(np.full(len(ci), kk))) / g.cell_areas[ci]
    # S = R[k+1] + ... + R[k+s], accumulated in order of s; the walk lists the steps of one
    # (cell, slot) consecutively, so step s follows step s - 1 in the flat arrays
    vals = R[i, kp]
    S = np.zeros(len(e))
    first = s == 1
    S[first] = vals[first]
    for step in range(2, cw):
        m = np.flatnonzero(s == step)
        S[m] = S[m - 1] + vals[m]
    signs = g.cell_signs
    W = np.zeros(g.trisk_weights.shape)
    W[e, slot] = signs[i, k] * signs[i, kp] * (0.5 - S)
    return W


def mpas_tables(grid: TRiSKGrid, vgrid: dict, *, radius: float = 6.37122e6, omega: float = 7.292e-5,
                kinetic_energy="cell", pv_flux: str = "iap", vertical_advection: str = "iap",
                trisk_weights: str = "iap", vertical_solver: str = "five_band") -> dict:
    """The arrays of MPASGassmannNonhydrostatic(grid, vgrid; ...) that slow_tendencies! reads,
    for flat ground (MPASGassmannNonhydrostatic.jl:152-307), coriolis(x) = 2 omega x[3]."""
    from .model import model_tables
    if pv_flux not in ("iap", "trisk"):
        raise ValueError("pv_flux must be iap or trisk")
    vertical = {"advective": 0, "vector_invariant": 1, "iap": 2}.get(vertical_advection)
    if vertical is None:
        raise ValueError("vertical_advection must be iap, vector_invariant or advective")
    if trisk_weights not in ("iap", "exact"):
        raise ValueError("trisk_weights must be iap or exact")
    if vertical_solver not in ("five_band", "tridiagonal"):
        raise ValueError("vertical_solver must be five_band or tridiagonal")
    if vertical_solver == "five_band" and vertical == 0:
        raise ValueError("vertical_solver = five_band needs the vector-invariant vertical advection")
    g = grid
    a = float(radius)
    sw = model_tables(g, omega=omega, pv_flux="trisk", kinetic_energy=kinetic_energy)
    nc, ne, nv = g.nc, g.ne, g.nv
    nlev = len(vgrid["dz"])
    ew = g.cell_distances / g.dual_lengths[:, None]                     # (ne, 2)
    # flat levels: every cell column is vgrid; edge columns from the edge weights
    zi = np.broadcast_to(vgrid["z_half"], (nc, nlev + 1))
    ze = ew[:, 0:1] * zi[g.edge_cells[:, 0] - 1] + ew[:, 1:2] * zi[g.edge_cells[:, 1] - 1]
    zfe = (ze[:, :nlev] + ze[:, 1:]) / 2
    dze = ze[:, 1:] - ze[:, :nlev]
    dzhe = np.zeros((ne, nlev + 1))
    dzhe[:, 1:nlev] = zfe[:, 1:] - zfe[:, :-1]
    if not np.all(dze > 0):
        raise ValueError("edge levels must increase")
    side = np.where(g.edge_cells[g.cell_edges - 1, 0] - 1 == np.arange(nc)[:, None], 0, 1)
    ce = g.cell_edges - 1
    inner = np.where(g.cell_signs != 0,
                     g.primal_lengths[ce] * g.cell_distances[ce, side] / g.cell_areas[:, None], 0.0)
    rh = g.vertex_areas[g.edge_vertices - 1]
    rh = rh / (rh[:, 0:1] + rh[:, 1:2])
    pv = trisk_pv_edges(g) if pv_flux == "iap" else np.zeros(g.trisk_edges.shape, dtype=np.int64)
    W = iap_trisk_weights(g) if trisk_weights == "iap" else g.trisk_weights
    ep = g.trisk_edges - 1
    trisk = W * g.primal_lengths[ep] / (2 * g.dual_lengths[:, None])
    self_e = np.broadcast_to(np.arange(ne)[:, None], ep.shape)
    zero = trisk == 0
    ti = np.stack([np.where(zero, self_e, ep),
                   np.where(zero, self_e, np.where(pv == 0, self_e, pv - 1)),
                   np.where(zero, self_e, np.where(pv == 0, ep, pv - 1))], axis=2) + 1
    t = {
        "nc": nc, "ne": ne, "nv": nv, "nlev": nlev,
        "cell_edges": g.cell_edges.copy(), "kinetic": sw["kinetic"], "inner": inner,
        "edge_cells": g.edge_cells.copy(), "edge_weight": ew, "edge_vertices": g.edge_vertices.copy(),
        "rhombus": rh, "inverse_dual": sw["inverse_dual"] / a, "edge_coriolis": 2 * omega * g.edge_points[:, 2],
        "vertex_edges": g.vertex_edges.copy(), "curl": sw["curl"] / a, "vertex_cells": g.vertex_cells.copy(),
        "vertex_weight": sw["vertex_height"], "coriolis": sw["coriolis"],
        "trisk": np.ascontiguousarray(trisk), "trisk_index": np.ascontiguousarray(ti.astype(np.int32)),
        "dz_cells": np.ascontiguousarray(np.broadcast_to(vgrid["dz"][:, None], (nlev, nc))),
        "dzh_cells": np.ascontiguousarray(np.broadcast_to(vgrid["dzh"][:, None], (nlev + 1, nc))),
        "wlow": np.ascontiguousarray(np.broadcast_to(vgrid["wlow"][:, None], (nlev + 1, nc))),
        "dz_edges": np.ascontiguousarray(dze.T), "dzh_edges": np.ascontiguousarray(dzhe.T),
        "iap_pv": pv_flux == "iap", "vertical": vertical, "five_band": vertical_solver == "five_band",
        "vk_cell_vertices": sw["vk_cell_vertices"], "vk_kites": sw["vk_kites"], "vk_weights": sw["vk_weights"],
    }
    return t


_INT_TABLES = ("cell_edges", "edge_cells", "edge_vertices", "vertex_edges", "vertex_cells", "vk_cell_vertices")
_REAL_TABLES = ("kinetic", "inner", "vk_kites", "edge_weight", "rhombus", "inverse_dual", "edge_coriolis", "curl",
                "vertex_weight", "vk_weights", "coriolis", "trisk", "dz_cells", "dzh_cells", "wlow", "dz_edges",
                "dzh_edges")
WORK_FIELDS = ("theta", "exner", "K", "Kv", "qv", "zetav", "rhov", "qe", "rhoe", "Fs", "eta", "tvn", "tw")


class MPASOperators:
    """slow_tendencies! of MPASGassmannNonhydrostatic on one GPU (flat ground). ``tables``:
    the dict of ``mpas_tables`` (or the same arrays taken from a reference model)."""

    def __init__(self, tables: dict, device: int = 0, levels_per_thread: int = 0):
        t = tables
        s = _lib.TriskMpasTables()
        s.nc, s.ne, s.nv, s.nlev = t["nc"], t["ne"], t["nv"], t["nlev"]
        s.cw, s.vw, s.nt = t["cell_edges"].shape[1], t["vertex_edges"].shape[1], t["trisk"].shape[1]
        s.iap_pv, s.vertical, s.five_band = int(bool(t["iap_pv"])), int(t["vertical"]), int(bool(t["five_band"]))
        s.vertex_kinetic = int(t.get("vk_weights") is not None)
        self._keep = []
        for name in _INT_TABLES + _REAL_TABLES:
            a = t.get(name)
            if a is None:
                setattr(s, name, None)
                continue
            if name == "trisk":
                a = a.T                      # edge-first, as the reference's (ne, nt) array
            a = np.ascontiguousarray(a, dtype=np.int64 if name in _INT_TABLES else np.float64)
            self._keep.append(a)
            setattr(s, name, a.ctypes.data)
        ti = np.ascontiguousarray(np.transpose(t["trisk_index"], (2, 1, 0)), dtype=np.int32)  # (ne, nt, 3) edge-first
        self._keep.append(ti)
        s.trisk_index = ti.ctypes.data
        h = C.c_void_p()
        check(lib.trisk_mpas_create(C.byref(s), int(device), int(levels_per_thread), C.byref(h)))
        self._h = h
        self.nc, self.ne, self.nv, self.nlev = t["nc"], t["ne"], t["nv"], t["nlev"]
        self.vertex_kinetic = bool(s.vertex_kinetic)
        self.levels_per_thread = int(levels_per_thread) or 8

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_mpas_destroy(self._h)
            self._h = None

    def shapes(self) -> dict:
        nc, ne, nv, nl = self.nc, self.ne, self.nv, self.nlev
        return {"theta": (nl, nc), "exner": (nl, nc), "K": (nl, nc), "Kv": (nl, nv), "qv": (nl, nv),
                "zetav": (nl, nv), "rhov": (nl, nv), "qe": (nl, ne), "rhoe": (nl, ne), "Fs": (nl, ne),
                "eta": (nl + 1, ne), "tvn": (nl, ne), "tw": (nl + 1, nc)}

    def work(self, device=None) -> dict:
        """Zeroed device work arrays of the right shapes (torch, float64)."""
        import torch
        dev = device if device is not None else torch.device("cuda")
        return {k: torch.zeros(v, dtype=torch.float64, device=dev) for k, v in self.shapes().items()}

    def slow_tendencies(self, vn, w, rho, rhotheta, out: dict, pressure: float = 1.0) -> dict:
        """slow_tendencies!(m, ys, pressure) with ys = (vn, w, rho, rhotheta) device tensors;
        ``out`` holds device tensors for the work arrays and tendencies (``work()``)."""
        f = self.fields(vn, w, rho, rhotheta, out)
        check(lib.trisk_mpas_slow_tendencies(self._h, C.byref(f), float(pressure)))
        return out

    def fields(self, vn, w, rho, rhotheta, out: dict) -> "_lib.TriskMpasFields":
        """The TriskMpasFields struct of these tensors (shapes and devices checked)."""
        f = _lib.TriskMpasFields()
        for name, shape in (("vn", (self.nlev, self.ne)), ("w", (self.nlev + 1, self.nc)),
                            ("rho", (self.nlev, self.nc)), ("rhotheta", (self.nlev, self.nc))):
            x = locals()[name]
            _check(x, shape, name)
            setattr(f, name, x.data_ptr())
        for name, shape in self.shapes().items():
            x = out.get(name)
            if x is None:
                if name == "Kv" and not self.vertex_kinetic:
                    continue
                raise ValueError(f"out[{name!r}] is missing")
            _check(x, shape, name)
            setattr(f, name, x.data_ptr())
        return f

    def launch_count(self) -> int:
        return lib.trisk_mpas_launch_count(self._h)


def _check(x, shape, name):
    if not hasattr(x, "data_ptr") or not x.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if str(x.dtype) != "torch.float64" or not x.is_contiguous() or tuple(x.shape) != tuple(shape):
        raise ValueError(f"{name} must be a contiguous float64 tensor of shape {shape}")


def algorithmic_bytes(t: dict) -> int:
    """DRAM bytes one slow_tendencies call must move with its five phases, each reading every
    array it touches once and writing its outputs once (FP64 fields, int32 / FP64 tables):

        vertices  vn, rho -> zeta_v, rho_v, q_v (+ K_v)
        cells     vn, rho, rho theta, w, dz, dzh (+ K_v) -> theta, pi, K (+ K without K_w)
        edges     q_v, zeta_v, rho_v, rho, vn, w, dzh_e -> q_e, rho_e, F_s, eta
        w         eta, vn, rho_e, K, dzh, wlow -> t_w   (advective: vn, w, dz)
        vn        F_s, q_e, eta, vn, theta, pi, K, w, rho, wlow, dz_e, dzh_e -> t_vn

    per level, plus every table once."""
    nc, ne, nv, nl = t["nc"], t["ne"], t["nv"], t["nlev"]
    vk = t.get("vk_weights") is not None
    vi = t["vertical"] > 0
    fb = bool(t["five_band"])
    mw = t["vertical"] == 2
    # vertices: vn, rho -> zeta_v, rho_v, q_v (+ K_v)
    per_level = ne + nc + (4 if vk else 3) * nv
    # cells: vn, rho, rho theta (+ K_v) (+ w, dz, dzh) -> theta, pi, K (+ K without K_w)
    per_level += ne + 2 * nc + (nv if vk else 0) + (3 * nc if vi else 0) + 3 * nc + (nc if fb else 0)
    # edges: zeta_v, rho_v (or q_v), rho, vn (+ w, dzh_e) -> q_e, rho_e, F_s (+ eta)
    per_level += (2 if t["iap_pv"] else 1) * nv + nc + ne + (nc + ne if vi else 0) + 3 * ne + (ne if vi else 0)
    # w: eta, vn, rho_e, K, dzh, wlow -> t_w   (advective: vn, w, dz -> t_w)
    per_level += (3 * ne + 3 * nc + nc) if vi else (ne + 2 * nc + nc)
    # vn: F_s, q_e, theta, pi, K, w, dz_e (+ eta, dzh_e; + rho, wlow with mass fluxes; advective: vn) -> t_vn
    per_level += 2 * ne + 4 * nc + ne + ((2 * ne) if vi else ne) + (2 * nc if mw else 0) + ne
    cw, vw, nt = t["cell_edges"].shape[1], t["vertex_edges"].shape[1], t["trisk"].shape[1]
    tables = nv * vw * (4 + 4 + 8 + 8 + (8 if vk else 0)) + 8 * nv
    tables += nc * cw * (4 + 8 + (12 if vk else 0)) + nc * cw * (4 + 8 + (0 if vi else 12))
    tables += ne * (2 * 4 + 2 * 4 + 2 * 8 + 2 * 8 + 8 + 8) + ne * nt * (8 + 12) + ne * (2 * 4 + 2 * 8 + 8)
    return int(8 * per_level * nl + tables)
