"""ICON triangle shallow water on the GPU, mirroring dmplex.jl's ICONShallowWater:

    ICONShallowWater(grid; gravity, coriolis, rbf_scale, divergence_damping, kinetic_gradient)
                                           src/FiniteVolumes/ICONShallowWater.jl:96-147
    tendency!(dy, y, m)                    :191-208 (+ divergence_damping! :210-218)
    rk4_step!(y, dt, tendency!, cache, m)  src/TimeSteppers/RungeKutta.jl:18-29
    rbf_coefficients(grid; scale)          src/FiniteVolumes/TRiSKGrid.jl:269-282
    bilinear_weights(grid)                 ICONShallowWater.jl:82-94

Normal velocities at the edges, heights at the triangles' circumcenters, vorticity at the
vertices; the state y = [u; h] in file numbering, FP64. The tables are built here (numpy)
from a TRiSKGrid of create_triangle_mesh, uploaded once; the tendency and the RK4 steps run
in the library's ICON kernels (trisk_icon_*).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .mesh import TRiSKGrid


def _arc_length(a, b):
    """atan(|a x b|, a . b) row-wise (TRiSKGrid.jl:2)."""
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=-1), np.einsum("...i,...i->...", a, b))


def bilinear_weights(g: TRiSKGrid) -> np.ndarray:
    """ICON's edge-to-cell weights (e_bln_c_s, ICONShallowWater.jl:82-94): per triangle the
    three weights that sum to one and have no first moment in the tangent plane. (nc, 3)."""
    c = g.centers
    if g.cell_edges.shape[1] != 3:
        raise ValueError("bilinear weights need a triangle mesh")
    axis = np.where((np.abs(c[:, 2]) < 0.9)[:, None], np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0]))
    a = np.cross(c, axis)
    a /= np.linalg.norm(a, axis=1, keepdims=True)
    b = np.cross(c, a)
    x = g.edge_points[g.cell_edges - 1]  # (nc, 3, 3)
    A = np.stack([np.ones((len(c), 3)), np.einsum("nkj,nj->nk", x, a), np.einsum("nkj,nj->nk", x, b)], axis=1)
    rhs = np.zeros((len(c), 3))
    rhs[:, 0] = 1.0
    return np.linalg.solve(A, rhs[..., None])[..., 0]


def rbf_coefficients(g: TRiSKGrid, scale: float = 0.5):
    """Vector-RBF tangential velocity (TRiSKGrid.jl:269-282): for edge e the other edges of
    its two cells, kernel 1/sqrt(1 + (r/scale)^2) of the great-circle distance times the dot
    product of the normals, normalized to reproduce a constant vector along r x n_e. Returns
    (edges (ne, 4) 1-based, weights (ne, 4))."""
    n, x = g.edge_normals, g.edge_points
    ne = g.ne
    ce, cs, ec = g.cell_edges - 1, g.cell_signs, g.edge_cells - 1
    if ce.shape[1] != 3 or np.any(cs == 0):
        raise ValueError("the RBF stencil needs triangles")
    parts = []
    for side in range(2):  # the cell's other two edges, in the cell's order
        sides = ce[ec[:, side]]                                   # (ne, 3)
        keep = sides != np.arange(ne)[:, None]
        if not np.all(keep.sum(1) == 2):
            raise ValueError("an edge is not a side of its cell")
        parts.append(sides[keep].reshape(ne, 2))
    stencil = np.concatenate(parts, axis=1)

    def kern(p, q):
        return 1.0 / np.sqrt(1.0 + (_arc_length(p, q) / scale) ** 2)

    ns, xs = n[stencil], x[stencil]                                              # (ne, 4, 3)
    A = np.einsum("eid,ejd->eij", ns, ns) * kern(xs[:, :, None, :], xs[:, None, :, :])
    t = np.cross(x, n)
    tn = np.einsum("ed,ekd->ek", t, ns)
    rhs = tn * kern(x[:, None, :], xs)
    L = np.linalg.cholesky(A)
    c = np.linalg.solve(np.swapaxes(L, 1, 2), np.linalg.solve(L, rhs[..., None]))[..., 0]
    c /= np.einsum("ek,ek->e", c, tn)[:, None]
    return stencil + 1, c


def icon_tables(g: TRiSKGrid, gravity: float = 1.0, omega: float = 1.0, rbf_scale: float = 0.5,
                kinetic_gradient: str = "icon") -> dict:
    """The coefficients of ICONShallowWater (ICONShallowWater.jl:96-127), 1-based indices,
    (entity, k) layout, coriolis(x) = 2 omega x[3]."""
    if kinetic_gradient not in ("icon", "centered"):
        raise ValueError(f"unknown kinetic_gradient {kinetic_gradient}")
    l, d, dc = g.primal_lengths, g.dual_lengths, g.cell_distances
    ce = g.cell_edges - 1
    divergence = g.cell_signs * l[ce] / g.cell_areas[:, None]
    edge_height = np.stack([dc[:, 1], dc[:, 0]], axis=1) / d[:, None]
    if kinetic_gradient == "icon":
        gradient = np.stack([dc[:, 1] / (dc[:, 0] * d), dc[:, 0] / (dc[:, 1] * d)], axis=1)
    else:
        gradient = np.stack([1 / d, 1 / d], axis=1)
    curl = g.vertex_signs * d[g.vertex_edges - 1] / g.vertex_areas[:, None]
    rbf_edges, rbf = rbf_coefficients(g, rbf_scale)
    return {
        "nc": g.nc, "ne": g.ne, "nv": g.nv, "vw": g.vertex_edges.shape[1], "gravity": float(gravity),
        "cell_edges": g.cell_edges.copy(), "divergence": divergence, "bilinear": bilinear_weights(g),
        "edge_cells": g.edge_cells.copy(), "edge_vertices": g.edge_vertices.copy(), "edge_height": edge_height,
        "gradient": gradient, "inverse_dual": 1.0 / d, "rbf_edges": rbf_edges, "rbf": rbf,
        "edge_coriolis": 2 * omega * g.edge_points[:, 2], "vertex_edges": g.vertex_edges.copy(), "curl": curl,
        "cell_areas": g.cell_areas.copy(),
    }


_TABLE_FIELDS = ("cell_edges", "divergence", "bilinear", "edge_cells", "edge_vertices", "edge_height", "gradient",
                 "inverse_dual", "rbf_edges", "rbf", "edge_coriolis", "vertex_edges", "curl", "cell_areas")


class ICONShallowWater:
    """The ICON triangle shallow-water model on one GPU (ICONShallowWater.jl:1-48).
    divergence_damping: nu_4 (a number, or one value per edge) of ICON's fourth-order
    divergence damping -nu_4 grad div grad div u (0: off)."""

    def __init__(self, grid, *, gravity: float = 1.0, omega: float = 1.0, rbf_scale: float = 0.5,
                 divergence_damping=0.0, kinetic_gradient: str = "icon", device: int = 0):
        if not isinstance(grid, TRiSKGrid):
            grid = TRiSKGrid(grid)
        self.grid = grid
        self.tables = icon_tables(grid, gravity, omega, rbf_scale, kinetic_gradient)
        nu = np.asarray(divergence_damping, dtype=np.float64)
        if nu.ndim == 0:
            nu = np.zeros(0) if nu == 0 else np.full(grid.ne, float(nu))
        elif nu.shape != (grid.ne,):
            raise ValueError("divergence_damping: a number or one value per edge")
        self.tables["divergence_damping"] = np.ascontiguousarray(nu)
        t = self.tables
        s = _lib.TriskIconTables()
        s.nc, s.ne, s.nv, s.vw, s.gravity = t["nc"], t["ne"], t["nv"], t["vw"], t["gravity"]
        self._keep = []
        for name in _TABLE_FIELDS:
            a = np.ascontiguousarray(t[name], dtype=np.int64 if t[name].dtype.kind == "i" else np.float64)
            self._keep.append(a)
            setattr(s, name, a.ctypes.data)
        s.divergence_damping = t["divergence_damping"].ctypes.data if len(nu) else None
        self._keep.append(t["divergence_damping"])
        h = C.c_void_p()
        check(lib.trisk_icon_create(C.byref(s), int(device), C.byref(h)))
        self._h = h
        self.nc, self.ne, self.nv = grid.nc, grid.ne, grid.nv

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_icon_destroy(self._h)
            self._h = None

    @property
    def state_size(self) -> int:
        return self.ne + self.nc

    def tendency(self, dy, y):
        """tendency!(dy, y, m) (ICONShallowWater.jl:191-208)."""
        check(lib.trisk_icon_tendency(self._h, _state(y, self), _state(dy, self)))
        return dy

    def rk4_step(self, y, dt: float, nsteps: int = 1):
        """rk4_step!(y, dt, tendency!, cache, m) in place, nsteps times."""
        check(lib.trisk_icon_rk4_step(self._h, _state(y, self), float(dt), int(nsteps)))
        return y

    def launch_count(self) -> int:
        """Kernels launched so far (a replayed RK4 step counts its graph's kernels)."""
        return int(lib.trisk_icon_launch_count(self._h))

    def algorithmic_bytes(self) -> dict:
        return algorithmic_bytes(self.tables)

    def total_mass(self, y) -> float:
        y = np.asarray(y)
        return float(self.grid.cell_areas @ y[self.ne:])


def algorithmic_bytes(tables: dict) -> dict:
    """The ICON path's byte model, in the form used for the TRiSK path: int32 indices (4 B) and
    FP64 weights (8 B) as uploaded (vertex tables padded to 6 edges), every table read once per
    tendency; the state N = 8 (ne + nc) bytes; per RK4 step 4 (T + 2N) + 15N (each tendency
    reads its state and writes its tendency, plus the RK4 vector passes)."""
    ne, nc, nv = tables["ne"], tables["nc"], tables["nv"]
    damping = len(tables.get("divergence_damping", ())) > 0
    per_edge = 4 * 4 + 8 * 4 + 4 * 2 + 8 * 2 + 8 + 4 * 2 + 8 * 2 + 8 + (8 if damping else 0)
    per_cell = 4 * 3 + 8 * 3 + 8 * 3
    per_vertex = (4 + 8) * 6
    T = ne * per_edge + nc * per_cell + nv * per_vertex
    N = 8 * (ne + nc)
    return {"tables": T, "state": N, "tendency": T + 2 * N, "rk4_step": 4 * (T + 2 * N) + 15 * N,
            "per_edge": per_edge, "per_cell": per_cell, "per_vertex": per_vertex}


def _state(y, m):
    if isinstance(y, np.ndarray):
        if y.dtype != np.float64 or not y.flags.c_contiguous or y.size != m.state_size:
            raise ValueError(f"state must be a contiguous float64 vector of length {m.state_size}")
    elif hasattr(y, "data_ptr"):
        if str(y.dtype) != "torch.float64" or not y.is_contiguous() or y.numel() != m.state_size:
            raise ValueError(f"state must be a contiguous float64 tensor of length {m.state_size}")
    else:
        raise TypeError("state must be a numpy array or a torch tensor")
    return ptr(y)
