"""Mesh generation and TRiSK grid tables (host set-up), mirroring dmplex.jl's

    create_hexagon_mesh(n; centroidal)     src/Grids/Hexagonal.jl:11-17
    plex_from_polygons(polygons, x)        src/Topology/Plex.jl:49-97
    TRiSKGrid(dm; centers)                 src/FiniteVolumes/TRiSKGrid.jl:76-162
    hilbert_permutation(dm)                src/Topology/Ordering.jl:85-92
    vertex_edge_areas(g)                   src/FiniteVolumes/TRiSKGrid.jl:179-191
    gassmann_coefficients(g)               src/FiniteVolumes/TRiSKGrid.jl:214-251

All work is done by the C++ builder in libtrisk_b200.so. Arrays are numpy copies in
the reference's own memory layout: a Julia column-major ``[k, entity]`` table is a
numpy ``(entity, k)`` array, and indices are 1-based as in Julia.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, view


class Plex:
    """CSR arrays of the mesh DAG (src/Topology/Plex.jl:23-34), 1-based points."""

    def __init__(self, p: _lib.TriskPlex):
        n = p.nc + p.ne + p.nv
        self.nc, self.ne, self.nv = p.nc, p.ne, p.nv
        self.cone_offsets = view(p.cone_offsets, (n + 1,), np.int64)
        self.cones = view(p.cones, (p.ncones,), np.int64)
        self.cone_orientations = view(p.cone_orientations, (p.ncones,), np.int64)
        self.support_offsets = view(p.support_offsets, (n + 1,), np.int64)
        self.supports = view(p.supports, (p.ncones,), np.int64)
        self.coordinates = view(p.coordinates, (p.nv, 3), np.float64)

    def cone(self, point: int) -> np.ndarray:
        """get_cone(dm, p) for a 1-based point."""
        return self.cones[self.cone_offsets[point - 1] - 1:self.cone_offsets[point] - 1]

    def support(self, point: int) -> np.ndarray:
        return self.supports[self.support_offsets[point - 1] - 1:self.support_offsets[point] - 1]


class HexMesh:
    """create_hexagon_mesh(subdivisions; centroidal): the Voronoi dual of the icosahedral
    mesh, with the icosahedral vertices (the generators) that the reference's examples
    pass as ``centers``."""

    _CREATE = "trisk_mesh_create_hexagon"

    def __init__(self, subdivisions: int, centroidal: bool = False, spring_beta: float | None = None):
        handle = C.c_void_p()
        beta = 0.0 if spring_beta is None else float(spring_beta)
        check(getattr(lib, self._CREATE)(int(subdivisions), int(bool(centroidal)), beta, C.byref(handle)))
        self.subdivisions, self.centroidal, self.spring_beta = int(subdivisions), bool(centroidal), spring_beta
        self._attach(handle)

    def _attach(self, handle) -> None:
        self._h = handle
        p = _lib.TriskPlex()
        check(lib.trisk_mesh_plex(self._h, C.byref(p)))
        self.plex = Plex(p)
        self.nc, self.ne, self.nv = p.nc, p.ne, p.nv
        g = C.c_void_p()
        check(lib.trisk_mesh_generators(self._h, C.byref(g)))
        self.generators = view(g.value, (self.nc, 3), np.float64)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_mesh_destroy(self._h)
            self._h = None

    def set_centers(self, centers: np.ndarray) -> None:
        """The cell centers (nc, 3) a TRiSKGrid of this mesh is built from
        (TRiSKGrid(dm; centers), TRiSKGrid.jl:76-78)."""
        c = np.ascontiguousarray(centers, dtype=np.float64)
        if c.shape != (self.nc, 3):
            raise ValueError(f"centers must have shape ({self.nc}, 3)")
        check(lib.trisk_mesh_set_centers(self._h, c.ctypes.data))
        self.generators = c.copy()

    def hilbert_permutation(self) -> np.ndarray:
        perm = np.zeros(self.nc, dtype=np.int64)
        check(lib.trisk_mesh_hilbert_permutation(self._h, perm.ctypes.data))
        return perm

    def orthogonality_defect(self) -> float:
        out = C.c_double()
        check(lib.trisk_mesh_orthogonality_defect(self._h, C.byref(out)))
        return out.value


def create_hexagon_mesh(subdivisions: int, centroidal: bool = False, spring_beta: float | None = None) -> HexMesh:
    return HexMesh(subdivisions, centroidal, spring_beta)


class TriangleMesh(HexMesh):
    """create_spherical_mesh(subdivisions; centroidal) with the triangles as cells and their
    circumcenters as cell centers (``generators``): the ICON C grid (src/Grids/
    Icosahedral.jl:22-61, CellCenters.jl:37-42)."""

    _CREATE = "trisk_mesh_create_triangles"


def create_triangle_mesh(subdivisions: int, centroidal: bool = False,
                         spring_beta: float | None = None) -> TriangleMesh:
    return TriangleMesh(subdivisions, centroidal, spring_beta)


class PolygonMesh(HexMesh):
    """plex_from_polygons(polygons, coordinates) (src/Topology/Plex.jl:49-97): a mesh from
    arbitrary polygons, as the grid-file readers build it. ``polygons``: a list of 1-based
    vertex sequences, an (nc, k) array, or a pair (sizes, flat vertex list); ``centers`` (nc, 3): the cell centers of its
    TRiSKGrid (default: the normalized vertex means; see gridfiles.cell_centers)."""

    def __init__(self, polygons, coordinates: np.ndarray, centers: np.ndarray | None = None):
        if isinstance(polygons, tuple) and len(polygons) == 2:      # (sizes, flat): CSR
            sizes = np.asarray(polygons[0], dtype=np.int64)
            flat = np.ascontiguousarray(polygons[1], dtype=np.int64)
        elif isinstance(polygons, np.ndarray) and polygons.ndim == 2:
            sizes = np.full(len(polygons), polygons.shape[1], dtype=np.int64)
            flat = np.ascontiguousarray(polygons, dtype=np.int64).ravel()
        else:
            sizes = np.array([len(p) for p in polygons], dtype=np.int64)
            flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int64) for p in polygons])
                                        if len(polygons) else np.zeros(0, np.int64))
        if sizes.sum() != len(flat):
            raise ValueError("polygon sizes do not match the vertex list")
        offsets = np.ascontiguousarray(np.concatenate([[1], 1 + np.cumsum(sizes)]), dtype=np.int64)
        x = np.ascontiguousarray(coordinates, dtype=np.float64)
        if x.ndim != 2 or x.shape[1] != 3:
            raise ValueError("coordinates must have shape (nv, 3)")
        c = None
        if centers is not None:
            c = np.ascontiguousarray(centers, dtype=np.float64)
            if c.shape != (len(sizes), 3):
                raise ValueError(f"centers must have shape ({len(sizes)}, 3)")
        handle = C.c_void_p()
        check(lib.trisk_mesh_from_polygons(offsets.ctypes.data, flat.ctypes.data, len(sizes), x.ctypes.data,
                                           len(x), None if c is None else c.ctypes.data, C.byref(handle)))
        self.subdivisions, self.centroidal, self.spring_beta = None, False, None
        self._attach(handle)


def plex_from_polygons(polygons, coordinates: np.ndarray, centers: np.ndarray | None = None) -> PolygonMesh:
    return PolygonMesh(polygons, coordinates, centers)


def icosahedral_mesh(subdivisions: int, centroidal: bool = False, spring_beta: float | None = None):
    """(coordinates (nv, 3), triangles (nt, 3) 1-based) of create_spherical_mesh before it
    becomes a Plex (src/Grids/Icosahedral.jl:22-58)."""
    nv, nt = 10 * 4 ** subdivisions + 2, 20 * 4 ** subdivisions
    x = np.zeros((nv, 3))
    t = np.zeros((nt, 3), dtype=np.int64)
    beta = 0.0 if spring_beta is None else float(spring_beta)
    check(lib.trisk_icosahedral_mesh(int(subdivisions), int(bool(centroidal)), beta, x.ctypes.data, t.ctypes.data))
    return x, t


def lloyd(x: np.ndarray, triangles: np.ndarray, fixed: int = 12, history: int = 16) -> int:
    """lloyd!(x, triangles; fixed=1:fixed, history) in place; returns the iterations used."""
    assert x.dtype == np.float64 and x.flags.c_contiguous and x.shape[1] == 3
    tri = np.ascontiguousarray(triangles, dtype=np.int64)
    it = C.c_int32()
    check(lib.trisk_lloyd(x.ctypes.data, len(x), tri.ctypes.data, len(tri), int(fixed), int(history), C.byref(it)))
    return it.value


class TRiSKGrid:
    """Geometry and padded neighbour tables (TRiSKGrid.jl:37-60), 1-based indices.

    ``TRiSKGrid(mesh)`` builds them with the library's builder (centers = the mesh's
    generators). ``TRiSKGrid.from_arrays(**arrays)`` wraps tables built elsewhere, e.g.
    copied out of a Julia ``TRiSKGrid``.
    """

    FIELDS = _lib.GRID_POINTERS

    def __init__(self, mesh: HexMesh | None = None, **arrays):
        if mesh is not None:
            g = _lib.TriskGrid()
            check(lib.trisk_mesh_grid(mesh._h, C.byref(g)))
            nc, ne, nv, cw, vw, tw = g.nc, g.ne, g.nv, g.cw, g.vw, g.tw
            f, i = np.float64, np.int64
            shapes = {
                "centers": ((nc, 3), f), "vertices": ((nv, 3), f), "edge_points": ((ne, 3), f),
                "edge_normals": ((ne, 3), f), "primal_lengths": ((ne,), f), "dual_lengths": ((ne,), f),
                "edge_cells": ((ne, 2), i), "edge_vertices": ((ne, 2), i), "cell_distances": ((ne, 2), f),
                "cell_areas": ((nc,), f), "vertex_areas": ((nv,), f),
                "cell_edges": ((nc, cw), i), "cell_signs": ((nc, cw), f), "cell_vertices": ((nc, cw), i),
                "cell_kites": ((nc, cw), f), "vertex_edges": ((nv, vw), i), "vertex_signs": ((nv, vw), f),
                "vertex_cells": ((nv, vw), i), "vertex_kites": ((nv, vw), f), "trisk_edges": ((ne, tw), i),
                "trisk_weights": ((ne, tw), f),
            }
            for name, (shape, dtype) in shapes.items():
                setattr(self, name, view(getattr(g, name), shape, dtype))
            self.mesh = mesh
        else:
            for name in self.FIELDS:
                setattr(self, name, np.ascontiguousarray(arrays[name]))
            self.mesh = None
        self.nc, self.ne, self.nv = len(self.centers), len(self.primal_lengths), len(self.vertices)

    @classmethod
    def from_arrays(cls, **arrays) -> "TRiSKGrid":
        return cls(None, **arrays)

    def struct(self) -> _lib.TriskGrid:
        """The TriskGrid C struct pointing at this object's arrays (kept alive by self)."""
        g = _lib.TriskGrid()
        g.nc, g.ne, g.nv = self.nc, self.ne, self.nv
        g.cw, g.vw, g.tw = self.cell_edges.shape[1], self.vertex_edges.shape[1], self.trisk_edges.shape[1]
        for name in self.FIELDS:
            a = getattr(self, name)
            want = np.int64 if a.dtype.kind in "iu" else np.float64
            if a.dtype != want or not a.flags.c_contiguous:
                a = np.ascontiguousarray(a, dtype=want)
                setattr(self, name, a)
            setattr(g, name, a.ctypes.data)
        return g

    def vertex_edge_areas(self):
        if self.mesh is None:
            raise ValueError("vertex_edge_areas needs a grid built from a mesh")
        bv = np.zeros((self.nv, self.vertex_edges.shape[1]))
        be = np.zeros((self.ne, 2))
        check(lib.trisk_mesh_vertex_edge_areas(self.mesh._h, bv.ctypes.data, be.ctypes.data))
        return bv, be

    def gassmann_coefficients(self):
        if self.mesh is None:
            raise ValueError("gassmann_coefficients needs a grid built from a mesh")
        E = np.zeros((self.ne, 12), dtype=np.int64)
        P = np.zeros((self.ne, 12), dtype=np.int64)
        W = np.zeros((self.ne, 12))
        check(lib.trisk_mesh_gassmann(self.mesh._h, E.ctypes.data, P.ctypes.data, W.ctypes.data))
        return E, P, W
