"""ICON and MPAS grid files as meshes, mirroring dmplex.jl's readers and the cell-center
rules a TRiSKGrid built on them uses:

    read_variable(ds, name)               src/Grids/FileGrids.jl:8-11
    lonlat_to_xyz(lon, lat)               FileGrids.jl:13
    rows_per_entity(table, n)             FileGrids.jl:16-20
    sort_ring(ids, coordinates, axis)     FileGrids.jl:28-32
    dual_polygons(rings, coords, centers) FileGrids.jl:40-42
    read_icon_grid(filename; dual)        FileGrids.jl:52-65
    read_mpas_grid(filename; dual)        FileGrids.jl:77-95
    read_grid(filename; dual)             FileGrids.jl:101-107
    cell_centers(dm; method)              src/Grids/CellCenters.jl:25-46
    voronoi_generators(dm; iterations)    CellCenters.jl:49-81
    check_plex(dm; closed)                src/Topology/Plex.jl:329-359
    hilbert_order(dm)                     src/Topology/Ordering.jl:44-82

A reader returns a PolygonMesh (the Plex of plex_from_polygons, built by the library) whose
``generators`` are ``cell_centers(mesh)``: what ``TRiSKGrid(read_grid(f))`` uses in the
reference, so ``TRiSKGrid(read_grid(f))`` here gives the same tables. Cells and vertices keep
the file's numbering; edges are numbered by first appearance, as in the reference.

Files are read with scipy's NetCDF reader: the classic (CDF-1) and 64-bit-offset (CDF-2)
formats. A NetCDF-4 (HDF5) file raises ValueError naming the conversion
(``nccopy -k classic``); no HDF5 library is part of this package's dependencies.
Variables are read raw, without fill values or scaling, like the reference's
``read_variable``. numpy holds a variable in the file's (ncdump) dimension order, the
reverse of Julia's; ``rows_per_entity`` is written for that order and picks the same rows
as the reference in every case, the square one included.
"""
from __future__ import annotations

import numpy as np

from .mesh import HexMesh, PolygonMesh

_HDF5_SIGNATURE = b"\x89HDF\r\n\x1a\n"


class _Dataset:
    """An open classic-NetCDF file (scipy.io.netcdf_file, raw values)."""

    def __init__(self, filename: str):
        with open(filename, "rb") as f:
            magic = f.read(8)
        if magic == _HDF5_SIGNATURE:
            raise ValueError(f"{filename} is a NetCDF-4 (HDF5) file; convert it with `nccopy -k classic` "
                             "(or -k 64-bit-offset) to read it")
        if magic[:3] != b"CDF":
            raise ValueError(f"{filename} is not a NetCDF file")
        from scipy.io import netcdf_file
        self.ds = netcdf_file(filename, "r", mmap=False, maskandscale=False)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.ds.close()

    def __contains__(self, name: str) -> bool:
        return name in self.ds.variables

    def attribute(self, name: str):
        # the global attributes as scipy keeps them (getattr would also find the file's
        # methods and fields for names such as "mode" or "filename")
        value = self.ds._attributes.get(name)
        if isinstance(value, bytes):
            value = value.decode("utf-8", "replace")
        return value


def read_variable(ds: _Dataset, name: str) -> np.ndarray:
    """The whole variable, raw (FileGrids.jl:8-11), in the file's dimension order."""
    return np.array(ds.ds.variables[name].data)


def lonlat_to_xyz(lon, lat) -> np.ndarray:
    """(cos(lat) cos(lon), cos(lat) sin(lon), sin(lat)) row-wise (FileGrids.jl:13)."""
    lon, lat = np.asarray(lon, dtype=np.float64), np.asarray(lat, dtype=np.float64)
    return np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)], axis=-1)


def rows_per_entity(table: np.ndarray, n: int) -> np.ndarray:
    """A connectivity table as (n, k), one row per entity (FileGrids.jl:16-20). ``table`` is in
    the file's dimension order: the reference's first test (Julia's first dimension = the
    file's last) is the file's last dimension here."""
    if table.ndim != 2:
        raise ValueError(f"connectivity table of shape {table.shape} is not a matrix")
    if table.shape[1] == n:
        return np.ascontiguousarray(table.T)
    if table.shape[0] == n:
        return table
    raise ValueError(f"connectivity table of size {table.shape} does not match {n} entities")


def _normalize(x: np.ndarray) -> np.ndarray:
    return x / np.sqrt(x[..., 0] * x[..., 0] + x[..., 1] * x[..., 1] + x[..., 2] * x[..., 2])[..., None]


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def sort_ring(ids, coordinates: np.ndarray, axis: np.ndarray) -> np.ndarray:
    """The points coordinates[ids] (1-based) counter-clockwise around ``axis`` seen from
    outside, starting from the angle of the first id (FileGrids.jl:28-32)."""
    ids = np.asarray(ids, dtype=np.int64)
    return _sort_rings(ids[None, :], np.ones((1, len(ids)), bool), coordinates, np.asarray(axis)[None, :])[0]


def _sort_rings(rings: np.ndarray, valid: np.ndarray, coordinates: np.ndarray, axes: np.ndarray) -> np.ndarray:
    """sort_ring for every row of a padded (n, k) table of 1-based ids; invalid entries go
    last. The sort is stable, like Julia's sortperm."""
    x = coordinates[np.where(valid, rings, 1) - 1]                   # (n, k, 3)
    e1 = x[:, 0, :] - axes                                           # first id at angle 0
    v = x - axes[:, None, :]
    angle = np.arctan2(_dot(np.cross(e1[:, None, :], v), axes[:, None, :]), _dot(e1[:, None, :], v))
    angle = np.where(valid, angle, np.inf)
    order = np.argsort(angle, axis=1, kind="stable")
    return np.take_along_axis(rings, order, axis=1)


def dual_polygons(rings, coordinates: np.ndarray, centers: np.ndarray) -> list:
    """Dual cells (FileGrids.jl:40-42): rings[v] lists the primal cells around primal vertex v
    (1-based), sorted counter-clockwise around that vertex."""
    sizes = np.array([len(r) for r in rings], dtype=np.int64)
    k = int(sizes.max()) if len(sizes) else 0
    table = np.ones((len(rings), k), dtype=np.int64)
    valid = np.arange(k)[None, :] < sizes[:, None]
    table[valid] = np.concatenate([np.asarray(r, dtype=np.int64) for r in rings])
    s = _sort_rings(table, valid, coordinates, _normalize(np.asarray(centers, dtype=np.float64)))
    return [s[v, :sizes[v]] for v in range(len(rings))]


# ---------------------------------------------------------------------------------------
# Plex queries on the CSR arrays (1-based points: cells 1..nc, edges nc+1..nc+ne, then
# vertices), vectorised over all cells / edges.

def _cone_table(mesh: HexMesh):
    """Per cone entry of every cell: (cell 0-based, edge 0-based, orientation, position
    in the cell, cone size of the cell)."""
    p = mesh.plex
    nc = p.nc
    off = p.cone_offsets[:nc + 1] - 1
    sizes = np.diff(off)
    cell = np.repeat(np.arange(nc), sizes)
    pos = np.arange(off[-1]) - np.repeat(off[:-1], sizes)
    edge = p.cones[:off[-1]] - nc - 1
    return cell, edge, p.cone_orientations[:off[-1]], pos, sizes


def _edge_vertices(mesh: HexMesh) -> np.ndarray:
    """(ne, 2) 0-based vertex indices of every edge's cone."""
    p = mesh.plex
    off = p.cone_offsets[p.nc:p.nc + p.ne] - 1
    return np.stack([p.cones[off], p.cones[off + 1]], axis=1) - p.nc - p.ne - 1


def cell_vertex_csr(mesh: HexMesh):
    """get_cell_vertices of all cells (Plex.jl:226-230) as (sizes, flat 1-based vertex
    list): corner i of a cell is where its cone edge i starts."""
    cell, edge, orient, pos, sizes = _cone_table(mesh)
    ev = _edge_vertices(mesh)
    return sizes, np.where(orient == 0, ev[edge, 0], ev[edge, 1]) + 1


def cell_vertex_table(mesh: HexMesh) -> list:
    """get_cell_vertices for every cell, one array per cell (see cell_vertex_csr)."""
    sizes, start = cell_vertex_csr(mesh)
    return np.split(start, np.cumsum(sizes)[:-1])


def _edge_cells(mesh: HexMesh) -> np.ndarray:
    """(ne, 2) 0-based (left, right) cells of every edge, -1 where missing (Plex.jl:210-218)."""
    cell, edge, orient, _, _ = _cone_table(mesh)
    lr = np.full((mesh.ne, 2), -1, dtype=np.int64)
    lr[edge[orient == 0], 0] = cell[orient == 0]
    lr[edge[orient != 0], 1] = cell[orient != 0]
    return lr


def check_plex(mesh: HexMesh, closed: bool = True) -> bool:
    """check_plex(dm; closed) (Plex.jl:329-359): cones and supports agree, every cell
    boundary is a closed loop of at least three edges turning counter-clockwise, every edge
    has at most one cell on each side (exactly one on a closed mesh), and a closed mesh has
    the Euler characteristic of the sphere (2) or of the doubly periodic plane (0). Raises
    ValueError naming the first violation."""
    p = mesh.plex
    n = p.nc + p.ne + p.nv
    # cone/support: the (point, cone point) pairs from both sides are the same multiset
    owner = np.repeat(np.arange(1, n + 1), np.diff(p.cone_offsets))
    held = np.repeat(np.arange(1, n + 1), np.diff(p.support_offsets))
    a = np.sort(owner * (n + 1) + p.cones)
    b = np.sort(p.supports * (n + 1) + held)
    if len(a) != len(b) or not np.array_equal(a, b):
        bad = np.setdiff1d(a, b)
        q = int(bad[0]) if len(bad) else int(a[0])
        raise ValueError(f"cone/support mismatch between {q // (n + 1)} and {q % (n + 1)}")
    cell, edge, orient, pos, sizes = _cone_table(mesh)
    small = np.flatnonzero(sizes < 3)
    if len(small):
        raise ValueError(f"cell {small[0] + 1} has fewer than three edges")
    ev = _edge_vertices(mesh)
    start = np.where(orient == 0, ev[edge, 0], ev[edge, 1])
    stop = np.where(orient == 0, ev[edge, 1], ev[edge, 0])
    first = np.cumsum(sizes) - sizes
    nxt = np.where(pos + 1 < sizes[cell], np.arange(len(cell)) + 1, first[cell])
    broken = np.flatnonzero(stop != start[nxt])
    if len(broken):
        raise ValueError(f"cell {cell[broken[0]] + 1} boundary is not a closed loop")
    x = p.coordinates
    xs, xn = x[start], x[start[nxt]]
    normal = np.zeros((p.nc, 3))
    total = np.zeros((p.nc, 3))
    np.add.at(normal, cell, np.cross(xs, xn))
    np.add.at(total, cell, xs)
    sphere = not np.all(x[:, 2] == 0.0)
    ref = _normalize(total) if sphere else np.broadcast_to(np.array([0.0, 0.0, 1.0]), total.shape)
    cw = np.flatnonzero(~(_dot(normal, ref) > 0))
    if len(cw):
        raise ValueError(f"cell {cw[0] + 1} is not counter-clockwise")
    nleft = np.bincount(edge[orient == 0], minlength=p.ne)
    nright = np.bincount(edge[orient != 0], minlength=p.ne)
    bad = np.flatnonzero((nleft > 1) | (nright > 1))
    if len(bad):
        raise ValueError(f"edge {p.nc + bad[0] + 1} has inconsistent cell orientations")
    if closed:
        bad = np.flatnonzero((nleft != 1) | (nright != 1))
        if len(bad):
            raise ValueError(f"edge {p.nc + bad[0] + 1} is a boundary edge of a closed mesh")
        chi = p.nv - p.ne + p.nc
        expected = 2 if sphere else 0
        if chi != expected:
            raise ValueError(f"Euler characteristic {chi} != {expected}")
    return True


def orthogonality_defect(mesh: HexMesh, centers: np.ndarray) -> float:
    """Largest |cos| between a primal edge and the great circle through its two cells'
    centers (CellCenters.jl:90-101); interior edges only."""
    lr = _edge_cells(mesh)
    ev = _edge_vertices(mesh)
    inner = np.all(lr >= 0, axis=1)
    x = mesh.plex.coordinates
    dual = _normalize(np.cross(centers[lr[inner, 0]], centers[lr[inner, 1]]))
    primal = _normalize(np.cross(x[ev[inner, 0]], x[ev[inner, 1]]))
    return float(np.abs(_dot(dual, primal)).max()) if inner.any() else 0.0


def _centroids(mesh: HexMesh) -> np.ndarray:
    rings = cell_vertex_table(mesh)
    x = mesh.plex.coordinates
    return np.array([_normalize(x[r - 1].sum(axis=0)) for r in rings])


def _circumcenters(mesh: HexMesh) -> np.ndarray:
    rings = cell_vertex_table(mesh)
    if any(len(r) != 3 for r in rings):
        raise ValueError("circumcenters need a triangle mesh")
    t = np.stack(rings) - 1
    x = mesh.plex.coordinates
    a, b, d = x[t[:, 0]], x[t[:, 1]], x[t[:, 2]]
    return _normalize(np.cross(b - a, d - a))  # counter-clockwise cells: points outward


def voronoi_generators(mesh: HexMesh, iterations: int = 4) -> np.ndarray:
    """The generators of the Voronoi diagram that fits the mesh best (CellCenters.jl:49-81):
    every interior edge with great-circle normal n between cells i and j asks
    (I - n n^T)(g_i - g_j) = 0 (two rows, on a tangent basis of the plane normal to n) and
    n . (g_i + g_j) = 0. The least-squares null vector of these homogeneous rows is found by
    inverse iteration on A^T A + 1e-10 max|diag| I from the cell centroids."""
    import scipy.sparse as sp
    from scipy.sparse.linalg import splu
    lr = _edge_cells(mesh)
    ev = _edge_vertices(mesh)
    inner = np.flatnonzero(np.all(lr >= 0, axis=1))
    x = mesh.plex.coordinates
    i, j = lr[inner, 0], lr[inner, 1]
    n = _normalize(np.cross(x[ev[inner, 0]], x[ev[inner, 1]]))
    pick = np.where((np.abs(n[:, 0]) < 0.9)[:, None], np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]))
    t1 = _normalize(np.cross(n, pick))
    t2 = np.cross(n, t1)
    m = len(inner)
    rows, cols, vals = [], [], []
    for r, (w, sj) in enumerate(((t1, -1.0), (t2, -1.0), (n, 1.0))):
        row = 3 * np.arange(m) + r
        for k in range(3):
            rows += [row, row]
            cols += [3 * i + k, 3 * j + k]
            vals += [w[:, k], sj * w[:, k]]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(3 * m, 3 * mesh.nc))
    B = (A.T @ A).tocsc()
    B = B + (1e-10 * np.abs(B.diagonal()).max()) * sp.identity(B.shape[0], format="csc")
    lu = splu(B.tocsc())
    centroids = _centroids(mesh)
    v = centroids.ravel().copy()
    for _ in range(int(iterations)):
        v = lu.solve(v)
        v /= np.linalg.norm(v)
    g = _normalize(v.reshape(-1, 3))
    if np.sum(_dot(g, centroids)) < 0:  # sign of the null vector
        g = -g
    return g


def cell_centers(mesh: HexMesh, method: str = "auto", tolerance: float = 1e-8) -> np.ndarray:
    """Cell centers on the unit sphere (CellCenters.jl:25-46): "circumcenter" (triangles),
    "voronoi", "centroid", or "auto" = circumcenters for a triangle mesh, else the Voronoi
    generators when they make the mesh orthogonal to ``tolerance``, else centroids."""
    if method == "auto":
        if all(len(r) == 3 for r in cell_vertex_table(mesh)):
            return _circumcenters(mesh)
        g = voronoi_generators(mesh)
        if orthogonality_defect(mesh, g) < tolerance:
            return g
        return _centroids(mesh)
    if method == "circumcenter":
        return _circumcenters(mesh)
    if method == "voronoi":
        return voronoi_generators(mesh)
    if method == "centroid":
        return _centroids(mesh)
    raise ValueError(f"unknown cell-center method {method!r}")


def _finish(polygons, coordinates, centers: str | None) -> PolygonMesh:
    mesh = PolygonMesh(polygons, coordinates)
    if centers is not None:
        mesh.set_centers(cell_centers(mesh, centers))
    return mesh


def read_icon_grid(filename: str, dual: bool = False, centers: str | None = "auto") -> PolygonMesh:
    """ICON triangular grid (``vlon``, ``vlat``, ``vertex_of_cell``; FileGrids.jl:52-65). With
    ``dual`` the hexagonal/pentagonal dual instead: vertices at the triangle centers (``clon``,
    ``clat``), cells from ``cells_of_vertex``; global grids only. ``centers``: the
    cell_centers method of the mesh's TRiSK grid (None: the normalized vertex means)."""
    with _Dataset(filename) as ds:
        vertices = lonlat_to_xyz(read_variable(ds, "vlon"), read_variable(ds, "vlat"))
        cell_points = lonlat_to_xyz(read_variable(ds, "clon"), read_variable(ds, "clat"))
        if not dual:
            table = rows_per_entity(read_variable(ds, "vertex_of_cell"), len(cell_points))
            return _finish(table.astype(np.int64), vertices, centers)
        table = rows_per_entity(read_variable(ds, "cells_of_vertex"), len(vertices)).astype(np.int64)
    inside = (table >= 1) & (table <= len(cell_points))
    if not np.all(inside.sum(axis=1) >= 5):
        raise ValueError("the dual of a regional ICON grid is not supported")
    rings = [row[keep] for row, keep in zip(table, inside)]
    return _finish(dual_polygons(rings, cell_points, vertices), cell_points, centers)


def read_mpas_grid(filename: str, dual: bool = False, centers: str | None = "auto") -> PolygonMesh:
    """MPAS Voronoi grid (``x/y/zVertex``, ``verticesOnCell``, ``nEdgesOnCell``; FileGrids.jl:
    77-95), coordinates projected onto the unit sphere. With ``dual`` the Delaunay
    triangulation instead: vertices at the generators (``x/y/zCell``), triangles from
    ``cellsOnVertex``, those touching a missing cell (regional grids) dropped."""
    with _Dataset(filename) as ds:
        flag = ds.attribute("on_a_sphere")
        if flag is not None and str(flag).strip() != "YES":
            raise ValueError(f"{filename} is a planar MPAS mesh")

        def xyz(prefix):
            return _normalize(np.stack([read_variable(ds, a + prefix).astype(np.float64) for a in "xyz"], axis=1))
        vertices, cell_points = xyz("Vertex"), xyz("Cell")
        if not dual:
            table = rows_per_entity(read_variable(ds, "verticesOnCell"), len(cell_points)).astype(np.int64)
            nedges = read_variable(ds, "nEdgesOnCell").astype(np.int64)
            if np.any(nedges > table.shape[1]):
                raise ValueError("nEdgesOnCell exceeds the width of verticesOnCell")
            return _finish([table[c, :nedges[c]] for c in range(len(table))], vertices, centers)
        table = rows_per_entity(read_variable(ds, "cellsOnVertex"), len(vertices)).astype(np.int64)
    keep = np.all((table >= 1) & (table <= len(cell_points)), axis=1)
    return _finish(table[keep], cell_points, centers)


def read_grid(filename: str, dual: bool = False, centers: str | None = "auto") -> PolygonMesh:
    """An ICON or MPAS grid file, told apart by its variables (FileGrids.jl:101-107)."""
    with _Dataset(filename) as ds:
        kind = "icon" if "vertex_of_cell" in ds else "mpas" if "verticesOnCell" in ds else None
    if kind == "icon":
        return read_icon_grid(filename, dual, centers)
    if kind == "mpas":
        return read_mpas_grid(filename, dual, centers)
    raise ValueError(f"{filename} is neither an ICON nor an MPAS grid file")


def hilbert_order(mesh: HexMesh) -> PolygonMesh:
    """The same mesh renumbered for locality (Ordering.jl:44-82): cells along the Hilbert
    curve of their centroids (hilbert_permutation), vertices in order of first appearance in
    the new cell order, edges by first appearance as plex_from_polygons numbers them. Cell c
    of the result is cell perm[c] of ``mesh``; its centers are the mesh's centers permuted
    the same way."""
    perm = mesh.hilbert_permutation() - 1
    sizes, verts = cell_vertex_csr(mesh)
    starts = np.cumsum(sizes) - sizes
    new_sizes = sizes[perm]
    # the vertex list of the permuted cells: cell perm[c]'s run, for c in order
    idx = np.repeat(starts[perm] - (np.cumsum(new_sizes) - new_sizes), new_sizes) + np.arange(new_sizes.sum())
    flat = verts[idx] - 1
    ids, at = np.unique(flat, return_index=True)
    if len(ids) != mesh.nv:
        raise ValueError("vertices without cells")
    first = np.empty(mesh.nv, dtype=np.int64)
    first[flat[np.sort(at)]] = np.arange(mesh.nv)    # new number = rank of first appearance
    x = np.empty_like(mesh.plex.coordinates)
    x[first] = mesh.plex.coordinates
    return PolygonMesh((new_sizes, first[flat] + 1), x, centers=mesh.generators[perm])
