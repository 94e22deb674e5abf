"""The grid geometry and the model's premultiplied coefficients, restated a second time in
numpy straight from the reference's Julia and compared with the library's C++ builder
(`TRiSKGrid`, `model_tables`), so that an error in that builder cannot hide behind the
oracle, which consumes the builder's tables.

Restated here, sharing no code with `dmplex_b200/csrc/mesh.cpp`:
- the TRiSKGrid geometry from the mesh's topology and coordinates: edge points, normals,
  primal and dual lengths, signed cell distances, kites, cell and vertex areas, vertex
  circulation signs, the vertex-cell lists and the TRiSK weights (TRiSKGrid.jl:83-160);
- `vertex_edge_areas` (TRiSKGrid.jl:179-191) and `gassmann_coefficients` (:214-251);
- the constructor's coefficients (TRiSKShallowWater.jl:103-158, serial distribution).

The topology itself (cell edges and corners in counter-clockwise order, edge cells and
vertices, vertex edges) is taken from the grid: it is integer, and its invariants are tested
in test_mesh.py. Index tables must agree exactly, and so must every floating-point table
whose formula has no great-circle length in it: the formulas and their association are the
reference's in both builders. The arc lengths (`atan2` of a cross and a dot product) come
from libm in the C++ builder and from numpy's `arctan2` here, which round the last bit
differently: the lengths and signed distances differ by under 1 ulp of the table's largest
entry (0.78 measured on hexagons 3 and 4), and the Gassmann weights, which multiply several
of them, by under 4 (3.74 measured).
"""
import numpy as np
import pytest

import dmplex_b200 as d
from conftest import trisk_grid

EPS = np.finfo(np.float64).eps


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], axis=-1)


def _norm(a):
    return np.sqrt(_dot(a, a))


def _normalize(a):
    with np.errstate(invalid="ignore", divide="ignore"):
        return a / _norm(a)[..., None]


def _arc_length(a, b):                       # TRiSKGrid.jl:2
    return np.arctan2(_norm(_cross(a, b)), _dot(a, b))


def _signed_triangle_area(a, b, c):          # TRiSKGrid.jl:5
    return 2 * np.arctan2(_dot(a, _cross(b, c)), 1 + _dot(a, b) + _dot(b, c) + _dot(c, a))


def _corner_counts(grid):
    return (grid.cell_signs != 0).sum(axis=1)


def restate_geometry(grid) -> dict:
    """TRiSKGrid.jl:83-160 on the grid's topology and coordinates; 0-based internally,
    returned 1-based like the grid."""
    x, g = grid.vertices, grid.centers
    ec, ev = grid.edge_cells - 1, grid.edge_vertices - 1
    xa, xb, gl, gr = x[ev[:, 0]], x[ev[:, 1]], g[ec[:, 0]], g[ec[:, 1]]
    m = _cross(_cross(xa, xb), _cross(gl, gr))
    m = np.where((_norm(m) > 1e-14)[:, None], _normalize(m), _normalize(xa + xb))
    m = np.where((_dot(m, xa + xb) < 0)[:, None], -m, m)
    normals = _normalize(_cross(xb, xa))
    l, dl = _arc_length(xa, xb), _arc_length(gl, gr)
    distances = np.stack([-np.sign(_dot(gl, normals)) * _arc_length(gl, m),
                          np.sign(_dot(gr, normals)) * _arc_length(gr, m)], axis=1)

    nc, nv, cw = grid.nc, grid.nv, grid.cell_edges.shape[1]
    ce, cv = grid.cell_edges - 1, grid.cell_vertices - 1
    count = _corner_counts(grid)
    kites = np.zeros((nc, cw))
    for n in np.unique(count):
        cells = np.flatnonzero(count == n)
        for k in range(n):
            v = cv[cells, k]
            kites[cells, k] = (_signed_triangle_area(g[cells], m[ce[cells, (k - 1) % n]], x[v]) +
                               _signed_triangle_area(g[cells], x[v], m[ce[cells, k]]))
    areas = np.zeros(nc)
    for k in range(cw):                      # sum.(cell_kites), in order
        areas = areas + kites[:, k]

    # vertex_cells / vertex_kites in push order: cells in order, corners in order
    cells_flat = np.repeat(np.arange(nc), cw)
    corner_flat = np.tile(np.arange(cw), nc)
    real = corner_flat < np.repeat(count, cw)
    owner = cv.reshape(-1)[real]
    order = np.argsort(owner, kind="stable")
    owner, push_cell, push_kite = owner[order], cells_flat[real][order], kites.reshape(-1)[real][order]
    vw = grid.vertex_edges.shape[1]
    slot = np.arange(len(owner)) - np.searchsorted(owner, owner, side="left")
    vertex_cells = np.ones((nv, vw), dtype=np.int64)
    vertex_kites = np.zeros((nv, vw))
    vertex_cells[owner, slot] = push_cell + 1
    vertex_kites[owner, slot] = push_kite
    vertex_areas = np.zeros(nv)
    for k in range(vw):
        vertex_areas = vertex_areas + vertex_kites[:, k]

    ve = grid.vertex_edges - 1
    present = grid.vertex_signs != 0
    vertex_signs = np.where(present, np.sign(_dot(normals[ve], _cross(x[:, None, :], m[ve]))), 0.0)

    # TRiSK weights: each cell in order walks counter-clockwise from every edge
    ne, tw = grid.ne, grid.trisk_edges.shape[1]
    pushes_e, pushes_cell, pushes_order, pushes_edge, pushes_w = [], [], [], [], []
    signs = grid.cell_signs
    for n in np.unique(count):
        cells = np.flatnonzero(count == n)
        R = kites[cells, :n] / areas[cells, None]
        for k in range(n):
            S = np.zeros(len(cells))
            for s in range(1, n):
                kk = (k + s) % n
                S = S + R[:, kk]
                pushes_e.append(ce[cells, k])
                pushes_cell.append(cells)
                pushes_order.append(np.full(len(cells), k * cw + s))
                pushes_edge.append(ce[cells, kk] + 1)
                pushes_w.append(signs[cells, k] * signs[cells, kk] * (0.5 - S))
    e_all = np.concatenate(pushes_e)
    key = np.lexsort((np.concatenate(pushes_order), np.concatenate(pushes_cell), e_all))
    e_sorted = e_all[key]
    slot = np.arange(len(e_sorted)) - np.searchsorted(e_sorted, e_sorted, side="left")
    trisk_edges = np.ones((ne, tw), dtype=np.int64)
    trisk_weights = np.zeros((ne, tw))
    trisk_edges[e_sorted, slot] = np.concatenate(pushes_edge)[key]
    trisk_weights[e_sorted, slot] = np.concatenate(pushes_w)[key]
    return dict(edge_points=m, edge_normals=normals, primal_lengths=l, dual_lengths=dl, cell_distances=distances,
                cell_kites=kites, cell_areas=areas, vertex_cells=vertex_cells, vertex_kites=vertex_kites,
                vertex_areas=vertex_areas, vertex_signs=vertex_signs, trisk_edges=trisk_edges,
                trisk_weights=trisk_weights)


def restate_vertex_edge_areas(grid):
    """TRiSKGrid.jl:179-191."""
    ec, cv, ce = grid.edge_cells - 1, grid.cell_vertices - 1, grid.cell_edges - 1
    count = _corner_counts(grid)

    def area(e, v):
        left = ec[e, 0]
        n = count[left]
        j = np.argmax(ce[left] == e[:, None], axis=1)
        assert (ce[left, j] == e).all()
        orientation = np.where(cv[left, (j + 1) % n] == v, 1.0, -1.0)
        return orientation * _signed_triangle_area(grid.centers[left], grid.centers[ec[e, 1]], grid.vertices[v])

    nv, vw = grid.vertex_edges.shape
    by_vertex = np.zeros((nv, vw))
    vs = np.arange(nv)
    for k in range(vw):
        live = grid.vertex_signs[:, k] != 0
        by_vertex[live, k] = area(grid.vertex_edges[live, k] - 1, vs[live])
    es = np.arange(grid.ne)
    by_edge = np.stack([area(es, grid.edge_vertices[:, s] - 1) for s in range(2)], axis=1)
    return by_vertex, by_edge


def restate_gassmann(grid):
    """TRiSKGrid.jl:214-251 (every vertex has three edges on a Voronoi mesh)."""
    ne = grid.ne
    l, dl, n, A = grid.primal_lengths, grid.dual_lengths, grid.edge_normals, grid.vertex_areas
    ev, ve = grid.edge_vertices - 1, grid.vertex_edges - 1
    assert (grid.vertex_signs != 0).all(), "Gassmann's reconstruction needs three edges per vertex"
    p, xv = grid.edge_points, grid.vertices
    es = np.arange(ne)

    def to_vertex(e, v):
        return _arc_length(p[e], xv[v])

    def rhombus(e):
        return A[ev[e, 0]] + A[ev[e, 1]]

    def other(e, v):
        return np.where(ev[e, 0] == v, ev[e, 1], ev[e, 0])

    def others(v, e):                        # the edges of v other than e, in order
        around = ve[v]
        keep = around != e[:, None]
        assert (keep.sum(axis=1) == 2).all()
        return around[keep].reshape(-1, 2)

    def metric(f):
        return _dot(n[f], _cross(_normalize(p[es] + p[f]), n[es]))

    area = l * dl
    edges = np.zeros((ne, 12), dtype=np.int64)
    pv_edges = np.zeros((ne, 12), dtype=np.int64)
    weights = np.zeros((ne, 12))
    k = 0
    for s in range(2):
        v = ev[:, s]
        inner = others(v, es)
        a = to_vertex(es, v) * dl / area
        for j in range(2):
            f, third = inner[:, j], inner[:, 1 - j]
            b = to_vertex(f, v) * dl[f]
            edges[:, k], pv_edges[:, k] = f + 1, third + 1
            weights[:, k] = metric(f) * (-a * b / A[v] + 2 / 3 * (a * l[f] * dl[f] / rhombus(f) + b / rhombus(es) +
                                                                 a * b / rhombus(third)))
            k += 1
            w = other(f, v)
            outer = others(w, f)
            for o in (outer[:, 0], outer[:, 1]):
                edges[:, k], pv_edges[:, k] = o + 1, f + 1
                weights[:, k] = 2 / 3 * metric(o) * a * to_vertex(o, w) * dl[o] / rhombus(f)
                k += 1
    return edges, pv_edges, weights


def restate_coefficients(grid, alpha: float, pv_flux: str) -> dict:
    """TRiSKShallowWater.jl:103-158 with the default coriolis (x -> 2x[3]) and the serial
    distribution (local numbering = global numbering)."""
    l, dl = grid.primal_lengths, grid.dual_lengths
    ce, ec, ev = grid.cell_edges - 1, grid.edge_cells - 1, grid.edge_vertices - 1
    s = grid.cell_signs
    cells = np.arange(grid.nc)[:, None]
    side = np.where(ec[ce, 0] == cells, 0, 1)
    live = s != 0
    Ai = grid.cell_areas[:, None]
    out = {
        "divergence": np.where(live, s * l[ce] / Ai, 0.0),
        "kinetic": np.where(live, alpha * l[ce] * grid.cell_distances[ce, side] / (2 * Ai), 0.0),
        "curl": grid.vertex_signs * dl[grid.vertex_edges - 1] / grid.vertex_areas[:, None],
        "vertex_height": grid.vertex_kites / grid.vertex_areas[:, None],
        "trisk": grid.trisk_weights * l[grid.trisk_edges - 1] / dl[:, None],
        "edge_height": alpha * grid.cell_distances / dl[:, None],
        "inverse_dual": 1 / dl,
        "coriolis": 2 * grid.vertices[:, 2],
    }
    if pv_flux != "trisk":
        r = grid.vertex_areas[ev]
        out["rhombus"] = r / (r[:, :1] + r[:, 1:])
        E, P, W = restate_gassmann(grid)
        out.update(g_edges=E, g_pv_edges=P, g_weights=W, g_coriolis=2 * grid.edge_points[:, 2])
    if alpha != 1:
        by_vertex, by_edge = restate_vertex_edge_areas(grid)
        out["vk_kites"] = (1 - alpha) * grid.cell_kites / Ai
        out["vk_weights"] = by_vertex / grid.vertex_areas[:, None]
        out["vk_height"] = (1 - alpha) * 2 * by_edge / (l * dl)[:, None]
    return out


def _ulps(got, want):
    """Largest difference in units of the last place of the table's largest entry."""
    scale = np.abs(want).max()
    return float(np.abs(got - want).max() / (EPS * scale)) if scale > 0 else float(np.abs(got).max())


GRIDS = [(3, False), (4, True)]


@pytest.mark.parametrize("level,centroidal", GRIDS)
def test_grid_geometry_restated_from_the_topology(level, centroidal):
    grid = trisk_grid(level, centroidal)
    mine = restate_geometry(grid)
    for name in ("vertex_cells", "trisk_edges"):
        assert np.array_equal(mine[name], getattr(grid, name)), name
    lengths = ("primal_lengths", "dual_lengths", "cell_distances")
    for name, want in mine.items():
        if want.dtype.kind == "f":
            worst = _ulps(getattr(grid, name), want)
            assert worst <= (1.0 if name in lengths else 0.0), (name, worst)
    # the cell signs point out of the cell: +1 on the left cell of an edge (the normal runs left to right)
    ce, ec = grid.cell_edges - 1, grid.edge_cells - 1
    live = grid.cell_signs != 0
    left = ec[ce, 0] == np.arange(grid.nc)[:, None]
    assert np.array_equal(grid.cell_signs[live], np.where(left, 1.0, -1.0)[live])


@pytest.mark.parametrize("level,centroidal", GRIDS)
@pytest.mark.parametrize("pv_flux,kinetic_energy,alpha", [("trisk", "cell", 1.0), ("gassmann", "vertex", 0.0),
                                                          ("gassmann_mean", "mixed", 3 / 8)])
def test_model_coefficients_restated_from_the_grid(level, centroidal, pv_flux, kinetic_energy, alpha):
    grid = trisk_grid(level, centroidal)
    tables = d.model_tables(grid, pv_flux=pv_flux, kinetic_energy=kinetic_energy)
    mine = restate_coefficients(grid, alpha, pv_flux)
    for name, want in mine.items():
        got = tables[name]
        assert got is not None and got.shape == want.shape, name
        if want.dtype.kind == "i":
            assert np.array_equal(got, want), name
        else:
            worst = _ulps(got, want)
            assert worst <= (4.0 if name == "g_weights" else 0.0), (name, worst)
    # the builder's padding: index 1, weight 0
    assert (tables["divergence"][grid.cell_signs == 0] == 0).all()
    assert (tables["cell_edges"][grid.cell_signs == 0] == 1).all()
    # tables the scheme does not use are not built
    if pv_flux == "trisk":
        assert tables["g_weights"] is None
    if alpha == 1:
        assert tables["vk_weights"] is None
