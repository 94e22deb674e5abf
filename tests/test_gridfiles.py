"""ICON and MPAS grid files (dmplex.jl's FileGrids readers), after the reference's own test
(test/grids.jl:1-87): an ICON-like file written from an icosahedral triangle mesh and an
MPAS-like file written from a hexagon mesh, in the variable layout of those models' grid
files, read back as the primal and the dual mesh. Here the round trip is also held to the
tables: the TRiSK grid of a file read back equals the grid of the mesh that wrote it, and the
tendency on it equals the original's."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import gridfiles as gf

RADIUS = 6.371229e6


def _xyz_to_lonlat(x):
    return np.arctan2(x[:, 1], x[:, 0]), np.arcsin(np.clip(x[:, 2], -1, 1))


def _ring_table(g, width, fill):
    """vertex_cells of a TRiSK grid with the padding (sign 0) replaced by ``fill``."""
    t = np.where(g.vertex_signs != 0, g.vertex_cells, fill)
    out = np.full((g.nv, width), fill, dtype=np.int32)
    out[:, :t.shape[1]] = t
    return out


def write_icon_file(path, mesh, transposed=False):
    """ICON grid-file layout: vlon/vlat, clon/clat (radians), vertex_of_cell(nv, cell) and
    cells_of_vertex(ne, vertex), padded with 0 around pentagons."""
    from scipy.io import netcdf_file
    g = d.TRiSKGrid(mesh)
    vlon, vlat = _xyz_to_lonlat(g.vertices)
    clon, clat = _xyz_to_lonlat(g.centers)
    with netcdf_file(path, "w") as f:
        f.createDimension("vertex", g.nv)
        f.createDimension("cell", g.nc)
        f.createDimension("nv", 3)
        f.createDimension("ne", 6)
        for name, values, dim in (("vlon", vlon, "vertex"), ("vlat", vlat, "vertex"),
                                  ("clon", clon, "cell"), ("clat", clat, "cell")):
            f.createVariable(name, "f8", (dim,))[:] = values
        voc = g.cell_vertices.astype(np.int32)
        cov = _ring_table(g, 6, 0)
        if transposed:
            f.createVariable("vertex_of_cell", "i4", ("cell", "nv"))[:] = voc
            f.createVariable("cells_of_vertex", "i4", ("vertex", "ne"))[:] = cov
        else:
            f.createVariable("vertex_of_cell", "i4", ("nv", "cell"))[:] = voc.T
            f.createVariable("cells_of_vertex", "i4", ("ne", "vertex"))[:] = cov.T


def write_mpas_file(path, mesh, on_a_sphere="YES", cells_on_vertex=None):
    """MPAS grid-file layout: x/y/z Vertex and Cell on a sphere of Earth's radius,
    verticesOnCell(nCells, maxEdges) padded with nVertices+1 as MPAS-Ocean files are,
    nEdgesOnCell, cellsOnVertex(nVertices, vertexDegree)."""
    from scipy.io import netcdf_file
    g = d.TRiSKGrid(mesh)
    with netcdf_file(path, "w") as f:
        f.on_a_sphere = on_a_sphere
        f.createDimension("nCells", g.nc)
        f.createDimension("nVertices", g.nv)
        f.createDimension("maxEdges", 6)
        f.createDimension("vertexDegree", 3)
        for name, pts, dim in (("Vertex", g.vertices, "nVertices"), ("Cell", mesh.generators, "nCells")):
            for k, axis in enumerate("xyz"):
                f.createVariable(axis + name, "f8", (dim,))[:] = RADIUS * pts[:, k]
        n = (g.cell_signs != 0).sum(axis=1)
        voc = np.full((g.nc, 6), g.nv + 1, dtype=np.int32)
        for c in range(g.nc):
            voc[c, :n[c]] = g.cell_vertices[c, :n[c]]
        f.createVariable("verticesOnCell", "i4", ("nCells", "maxEdges"))[:] = voc
        f.createVariable("nEdgesOnCell", "i4", ("nCells",))[:] = n
        cov = _ring_table(g, 3, 0) if cells_on_vertex is None else cells_on_vertex
        f.createVariable("cellsOnVertex", "i4", ("nVertices", "vertexDegree"))[:] = cov


def _sphere_area(mesh):
    return d.TRiSKGrid(mesh).cell_areas.sum()


def _same_grid(a, b, rtol=0.0):
    for name in d.TRiSKGrid.FIELDS:
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        if rtol == 0.0 or x.dtype.kind in "iu":
            assert np.array_equal(x, y), name
        else:
            assert np.allclose(x, y, rtol=rtol, atol=rtol), name


def test_icon_reader(tmp_path):
    tri = d.create_triangle_mesh(2)
    for transposed in (False, True):
        path = tmp_path / f"icon{int(transposed)}.nc"
        write_icon_file(path, tri, transposed)
        m = gf.read_grid(str(path))
        assert gf.check_plex(m)
        assert (m.nc, m.ne, m.nv) == (tri.nc, tri.ne, tri.nv)
        assert np.allclose(m.plex.coordinates, tri.plex.coordinates, rtol=0, atol=1e-15)
        assert np.array_equal(m.plex.cones, tri.plex.cones)  # same polygons: same Plex
        _same_grid(d.TRiSKGrid(m), d.TRiSKGrid(tri), rtol=1e-13)
    dual = gf.read_icon_grid(str(path), dual=True)
    assert gf.check_plex(dual)
    assert dual.nc == tri.nv
    sizes = np.array([len(r) for r in gf.cell_vertex_table(dual)])
    assert np.sum(sizes == 5) == 12 and np.all((sizes == 5) | (sizes == 6))
    assert abs(_sphere_area(dual) - 4 * np.pi) < 1e-12
    # the dual of the ICON grid is the hexagon mesh of the same level (up to numbering)
    hexa = d.create_hexagon_mesh(2)
    assert dual.ne == hexa.ne and dual.nv == hexa.nv
    assert np.allclose(np.sort(d.TRiSKGrid(dual).cell_areas), np.sort(d.TRiSKGrid(hexa).cell_areas), rtol=1e-12)
    assert gf.orthogonality_defect(dual, dual.generators) < 1e-8


def test_mpas_reader(tmp_path):
    hexa = d.create_hexagon_mesh(2)
    path = tmp_path / "mpas.nc"
    write_mpas_file(path, hexa)
    m = gf.read_grid(str(path))
    assert gf.check_plex(m)
    assert m.nc == hexa.nc
    assert np.allclose(np.linalg.norm(m.plex.coordinates, axis=1), 1.0, rtol=0, atol=1e-15)
    assert np.array_equal(m.plex.cones, hexa.plex.cones)
    # the Voronoi generators recovered from the Plex alone are the file's generators
    assert np.abs(m.generators - hexa.generators).max() < 1e-12
    assert m.orthogonality_defect() < 1e-8
    _same_grid(d.TRiSKGrid(m), d.TRiSKGrid(hexa), rtol=1e-10)
    delaunay = gf.read_mpas_grid(str(path), dual=True)
    assert gf.check_plex(delaunay)
    assert delaunay.nc == hexa.nv
    assert all(len(r) == 3 for r in gf.cell_vertex_table(delaunay))
    assert abs(_sphere_area(delaunay) - 4 * np.pi) < 1e-12


def test_tendency_on_a_read_grid(tmp_path):
    """The oracle's tendency on the TRiSK tables of a grid read from an MPAS file is the
    tendency on the generated mesh up to the round-off of the geometry: the file holds the
    coordinates times Earth's radius, renormalized on reading, and the cell centers are the
    Voronoi generators recovered by inverse iteration (1e-15 apart). The gravity term's
    cancellation lifts that to about 1e-11 relative; 1e-10 is the bar."""
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    hexa = d.create_hexagon_mesh(3)
    path = tmp_path / "mpas3.nc"
    write_mpas_file(path, hexa)
    g0, g1 = d.TRiSKGrid(hexa), d.TRiSKGrid(gf.read_grid(str(path)))
    si = w.si_parameters()
    y = w.synthetic_state(g0, seed=2)
    a = Oracle(d.model_tables(g0, pv_flux="gassmann", kinetic_energy="vertex", **si)).tendency(y)
    b = Oracle(d.model_tables(g1, pv_flux="gassmann", kinetic_energy="vertex", **si)).tendency(y)
    assert 0 < np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(a)


def test_regional_and_invalid_files(tmp_path):
    tri, hexa = d.create_triangle_mesh(1), d.create_hexagon_mesh(1)
    # a regional MPAS grid: triangles that touch a missing cell are dropped
    g = d.TRiSKGrid(hexa)
    cov = _ring_table(g, 3, 0)
    cov[cov == 1] = 0
    path = tmp_path / "regional.nc"
    write_mpas_file(path, hexa, cells_on_vertex=cov)
    part = gf.read_mpas_grid(str(path), dual=True, centers=None)
    assert part.nc == hexa.nv - np.sum(np.any(_ring_table(g, 3, 0) == 1, axis=1))
    assert gf.check_plex(part, closed=False)
    with pytest.raises(ValueError, match="boundary edge"):
        gf.check_plex(part)
    # the dual of a regional ICON grid is refused
    path = tmp_path / "icon.nc"
    write_icon_file(path, tri)
    from scipy.io import netcdf_file
    with netcdf_file(path, "a") as f:
        cov = f.variables["cells_of_vertex"]
        t = cov[:].copy()
        t[:, 0] = 0
        cov[:] = t
    assert gf.check_plex(gf.read_icon_grid(str(path)))
    with pytest.raises(ValueError, match="regional"):
        gf.read_icon_grid(str(path), dual=True)
    # planar MPAS, a file of neither kind, an HDF5 file, a file of something else
    path = tmp_path / "planar.nc"
    write_mpas_file(path, hexa, on_a_sphere="NO")
    with pytest.raises(ValueError, match="planar"):
        gf.read_grid(str(path))
    path = tmp_path / "other.nc"
    with netcdf_file(path, "w") as f:
        f.createDimension("x", 3)
        f.createVariable("temperature", "f8", ("x",))[:] = 0.0
    with pytest.raises(ValueError, match="neither"):
        gf.read_grid(str(path))
    path = tmp_path / "netcdf4.nc"
    path.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    with pytest.raises(ValueError, match="nccopy"):
        gf.read_grid(str(path))
    path = tmp_path / "text.nc"
    path.write_bytes(b"not a grid")
    with pytest.raises(ValueError, match="not a NetCDF"):
        gf.read_grid(str(path))


def test_polygon_mesh_errors():
    x, t = d.icosahedral_mesh(1)
    m = d.PolygonMesh(t, x)
    assert gf.check_plex(m)
    assert np.array_equal(gf.cell_centers(m), d.create_triangle_mesh(1).generators)
    bad = t.copy()
    bad[3, 1] = len(x) + 1
    with pytest.raises(d.TriskError, match="outside"):
        d.PolygonMesh(bad, x)
    with pytest.raises(d.TriskError, match="fewer than three"):
        d.PolygonMesh([t[0], t[1][:2]], x)
    # a triangle twice: its edges get two cells on one side
    with pytest.raises(ValueError, match="inconsistent"):
        gf.check_plex(d.PolygonMesh(np.concatenate([t, t[:1]]), x))
    with pytest.raises(ValueError, match="Euler characteristic 4"):  # two disjoint spheres
        gf.check_plex(d.PolygonMesh(np.concatenate([t, t + len(x)]), np.concatenate([x, x])))
    with pytest.raises(ValueError):
        gf.cell_centers(m, "barycentric")
    with pytest.raises(ValueError, match="triangle"):
        gf.cell_centers(d.create_hexagon_mesh(1), "circumcenter")


def test_sort_ring():
    """sort_ring: counter-clockwise seen from outside, by the angle from the first id in
    (-pi, pi] (the first id at 0), so ids at negative angles come first."""
    axis = np.array([0.0, 0.0, 1.0])
    ang = np.array([0.0, 2.0, 4.0, 1.0, 3.0, 5.0])
    pts = np.stack([0.5 * np.cos(ang), 0.5 * np.sin(ang), np.full(6, 1.0)], axis=1)
    ids = np.array([4, 1, 2, 3, 5, 6])
    rel = np.angle(np.exp(1j * (ang[ids - 1] - ang[3])))   # 0, -1, 1, 3, 2, -2.28
    assert list(gf.sort_ring(ids, pts, axis)) == [6, 1, 4, 2, 5, 3]
    assert list(gf.sort_ring(ids, pts, axis)) == list(ids[np.argsort(rel)])
    rings = [ids, ids[:3]]
    out = gf.dual_polygons(rings, pts, np.stack([axis, 2 * axis]))
    assert list(out[0]) == [6, 1, 4, 2, 5, 3] and list(out[1]) == [1, 4, 2]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["mpas", "icon_dual"])
def test_gpu_model_on_a_read_grid(require_gpu, tmp_path, kind):
    """The library's kernels on a grid read from a file (its own numbering, Hilbert
    reordering on) match the oracle on the same tables bit for bit, tendency and RK4."""
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    path = tmp_path / "grid.nc"
    if kind == "mpas":
        write_mpas_file(path, d.create_hexagon_mesh(4))
        mesh = gf.read_grid(str(path))
    else:
        write_icon_file(path, d.create_triangle_mesh(4))
        mesh = gf.read_grid(str(path), dual=True)
    g = d.TRiSKGrid(mesh)
    si = w.si_parameters()
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    o = Oracle(d.model_tables(g, pv_flux="gassmann", kinetic_energy="vertex", **si))
    y = w.synthetic_state(g, seed=4)
    dy = np.zeros_like(y)
    d.tendency(dy, y, m)
    assert np.array_equal(dy, o.tendency(y))
    ref = o.rk4_step(y.copy(), 300.0, 3)
    d.rk4_step(y, 300.0, d.tendency, d.RK4Cache(y), m, nsteps=3)
    assert np.array_equal(y, ref)


def test_hilbert_order():
    """hilbert_order(dm) (Ordering.jl:44-82): cells along the Hilbert curve, vertices and
    edges by first appearance; the same mesh otherwise."""
    m = d.create_hexagon_mesh(3)
    h = gf.hilbert_order(m)
    assert gf.check_plex(h)
    perm = m.hilbert_permutation() - 1
    g0, g1 = d.TRiSKGrid(m), d.TRiSKGrid(h)
    assert np.allclose(g1.cell_areas, g0.cell_areas[perm], rtol=1e-13, atol=0)
    assert np.array_equal(h.generators, m.generators[perm])
    flat = np.concatenate(gf.cell_vertex_table(h)) - 1
    assert np.array_equal(np.unique(flat, return_index=True)[1], np.sort(np.unique(flat, return_index=True)[1]))
    assert h.orthogonality_defect() < 1e-12
