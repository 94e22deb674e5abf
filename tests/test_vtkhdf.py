"""VTKHDF output (dmplex.jl's write_vtkhdf, src/Outputs/VTKHDF.jl:8-23) and the cell
vorticity the TRiSK example writes (examples/trisk_galewsky.jl:119-125, 180-191). The files
are read back by a reader written from the HDF5 file-format specification
(hdf5_spec_reader.py): no HDF5 library is in the image."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import gridfiles as gf
from dmplex_b200 import vtkhdf
from hdf5_spec_reader import read_hdf5


def _vtk(path):
    root, _ = read_hdf5(path)
    kind, members, attrs = root["VTKHDF"]
    assert kind == "group"
    return members, attrs


@pytest.mark.parametrize("kind", ["hexagon", "triangle"])
def test_vtkhdf_mesh(tmp_path, kind):
    mesh = d.create_hexagon_mesh(2) if kind == "hexagon" else d.create_triangle_mesh(2)
    rng = np.random.default_rng(1)
    data = rng.standard_normal(mesh.nc)
    vec = rng.standard_normal((mesh.nc, 3)).astype(np.float32)
    path = str(tmp_path / f"{kind}.vtkhdf")
    assert vtkhdf.write_vtkhdf(path, mesh, vorticity=data, wind=vec) == path
    m, attrs = _vtk(path)
    assert list(attrs["Version"]) == [1, 0] and attrs["Version"].dtype == np.int64
    assert attrs["Type"][()] == b"UnstructuredGrid"
    ds = {k: v[1] for k, v in m.items() if v[0] == "dataset"}
    assert ds["NumberOfPoints"].tolist() == [mesh.nv] and ds["NumberOfCells"].tolist() == [mesh.nc]
    rings = gf.cell_vertex_table(mesh)
    conn = ds["Connectivity"]
    assert ds["NumberOfConnectivityIds"].tolist() == [len(conn)]
    assert conn.dtype == np.int64 and ds["Offsets"].dtype == np.int64 and ds["Types"].dtype == np.uint8
    off = ds["Offsets"]
    assert off[0] == 0 and off[-1] == len(conn) and len(off) == mesh.nc + 1
    for c in (0, 1, mesh.nc - 1):
        assert list(conn[off[c]:off[c + 1]] + 1) == list(rings[c])
    assert np.array_equal(ds["Points"], mesh.plex.coordinates)
    want = vtkhdf.VTK_TRIANGLE if kind == "triangle" else vtkhdf.VTK_POLYGON
    assert np.all(ds["Types"] == want)
    cells = m["CellData"][1]
    assert np.array_equal(cells["vorticity"][1], data)
    assert cells["wind"][1].dtype == np.float32 and np.array_equal(cells["wind"][1], vec)
    assert "PointData" not in m
    with pytest.raises(ValueError):
        vtkhdf.write_vtkhdf(path, mesh, vorticity=data[:-1])


def test_hdf5_groups_and_types(tmp_path):
    """Groups of more than one symbol-table node (8 entries), nested groups, empty and scalar
    datasets, every integer width, float32/64, string attributes; the member limit."""
    many = {f"field{i:03d}": np.arange(i, dtype=np.int32) for i in range(37)}
    tree = {
        "many": many,
        "nested": ({"inner": {"x": np.array(2.5)}, "u8": np.arange(5, dtype=np.uint8)},
                   {"note": np.array(b"hello", dtype="S6"), "pair": np.array([1.5, -2.0])}),
        "types": {f"{t}": np.arange(6, dtype=t).reshape(2, 3) for t in
                  ("int8", "uint16", "int32", "uint64", "float32", "float64")},
        "empty": np.zeros((0, 3)),
    }
    path = str(tmp_path / "t.h5")
    vtkhdf.write_hdf5(path, tree)
    root, _ = read_hdf5(path)
    got = root["many"][1]
    assert sorted(got) == sorted(many)
    for k, v in many.items():
        assert np.array_equal(got[k][1], v) and got[k][1].dtype == np.int32
    kind, nested, attrs = root["nested"]
    assert attrs["note"][()] == b"hello" and list(attrs["pair"]) == [1.5, -2.0]
    assert nested["inner"][1]["x"][1][()] == 2.5 and nested["inner"][1]["x"][1].shape == ()
    assert np.array_equal(nested["u8"][1], np.arange(5, dtype=np.uint8))
    for t, (_, a, _) in root["types"][1].items():
        assert a.dtype == np.dtype(t).newbyteorder("<") and np.array_equal(a, np.arange(6, dtype=t).reshape(2, 3))
    assert root["empty"][1].shape == (0, 3)
    with pytest.raises(ValueError, match="at most"):
        vtkhdf.write_hdf5(path, {f"g{i}": np.zeros(1) for i in range(257)})


def test_cell_vorticity():
    """Solid-body rotation u = U0 (-y, x, 0): relative vorticity 2 U0 z, to a truncation error
    that falls with resolution."""
    u0 = 0.2

    def error(n):
        g = d.TRiSKGrid(d.create_hexagon_mesh(n))
        vel = u0 * np.stack([-g.edge_points[:, 1], g.edge_points[:, 0], np.zeros(g.ne)], axis=1)
        zeta = vtkhdf.cell_vorticity(g, np.einsum("ij,ij->i", vel, g.edge_normals))
        return np.abs(zeta - 2 * u0 * g.centers[:, 2]).max()
    e3, e4 = error(3), error(4)
    assert 0 < e4 < 0.02 * u0 and e4 < 0.6 * e3
