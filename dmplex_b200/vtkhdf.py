"""VTKHDF output of a surface mesh with cell data, mirroring dmplex.jl's

    write_vtkhdf(filename, dm; cell_data...)   src/Outputs/VTKHDF.jl:1-23
    cell_vorticity(g, u)                       examples/trisk_galewsky.jl:119-125

The file is a VTKHDF UnstructuredGrid (one piece) that ParaView and VTK open directly:
group ``/VTKHDF`` with the attributes ``Version`` = (1, 0) and ``Type`` = "UnstructuredGrid",
the datasets NumberOfPoints, NumberOfCells, NumberOfConnectivityIds (one entry each),
Points (np, 3) float64, Offsets (nc + 1) and Connectivity (0-based point ids) int64, Types
(nc) uint8 (5 triangle, 9 quad, 7 polygon, as VTKHDF.jl:12-15 picks them), and one dataset
per keyword under ``/VTKHDF/CellData`` (``/VTKHDF/PointData`` for point data).

No HDF5 library is needed: ``_H5File`` writes the HDF5 file format itself, in its oldest and
simplest form, which every HDF5 release reads — superblock version 0, version-1 object
headers, groups as a symbol table (a local heap of names, one leaf of a version-1 B-tree, and
symbol-table nodes of at most 2K = 8 entries each), contiguous datasets of little-endian
integers and IEEE floats, attributes in version-1 attribute messages. No structure of this
form carries a checksum.
"""
from __future__ import annotations

import struct

import numpy as np

from .mesh import HexMesh, TRiSKGrid

UNDEF = 0xFFFFFFFFFFFFFFFF   # the undefined address
_FREE_NULL = 1               # end of a local heap's free list (the library's on-disk value)
_LEAF_K, _NODE_K = 4, 16     # group leaf-node K and internal-node K of the superblock
_SNOD_ENTRIES = 2 * _LEAF_K
_BTREE_CHILDREN = 2 * _NODE_K
_BTREE_SIZE = 24 + (_BTREE_CHILDREN + 1) * 8 + _BTREE_CHILDREN * 8
_SNOD_SIZE = 8 + _SNOD_ENTRIES * 40

VTK_TRIANGLE, VTK_POLYGON, VTK_QUAD = 5, 7, 9


def _pad8(b: bytes) -> bytes:
    return b + bytes(-len(b) % 8)


def _datatype(dtype: np.dtype) -> bytes:
    """Datatype message body (version 1): fixed-point, IEEE floating-point or a fixed-length
    null-terminated ASCII string ('S' dtypes)."""
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        flags = 0x08 if dt.kind == "i" else 0x00          # bit 0 = 0: little endian; bit 3: signed
        return struct.pack("<B3BI", 0x10 | 0, flags, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "f":
        bits = 8 * dt.itemsize
        exp_loc, exp_size, mant_size, bias = {64: (52, 11, 52, 1023), 32: (23, 8, 23, 127)}[bits]
        # byte 0: little endian, no padding, mantissa normalization 2 (implied leading 1)
        return (struct.pack("<B3BI", 0x10 | 1, 0x20, bits - 1, 0, dt.itemsize)
                + struct.pack("<HHBBBBI", 0, bits, exp_loc, exp_size, 0, mant_size, bias))
    if dt.kind == "S":
        return struct.pack("<B3BI", 0x10 | 3, 0x00, 0, 0, dt.itemsize)  # null terminated, ASCII
    raise TypeError(f"no HDF5 datatype for {dt}")


def _dataspace(shape) -> bytes:
    """Dataspace message body (version 1; rank 0 is a scalar), no maximum dimensions."""
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", int(n)) for n in shape)


def _message(mtype: int, body: bytes) -> bytes:
    body = _pad8(body)
    return struct.pack("<HHB3x", mtype, len(body), 0) + body


def _attribute(name: str, value: np.ndarray) -> bytes:
    """Attribute message (version 1): the name, datatype and dataspace fields are each padded
    to 8 bytes, their sizes given unpadded."""
    n = name.encode("ascii") + b"\0"
    dt, ds = _datatype(value.dtype), _dataspace(value.shape)
    body = struct.pack("<BBHHH", 1, 0, len(n), len(dt), len(ds)) + _pad8(n) + _pad8(dt) + _pad8(ds)
    return _message(0x000C, body + value.astype(value.dtype.newbyteorder("<")).tobytes())


class _H5File:
    """Append-only builder: every structure is placed at an 8-byte aligned address after the
    96-byte superblock, children before the group that names them."""

    def __init__(self):
        self.buf = bytearray(96)

    def put(self, data: bytes) -> int:
        self.buf += bytes(-len(self.buf) % 8)
        addr = len(self.buf)
        self.buf += data
        return addr

    def object_header(self, messages: list) -> int:
        body = b"".join(messages)
        return self.put(struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body)

    def dataset(self, data: np.ndarray, attrs: dict | None = None) -> tuple:
        data = np.asarray(data)
        if not data.flags.c_contiguous:
            data = data.copy(order="C")  # (np.ascontiguousarray would make a scalar 1-D)
        raw = data.astype(data.dtype.newbyteorder("<")).tobytes()
        addr = self.put(raw) if raw else UNDEF
        msgs = [_message(0x0001, _dataspace(data.shape)), _message(0x0003, _datatype(data.dtype)),
                _message(0x0005, struct.pack("<BBBB", 2, 2, 2, 0)),        # fill value: late, if set, undefined
                _message(0x0008, struct.pack("<BBQQ", 3, 1, addr, len(raw)))]  # contiguous layout
        msgs += [_attribute(k, np.asarray(v)) for k, v in (attrs or {}).items()]
        return self.object_header(msgs), None

    def group(self, members: dict, attrs: dict | None = None) -> tuple:
        """members: name -> (object header address, (B-tree, heap) of a member group or None)."""
        names = sorted(members, key=lambda s: s.encode("utf-8"))
        if len(names) > _SNOD_ENTRIES * _BTREE_CHILDREN:
            raise ValueError(f"a group holds at most {_SNOD_ENTRIES * _BTREE_CHILDREN} members here")
        heap = bytearray(8)                         # offset 0: the empty name
        offsets = {}
        for name in names:
            offsets[name] = len(heap)
            heap += _pad8(name.encode("utf-8") + b"\0")
        heap_data = self.put(bytes(heap))
        heap_addr = self.put(b"HEAP" + struct.pack("<B3xQQQ", 0, len(heap), _FREE_NULL, heap_data))
        chunks = [names[i:i + _SNOD_ENTRIES] for i in range(0, len(names), _SNOD_ENTRIES)]
        children = []
        for chunk in chunks:
            entries = b""
            for name in chunk:
                header, cache = members[name]
                if cache is None:
                    entries += struct.pack("<QQI4x16x", offsets[name], header, 0)
                else:
                    entries += struct.pack("<QQI4xQQ", offsets[name], header, 1, *cache)
            node = b"SNOD" + struct.pack("<BBH", 1, 0, len(chunk)) + entries
            children.append(self.put(node + bytes(_SNOD_SIZE - len(node))))
        tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(children), UNDEF, UNDEF) + struct.pack("<Q", 0)
        for chunk, child in zip(chunks, children):   # key i+1: the last name of child i
            tree += struct.pack("<QQ", child, offsets[chunk[-1]])
        btree = self.put(tree + bytes(_BTREE_SIZE - len(tree)))
        msgs = [_message(0x0011, struct.pack("<QQ", btree, heap_addr))]
        msgs += [_attribute(k, np.asarray(v)) for k, v in (attrs or {}).items()]
        return self.object_header(msgs), (btree, heap_addr)

    def finish(self, root: tuple) -> bytes:
        header, (btree, heap) = root
        sb = b"\x89HDF\r\n\x1a\n" + struct.pack("<8B", 0, 0, 0, 0, 0, 8, 8, 0)
        sb += struct.pack("<HHI", _LEAF_K, _NODE_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
        sb += struct.pack("<QQI4xQQ", 0, header, 1, btree, heap)  # root group symbol-table entry
        assert len(sb) == 96
        self.buf[:96] = sb
        return bytes(self.buf)


def write_hdf5(filename: str, tree: dict) -> str:
    """Write a tree of groups and datasets: ``tree`` maps a name to an ndarray (a dataset), to
    a dict (a group), or to a pair (dict, attributes) for a group with attributes."""
    f = _H5File()

    def build(members: dict, attrs=None):
        out = {}
        for name, value in members.items():
            if isinstance(value, tuple):
                out[name] = build(*value)
            elif isinstance(value, dict):
                out[name] = build(value)
            else:
                out[name] = f.dataset(np.asarray(value))
        return f.group(out, attrs)

    data = f.finish(build(tree))
    with open(filename, "wb") as fh:
        fh.write(data)
    return filename


def _polygons(mesh) -> list:
    from .gridfiles import cell_vertex_table
    return cell_vertex_table(mesh)


def write_vtkhdf(filename: str, mesh: HexMesh, point_data: dict | None = None, **cell_data) -> str:
    """write_vtkhdf(filename, dm; cell_data...) (VTKHDF.jl:8-23): the cells of ``mesh`` as
    VTK triangles, quads or polygons over its vertices, with one float dataset per keyword
    (length nc, or (nc, k) for vectors). Returns ``filename``."""
    rings = _polygons(mesh)
    sizes = np.array([len(r) for r in rings], dtype=np.int64)
    conn = np.concatenate(rings).astype(np.int64) - 1
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    types = np.where(sizes == 3, VTK_TRIANGLE, np.where(sizes == 4, VTK_QUAD, VTK_POLYGON)).astype(np.uint8)
    points = np.ascontiguousarray(mesh.plex.coordinates, dtype=np.float64)
    cells = {}
    for name, values in cell_data.items():
        v = np.asarray(values)
        if v.shape[:1] != (mesh.nc,):
            raise ValueError(f"cell data {name!r} needs {mesh.nc} rows, got shape {v.shape}")
        cells[name] = v if v.dtype.kind in "iuf" else v.astype(np.float64)
    vtk = {
        "NumberOfPoints": np.array([len(points)], dtype=np.int64),
        "NumberOfCells": np.array([mesh.nc], dtype=np.int64),
        "NumberOfConnectivityIds": np.array([len(conn)], dtype=np.int64),
        "Points": points, "Offsets": offsets, "Connectivity": conn, "Types": types,
    }
    if cells:
        vtk["CellData"] = cells
    if point_data:
        for name, v in point_data.items():
            if np.shape(v)[:1] != (len(points),):
                raise ValueError(f"point data {name!r} needs {len(points)} rows")
        vtk["PointData"] = {k: np.asarray(v) for k, v in point_data.items()}
    attrs = {"Version": np.array([1, 0], dtype=np.int64), "Type": np.array(b"UnstructuredGrid", dtype="S17")}
    return write_hdf5(filename, {"VTKHDF": (vtk, attrs)})


def cell_vorticity(grid: TRiSKGrid, u: np.ndarray) -> np.ndarray:
    """Relative vorticity at the cells from the normal velocities: the vertex vorticities
    (circulation / dual area) averaged over each cell with its kite areas
    (trisk_galewsky.jl:119-125)."""
    u = np.asarray(u, dtype=np.float64)[:grid.ne]
    zeta = np.zeros(grid.nv)
    for k in range(grid.vertex_edges.shape[1]):
        e = grid.vertex_edges[:, k] - 1
        zeta = zeta + grid.vertex_signs[:, k] * grid.dual_lengths[e] * u[e]
    zeta = zeta / grid.vertex_areas
    out = np.zeros(grid.nc)
    for k in range(grid.cell_vertices.shape[1]):
        out = out + grid.cell_kites[:, k] * zeta[grid.cell_vertices[:, k] - 1]
    return out / grid.cell_areas
