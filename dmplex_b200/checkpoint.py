"""Checkpoint and resume of a run's state.

The reference has no checkpoint: its state is the flat vector y = [u; h] (or, for an
ensemble, one such vector per member) in the numbering of its mesh. A checkpoint here is that
state in a raw binary file with a header that says what it belongs to, so that a resumed run
continues bit for bit where the interrupted one stopped:

    magic        8 bytes   b"TRSKSTAT"
    version      uint32    1
    header_len   uint32    bytes of the JSON header that follows
    header       UTF-8 JSON: kind, nc, ne, nv, state_size, members, step, time, mesh (the
                 fingerprint of the mesh numbering), meta (free-form)
    padding      to a multiple of 8 bytes
    payload      members x state_size float64, little endian
    crc32        uint32 of the payload

The mesh fingerprint is a SHA-256 over the sizes and the neighbour tables of the TRiSK grid:
a state is only meaningful in the numbering it was computed in, so loading it against a
different mesh (or a renumbered one) is refused. Files are written to a temporary name and
renamed into place, so an interrupted write never leaves a truncated checkpoint under the
final name.
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import zlib

import numpy as np

MAGIC = b"TRSKSTAT"
VERSION = 1


def mesh_fingerprint(grid) -> str:
    """SHA-256 (hex) of the sizes and neighbour tables of a TRiSKGrid: equal for the same mesh
    in the same numbering, different after any renumbering."""
    h = hashlib.sha256()
    h.update(struct.pack("<qqq", int(grid.nc), int(grid.ne), int(grid.nv)))
    for name in ("edge_cells", "edge_vertices", "cell_edges", "vertex_edges"):
        a = np.ascontiguousarray(getattr(grid, name), dtype="<i8")
        h.update(name.encode())
        h.update(struct.pack("<qq", *a.shape))
        h.update(a.tobytes())
    return h.hexdigest()


def _host(y) -> np.ndarray:
    if hasattr(y, "detach"):
        y = y.detach().cpu().numpy()
    y = np.asarray(y)
    if y.dtype != np.float64:
        raise ValueError("the state must be float64")
    return np.ascontiguousarray(y)


def save_state(path: str, y, grid, *, step: int = 0, time: float = 0.0, kind: str = "trisk",
               meta: dict | None = None) -> None:
    """Write the state ``y`` (one state vector, or members x state_size; numpy or a torch
    tensor on any device) of a run on ``grid`` after ``step`` steps (model time ``time``)."""
    a = _host(y)
    if a.ndim not in (1, 2):
        raise ValueError("the state must be a vector or a members x state matrix")
    members, size = (1, a.shape[0]) if a.ndim == 1 else a.shape
    if size != grid.ne + grid.nc and kind in ("trisk", "icon"):
        raise ValueError(f"a {kind} state has ne + nc = {grid.ne + grid.nc} values, not {size}")
    header = {"kind": kind, "nc": int(grid.nc), "ne": int(grid.ne), "nv": int(grid.nv), "state_size": int(size),
              "members": int(members), "ndim": int(a.ndim), "step": int(step), "time": float(time),
              "mesh": mesh_fingerprint(grid), "meta": meta or {}}
    hb = json.dumps(header, sort_keys=True).encode("utf-8")
    head = MAGIC + struct.pack("<II", VERSION, len(hb)) + hb
    head += bytes(-len(head) % 8)
    payload = a.astype("<f8", copy=False).tobytes()
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "wb") as f:
        f.write(head)
        f.write(payload)
        f.write(struct.pack("<I", zlib.crc32(payload) & 0xFFFFFFFF))
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def load_state(path: str, grid=None) -> tuple[np.ndarray, dict]:
    """(state, header) of a checkpoint. With ``grid`` the checkpoint must belong to that mesh
    in that numbering. Raises ValueError for a file that is not a checkpoint, of another
    version, truncated, corrupted (CRC) or of another mesh."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 16 or data[:8] != MAGIC:
        raise ValueError(f"{path} is not a state checkpoint")
    version, hlen = struct.unpack_from("<II", data, 8)
    if version != VERSION:
        raise ValueError(f"{path}: checkpoint version {version}, this library reads {VERSION}")
    if 16 + hlen > len(data):
        raise ValueError(f"{path} is truncated")
    header = json.loads(data[16:16 + hlen].decode("utf-8"))
    start = 16 + hlen
    start += -start % 8
    n = header["members"] * header["state_size"]
    end = start + 8 * n
    if end + 4 != len(data):
        raise ValueError(f"{path} is truncated or has trailing bytes")
    payload = data[start:end]
    (crc,) = struct.unpack_from("<I", data, end)
    if zlib.crc32(payload) & 0xFFFFFFFF != crc:
        raise ValueError(f"{path}: the state fails its CRC check")
    if grid is not None and header["mesh"] != mesh_fingerprint(grid):
        raise ValueError(f"{path} belongs to a different mesh or numbering")
    y = np.frombuffer(payload, dtype="<f8").astype(np.float64)
    if header.get("ndim", 1) == 2:
        y = y.reshape(header["members"], header["state_size"])
    return y, header


class RunLog:
    """JSON-lines run log: one object per record, with the fields the reference's examples print
    (mass, energy and enstrophy change, L2 height change, ms per step) plus whatever the
    caller adds (GB/s, roofline fraction, ...). Each line is flushed when written."""

    def __init__(self, path: str, **fixed):
        self.path = path
        self.fixed = fixed
        self._f = open(path, "a", encoding="utf-8")

    def write(self, **record) -> None:
        rec = dict(self.fixed)
        rec.update({k: (float(v) if isinstance(v, (np.floating, np.integer)) else v) for k, v in record.items()})
        self._f.write(json.dumps(rec, sort_keys=True) + "\n")
        self._f.flush()

    def close(self) -> None:
        if not self._f.closed:
            self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def read_run_log(path: str) -> list:
    with open(path, encoding="utf-8") as f:
        return [json.loads(line) for line in f if line.strip()]
