"""ctypes binding of the CPU oracle (oracle/libtrisk_oracle.so).

TEST INFRASTRUCTURE: imported only by tests/, the smoke check and bench.py's CPU-baseline
leg, as the checker. It restates the reference kernels in plain C (see trisk_oracle.h for
the cited reference lines and for how parity is pinned); the product never calls it.

The oracle takes the same premultiplied tables the model exports
(``TRiSKShallowWater.coefficients()``): 1-based Int64, numpy ``(entity, k)`` layout.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrisk_oracle.so")

POINTERS = (
    "cell_edges", "divergence", "kinetic", "edge_cells", "edge_height", "edge_vertices", "inverse_dual",
    "vertex_edges", "curl", "vertex_cells", "vertex_height", "coriolis", "trisk_edges", "trisk",
    "cell_areas", "vertex_areas", "g_edges", "g_pv_edges", "g_weights", "rhombus", "g_coriolis",
    "vk_cell_vertices", "vk_kites", "vk_weights", "vk_height",
)
INDEX = {"cell_edges", "edge_cells", "edge_vertices", "vertex_edges", "vertex_cells", "trisk_edges", "g_edges",
         "g_pv_edges", "vk_cell_vertices"}


class OracleModelStruct(C.Structure):
    _fields_ = [("nc", C.c_int64), ("ne", C.c_int64), ("nv", C.c_int64), ("cw", C.c_int32), ("vw", C.c_int32),
                ("tw", C.c_int32), ("pv_flux", C.c_int32), ("alpha", C.c_double),
                ("gravity", C.c_double)] + [(n, C.c_void_p) for n in POINTERS]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    sources = [os.path.join(HERE, f) for f in ("trisk_oracle.c", "trisk_oracle.h", "mpas_oracle.c", "mpas_oracle.h",
                                               "icon_oracle.c", "icon_oracle.h")]
    if not os.path.exists(LIB_PATH) or any(os.path.getmtime(f) > os.path.getmtime(LIB_PATH)
                                           for f in sources if os.path.exists(f)):
        build()
    lib = C.CDLL(LIB_PATH)
    p, d = C.c_void_p, C.c_double
    for name, res, args in [
        ("oracle_model_size", C.c_int, []),
        ("oracle_work_create", p, [p]),
        ("oracle_work_destroy", None, [p]),
        ("oracle_set_threads", None, [C.c_int]),
        ("oracle_threads", C.c_int, []),
        ("oracle_tendency", None, [p, p, p, p]),
        ("oracle_rk4_step", None, [p, p, p, d, p]),
        ("oracle_kinetic_energy", None, [p, p, p, p]),
        ("oracle_vertex_pv", None, [p, p, p, p]),
        ("oracle_mass_flux", None, [p, p, p, p]),
        ("oracle_total_mass", d, [p, p]),
        ("oracle_total_energy", d, [p, p, p]),
        ("oracle_potential_enstrophy", d, [p, p, p]),
        ("oracle_relative_vorticity", None, [p, p, p]),
        ("oracle_tangential_velocity", None, [p, p, p]),
        ("mpas_oracle_set_threads", None, [C.c_int]),
        ("mpas_oracle_tables_size", C.c_int, []),
        ("mpas_oracle_fields_size", C.c_int, []),
        ("mpas_oracle_slow_tendencies", None, [p, p, d]),
        ("icon_oracle_set_threads", None, [C.c_int]),
        ("icon_oracle_tables_size", C.c_int, []),
        ("icon_oracle_tendency", None, [p, p, p]),
        ("icon_oracle_rk4_step", None, [p, p, d, C.c_int64]),
    ]:
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    if lib.oracle_model_size() != C.sizeof(OracleModelStruct):
        raise ImportError("oracle_model layout mismatch")
    return lib


_lib = _load()


class OracleWorkStruct(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("K", "B", "F", "zv", "hv", "qv", "qe", "Kv")]


class Oracle:
    """The reference's serial TRiSK model restated on the CPU."""

    def __init__(self, coefficients: dict, threads: int = 1):
        c = coefficients
        self.nc, self.ne, self.nv = int(c["nc"]), int(c["ne"]), int(c["nv"])
        self.alpha = float(c["alpha"])
        self._keep = []
        s = OracleModelStruct()
        s.nc, s.ne, s.nv = self.nc, self.ne, self.nv
        s.cw, s.vw, s.tw = int(c["cw"]), int(c["vw"]), int(c["tw"])
        s.pv_flux, s.alpha, s.gravity = int(c["pv_flux"]), float(c["alpha"]), float(c["gravity"])
        for name in POINTERS:
            a = c.get(name)
            if a is None:
                continue
            a = np.ascontiguousarray(a, dtype=np.int64 if name in INDEX else np.float64)
            self._keep.append(a)
            setattr(s, name, a.ctypes.data)
        self._s = s
        self._w = _lib.oracle_work_create(C.byref(s))
        self.threads = threads

    def __del__(self):
        if getattr(self, "_w", None):
            _lib.oracle_work_destroy(self._w)
            self._w = None

    def _threads(self):
        _lib.oracle_set_threads(int(self.threads))

    @property
    def n(self) -> int:
        return self.ne + self.nc

    def work(self) -> dict:
        w = C.cast(self._w, C.POINTER(OracleWorkStruct)).contents
        sizes = {"K": self.nc, "B": self.nc, "F": self.ne, "zv": self.nv, "hv": self.nv, "qv": self.nv,
                 "qe": self.ne, "Kv": self.nv if self.alpha != 1.0 else 1}
        return {k: np.ctypeslib.as_array(getattr(w, k), shape=(n,)).copy() for k, n in sizes.items()}

    def tendency(self, y: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.zeros_like(y)
        self._threads()
        _lib.oracle_tendency(C.byref(self._s), self._w, y.ctypes.data, dy.ctypes.data)
        return dy

    def rk4_step(self, y: np.ndarray, dt: float, nsteps: int = 1) -> np.ndarray:
        """In place on a contiguous float64 y."""
        assert y.dtype == np.float64 and y.flags.c_contiguous
        cache = np.zeros(5 * self.n)
        self._threads()
        for _ in range(nsteps):
            _lib.oracle_rk4_step(C.byref(self._s), self._w, y.ctypes.data, float(dt), cache.ctypes.data)
        return y

    def kinetic_energy(self, y) -> np.ndarray:
        """K at the cells from kinetic_energy!(m, u, h) (TRiSKShallowWater.jl:332-340)."""
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._threads()
        _lib.oracle_kinetic_energy(C.byref(self._s), self._w, y.ctypes.data, y[self.ne:].ctypes.data)
        return self.work()["K"]

    def total_mass(self, y) -> float:
        y = np.ascontiguousarray(y, dtype=np.float64)
        return _lib.oracle_total_mass(C.byref(self._s), y.ctypes.data)

    def total_energy(self, y) -> float:
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._threads()
        return _lib.oracle_total_energy(C.byref(self._s), self._w, y.ctypes.data)

    def potential_enstrophy(self, y) -> float:
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._threads()
        return _lib.oracle_potential_enstrophy(C.byref(self._s), self._w, y.ctypes.data)

    def relative_vorticity(self, y) -> np.ndarray:
        y = np.ascontiguousarray(y, dtype=np.float64)
        z = np.zeros(self.nv)
        _lib.oracle_relative_vorticity(C.byref(self._s), y.ctypes.data, z.ctypes.data)
        return z

    def tangential_velocity(self, u) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64)
        v = np.zeros(self.ne)
        _lib.oracle_tangential_velocity(C.byref(self._s), u.ctypes.data, v.ctypes.data)
        return v
