"""CPU oracle of the ICON triangle shallow-water path (test infrastructure, never shipped).

A numpy restatement of dmplex.jl's ICONShallowWater kernels and rk4_step!, vectorised over
entities with each per-entity sum in the reference's order (numpy does not contract to FMA):

    icon_edge_kernel!          src/FiniteVolumes/ICONShallowWater.jl:149-159
    edge_sum_kernel!           src/FiniteVolumes/TRiSKShallowWater.jl:305-312 (K, zeta_v)
    icon_momentum_kernel!      ICONShallowWater.jl:161-171
    continuity_kernel!         TRiSKShallowWater.jl:298-305
    divergence_damping!        ICONShallowWater.jl:210-218 (edge_gradient_kernel! :173-176)
    rk4_step!                  src/TimeSteppers/RungeKutta.jl:18-29
    total_mass, total_energy   TRiSKShallowWater.jl:397-411 (K from kinetic_energy!, :184-189)

It works on the tables of dmplex_b200.icon.icon_tables (1-based, (entity, k)), the same the
library uploads. ``IconOracleC`` runs the same restatement in C with OpenMP
(oracle/icon_oracle.c), bit for bit the same. Its correctness is pinned by the reference's own ICON test assertions
(test/finite_volumes.jl:112-166) in tests/test_icon.py, and by the ICON figures it publishes
(docs/STATUS.md:40-55: TC2 errors on bisection and spring triangles, the Galewsky failure mode
of ICON's kinetic-energy gradient) in tests/test_published.py.
"""
from __future__ import annotations

import numpy as np


class IconOracle:
    def __init__(self, tables: dict):
        t = tables
        self.t = t
        self.ne, self.nc, self.nv = t["ne"], t["nc"], t["nv"]
        self.ce = t["cell_edges"] - 1
        self.ec = t["edge_cells"] - 1
        self.ev = t["edge_vertices"] - 1
        self.re = t["rbf_edges"] - 1
        self.ve = t["vertex_edges"] - 1
        self.nu = t.get("divergence_damping")
        if self.nu is not None and len(self.nu) == 0:
            self.nu = None

    @staticmethod
    def _edge_sum(w, idx, x):
        s = np.zeros(len(w))
        for k in range(w.shape[1]):
            s = s + w[:, k] * x[idx[:, k]]
        return s

    def kinetic_energy(self, u, h):
        """v, Ke, F at the edges and K at the cells (kinetic_energy!)."""
        t = self.t
        v = self._edge_sum(t["rbf"], self.re, u)
        Ke = (u * u + v * v) / 2
        F = (t["edge_height"][:, 0] * h[self.ec[:, 0]] + t["edge_height"][:, 1] * h[self.ec[:, 1]]) * u
        K = self._edge_sum(t["bilinear"], self.ce, Ke)
        return v, Ke, F, K

    def _continuity(self, F):
        return -self._edge_sum(self.t["divergence"], self.ce, F)

    def _gradient(self, D, scale):
        return scale * (D[self.ec[:, 1]] - D[self.ec[:, 0]]) * self.t["inverse_dual"]

    def tendency(self, y):
        t = self.t
        ne = self.ne
        u, h = y[:ne], y[ne:]
        v, Ke, F, K = self.kinetic_energy(u, h)
        zv = self._edge_sum(t["curl"], self.ve, u)
        zeta = (zv[self.ev[:, 0]] + zv[self.ev[:, 1]]) / 2
        g0, g1 = t["gradient"][:, 0], t["gradient"][:, 1]
        l, r = self.ec[:, 0], self.ec[:, 1]
        gradK = Ke * (g0 - g1) + g1 * K[r] - g0 * K[l]
        du = (t["edge_coriolis"] + zeta) * v - gradK - t["gravity"] * (h[r] - h[l]) * t["inverse_dual"]
        dh = self._continuity(F)
        if self.nu is not None:
            D = self._continuity(u)
            G = self._gradient(D, 1.0)
            D = self._continuity(G)
            G = self._gradient(D, -1.0)
            du = du + self.nu * G
        return np.concatenate([du, dh])

    def rk4_step(self, y, dt, nsteps=1):
        half, sixth = dt / 2, dt / 6
        for _ in range(nsteps):
            k1 = self.tendency(y)
            k2 = self.tendency(y + half * k1)
            k3 = self.tendency(y + half * k2)
            k4 = self.tendency(y + dt * k3)
            y += sixth * (k1 + 2 * k2 + 2 * k3 + k4)
        return y

    def total_mass(self, y):
        return float(np.sum(self.t["cell_areas"] * y[self.ne:]))

    def total_energy(self, y):
        u, h = y[:self.ne], y[self.ne:]
        K = self.kinetic_energy(u, h)[3]
        return float(np.sum(self.t["cell_areas"] * h * (K + self.t["gravity"] * h / 2)))


_INDEX = ("cell_edges", "edge_cells", "edge_vertices", "rbf_edges", "vertex_edges")
_REAL = ("divergence", "bilinear", "edge_height", "gradient", "inverse_dual", "rbf", "edge_coriolis", "curl",
         "cell_areas")


class IconOracleC:
    """tendency and rk4_step of IconOracle in C with OpenMP (oracle/icon_oracle.c), bit for bit
    the same, on ``threads`` host threads."""

    def __init__(self, tables: dict, threads: int = 1):
        import ctypes as C
        from oracle.oracle import _lib

        class Tables(C.Structure):
            _fields_ = ([(n, C.c_int64) for n in ("nc", "ne", "nv")] + [("vw", C.c_int32), ("reserved", C.c_int32),
                                                                       ("gravity", C.c_double)]
                        + [(n, C.c_void_p) for n in _INDEX + _REAL + ("divergence_damping",)])
        if _lib.icon_oracle_tables_size() != C.sizeof(Tables):
            raise RuntimeError("oracle struct layout mismatch")
        t = tables
        s = Tables()
        s.nc, s.ne, s.nv, s.vw, s.gravity = t["nc"], t["ne"], t["nv"], t["vw"], t["gravity"]
        self._keep = []
        for name in _INDEX + _REAL:
            a = np.ascontiguousarray(t[name], dtype=np.int64 if name in _INDEX else np.float64)
            self._keep.append(a)
            setattr(s, name, a.ctypes.data)
        nu = t.get("divergence_damping")
        if nu is not None and len(nu):
            a = np.ascontiguousarray(nu, dtype=np.float64)
            self._keep.append(a)
            s.divergence_damping = a.ctypes.data
        self._s, self._lib, self.threads = s, _lib, int(threads)
        self.ne, self.nc = t["ne"], t["nc"]
        self.cell_areas = np.ascontiguousarray(t["cell_areas"], dtype=np.float64)

    def tendency(self, y):
        import ctypes as C
        y = np.ascontiguousarray(y, dtype=np.float64)
        dy = np.empty_like(y)
        self._lib.icon_oracle_set_threads(self.threads)
        self._lib.icon_oracle_tendency(C.byref(self._s), y.ctypes.data, dy.ctypes.data)
        return dy

    def rk4_step(self, y, dt, nsteps=1):
        import ctypes as C
        if y.dtype != np.float64 or not y.flags.c_contiguous:
            raise ValueError("y must be a contiguous float64 array")
        self._lib.icon_oracle_set_threads(self.threads)
        self._lib.icon_oracle_rk4_step(C.byref(self._s), y.ctypes.data, float(dt), int(nsteps))
        return y

    def total_mass(self, y):
        return float(np.sum(self.cell_areas * y[self.ne:]))
