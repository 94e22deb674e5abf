"""TRiSK shallow-water model on the GPU, mirroring dmplex.jl's interface:

    TRiSKShallowWater(grid; gravity, coriolis, pv_flux, kinetic_energy)
                                           src/FiniteVolumes/TRiSKShallowWater.jl:94-170
    tendency!(dy, y, m)                    :379-394      -> tendency(dy, y, m)
    rk4_step!(y, dt, tendency!, cache, m)  RungeKutta.jl:18-29 -> rk4_step(y, dt, tendency, cache, m)
    total_mass / total_energy / potential_enstrophy / relative_vorticity   :397-426
    initial_state(m, velocity, height)     :184-188
    velocity_dofs / height_dofs            :173-174

The state ``y = [u; h]`` is FP64 in file (Plex) numbering: a numpy array (host) or a
CUDA float64 torch tensor (device). Every call goes to libtrisk_b200.so; there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, ptr, view
from .mesh import HexMesh, TRiSKGrid

PV_FLUX = {"trisk": 0, "gassmann": 1, "gassmann_mean": 2}
KINETIC_ENERGY = {"cell": 1.0, "mixed": 3 / 8, "vertex": 0.0}


def _pv_code(pv_flux) -> int:
    key = str(pv_flux).lstrip(":")
    if key not in PV_FLUX:
        raise ValueError("pv_flux must be :trisk, :gassmann or :gassmann_mean")
    return PV_FLUX[key]


def _alpha(kinetic_energy) -> float:
    if isinstance(kinetic_energy, (int, float, np.floating)) and not isinstance(kinetic_energy, bool):
        return float(kinetic_energy)
    key = str(kinetic_energy).lstrip(":")
    if key not in KINETIC_ENERGY:
        raise ValueError("kinetic_energy must be :cell, :mixed, :vertex or a weight")
    return KINETIC_ENERGY[key]


class TRiSKShallowWater:
    """Nonlinear rotating shallow water on the C grid of a Voronoi mesh (TRiSK or
    Gassmann PV flux, cell/vertex/mixed kinetic energy), on one GPU."""

    def __init__(self, grid, *, gravity: float = 1.0, coriolis=None, omega: float = 1.0,
                 pv_flux="trisk", kinetic_energy="cell", reorder: bool = True, device: int = 0,
                 use_graph: bool = True, use_pdl: bool = True, block: int = 0, _coefficients=None):
        if isinstance(grid, HexMesh):
            grid = TRiSKGrid(grid)
        self.grid = grid
        self.pv_flux = str(pv_flux).lstrip(":")
        self.alpha = _alpha(kinetic_energy)
        pv = _pv_code(pv_flux)
        cfg = _lib.TriskConfig()
        cfg.pv_flux, cfg.reorder, cfg.alpha, cfg.gravity, cfg.omega = pv, int(reorder), self.alpha, gravity, omega
        cfg.device, cfg.use_graph, cfg.use_pdl, cfg.block = device, int(use_graph), int(use_pdl), block
        keep = []
        if coriolis is not None and grid is not None:  # coriolis(x) at the vertices and the edge points
            fv = np.ascontiguousarray(coriolis(grid.vertices), dtype=np.float64)
            fe = np.ascontiguousarray(coriolis(grid.edge_points), dtype=np.float64)
            keep += [fv, fe]
            cfg.coriolis_vertices, cfg.coriolis_edges = fv.ctypes.data, fe.ctypes.data
        handle = C.c_void_p()
        if _coefficients is None:
            gs = grid.struct()
            check(lib.trisk_model_create(C.byref(gs), C.byref(cfg), C.byref(handle)))
        else:
            cs, arrays = _coefficients_struct(_coefficients, pv, self.alpha, gravity)
            keep += arrays
            if grid is not None and reorder:
                pos = np.ascontiguousarray(grid.centers, dtype=np.float64)
                keep.append(pos)
                cfg.cell_positions = pos.ctypes.data
            check(lib.trisk_model_create_from_coefficients(C.byref(cs), C.byref(cfg), C.byref(handle)))
        self._h = handle
        sizes = np.zeros(3, dtype=np.int64)
        check(lib.trisk_model_sizes(self._h, sizes.ctypes.data))
        self.nc, self.ne, self.nv = (int(x) for x in sizes)
        self.gravity = gravity

    @classmethod
    def from_coefficients(cls, coefficients: dict, grid=None, **kwargs) -> "TRiSKShallowWater":
        """Model from the premultiplied tables of an existing reference model (the arrays
        of a Julia ``TRiSKShallowWater``: 1-based, ``(entity, k)`` numpy layout)."""
        return cls(grid, _coefficients=coefficients, **kwargs)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.trisk_model_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def state_size(self) -> int:
        return self.ne + self.nc

    def coefficients(self) -> dict:
        """The model's premultiplied tables (file numbering, 1-based), as numpy copies."""
        c = _lib.TriskCoefficients()
        check(lib.trisk_model_coefficients(self._h, C.byref(c)))
        return _coefficients_dict(c)

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib.trisk_model_stream(self._h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        return int(lib.trisk_launch_count(self._h))

    def algorithmic_bytes(self) -> dict:
        out = np.zeros(4)
        check(lib.trisk_model_bytes(self._h, out.ctypes.data))
        return {"vertex": out[0], "flux": out[1], "tend": out[2], "rk4_step": out[3]}

    def profile_phases(self, y_device, dt: float, nsteps: int) -> dict:
        ms = np.zeros(3)
        check(lib.trisk_profile_phases(self._h, ptr(y_device), float(dt), int(nsteps), ms.ctypes.data))
        return {"vertex": ms[0], "flux": ms[1], "tend": ms[2]}

    def info(self) -> dict:
        pv = C.c_int32()
        block = np.zeros(3, dtype=np.int32)
        saved = C.c_double()
        check(lib.trisk_model_info(self._h, C.byref(pv), block.ctypes.data, C.byref(saved)))
        keep, window = C.c_int64(), C.c_int32()
        check(lib.trisk_model_get_l2_residency(self._h, C.byref(keep), C.byref(window)))
        return {"pv_mode": pv.value, "block": block.tolist(), "derived_pv_bytes_saved": saved.value,
                "l2_resident_table_bytes": keep.value, "l2_window": bool(window.value)}

    def autotune(self, y_device, dt: float, steps: int = 20) -> float:
        """Picks the fastest phase block sizes and L2-resident table prefix for this mesh and
        scheme; returns ms/step."""
        best = C.c_double()
        check(lib.trisk_autotune(self._h, ptr(y_device), float(dt), int(steps), C.byref(best)))
        return best.value

    def set_block(self, block) -> None:
        """Threads per block of the (vertex, flux, tend) phases, e.g. an autotune result."""
        b = np.ascontiguousarray(block, dtype=np.int32)
        if b.shape != (3,):
            raise ValueError("three block sizes")
        check(lib.trisk_model_set_block(self._h, b.ctypes.data))

    @property
    def persistent(self) -> bool:
        """Whether the RK4 steps run as one cooperative launch (the autotuner may choose it)."""
        on = C.c_int32()
        check(lib.trisk_model_get_persistent(self._h, C.byref(on)))
        return bool(on.value)

    def set_persistent(self, on: bool) -> None:
        """RK4 steps as one cooperative launch with grid barriers between the phases (meshes
        that stay in L2), or as the CUDA graph of twelve launches per step."""
        check(lib.trisk_model_set_persistent(self._h, int(bool(on))))

    def set_l2_residency(self, nbytes: int, window: bool = False) -> None:
        """Keeps the first nbytes of the packed tables in L2 (evict-last loads; with window
        also a persisting access-policy window). 0 streams every table."""
        check(lib.trisk_model_set_l2_residency(self._h, int(nbytes), int(bool(window))))

    def rk4_async(self, y_device, dt: float, nsteps: int = 1) -> None:
        check(lib.trisk_rk4_step_async(self._h, ptr(y_device), float(dt), int(nsteps)))

    def synchronize(self) -> None:
        check(lib.trisk_synchronize(self._h))


def l2_info(device: int = 0) -> dict:
    """L2 size, largest persisting set-aside, largest access-policy window and the current
    persisting limit of a CUDA device, in bytes."""
    out = np.zeros(4, dtype=np.int64)
    check(lib.trisk_l2_info(int(device), out.ctypes.data))
    return dict(zip(("l2_bytes", "max_persisting_bytes", "max_window_bytes", "persisting_limit"), out.tolist()))


def _coefficients_dict(c: _lib.TriskCoefficients) -> dict:
    nc, ne, nv, cw, vw, tw = c.nc, c.ne, c.nv, c.cw, c.vw, c.tw
    shapes = {
        "cell_edges": (nc, cw), "divergence": (nc, cw), "kinetic": (nc, cw), "edge_cells": (ne, 2),
        "edge_height": (ne, 2), "edge_vertices": (ne, 2), "inverse_dual": (ne,), "vertex_edges": (nv, vw),
        "curl": (nv, vw), "vertex_cells": (nv, vw), "vertex_height": (nv, vw), "coriolis": (nv,),
        "trisk_edges": (ne, tw), "trisk": (ne, tw), "cell_areas": (nc,), "vertex_areas": (nv,),
        "g_edges": (ne, 12), "g_pv_edges": (ne, 12), "g_weights": (ne, 12), "rhombus": (ne, 2),
        "g_coriolis": (ne,), "vk_cell_vertices": (nc, cw), "vk_kites": (nc, cw), "vk_weights": (nv, vw),
        "vk_height": (ne, 2),
    }
    out = {"nc": nc, "ne": ne, "nv": nv, "cw": cw, "vw": vw, "tw": tw, "pv_flux": c.pv_flux,
           "alpha": c.alpha, "gravity": c.gravity}
    for name, shape in shapes.items():
        address = getattr(c, name)
        dtype = np.int64 if name in _lib.INDEX_TABLES else np.float64
        out[name] = view(address, shape, dtype) if address else None
    return out


def model_tables(grid, *, gravity: float = 1.0, coriolis=None, omega: float = 1.0, pv_flux="trisk",
                 kinetic_energy="cell") -> dict:
    """The premultiplied tables of TRiSKShallowWater(grid; ...) built on the host, without a
    GPU (TRiSKShallowWater.jl:103-158): the same arrays ``TRiSKShallowWater.coefficients()``
    returns."""
    if isinstance(grid, HexMesh):
        grid = TRiSKGrid(grid)
    cfg = _lib.TriskConfig()
    cfg.pv_flux, cfg.alpha, cfg.gravity, cfg.omega = _pv_code(pv_flux), _alpha(kinetic_energy), gravity, omega
    keep = []
    if coriolis is not None:
        fv = np.ascontiguousarray(coriolis(grid.vertices), dtype=np.float64)
        fe = np.ascontiguousarray(coriolis(grid.edge_points), dtype=np.float64)
        keep += [fv, fe]
        cfg.coriolis_vertices, cfg.coriolis_edges = fv.ctypes.data, fe.ctypes.data
    gs = grid.struct()
    handle = C.c_void_p()
    check(lib.trisk_tables_create(C.byref(gs), C.byref(cfg), C.byref(handle)))
    try:
        c = _lib.TriskCoefficients()
        check(lib.trisk_tables_view(handle, C.byref(c)))
        return _coefficients_dict(c)
    finally:
        lib.trisk_tables_destroy(handle)


def _coefficients_struct(coeffs: dict, pv: int, alpha: float, gravity: float):
    cs = _lib.TriskCoefficients()
    nc, cw = np.asarray(coeffs["cell_edges"]).shape
    ne = len(coeffs["inverse_dual"])
    nv, vw = np.asarray(coeffs["vertex_edges"]).shape
    tw = np.asarray(coeffs["trisk_edges"]).shape[1] if coeffs.get("trisk_edges") is not None else 10
    cs.nc, cs.ne, cs.nv, cs.cw, cs.vw, cs.tw = nc, ne, nv, cw, vw, tw
    cs.pv_flux, cs.alpha, cs.gravity = pv, alpha, gravity
    keep = []
    for name in _lib.COEFFICIENT_POINTERS:
        a = coeffs.get(name)
        if a is None:
            continue
        dtype = np.int64 if name in _lib.INDEX_TABLES else np.float64
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        setattr(cs, name, a.ctypes.data)
    return cs, keep


def velocity_dofs(m: TRiSKShallowWater) -> slice:
    return slice(0, m.ne)


def height_dofs(m: TRiSKShallowWater) -> slice:
    return slice(m.ne, m.ne + m.nc)


def _state(y, m: TRiSKShallowWater):
    if isinstance(y, np.ndarray):
        if y.dtype != np.float64 or not y.flags.c_contiguous or y.size != m.state_size:
            raise ValueError(f"state must be a contiguous float64 vector of length {m.state_size}")
    elif hasattr(y, "data_ptr"):
        if str(y.dtype) != "torch.float64" or not y.is_contiguous() or y.numel() != m.state_size:
            raise ValueError(f"state must be a contiguous float64 tensor of length {m.state_size}")
    else:
        raise TypeError("state must be a numpy array or a torch tensor")
    return ptr(y)


def tendency(dy, y, m: TRiSKShallowWater):
    """tendency!(dy, y, m): writes the tendency of y into dy and returns dy."""
    check(lib.trisk_tendency(m.handle, _state(y, m), _state(dy, m)))
    return dy


class RK4Cache:
    """Work arrays of rk4_step! (RungeKutta.jl:2-10). The library keeps its stage vectors
    on the device, so the cache only records the state size."""

    def __init__(self, y):
        self.n = int(np.prod(getattr(y, "shape", (len(y),))))


def rk4_step(y, dt: float, tendency_fn, cache: RK4Cache, m: TRiSKShallowWater, nsteps: int = 1):
    """rk4_step!(y, dt, tendency!, cache, m): classical RK4 in place (nsteps of them)."""
    if tendency_fn is not tendency:
        raise TypeError("rk4_step integrates the library's own TRiSK tendency")
    if cache.n != m.state_size:
        raise ValueError("cache does not match the state size")
    check(lib.trisk_rk4_step(m.handle, _state(y, m), float(dt), int(nsteps)))
    return y


def _diagnostics(m, y, which):
    out = [C.c_double(), C.c_double(), C.c_double()]
    args = [C.byref(out[k]) if k == which else None for k in range(3)]
    check(lib.trisk_diagnostics(m.handle, _state(y, m), *args))
    return out[which].value


def total_mass(m: TRiSKShallowWater, y) -> float:
    return _diagnostics(m, y, 0)


def total_energy(m: TRiSKShallowWater, y) -> float:
    return _diagnostics(m, y, 1)


def potential_enstrophy(m: TRiSKShallowWater, y) -> float:
    return _diagnostics(m, y, 2)


def relative_vorticity(m: TRiSKShallowWater, y) -> np.ndarray:
    zeta = np.zeros(m.nv)
    check(lib.trisk_relative_vorticity(m.handle, _state(y, m), zeta.ctypes.data))
    return zeta


def initial_state(m: TRiSKShallowWater, velocity, height) -> np.ndarray:
    """[u; h]: normal components of velocity(x) at the edge points and height(x) at the
    generators (TRiSKShallowWater.jl:184-188). velocity and height take (n, 3) arrays."""
    g = m.grid
    u = np.einsum("ij,ij->i", np.asarray(velocity(g.edge_points), dtype=np.float64), g.edge_normals)
    h = np.asarray(height(g.centers), dtype=np.float64)
    return np.ascontiguousarray(np.concatenate([u, h]))
