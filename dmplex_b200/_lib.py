"""ctypes binding of libtrisk_b200.so (declared in include/trisk_b200.h).

The library is built in-tree (``make -C dmplex_b200``) and loaded from
``dmplex_b200/lib``. There is no fallback: if the library is missing or a GPU
call fails, the error propagates.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtrisk_b200.so")

_i32, _i64, _f64, _p = C.c_int32, C.c_int64, C.c_double, C.c_void_p

TRISK_OK = 0
STATUS_NAMES = {
    1: "argument",
    2: "table",
    3: "cuda",
    4: "nonfinite",
    5: "timeout",
    6: "unsupported",
    7: "mesh",
}


class TriskError(RuntimeError):
    """A non-zero status of the C ABI, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"trisk status {status} ({STATUS_NAMES.get(status, '?')}): {message}")
        self.status = status


class TriskIconTables(C.Structure):
    _fields_ = [("nc", _i64), ("ne", _i64), ("nv", _i64), ("vw", _i32), ("gravity", _f64)] + [
        (n, _p) for n in ("cell_edges", "divergence", "bilinear", "edge_cells", "edge_vertices", "edge_height",
                          "gradient", "inverse_dual", "rbf_edges", "rbf", "edge_coriolis", "vertex_edges", "curl",
                          "cell_areas", "divergence_damping")
    ]


class TriskMpasTables(C.Structure):
    _fields_ = [("nc", _i64), ("ne", _i64), ("nv", _i64), ("nlev", _i64)] + [
        (n, _i32) for n in ("cw", "vw", "nt", "vertex_kinetic", "iap_pv", "vertical", "five_band", "reserved")
    ] + [
        (n, _p) for n in ("cell_edges", "edge_cells", "edge_vertices", "vertex_edges", "vertex_cells",
                          "vk_cell_vertices", "kinetic", "inner", "vk_kites", "edge_weight", "rhombus",
                          "inverse_dual", "edge_coriolis", "curl", "vertex_weight", "vk_weights", "coriolis",
                          "trisk", "dz_cells", "dzh_cells", "wlow", "dz_edges", "dzh_edges", "trisk_index")
    ]


class TriskMpasFields(C.Structure):
    _fields_ = [(n, _p) for n in ("vn", "w", "rho", "rhotheta", "theta", "exner", "K", "Kv", "qv", "zetav", "rhov",
                                  "qe", "rhoe", "Fs", "eta", "tvn", "tw")]


class TriskPlex(C.Structure):
    _fields_ = [("nc", _i64), ("ne", _i64), ("nv", _i64), ("ncones", _i64)] + [
        (n, _p)
        for n in ("cone_offsets", "cones", "cone_orientations", "support_offsets", "supports", "coordinates")
    ]


GRID_POINTERS = (
    "centers", "vertices", "edge_points", "edge_normals", "primal_lengths", "dual_lengths",
    "edge_cells", "edge_vertices", "cell_distances", "cell_areas", "vertex_areas",
    "cell_edges", "cell_signs", "cell_vertices", "cell_kites",
    "vertex_edges", "vertex_signs", "vertex_cells", "vertex_kites",
    "trisk_edges", "trisk_weights",
)


class TriskGrid(C.Structure):
    _fields_ = [("nc", _i64), ("ne", _i64), ("nv", _i64), ("cw", _i32), ("vw", _i32), ("tw", _i32),
                ("pad_", _i32)] + [(n, _p) for n in GRID_POINTERS]


class TriskConfig(C.Structure):
    _fields_ = [("pv_flux", _i32), ("reorder", _i32), ("alpha", _f64), ("gravity", _f64), ("omega", _f64),
                ("coriolis_vertices", _p), ("coriolis_edges", _p), ("cell_positions", _p), ("device", _i32),
                ("use_graph", _i32), ("use_pdl", _i32), ("block", _i32)]


COEFFICIENT_POINTERS = (
    "cell_edges", "divergence", "kinetic", "edge_cells", "edge_height", "edge_vertices", "inverse_dual",
    "vertex_edges", "curl", "vertex_cells", "vertex_height", "coriolis", "trisk_edges", "trisk",
    "cell_areas", "vertex_areas", "g_edges", "g_pv_edges", "g_weights", "rhombus", "g_coriolis",
    "vk_cell_vertices", "vk_kites", "vk_weights", "vk_height",
)
INDEX_TABLES = {"cell_edges", "edge_cells", "edge_vertices", "vertex_edges", "vertex_cells", "trisk_edges",
                "g_edges", "g_pv_edges", "vk_cell_vertices"}


class TriskCoefficients(C.Structure):
    _fields_ = [("nc", _i64), ("ne", _i64), ("nv", _i64), ("cw", _i32), ("vw", _i32), ("tw", _i32),
                ("pv_flux", _i32), ("alpha", _f64), ("gravity", _f64)] + [(n, _p) for n in COEFFICIENT_POINTERS]


class TriskHalo(C.Structure):
    _fields_ = [("ne_owned", _i64), ("nc_owned", _i64), ("nneighbors", _i32), ("pad_", _i32),
                ("send_offsets", _p), ("send_index", _p), ("recv_offsets", _p), ("recv_index", _p)]


# int (*)(void* user, const double* send, int64_t nsend, double* recv, int64_t nrecv, void* stream)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, _p, _p, _i64, _p, _i64, _p)
EXCHANGE_HOST, EXCHANGE_DEVICE, EXCHANGE_DEVICE_GRAPH = 0, 1, 2


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C dmplex_b200` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "trisk_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
        "trisk_abi_version": (_i32, []),
        "trisk_struct_size": (_i32, [_i32]),
        "trisk_mesh_create_hexagon": (C.c_int, [_i32, _i32, _f64, C.POINTER(_p)]),
        "trisk_mesh_create_triangles": (C.c_int, [_i32, _i32, _f64, C.POINTER(_p)]),
        "trisk_mesh_from_polygons": (C.c_int, [_p, _p, _i64, _p, _i64, _p, C.POINTER(_p)]),
        "trisk_mesh_set_centers": (C.c_int, [_p, _p]),
        "trisk_icon_create": (C.c_int, [_p, _i32, C.POINTER(_p)]),
        "trisk_icon_destroy": (None, [_p]),
        "trisk_icon_tendency": (C.c_int, [_p, _p, _p]),
        "trisk_icon_rk4_step": (C.c_int, [_p, _p, _f64, _i64]),
        "trisk_icon_launch_count": (_i64, [_p]),
        "trisk_mpas_create": (C.c_int, [_p, _i32, _i32, C.POINTER(_p)]),
        "trisk_mpas_destroy": (None, [_p]),
        "trisk_mpas_slow_tendencies": (C.c_int, [_p, _p, _f64]),
        "trisk_mpas_slow_tendencies_async": (C.c_int, [_p, _p, _f64]),
        "trisk_mpas_stream": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_mpas_synchronize": (C.c_int, [_p]),
        "trisk_mpas_launch_count": (_i64, [_p]),
        "trisk_icosahedral_mesh": (C.c_int, [_i32, _i32, _f64, _p, _p]),
        "trisk_lloyd": (C.c_int, [_p, _i64, _p, _i64, _i32, _i32, C.POINTER(_i32)]),
        "trisk_mesh_destroy": (None, [_p]),
        "trisk_mesh_plex": (C.c_int, [_p, C.POINTER(TriskPlex)]),
        "trisk_mesh_generators": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_mesh_grid": (C.c_int, [_p, C.POINTER(TriskGrid)]),
        "trisk_mesh_hilbert_permutation": (C.c_int, [_p, _p]),
        "trisk_mesh_orthogonality_defect": (C.c_int, [_p, C.POINTER(_f64)]),
        "trisk_mesh_vertex_edge_areas": (C.c_int, [_p, _p, _p]),
        "trisk_mesh_gassmann": (C.c_int, [_p, _p, _p, _p]),
        "trisk_model_create": (C.c_int, [C.POINTER(TriskGrid), C.POINTER(TriskConfig), C.POINTER(_p)]),
        "trisk_model_create_from_coefficients": (C.c_int, [C.POINTER(TriskCoefficients), C.POINTER(TriskConfig),
                                                           C.POINTER(_p)]),
        "trisk_model_destroy": (None, [_p]),
        "trisk_tables_create": (C.c_int, [C.POINTER(TriskGrid), C.POINTER(TriskConfig), C.POINTER(_p)]),
        "trisk_tables_view": (C.c_int, [_p, C.POINTER(TriskCoefficients)]),
        "trisk_tables_destroy": (None, [_p]),
        "trisk_model_coefficients": (C.c_int, [_p, C.POINTER(TriskCoefficients)]),
        "trisk_model_sizes": (C.c_int, [_p, _p]),
        "trisk_tendency": (C.c_int, [_p, _p, _p]),
        "trisk_rk4_step": (C.c_int, [_p, _p, _f64, _i64]),
        "trisk_rk4_step_async": (C.c_int, [_p, _p, _f64, _i64]),
        "trisk_synchronize": (C.c_int, [_p]),
        "trisk_diagnostics": (C.c_int, [_p, _p, _p, _p, _p]),
        "trisk_relative_vorticity": (C.c_int, [_p, _p, _p]),
        "trisk_model_stream": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_launch_count": (_i64, [_p]),
        "trisk_model_bytes": (C.c_int, [_p, _p]),
        "trisk_profile_phases": (C.c_int, [_p, _p, _f64, _i64, _p]),
        "trisk_weighted_sum_noalloc": (C.c_int, [_p, _p, _i64, _p, _p]),
        "trisk_model_info": (C.c_int, [_p, C.POINTER(_i32), _p, C.POINTER(_f64)]),
        "trisk_closure_create": (C.c_int, [_i32, _p, C.POINTER(_p)]),
        "trisk_closure_destroy": (None, [_p]),
        "trisk_closure_param_count": (_i32, []),
        "trisk_closure_get_params": (C.c_int, [_p, _p]),
        "trisk_closure_set_params": (C.c_int, [_p, _p]),
        "trisk_closure_forward": (C.c_int, [_p, _p, _i64, _p]),
        "trisk_closure_gradients": (C.c_int, [_p, _p, _p, _i64, _p, C.POINTER(C.c_float)]),
        "trisk_closure_adam": (C.c_int, [_p, C.c_float, C.c_float, C.c_float, C.c_float]),
        "trisk_closure_synchronize": (C.c_int, [_p]),
        "trisk_closure_stream": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_closure_expire_wait_once": (C.c_int, [_p, _i64]),
        "trisk_closure_info": (C.c_int, [_p, C.POINTER(_i32), C.POINTER(_i32)]),
        "trisk_ensemble_create": (C.c_int, [_p, _p, _p, _p, _i32, C.POINTER(_p)]),
        "trisk_ensemble_create_precision": (C.c_int, [_p, _p, _p, _p, _i32, _i32, C.POINTER(_p)]),
        "trisk_ensemble_set_block": (C.c_int, [_p, _p]),
        "trisk_ensemble_get_block": (C.c_int, [_p, _p]),
        "trisk_ensemble_autotune": (C.c_int, [_p, _i32, C.POINTER(_f64)]),
        "trisk_ensemble_destroy": (None, [_p]),
        "trisk_ensemble_set_member": (C.c_int, [_p, _i32, _i32, _p]),
        "trisk_ensemble_get_member": (C.c_int, [_p, _i32, _i32, _p]),
        "trisk_ensemble_run_async": (C.c_int, [_p, _i64]),
        "trisk_ensemble_synchronize": (C.c_int, [_p]),
        "trisk_ensemble_steps": (C.c_int, [_p, _p]),
        "trisk_ensemble_reset": (C.c_int, [_p]),
        "trisk_ensemble_stream": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_ensemble_launch_count": (_i64, [_p]),
        "trisk_ensemble_bytes": (C.c_int, [_p, C.POINTER(_f64)]),
        "trisk_ensemble_energy": (C.c_int, [_p, _i32, _p]),
        "trisk_ensemble_set_closure": (C.c_int, [_p, _i32, _p, _p, _p, _i32]),
        "trisk_dist_create": (C.c_int, [C.POINTER(TriskCoefficients), C.POINTER(TriskConfig), C.POINTER(TriskHalo),
                                        C.POINTER(_p)]),
        "trisk_dist_destroy": (None, [_p]),
        "trisk_dist_set_exchange": (C.c_int, [_p, EXCHANGE_FN, _p, _i32]),
        "trisk_dist_tendency": (C.c_int, [_p, _p, _p]),
        "trisk_dist_rk4_step": (C.c_int, [_p, _p, _f64, _i64]),
        "trisk_dist_stream": (C.c_int, [_p, C.POINTER(_p)]),
        "trisk_dist_launch_count": (_i64, [_p]),
        "trisk_ensemble_set_slices": (C.c_int, [_p, _p]),
        "trisk_ensemble_get_slices": (C.c_int, [_p, _p]),
        "trisk_ensemble_set_members_per_thread": (C.c_int, [_p, _i32]),
        "trisk_ensemble_get_members_per_thread": (C.c_int, [_p, C.POINTER(_i32)]),
        "trisk_ensemble_closure_mask": (C.c_int, [_p, _i32, _p]),
        "trisk_ensemble_features": (C.c_int, [_p, _i32, _p, _p, _p]),
        "trisk_ensemble_closure_check": (C.c_int, [_p]),
        "trisk_autotune": (C.c_int, [_p, _p, _f64, _i32, C.POINTER(_f64)]),
        "trisk_model_set_block": (C.c_int, [_p, _p]),
        "trisk_model_set_l2_residency": (C.c_int, [_p, _i64, _i32]),
        "trisk_model_get_l2_residency": (C.c_int, [_p, C.POINTER(_i64), C.POINTER(_i32)]),
        "trisk_l2_info": (C.c_int, [_i32, _p]),
        "trisk_model_set_persistent": (C.c_int, [_p, _i32]),
        "trisk_model_get_persistent": (C.c_int, [_p, C.POINTER(_i32)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for which, cls in enumerate((TriskGrid, TriskCoefficients, TriskConfig, TriskPlex, TriskIconTables,
                                  TriskMpasTables, TriskMpasFields, TriskHalo)):
        if lib.trisk_struct_size(which) != C.sizeof(cls):
            raise ImportError(f"{cls.__name__}: binding size {C.sizeof(cls)} != library size "
                              f"{lib.trisk_struct_size(which)}")
    return lib


lib = _load()

# Names the C ABI exports (include/trisk_b200.h); the CPU test suite checks them.
EXPORTED = tuple(n for n in dir(lib) if n.startswith("trisk_"))


def last_error() -> str:
    buf = C.create_string_buffer(4096)
    lib.trisk_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != TRISK_OK:
        raise TriskError(status, last_error())


def ptr(a) -> int | None:
    """Address of a numpy array, a torch tensor or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")


def view(address: int, shape, dtype) -> np.ndarray:
    """numpy copy of library-owned host memory."""
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype=dtype)
    ctype = {np.float64: C.c_double, np.int64: C.c_int64}[np.dtype(dtype).type]
    buf = (ctype * n).from_address(address)
    return np.ctypeslib.as_array(buf).reshape(shape).copy()
