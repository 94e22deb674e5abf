"""dmplex_b200: the TRiSK C-grid shallow-water hot path of dmplex.jl on NVIDIA B200.

The package is a thin host layer over libtrisk_b200.so (C ABI in include/trisk_b200.h):
mesh generation and table construction in C++, the tendency and the RK4 step as
hand-written sm_100a kernels. Names follow the reference (dmplex.jl); Julia's
mutating ``f!`` functions are ``f`` here.
"""
from ._lib import TriskError
from .ensemble import Ensemble
from .checkpoint import RunLog, load_state, save_state
from .gridfiles import check_plex, hilbert_order, read_grid, read_icon_grid, read_mpas_grid
from .vtkhdf import cell_vorticity, write_vtkhdf
from .mesh import (HexMesh, Plex, PolygonMesh, TRiSKGrid, TriangleMesh, create_hexagon_mesh, create_triangle_mesh,
                   icosahedral_mesh, lloyd, plex_from_polygons)
from .model import (RK4Cache, TRiSKShallowWater, height_dofs, initial_state, model_tables, potential_enstrophy,
                    relative_vorticity, rk4_step, tendency, total_energy, total_mass, velocity_dofs)

__all__ = [
    "TriskError", "Ensemble", "save_state", "load_state", "RunLog", "HexMesh", "Plex", "PolygonMesh", "plex_from_polygons", "check_plex", "hilbert_order", "read_grid",
    "read_icon_grid", "read_mpas_grid", "write_vtkhdf", "cell_vorticity", "TRiSKGrid", "TriangleMesh", "create_triangle_mesh", "create_hexagon_mesh", "icosahedral_mesh", "lloyd", "RK4Cache", "TRiSKShallowWater",
    "height_dofs", "initial_state", "model_tables", "potential_enstrophy", "relative_vorticity", "rk4_step", "tendency",
    "total_energy", "total_mass", "velocity_dofs",
]
