import functools
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


@functools.lru_cache(maxsize=None)
def hexagon_mesh(n: int, centroidal: bool = False, spring_beta=None):
    import dmplex_b200 as d
    return d.create_hexagon_mesh(n, centroidal=centroidal, spring_beta=spring_beta)


@functools.lru_cache(maxsize=None)
def trisk_grid(n: int, centroidal: bool = False, spring_beta=None):
    import dmplex_b200 as d
    return d.TRiSKGrid(hexagon_mesh(n, centroidal, spring_beta))


@functools.lru_cache(maxsize=None)
def tables(n: int, pv_flux="trisk", kinetic_energy="cell", centroidal=False, spring_beta=None, gravity=1.0,
           omega=1.0):
    import dmplex_b200 as d
    return d.model_tables(trisk_grid(n, centroidal, spring_beta), pv_flux=pv_flux, kinetic_energy=kinetic_energy,
                          gravity=gravity, omega=omega)


def oracle_for(n, pv_flux="trisk", kinetic_energy="cell", centroidal=False, spring_beta=None, gravity=1.0,
               threads=1):
    from oracle.oracle import Oracle
    return Oracle(tables(n, pv_flux, kinetic_energy, centroidal, spring_beta, gravity), threads=threads)


# Williamson test case 2 of the reference's tests (test/finite_volumes.jl:80-82)
U0 = 0.2


def tc2_velocity(x):
    x = np.asarray(x)
    return U0 * np.stack([-x[:, 1], x[:, 0], np.zeros(len(x))], axis=1)


def tc2_height(x):
    x = np.asarray(x)
    return 1 - (U0 + U0 ** 2 / 2) * x[:, 2] ** 2


def tc2_state(grid):
    u = np.einsum("ij,ij->i", tc2_velocity(grid.edge_points), grid.edge_normals)
    return np.ascontiguousarray(np.concatenate([u, tc2_height(grid.centers)]))


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not gpu_available():
        pytest.fail("this test needs a CUDA GPU")
