"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py from the CPU oracle):
the mesh generator and the oracle reproduce them exactly on the CPU, and the CUDA path
reproduces them through the C ABI on the GPU — bit for bit, which is stricter than the
1e-12 relative L2 per step the drop-in is held to (also asserted)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import make_golden as mg  # noqa: E402

CASES = [pytest.param(pv, ke, dt, id=f"{pv}-{ke}") for pv, ke, dt in mg.CASES]


def _golden(pv, ke):
    z = np.load(mg.path(pv, ke))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("pv,ke,dt", CASES)
def test_oracle_reproduces_golden(pv, ke, dt):
    g = _golden(pv, ke)
    now = mg.case_data(pv, ke, dt)
    assert np.array_equal(now["mesh"][:3], g["mesh"][:3])
    assert np.allclose(now["mesh"][3:], g["mesh"][3:], rtol=1e-14, atol=0)
    for k in ("y", "dy", "y1"):
        assert np.array_equal(now[k], g[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("pv,ke,dt", CASES)
def test_gpu_reproduces_golden(require_gpu, pv, ke, dt):
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    g = _golden(pv, ke)
    grid = d.TRiSKGrid(d.create_hexagon_mesh(mg.LEVEL, centroidal=True))
    m = d.TRiSKShallowWater(grid, pv_flux=pv, kinetic_energy=ke, **w.si_parameters())
    y = g["y"].copy()
    dy = np.zeros_like(y)
    d.tendency(dy, y, m)
    assert np.linalg.norm(dy - g["dy"]) <= 1e-12 * np.linalg.norm(g["dy"])
    assert np.array_equal(dy, g["dy"])
    d.rk4_step(y, float(g["dt"]), d.tendency, d.RK4Cache(y), m)
    assert np.linalg.norm(y - g["y1"]) <= 1e-12 * np.linalg.norm(g["y1"])
    assert np.array_equal(y, g["y1"])
