"""Pins the CPU oracle to the reference. The reference ships no golden vectors for this
path and cannot run here (no Julia), so the oracle is held to the properties the
reference's own tests assert for TRiSKShallowWater:

    test/finite_volumes.jl:79-110   Williamson test case 2 (energy-conserving
                                    semi-discretization, mass and energy after RK4, L2
                                    error bound, convergence ratio)
    test/finite_volumes.jl:184-229  vertex kinetic energy (conservation, accuracy order)
    test/shallow_water.jl:34-41     RK4 order
"""
import numpy as np
import pytest

from conftest import U0, oracle_for, tc2_state, tc2_velocity, trisk_grid


@pytest.mark.parametrize("pv_flux", ["trisk", "gassmann", "gassmann_mean"])
def test_williamson_tc2(pv_flux):
    errors = []
    for n in (3, 4):
        g = trisk_grid(n)
        o = oracle_for(n, pv_flux)
        y = tc2_state(g)
        y0 = y.copy()
        # the semi-discretization conserves energy (:89-95)
        rng = np.random.default_rng(3)
        z = y + 0.01 * rng.standard_normal(len(y))
        dz = o.tendency(z)
        eps = 1e-6
        dEdt = (o.total_energy(z + eps * dz) - o.total_energy(z - eps * dz)) / (2 * eps)
        assert abs(dEdt) < 1e-8 * np.linalg.norm(dz)
        mass0, energy0 = o.total_mass(y), o.total_energy(y)
        dt = 0.2 * np.sqrt(4 * np.pi / g.nc)
        o.rk4_step(y, dt, int(np.ceil(1 / dt)))
        assert abs(o.total_mass(y) - mass0) < 1e-13
        assert abs(o.total_energy(y) - energy0) / energy0 < 1e-8
        dh = (y - y0)[g.ne:]
        errors.append(np.sqrt((g.cell_areas * dh ** 2).sum() / (4 * np.pi)))
    assert errors[0] < 2e-3
    assert errors[1] < errors[0] / 2.5


def test_vertex_kinetic_energy():
    """test/finite_volumes.jl:201-228 on the spring hexagon mesh of level 4."""
    g = trisk_grid(4, False, 1.2)
    results = []
    for ke in ("cell", "mixed", "vertex"):
        o = oracle_for(4, "trisk", ke, False, 1.2)
        y = tc2_state(g)
        y0 = y.copy()
        rng = np.random.default_rng(3)
        z = y + 0.01 * rng.standard_normal(len(y))
        dz = o.tendency(z)
        eps = 1e-6
        dEdt = (o.total_energy(z + eps * dz) - o.total_energy(z - eps * dz)) / (2 * eps)
        assert abs(dEdt) < 1e-8 * np.linalg.norm(dz)
        K = o.kinetic_energy(y)
        exact = (tc2_velocity(g.centers) ** 2).sum(axis=1) / 2
        kerror = np.abs(K - exact).max() / (U0 ** 2 / 2)
        dt = 0.2 * np.sqrt(4 * np.pi / g.nc)
        o.rk4_step(y, dt, int(np.ceil(1 / dt)))
        results.append((kerror, np.abs((y - y0)[g.ne:]).max()))
    (kc, hc), (km, hm), (kv, hv) = results
    assert kv < kc / 2
    assert hv < hc / 2.5
    assert hv < hm < hc


def test_rk4_order():
    """The RK4 step is fourth order: its local error falls by ~2^5 when dt halves
    (the property test/shallow_water.jl:34-41 checks on an oscillator)."""
    g = trisk_grid(3)
    o = oracle_for(3, "trisk", "cell")
    y0 = tc2_state(g)
    y0[g.ne:] += 0.01 * np.cos(3 * g.centers[:, 0])

    def local_error(dt):
        a = y0.copy()
        o.rk4_step(a, dt, 1)
        b = y0.copy()
        o.rk4_step(b, dt / 2, 2)
        return np.abs(a - b).max()

    e1, e2 = local_error(0.2), local_error(0.1)
    assert 20 < e1 / e2 < 45


def test_oracle_threads_bitwise():
    """The OpenMP oracle (the timed CPU baseline) computes the same numbers as the serial one."""
    g = trisk_grid(4, True)
    for pv, ke in [("trisk", "cell"), ("gassmann", "vertex"), ("gassmann_mean", "mixed")]:
        y = tc2_state(g)
        o1 = oracle_for(4, pv, ke, True, threads=1)
        o8 = oracle_for(4, pv, ke, True, threads=4)
        assert np.array_equal(o1.tendency(y), o8.tendency(y))
        a, b = y.copy(), y.copy()
        o1.rk4_step(a, 0.01, 3)
        o8.rk4_step(b, 0.01, 3)
        assert np.array_equal(a, b)


def test_gassmann_more_accurate_than_trisk():
    """STATUS: Gassmann's reconstruction gives 2-4x smaller TC2 L2 height errors than TRiSK
    on the hexagon mesh (docs/STATUS.md:25-26)."""
    g = trisk_grid(4)
    errs = {}
    for pv in ("trisk", "gassmann"):
        o = oracle_for(4, pv)
        y = tc2_state(g)
        y0 = y.copy()
        dt = 0.2 * np.sqrt(4 * np.pi / g.nc)
        o.rk4_step(y, dt, int(np.ceil(1 / dt)))
        dh = (y - y0)[g.ne:]
        errs[pv] = np.sqrt((g.cell_areas * dh ** 2).sum() / (4 * np.pi))
    assert errs["gassmann"] < errs["trisk"] / 1.5
