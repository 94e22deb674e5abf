"""Parity of the sm_100a path with the CPU oracle, through the C ABI (libtrisk_b200.so).

Bar: the plain FP64 path matches the oracle to 1e-12 relative L2 per tendency and per RK4
step (the tolerance of the task's target), and, because every per-entity sum keeps the
reference's order and the library is built without FMA contraction, it is in fact
bit-identical; both are asserted. Diagnostics match to 1e-12 relative (their reductions
sum in a different order).
"""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import workloads as w
from conftest import oracle_for, tables, tc2_state, trisk_grid

pytestmark = pytest.mark.gpu

RTOL = 1e-12
SCHEMES = [("trisk", "cell"), ("trisk", "vertex"), ("trisk", "mixed"), ("gassmann", "cell"),
           ("gassmann", "vertex"), ("gassmann_mean", "mixed"), ("gassmann_mean", "vertex")]


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def perturbed_tc2(g, seed=7):
    y = tc2_state(g)
    rng = np.random.default_rng(seed)
    y[:g.ne] += 0.02 * rng.standard_normal(g.ne)
    y[g.ne:] += 0.01 * rng.standard_normal(g.nc)
    return y


@pytest.mark.parametrize("pv,ke", SCHEMES)
@pytest.mark.parametrize("reorder", [True, False])
def test_tendency_parity(require_gpu, pv, ke, reorder):
    n = 4
    g = trisk_grid(n, True)
    m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, reorder=reorder)
    o = oracle_for(n, pv, ke, True)
    y = perturbed_tc2(g)
    dy = np.zeros_like(y)
    d.tendency(dy, y, m)
    ref = o.tendency(y)
    assert rel_l2(dy, ref) <= RTOL
    assert np.array_equal(dy, ref)


@pytest.mark.parametrize("pv,ke", [("trisk", "cell"), ("gassmann", "vertex"), ("gassmann_mean", "mixed")])
def test_rk4_parity_per_step(require_gpu, pv, ke):
    n = 5
    g = trisk_grid(n, True)
    t = tables(n, pv, ke, True, None, **w.si_parameters())
    from oracle.oracle import Oracle
    o = Oracle(t, threads=8)
    m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **w.si_parameters())
    y = w.synthetic_state(g, seed=3)
    ref = y.copy()
    cache = d.RK4Cache(y)
    for _ in range(20):
        d.rk4_step(y, 300.0, d.tendency, cache, m)
        o.rk4_step(ref, 300.0, 1)
        assert rel_l2(y, ref) <= RTOL
    assert np.array_equal(y, ref)


def test_multi_step_call_matches_single_steps(require_gpu):
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex")
    y = perturbed_tc2(g)
    a, b = y.copy(), y.copy()
    d.rk4_step(a, 0.01, d.tendency, d.RK4Cache(a), m, nsteps=10)
    for _ in range(10):
        d.rk4_step(b, 0.01, d.tendency, d.RK4Cache(b), m)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("pv,ke", [("trisk", "cell"), ("gassmann", "vertex"), ("gassmann_mean", "mixed")])
def test_one_launch_rk4_step_bitwise(require_gpu, pv, ke):
    """The one-launch RK4 step (one cooperative launch for all steps of a call, grid barriers
    between the twelve phases of a step) against the oracle and against the twelve-launch
    graph step: bit for bit, and one launch per call besides the state's renumbering."""
    from oracle.oracle import Oracle
    si = w.si_parameters()
    g = trisk_grid(5, True)
    o = Oracle(tables(5, pv, ke, True, None, **si), threads=8)
    graph = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si)
    one = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si)
    one.set_persistent(True)
    assert one.persistent and not graph.persistent
    y = w.synthetic_state(g, seed=4)
    a, b, ref = y.copy(), y.copy(), y.copy()
    before = one.launch_count()
    d.rk4_step(a, 300.0, d.tendency, d.RK4Cache(a), one, nsteps=7)
    assert one.launch_count() - before == 1 + 2
    d.rk4_step(b, 300.0, d.tendency, d.RK4Cache(b), graph, nsteps=7)
    o.rk4_step(ref, 300.0, 7)
    assert np.array_equal(a, b) and np.array_equal(a, ref)
    one.set_persistent(False)  # back to the graph: still the same numbers
    d.rk4_step(a, 300.0, d.tendency, d.RK4Cache(a), one, nsteps=2)
    d.rk4_step(b, 300.0, d.tendency, d.RK4Cache(b), graph, nsteps=2)
    assert np.array_equal(a, b)


def test_one_launch_step_reports_nonfinite(require_gpu):
    g = trisk_grid(3)
    m = d.TRiSKShallowWater(g)
    m.set_persistent(True)
    y = tc2_state(g)
    y[5] = np.nan
    with pytest.raises(d.TriskError) as e:
        d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m, nsteps=3)
    assert e.value.status == 4
    y = tc2_state(g)
    d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m)
    assert np.isfinite(y).all()


@pytest.mark.parametrize("use_graph,use_pdl,block", [(False, False, 256), (True, False, 128), (False, True, 64)])
def test_launch_modes_bitwise(require_gpu, use_graph, use_pdl, block):
    g = trisk_grid(4, True)
    y = perturbed_tc2(g)
    ref = y.copy()
    d.rk4_step(ref, 0.01, d.tendency, d.RK4Cache(ref), d.TRiSKShallowWater(g, pv_flux="trisk"), nsteps=5)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", use_graph=use_graph, use_pdl=use_pdl, block=block)
    d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m, nsteps=5)
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("pv,ke", [("trisk", "cell"), ("gassmann", "mixed")])
def test_diagnostics(require_gpu, pv, ke):
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke)
    o = oracle_for(4, pv, ke, True)
    y = perturbed_tc2(g)
    assert abs(d.total_mass(m, y) - o.total_mass(y)) <= RTOL * abs(o.total_mass(y))
    assert abs(d.total_energy(m, y) - o.total_energy(y)) <= RTOL * abs(o.total_energy(y))
    assert abs(d.potential_enstrophy(m, y) - o.potential_enstrophy(y)) <= RTOL * abs(o.potential_enstrophy(y))
    assert np.array_equal(d.relative_vorticity(m, y), o.relative_vorticity(y))


def test_williamson_tc2_gpu(require_gpu):
    """The reference's TC2 assertions (test/finite_volumes.jl:97-109) through the GPU path."""
    for pv in ("trisk", "gassmann", "gassmann_mean"):
        errors = []
        for n in (3, 4):
            g = trisk_grid(n)
            m = d.TRiSKShallowWater(g, pv_flux=pv)
            y = tc2_state(g)
            y0 = y.copy()
            mass0, energy0 = d.total_mass(m, y), d.total_energy(m, y)
            dt = 0.2 * np.sqrt(4 * np.pi / g.nc)
            d.rk4_step(y, dt, d.tendency, d.RK4Cache(y), m, nsteps=int(np.ceil(1 / dt)))
            assert abs(d.total_mass(m, y) - mass0) < 1e-13
            assert abs(d.total_energy(m, y) - energy0) / energy0 < 1e-8
            dh = (y - y0)[g.ne:]
            errors.append(np.sqrt((g.cell_areas * dh ** 2).sum() / (4 * np.pi)))
        assert errors[0] < 2e-3 and errors[1] < errors[0] / 2.5


def test_device_pointers(require_gpu):
    import torch
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="mixed")
    y = perturbed_tc2(g)
    dy_host = np.zeros_like(y)
    d.tendency(dy_host, y, m)
    yd = torch.from_numpy(y).cuda()
    dyd = torch.zeros_like(yd)
    d.tendency(dyd, yd, m)
    assert np.array_equal(dyd.cpu().numpy(), dy_host)
    a = y.copy()
    d.rk4_step(a, 0.01, d.tendency, d.RK4Cache(a), m, nsteps=3)
    d.rk4_step(yd, 0.01, d.tendency, d.RK4Cache(yd), m, nsteps=3)
    assert np.array_equal(yd.cpu().numpy(), a)
    m.rk4_async(yd, 0.01, 2)
    m.synchronize()
    d.rk4_step(a, 0.01, d.tendency, d.RK4Cache(a), m, nsteps=2)
    assert np.array_equal(yd.cpu().numpy(), a)


def test_device_inputs_ordered_after_default_stream(require_gpu):
    """A device state written on PyTorch's (legacy default) stream just before the call is
    read after that write; an output buffer still being read there is written after it."""
    import torch
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex")
    y = perturbed_tc2(g)
    expect = np.zeros_like(y)
    d.tendency(expect, y, m)
    src = torch.from_numpy(y).cuda()
    yd = torch.zeros_like(src)
    dyd = torch.full_like(src, 7.0)
    torch.cuda.synchronize()
    torch.cuda._sleep(20_000_000)  # keeps the default stream busy for several milliseconds
    yd.copy_(src)
    seen = dyd * 1.0               # queued read of the output buffer's old contents
    d.tendency(dyd, yd, m)
    assert np.array_equal(dyd.cpu().numpy(), expect)
    assert bool((seen == 7.0).all())


def test_nonfinite_state_is_reported(require_gpu):
    g = trisk_grid(3)
    m = d.TRiSKShallowWater(g)
    y = tc2_state(g)
    y[5] = np.nan
    with pytest.raises(d.TriskError) as e:
        d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m)
    assert e.value.status == 4
    y = tc2_state(g)  # the model stays usable
    d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m)
    assert np.isfinite(y).all()


def test_launch_count(require_gpu):
    g = trisk_grid(3)
    m = d.TRiSKShallowWater(g)
    y = tc2_state(g)
    d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m)  # graph capture on the first call
    before = m.launch_count()
    d.rk4_step(y, 0.01, d.tendency, d.RK4Cache(y), m, nsteps=4)
    assert m.launch_count() - before == 4 * 12 + 2  # 3 phases x 4 stages per step + 2 permutations


def test_from_coefficients_matches(require_gpu):
    """A model made from the reference model's own premultiplied arrays gives the same
    results as one built from the grid."""
    g = trisk_grid(4, True)
    t = tables(4, "gassmann", "vertex", True)
    a = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex")
    b = d.TRiSKShallowWater.from_coefficients(t, grid=g, pv_flux="gassmann", kinetic_energy="vertex")
    y = perturbed_tc2(g)
    ya, yb = np.zeros_like(y), np.zeros_like(y)
    d.tendency(ya, y, a)
    d.tendency(yb, y, b)
    assert np.array_equal(ya, yb)


def test_gassmann_pv_modes(require_gpu):
    """Gassmann tables in gassmann_coefficients' own order let the kernel derive the PV
    edges (mode 3); a reordered table (entries 0 and 1 of each block swapped) has no such
    structure, is uploaded explicitly (mode 1) and still matches the oracle bit for bit."""
    from oracle.oracle import Oracle
    g = trisk_grid(4, True)
    t = dict(tables(4, "gassmann", "vertex", True))
    y = perturbed_tc2(g)
    a = d.TRiSKShallowWater.from_coefficients(t, grid=g, pv_flux="gassmann", kinetic_energy="vertex")
    assert a.info()["pv_mode"] == 3
    perm = np.arange(12)
    perm[[0, 1, 6, 7]] = [1, 0, 7, 6]
    for name in ("g_edges", "g_pv_edges", "g_weights"):
        t[name] = np.ascontiguousarray(t[name][:, perm])
    b = d.TRiSKShallowWater.from_coefficients(t, grid=g, pv_flux="gassmann", kinetic_energy="vertex")
    assert b.info()["pv_mode"] == 1
    dy = np.zeros_like(y)
    d.tendency(dy, y, b)
    assert np.array_equal(dy, Oracle(t).tendency(y))


def test_autotune_keeps_results(require_gpu):
    import torch
    g = trisk_grid(5, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex")
    y = perturbed_tc2(g)
    ref = y.copy()
    d.rk4_step(ref, 0.002, d.tendency, d.RK4Cache(ref), m, nsteps=4)
    yd = torch.from_numpy(y).cuda()
    ms = m.autotune(yd, 0.002, 5)
    assert ms > 0 and all(b in (64, 128, 256) for b in m.info()["block"])
    assert np.array_equal(yd.cpu().numpy(), y)  # the autotuner leaves the state alone
    d.rk4_step(yd, 0.002, d.tendency, d.RK4Cache(yd), m, nsteps=4)
    assert np.array_equal(yd.cpu().numpy(), ref)
    # fixed block sizes: same numbers, and bad sizes are rejected
    m.set_block([64, 256, 96])
    assert m.info()["block"] == [64, 256, 96]
    yd = torch.from_numpy(y).cuda()
    d.rk4_step(yd, 0.002, d.tendency, d.RK4Cache(yd), m, nsteps=4)
    assert np.array_equal(yd.cpu().numpy(), ref)
    for bad in ([32, 128, 128], [128, 100, 128], [128, 128, 512]):
        with pytest.raises(d.TriskError):
            m.set_block(bad)


def test_l2_residency_keeps_results(require_gpu):
    """The L2-resident table prefix (evict-last loads, with or without a persisting window)
    changes only where tables are cached: results stay bit-identical."""
    import torch
    from dmplex_b200.model import l2_info
    g = trisk_grid(5, True)
    si = w.si_parameters()
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    y = w.synthetic_state(g, seed=4)
    ref = y.copy()
    d.rk4_step(ref, 300.0, d.tendency, d.RK4Cache(ref), m, nsteps=3)
    info = l2_info(0)
    assert info["l2_bytes"] > 0 and info["max_window_bytes"] >= 0
    for keep, window in ((1 << 20, False), (8 << 20, True), (1 << 40, False)):
        m.set_l2_residency(keep, window)
        got = m.info()
        assert 0 < got["l2_resident_table_bytes"] <= keep and got["l2_window"] == window
        yd = torch.from_numpy(y).cuda()
        d.rk4_step(yd, 300.0, d.tendency, d.RK4Cache(yd), m, nsteps=3)
        assert np.array_equal(yd.cpu().numpy(), ref)
    m.set_l2_residency(0)
    assert m.info()["l2_resident_table_bytes"] == 0
    with pytest.raises(d.TriskError):
        m.set_l2_residency(-1)


@pytest.mark.slow
def test_config_level7_gassmann_vertex(require_gpu):
    """The drop-in configuration at full size (hexagon 7, Gassmann PV flux, vertex kinetic
    energy, dt = 75 s): bit parity with the oracle for 3 steps, then mass conservation to
    round-off over 200 steps."""
    from oracle.oracle import Oracle
    g = d.TRiSKGrid(d.create_hexagon_mesh(7, centroidal=True))
    si = w.si_parameters()
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    o = Oracle(d.model_tables(g, pv_flux="gassmann", kinetic_energy="vertex", **si), threads=8)
    y = w.synthetic_state(g, seed=11)
    ref = y.copy()
    for _ in range(3):
        d.rk4_step(y, 75.0, d.tendency, d.RK4Cache(y), m)
        o.rk4_step(ref, 75.0, 1)
        assert rel_l2(y, ref) <= RTOL
    assert np.array_equal(y, ref)
    mass0 = d.total_mass(m, y)
    d.rk4_step(y, 75.0, d.tendency, d.RK4Cache(y), m, nsteps=200)
    assert abs(d.total_mass(m, y) - mass0) / mass0 < 1e-14
