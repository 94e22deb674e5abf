"""The horizontal operators of the 3-D MPAS-Gassmann dycore (slow_tendencies! for flat ground).
The CPU oracle is pinned by the reference's own operator test (test/extruded.jl:54-106): the
PV edges of ICON-IAP are symmetric in (e, e'), the PV flux does no work, and the vorticity
term exchanges horizontal and vertical kinetic energy without loss; and by its rest test
(:24-40: a horizontally homogeneous column at rest has no tendency). The GPU kernels match
the oracle bit for bit, except the Exner pressure (CUDA's pow against the C library's, within
4 ulp) and the pressure-gradient part of t_vn that it feeds, held to 1e-12 relative L2. The
oracle's C port (the timed CPU baseline) equals its numpy form bit for bit."""
import functools

import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import mpas
from oracle.mpas_oracle import MpasOracle


@functools.lru_cache(maxsize=None)
def hex_grid(n):
    return d.TRiSKGrid(d.create_hexagon_mesh(n))


def test_pv_edges_symmetric():
    """test/extruded.jl:58-64: the PV usage of i_cori_method = 4 is symmetric in (e, e')."""
    g = hex_grid(2)
    P = mpas.trisk_pv_edges(g)
    T = g.trisk_edges
    for e in range(g.ne):
        for k in range(T.shape[1]):
            if g.trisk_weights[e, k] == 0:
                continue
            ep = T[e, k] - 1
            back = np.flatnonzero(T[ep] - 1 == e)
            assert P[e, k] in P[ep, back]
    assert np.any(P > 0) and np.any((P == 0) & (g.trisk_weights != 0))  # rhombus PV and opposite-edge means


def test_iap_weights_close_to_exact():
    g = hex_grid(3)
    W = mpas.iap_trisk_weights(g)
    n = (g.cell_signs != 0).sum(axis=1)
    used = (n[g.edge_cells[:, 0] - 1] - 1) + (n[g.edge_cells[:, 1] - 1] - 1)
    pad = np.arange(W.shape[1])[None, :] >= used[:, None]
    assert np.all(W[pad] == 0) and np.all(W[~pad] != 0)
    assert np.abs(W - g.trisk_weights).max() < 0.02


def _random_state(g, v, rng, nl):
    ne, nc = g.ne, g.nc
    vn = rng.standard_normal((nl, ne))
    w = rng.standard_normal((nl + 1, nc))
    w[0] = 0
    w[-1] = 0
    rho = 1 + 0.3 * rng.random((nl, nc))
    return vn, w, rho


@pytest.mark.parametrize("pv_flux,vertical_advection", [("iap", "iap"), ("trisk", "vector_invariant")])
def test_oracle_energy_properties(pv_flux, vertical_advection):
    """test/extruded.jl:54-106 with radius 1 and the exact TRiSK weights."""
    g = hex_grid(2)
    nl = 6
    v = mpas.vertical_grid(nl, 10000.0, stretch=3)
    t = mpas.mpas_tables(g, v, radius=1.0, pv_flux=pv_flux, vertical_advection=vertical_advection,
                         trisk_weights="exact")
    o = MpasOracle(t)
    rng = np.random.default_rng(1)
    vn, w, rho = _random_state(g, v, rng, nl)
    Ae = g.primal_lengths * g.dual_lengths
    ew = g.cell_distances / g.dual_lengths[:, None]
    rhoe = ew[:, 0] * rho[:, g.edge_cells[:, 0] - 1] + ew[:, 1] * rho[:, g.edge_cells[:, 1] - 1]
    rhoh = np.zeros((nl + 1, g.nc))
    for j in range(1, nl):
        rhoh[j] = v["wlow"][j] * rho[j - 1] + (1 - v["wlow"][j]) * rho[j]
    K, pi, theta = np.zeros((nl, g.nc)), np.zeros((nl, g.nc)), np.ones((nl, g.nc))
    qv, zv, rv = o.vertex_pv(vn, rho)
    qe = o.edge_pv(qv, zv, rv)
    re, Fs = o.edge_density(vn, rho)
    assert np.array_equal(re, rhoe)
    # the PV flux does no work
    tv = o.vn_tendency(vn, Fs, np.zeros_like(w), rho, theta, pi, K, qe, np.zeros((nl + 1, g.ne)), 1.0)
    work = (Ae[:, None] * (Fs * tv).T) @ v["dz"]
    assert abs(work.sum()) < 1e-12 * (Ae[:, None] * np.abs(Fs * tv).T @ v["dz"]).sum()
    # the vorticity term exchanges horizontal and vertical kinetic energy without loss
    mw = vertical_advection == "iap"
    eta = o.eta(vn, w)
    tw = o.w_tendency_vi(eta, vn, re, K, mw)
    tv = o.vn_tendency(vn, Fs, w, rho, theta, pi, K, np.zeros_like(qe), eta, 1.0)
    a = ((Ae[:, None] * ((rhoe if mw else 1) * vn * tv).T) @ v["dz"]).sum()
    b = ((g.cell_areas[:, None] * ((rhoh if mw else 1) * w * tw).T) @ v["dzh"]).sum()
    assert abs(a + b) < 1e-12 * abs(a)


def _column_state(g, v, nl, rng=None, amplitude=0.0):
    """A stratified column (rho, rho theta from a fixed profile), plus a perturbation."""
    z = v["z_full"]
    rho = np.repeat((1.2 * np.exp(-z / 8000.0))[:, None], g.nc, axis=1)
    theta = np.repeat((290.0 * np.exp(z / 30000.0))[:, None], g.nc, axis=1)
    vn = np.zeros((nl, g.ne))
    w = np.zeros((nl + 1, g.nc))
    if amplitude:
        vn = amplitude * 10 * rng.standard_normal((nl, g.ne))
        w[1:nl] = amplitude * 0.1 * rng.standard_normal((nl - 1, g.nc))
        rho = rho * (1 + amplitude * 0.01 * rng.standard_normal(rho.shape))
        theta = theta * (1 + amplitude * 0.01 * rng.standard_normal(theta.shape))
    return vn, w, rho, rho * theta


def test_oracle_rest_state():
    """A horizontally homogeneous column at rest has no horizontal or vertical tendency
    from these operators (test/extruded.jl:24-40 keeps such a column at rest)."""
    g = hex_grid(2)
    nl = 10
    v = mpas.vertical_grid(nl, 30000.0, stretch=3)
    for kw in (dict(), dict(pv_flux="trisk", vertical_advection="advective", vertical_solver="tridiagonal",
                            kinetic_energy="mixed")):
        o = MpasOracle(mpas.mpas_tables(g, v, **kw))
        out = o.slow_tendencies(*_column_state(g, v, nl))
        assert np.all(out["tvn"] == 0)
        assert np.all(out["tw"] == 0)
        assert np.all(out["K"] == 0)


def test_tables_arguments():
    g = hex_grid(1)
    v = mpas.vertical_grid(4, 1000.0)
    for bad in (dict(pv_flux="x"), dict(vertical_advection="x"), dict(trisk_weights="x"),
                dict(vertical_solver="x"), dict(vertical_advection="advective")):
        with pytest.raises(ValueError):
            mpas.mpas_tables(g, v, **bad)
    with pytest.raises(ValueError):
        mpas.vertical_grid_from_levels([0.0, 1.0, 1.0])
    vg = mpas.vertical_grid(5, 1000.0, stretch=2)
    assert abs(vg["z_half"][-1] - 1000.0) < 1e-9 and abs(vg["dz"][-1] / vg["dz"][0] - 2) < 1e-12


CONFIGS = [
    dict(),                                                                   # ICON-IAP defaults, five-band
    dict(pv_flux="trisk", vertical_advection="vector_invariant", vertical_solver="tridiagonal",
         kinetic_energy="mixed", trisk_weights="exact"),
    dict(pv_flux="iap", vertical_advection="advective", vertical_solver="tridiagonal", kinetic_energy="vertex"),
]


def _gpu_case(cfg, lpt, nl=10, n=4, pressure=1.0, seed=3):
    import torch
    g = hex_grid(n)
    v = mpas.vertical_grid(nl, 30000.0, stretch=3)
    t = mpas.mpas_tables(g, v, **cfg)
    o = MpasOracle(t)
    ops = mpas.MPASOperators(t, levels_per_thread=lpt)
    rng = np.random.default_rng(seed)
    state = _column_state(g, v, nl, rng, amplitude=1.0)
    ref = o.slow_tendencies(*state, pressure=pressure)
    dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in state]
    out = ops.work()
    ops.slow_tendencies(*dev, out=out, pressure=pressure)
    got = {k: x.cpu().numpy() for k, x in out.items()}
    return t, ref, got, ops


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", CONFIGS, ids=["iap", "trisk-vi", "advective"])
@pytest.mark.parametrize("lpt", [8, 1, 16])
def test_gpu_matches_oracle(require_gpu, cfg, lpt):
    t, ref, got, ops = _gpu_case(cfg, lpt)
    exact = ["theta", "K", "qv", "zetav", "rhov", "qe", "rhoe", "Fs", "tw"]
    if t["vertical"] > 0:
        exact.append("eta")
    if ops.vertex_kinetic:
        exact.append("Kv")
    for name in exact:
        assert np.array_equal(got[name], ref[name]), name
    # CUDA's pow is within 2 ulp, the C library's (the oracle's) within about half an ulp
    assert np.all(np.abs(got["exner"] - ref["exner"]) <= 4 * np.spacing(np.abs(ref["exner"])))
    rel = np.linalg.norm(got["tvn"] - ref["tvn"]) / np.linalg.norm(ref["tvn"])
    assert rel <= 1e-12
    assert ops.launch_count() == 5


@pytest.mark.gpu
def test_gpu_without_pressure_is_bitwise(require_gpu):
    """With pressure = 0 (slow_tendencies!(m, ys, 0), the corrector of ICON-IAP) t_vn does
    not read the Exner pressure and equals the oracle bit for bit."""
    t, ref, got, ops = _gpu_case(CONFIGS[0], 8, pressure=0.0)
    assert np.array_equal(got["tvn"], ref["tvn"])


@pytest.mark.gpu
def test_gpu_argument_errors(require_gpu):
    import torch
    g = hex_grid(2)
    nl = 4
    t = mpas.mpas_tables(g, mpas.vertical_grid(nl, 1000.0))
    ops = mpas.MPASOperators(t)
    out = ops.work()
    state = [torch.zeros(s, dtype=torch.float64, device="cuda") for s in
             ((nl, g.ne), (nl + 1, g.nc), (nl, g.nc), (nl, g.nc))]
    with pytest.raises(ValueError):
        ops.slow_tendencies(state[0][:-1], *state[1:], out=out)
    with pytest.raises(TypeError):
        ops.slow_tendencies(state[0].cpu(), *state[1:], out=out)
    with pytest.raises(d.TriskError):
        mpas.MPASOperators(t, levels_per_thread=3)
    bad = dict(t)
    bad["trisk_index"] = t["trisk_index"].copy()
    bad["trisk_index"][0, 0, 0] = g.ne + 5
    with pytest.raises(d.TriskError):
        mpas.MPASOperators(bad)


def test_operators_fail_loudly_without_a_gpu():
    """On a machine without a CUDA device the library refuses to create the operators (no
    CPU fallback)."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    g = hex_grid(1)
    t = mpas.mpas_tables(g, mpas.vertical_grid(4, 1000.0))
    with pytest.raises(d.TriskError, match="CUDA"):
        mpas.MPASOperators(t)


@pytest.mark.parametrize("cfg", CONFIGS, ids=["iap", "trisk-vi", "advective"])
def test_c_oracle_matches_numpy_oracle(cfg):
    from oracle.mpas_oracle import MpasOracleC
    g = hex_grid(3)
    nl = 10
    v = mpas.vertical_grid(nl, 30000.0, stretch=3)
    t = mpas.mpas_tables(g, v, **cfg)
    state = _column_state(g, v, nl, np.random.default_rng(3), amplitude=1.0)
    for pressure in (1.0, 0.0):
        ref = MpasOracle(t).slow_tendencies(*state, pressure=pressure)
        for threads in (1, 4):
            got = MpasOracleC(t, threads=threads).slow_tendencies(*state, pressure=pressure)
            assert sorted(got) == sorted(k for k in ref if k != "Kv" or t.get("vk_weights") is not None)
            for name in got:
                assert np.array_equal(got[name], ref[name]), name
