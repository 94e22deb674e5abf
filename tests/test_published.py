"""The oracle against the figures the reference publishes for this path (docs/STATUS.md), beyond
its test suite: the kinetic-energy error of a solid-body rotation for the cell and vertex forms
on plain, spring-dynamics and centroidal hexagon meshes (:95-96), the TRiSK tangential
reconstruction error on the three meshes (:61-62), and Williamson test case 2 at t = 1 — max
and L2 height errors on spring hexagons for the cell, mixed and vertex kinetic energy
(:96-98) and the L2 error on centroidal hexagons (:63-64); for the ICON model, the mesh
asymmetry and TC2 error on bisection and spring triangles (:40-55). Each published figure is checked to
its significant digits as printed: ours must round to it, within half a unit of its last digit
plus 1 % for the rounding of the geometry. These pin the mesh generators, the TRiSK tables,
the kinetic-energy forms and the time stepping together; the GPU path equals the oracle bit
for bit."""
import functools
import os

import numpy as np
import pytest

import dmplex_b200 as d
from oracle.oracle import Oracle

MESHES = {"plain": {}, "spring": {"spring_beta": 1.2}, "scvt": {"centroidal": True}}


@functools.lru_cache(maxsize=None)
def grid(kind, n):
    return d.TRiSKGrid(d.create_hexagon_mesh(n, **MESHES[kind]))


def close(ours, published: str):
    """ours rounds to the figure `published` as printed (its significant digits), with 1 %
    more for the rounding of the geometry."""
    mantissa = published.lower().split("e")[0].replace("-", "").replace(".", "").lstrip("0")
    value = float(published)
    unit = 10.0 ** (np.floor(np.log10(abs(value))) - max(len(mantissa), 1) + 1)
    return abs(ours - value) <= 0.5 * unit + 0.01 * abs(value)


# K error of a solid-body rotation (max |K_i - |u(x_i)|^2/2| / max |u|^2/2), in %
K_ERROR = {("spring", "cell"): ("1.5", "1.4", "1.25"), ("scvt", "cell"): ("2.0", "2.0", "2.0"),
           ("plain", "cell"): ("5.8", "5.8", "5.8"), ("spring", "vertex"): ("0.60", "0.27", "0.13"),
           ("scvt", "vertex"): ("0.50", "0.21", "0.09"), ("plain", "vertex"): ("0.71", "0.33", "0.16")}


@pytest.mark.parametrize("kind,form", sorted(K_ERROR))
def test_kinetic_energy_error(kind, form):
    w = np.array([0.0, 0.0, 1.0])
    for n, published in zip((4, 5, 6), K_ERROR[kind, form]):
        g = grid(kind, n)
        u = np.einsum("ij,ij->i", np.cross(w, g.edge_points), g.edge_normals)
        K = Oracle(d.model_tables(g, kinetic_energy=form)).kinetic_energy(np.concatenate([u, np.ones(g.nc)]))
        exact = 0.5 * np.sum(np.cross(w, g.centers) ** 2, axis=1)
        ours = 100 * np.abs(K[:g.nc] - exact).max() / exact.max()
        assert close(ours, published), (kind, form, n, ours, published)


def test_tangential_error_on_the_three_meshes():
    """max |v_TRiSK - v| for the solid-body rotation about the axis, levels 5 and 6: spring
    0.014 / 0.016, SCVT 0.0071 / 0.0072; plain "0.11" there (0.118 here, which another line of
    the same document, :25-26, gives as 0.12 for levels 3-6)."""
    w = np.array([0.0, 0.0, 1.0])
    published = {"spring": ("0.014", "0.016"), "scvt": ("0.0071", "0.0072"), "plain": ("0.11", "0.11")}
    for kind, values in published.items():
        for n, pub in zip((5, 6), values):
            g = grid(kind, n)
            solid = np.einsum("ij,ij->i", np.cross(w, g.edge_points), g.edge_normals)
            tang = np.einsum("ij,ij->i", np.cross(w, g.edge_points), np.cross(g.edge_points, g.edge_normals))
            ours = np.abs(Oracle(d.model_tables(g)).tangential_velocity(solid) - tang).max()
            if kind == "plain":
                assert 0.11 <= ours < 0.125
            else:
                assert close(ours, pub), (kind, n, ours, pub)


def tc2_errors(g, form):
    """(max, L2) height error of Williamson case 2 at t = 1 with the example's dt."""
    u0 = 0.2
    x = g.edge_points
    u = u0 * np.einsum("ij,ij->i", np.stack([-x[:, 1], x[:, 0], np.zeros(len(x))], axis=1), g.edge_normals)
    y = np.concatenate([u, 1 - (u0 + u0 ** 2 / 2) * g.centers[:, 2] ** 2])
    y0 = y.copy()
    o = Oracle(d.model_tables(g, kinetic_energy=form), threads=os.cpu_count() or 1)
    dt = min(0.2 * np.sqrt(4 * np.pi / g.nc), 0.4 * float(g.dual_lengths.min()))
    o.rk4_step(y, dt, int(np.ceil(1 / dt)))
    dh = (y - y0)[g.ne:]
    return np.abs(dh).max(), np.sqrt(np.sum(g.cell_areas * dh ** 2) / (4 * np.pi))


# spring hexagons 4/5/6: max errors per K form, L2 for cell and vertex
TC2_SPRING_MAX = {"cell": ("4.9e-4", "3.2e-4", "2.6e-4"), "mixed": ("2.6e-4", "1.4e-4", "1.0e-4"),
                  "vertex": ("1.75e-4", "7.2e-5", "3.8e-5")}
TC2_SPRING_L2 = {"cell": ("1.4e-4", "3.9e-5", "1.2e-5"), "vertex": ("9.0e-5", "2.2e-5", "5.7e-6")}


@pytest.mark.parametrize("form", ["cell", "mixed", "vertex"])
def test_tc2_on_spring_hexagons(form):
    for i, n in enumerate((4, 5, 6)):
        mx, l2 = tc2_errors(grid("spring", n), form)
        assert close(mx, TC2_SPRING_MAX[form][i]), (form, n, mx)
        if form in TC2_SPRING_L2:
            assert close(l2, TC2_SPRING_L2[form][i]), (form, n, l2)


def test_tc2_on_centroidal_hexagons():
    """L2 1.4e-4 / 4.0e-5 / 1.3e-5 for hexagon 4-6 with the cell K, max 3.5e-4 on hexagon 6."""
    for n, pub in zip((4, 5, 6), ("1.4e-4", "4.0e-5", "1.3e-5")):
        mx, l2 = tc2_errors(grid("scvt", n), "cell")
        assert close(l2, pub), (n, l2)
    assert close(mx, "3.5e-4")


@pytest.mark.slow
def test_level7_figures():
    """Hexagon 7: TC2 L2 5.4e-6 on the centroidal mesh; tangential error 0.018 (spring) and
    0.0073 (SCVT)."""
    mx, l2 = tc2_errors(grid("scvt", 7), "cell")
    assert close(l2, "5.4e-6")
    w = np.array([0.0, 0.0, 1.0])
    for kind, pub in (("spring", "0.018"), ("scvt", "0.0073")):
        g = grid(kind, 7)
        solid = np.einsum("ij,ij->i", np.cross(w, g.edge_points), g.edge_normals)
        tang = np.einsum("ij,ij->i", np.cross(w, g.edge_points), np.cross(g.edge_points, g.edge_normals))
        assert close(np.abs(Oracle(d.model_tables(g)).tangential_velocity(solid) - tang).max(), pub)


# the ICON triangle model (docs/STATUS.md:40-55)
def _triangles(kind, n):
    return d.TRiSKGrid(d.create_triangle_mesh(n, **({"spring_beta": 1.2} if kind == "spring" else {})))


def _asymmetry(g):
    """max |d_l - d_r| / d over the edges: how far the circumcenters sit from symmetric."""
    return (np.abs(g.cell_distances[:, 0] - g.cell_distances[:, 1]) / g.dual_lengths).max()


def _icon_tc2_l2(g):
    from dmplex_b200 import icon
    from oracle.icon_oracle import IconOracleC
    o = IconOracleC(icon.icon_tables(g), threads=os.cpu_count() or 1)
    u0 = 0.2
    x = g.edge_points
    u = u0 * np.einsum("ij,ij->i", np.stack([-x[:, 1], x[:, 0], np.zeros(len(x))], axis=1), g.edge_normals)
    y = np.concatenate([u, 1 - (u0 + u0 ** 2 / 2) * g.centers[:, 2] ** 2])
    y0 = y.copy()
    dt = min(0.2 * np.sqrt(4 * np.pi / g.nc), 0.4 * float(g.dual_lengths.min()))
    o.rk4_step(y, dt, int(np.ceil(1 / dt)))
    dh = (y - y0)[g.ne:]
    return np.sqrt(np.sum(g.cell_areas * dh ** 2) / (4 * np.pi))


def test_icon_on_bisection_and_spring_triangles():
    """Plain bisection keeps max |d_l - d_r|/d = 0.19 at every level; TC2 L2 8.5e-5 on 1280
    cells, 1.9e-5 / 7.0e-6 on triangle 4/5 (convergence stalls); with spring dynamics
    (beta = 1.2) TC2 2.3e-5 / 5.6e-6 on triangle 4/5 (second order)."""
    for n in (3, 4, 5):
        assert close(_asymmetry(_triangles("plain", n)), "0.19")
    for n, pub in ((3, "8.5e-5"), (4, "1.9e-5"), (5, "7.0e-6")):
        assert close(_icon_tc2_l2(_triangles("plain", n)), pub), n
    for n, pub in ((4, "2.3e-5"), (5, "5.6e-6")):
        assert close(_icon_tc2_l2(_triangles("spring", n)), pub), n


@pytest.mark.slow
@pytest.mark.skipif(not os.environ.get("TRISK_LONG_TESTS"), reason="long: set TRISK_LONG_TESTS=1")
def test_icon_level6_and_7_figures():
    """TC2 L2 3.9e-6 (plain) and 1.4e-6 (spring) on triangle 6; spring asymmetry 0.10 / 0.089
    on levels 6 / 7."""
    assert close(_icon_tc2_l2(_triangles("plain", 6)), "3.9e-6")
    g6 = _triangles("spring", 6)
    assert close(_icon_tc2_l2(g6), "1.4e-6")
    assert close(_asymmetry(g6), "0.10") and close(_asymmetry(_triangles("spring", 7)), "0.089")


@pytest.mark.slow
@pytest.mark.skipif(not os.environ.get("TRISK_LONG_TESTS"), reason="long: set TRISK_LONG_TESTS=1")
def test_icon_galewsky_on_bisection_triangles():
    """The Galewsky jet on plain triangle 5 blows up before day 3 with ICON's kinetic-energy
    gradient and stays stable with the centered one (:44-50)."""
    from dmplex_b200 import icon, run
    from dmplex_b200.cases import Galewsky
    from oracle.icon_oracle import IconOracleC
    case = Galewsky(3.0)
    g = _triangles("plain", 5)
    dt, n = case.steps(g)
    for gradient, survives in (("icon", False), ("centered", True)):
        t = icon.icon_tables(g, gravity=case.gravity, kinetic_gradient=gradient)
        t["divergence_damping"] = case.icon_damping(g, dt)
        o = IconOracleC(t, threads=os.cpu_count() or 1)
        y = run.edge_and_cell_state(g, case)
        with np.errstate(all="ignore"):
            o.rk4_step(y, dt, n)
        assert bool(np.isfinite(y).all() and np.abs(y[:g.ne]).max() < 1.0) == survives, gradient


# the same published ICON figures through the library's CUDA path: seconds on a B200, so they
# are default GPU tests (the CPU forms above take minutes and need TRISK_LONG_TESTS)
def _icon_tc2_l2_gpu(g):
    from dmplex_b200 import icon
    m = icon.ICONShallowWater(g)
    u0 = 0.2
    x = g.edge_points
    u = u0 * np.einsum("ij,ij->i", np.stack([-x[:, 1], x[:, 0], np.zeros(len(x))], axis=1), g.edge_normals)
    y = np.concatenate([u, 1 - (u0 + u0 ** 2 / 2) * g.centers[:, 2] ** 2])
    y0 = y.copy()
    dt = min(0.2 * np.sqrt(4 * np.pi / g.nc), 0.4 * float(g.dual_lengths.min()))
    m.rk4_step(y, dt, int(np.ceil(1 / dt)))
    dh = (y - y0)[g.ne:]
    return np.sqrt(np.sum(g.cell_areas * dh ** 2) / (4 * np.pi))


@pytest.mark.gpu
def test_icon_level6_and_7_figures_on_the_gpu(require_gpu):
    """TC2 L2 3.9e-6 (plain) and 1.4e-6 (spring) on triangle 6 through the ICON kernels; spring
    asymmetry 0.10 / 0.089 on levels 6 / 7 (docs/STATUS.md:40-55)."""
    assert close(_icon_tc2_l2_gpu(_triangles("plain", 6)), "3.9e-6")
    g6 = _triangles("spring", 6)
    assert close(_icon_tc2_l2_gpu(g6), "1.4e-6")
    assert close(_asymmetry(g6), "0.10") and close(_asymmetry(_triangles("spring", 7)), "0.089")


@pytest.mark.gpu
def test_icon_galewsky_on_bisection_triangles_on_the_gpu(require_gpu):
    """The published failure mode through the ICON kernels: the Galewsky jet on plain triangle 5
    blows up before day 3 with ICON's kinetic-energy gradient (the library reports the
    non-finite state) and stays stable with the centered one (:44-50)."""
    from dmplex_b200 import icon, run
    from dmplex_b200.cases import Galewsky
    case = Galewsky(3.0)
    g = _triangles("plain", 5)
    dt, n = case.steps(g)
    for gradient, survives in (("icon", False), ("centered", True)):
        m = icon.ICONShallowWater(g, gravity=case.gravity, kinetic_gradient=gradient,
                                  divergence_damping=case.icon_damping(g, dt))
        y = run.edge_and_cell_state(g, case)
        try:
            m.rk4_step(y, dt, n)
            stable = bool(np.isfinite(y).all() and np.abs(y[:g.ne]).max() < 1.0)
        except d.TriskError as err:
            assert err.status == 4
            stable = False
        assert stable == survives, gradient
