"""Host-side helpers of bench.py and the byte model of the MPAS-Gassmann roofline, on CPU."""
import dmplex_b200 as d
from dmplex_b200 import mpas


def test_optional_leg_reports_errors():
    import bench

    def fails():
        raise RuntimeError("boom")
    assert bench.optional_leg(lambda x: x + 1, 1) == 2
    assert bench.optional_leg(fails) == {"error": "RuntimeError: boom"}


def test_mpas_algorithmic_bytes():
    """The byte model is affine in the number of layers, and no smaller than reading the
    state once and writing every output once."""
    g = d.TRiSKGrid(d.create_hexagon_mesh(2))

    def count(nl, **kw):
        return mpas.algorithmic_bytes(mpas.mpas_tables(g, mpas.vertical_grid(nl, 10000.0), **kw))
    for kw in ({}, {"kinetic_energy": "mixed", "pv_flux": "trisk", "vertical_advection": "advective",
                    "vertical_solver": "tridiagonal"}):
        b4, b8, b12 = count(4, **kw), count(8, **kw), count(12, **kw)
        assert b12 - b8 == b8 - b4 > 0
        nc, ne, nv = g.nc, g.ne, g.nv
        state = ne + 2 * nc + nc                        # vn, rho, rho theta, w
        outputs = 3 * nc + 3 * nv + 3 * ne + ne + nc     # theta pi K, q_v zeta_v rho_v, q_e rho_e F_s, t_vn, t_w
        assert (b8 - b4) / 4 >= 8 * (state + outputs)
