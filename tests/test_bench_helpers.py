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


def test_leg_summary_is_compact_and_keeps_errors():
    """The key figures of every leg close the JSON line in a few hundred bytes; a failed leg
    keeps its error there."""
    import json

    import bench
    line = {"value": 1.3e9, "ms_per_step": 0.1238, "timing": {"spread": 0.01},
            "roofline": {"frac": 1.03, "frac_on_implementation_bytes": 0.86, "step_frac": 1.04},
            "e2e": {"value": 4.6e8},
            "ensemble": {"value": 2.38e9, "gpu_seconds_per_simulated_day": 1.2, "frac": 0.41,
                         "fp32_state": {"gpu_seconds_per_simulated_day": 0.98, "frac": 0.3}, "steps": [1] * 50},
            "closure": {"error": "RuntimeError: boom"}, "icon": None}
    s = bench.leg_summary(line)
    assert s["headline"]["k_tend_frac_on_implementation_bytes"] == 0.86
    assert s["ensemble"]["fp32_state_gpu_seconds_per_simulated_day"] == 0.98 and "steps" not in s["ensemble"]
    assert s["closure"] == {"error": "RuntimeError: boom"} and s["icon"] is None
    assert len(json.dumps(s)) < 1500


def test_ensemble_leg_flags(monkeypatch):
    """The ensemble leg runs the configured groups, scheme, precision and autotuner choice;
    the defaults are the batched benchmark's (Gassmann PV flux, vertex kinetic energy, FP64
    and FP32 state, autotuned)."""
    import sys

    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.ensemble_scheme, a.ensemble_state, a.ensemble_no_autotune) == ("gassmann/vertex", "both", False)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--ensemble-groups", "6x128", "--ensemble-scheme", "trisk/cell",
                                      "--ensemble-state", "32", "--ensemble-no-autotune"])
    a = bench.parse()
    assert (a.ensemble_groups, a.ensemble_scheme, a.ensemble_state, a.ensemble_no_autotune) == \
        ("6x128", "trisk/cell", "32", True)
