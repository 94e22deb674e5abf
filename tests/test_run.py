"""The shallow-water driver (the counterpart of the reference's examples/trisk_shallow_water.jl
and examples/trisk_galewsky.jl): its flags, a whole run with the CPU oracle standing in for
the GPU model (diagnostics, run log, checkpoints, VTKHDF output), a resumed run equal to the
uninterrupted one bit for bit, the Galewsky jet's set-up, and on the GPU the same runs through
the library's TRiSK and ICON models."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import run
from dmplex_b200.checkpoint import load_state, read_run_log, save_state
from oracle.oracle import Oracle

from hdf5_spec_reader import read_hdf5


class OracleEngine:
    """The CPU oracle behind the driver's engine interface (test infrastructure)."""

    def __init__(self, grid, cfg, case, dt):
        self.grid, self.case = grid, case
        self.o = Oracle(d.model_tables(grid, gravity=case.gravity, omega=1.0, pv_flux=cfg["pv_flux"],
                                       kinetic_energy=cfg["kinetic_energy"]))

    def initial_state(self):
        return run.edge_and_cell_state(self.grid, self.case)

    def step(self, y, dt, n):
        self.o.rk4_step(y, dt, n)

    def diagnostics(self, y):
        return {"mass": self.o.total_mass(y), "energy": self.o.total_energy(y),
                "enstrophy": self.o.potential_enstrophy(y)}

    def cell_field(self, y, y0):
        from dmplex_b200.vtkhdf import cell_vorticity
        return "vorticity", self.case.vorticity_scale * cell_vorticity(self.grid, y)


def test_parse():
    c = run.parse([])
    assert (c["mesh"], c["resolution"], c["pv_flux"], c["kinetic_energy"], c["icon"]) == ("hexagon", 5, "trisk",
                                                                                          "cell", False)
    c = run.parse(["triangle", "6", "--icon", "--centered-k", "--spring"])
    assert (c["mesh"], c["resolution"], c["icon"], c["kinetic_gradient"], c["spring_beta"]) == (
        "triangle", 6, True, "centered", 1.2)
    c = run.parse(["hexagon", "4", "--gassmann-mean", "--kinetic=0.375", "--scvt", "--spring=1.1", "--every=7"])
    assert (c["pv_flux"], c["kinetic_energy"], c["centroidal"], c["spring_beta"], c["every"]) == (
        "gassmann_mean", 0.375, True, 1.1, 7)
    assert run.parse(["--kinetic=vertex", "--gassmann"])["kinetic_energy"] == "vertex"
    c = run.parse(["--case=galewsky", "hexagon", "7", "2.5", "false", "--gassmann-mean"])
    assert (c["case"], c["resolution"], c["days"], c["perturbed"], c["pv_flux"]) == (
        "galewsky", 7, 2.5, False, "gassmann_mean")
    c = run.parse(["--case=galewsky"])
    assert (c["resolution"], c["days"], c["perturbed"]) == (6, 6.0, True)
    for bad in (["--bogus"], ["--case=unknown"], ["hexagon", "3", "1.0"], ["--case=galewsky", "hexagon", "3", "1",
                                                                            "maybe"]):
        with pytest.raises(ValueError):
            run.parse(bad)
    with pytest.raises(ValueError):
        run.load_mesh(run.parse(["no_such_file.nc"]))


def test_driver_with_the_oracle(tmp_path, capsys):
    args = ["hexagon", "3", "--gassmann", "--kinetic=vertex", f"--log={tmp_path / 'run.jsonl'}",
            f"--checkpoint={tmp_path / 'end.bin'}", f"--vtkhdf={tmp_path / 'out.vtkhdf'}"]
    last = run.main(args, engine=OracleEngine)
    assert abs(last["mass"]) < 1e-13 and abs(last["energy"]) < 1e-6 and last["h_l2"] < 2e-3
    recs = read_run_log(str(tmp_path / "run.jsonl"))
    assert len(recs) == 4 and recs[-1]["step"] == last["step"] and recs[0]["pv_flux"] == "gassmann"
    assert "cells" in capsys.readouterr().out
    y, h = load_state(str(tmp_path / "end.bin"))
    assert h["step"] == last["step"] and h["meta"]["config"]["pv_flux"] == "gassmann"
    root, _ = read_hdf5(str(tmp_path / "out.vtkhdf"))
    assert root["VTKHDF"][1]["CellData"][1]["vorticity"][1].shape == (642,)

    # a run resumed from a checkpoint of the same configuration after 5 steps ends in the
    # same state, bit for bit
    cfg = run.parse(args)
    case = run.make_case(cfg)
    g = d.TRiSKGrid(run.load_mesh(cfg))
    dt, _ = case.steps(g)
    eng = OracleEngine(g, cfg, case, dt)
    y = eng.initial_state()
    eng.step(y, dt, 5)
    save_state(str(tmp_path / "mid.bin"), y, g, step=5, time=5 * dt, meta={"config": run.config_meta(cfg)})
    run.main(["hexagon", "3", "--gassmann", "--kinetic=vertex", f"--resume={tmp_path / 'mid.bin'}",
              f"--checkpoint={tmp_path / 'resumed.bin'}"], engine=OracleEngine)
    z, hz = load_state(str(tmp_path / "resumed.bin"))
    end, _ = load_state(str(tmp_path / "end.bin"))
    assert hz["step"] == h["step"] and np.array_equal(z, end)
    # the checkpoint of another configuration is refused
    with pytest.raises(ValueError, match="another configuration"):
        run.main(["hexagon", "3", f"--resume={tmp_path / 'mid.bin'}"], engine=OracleEngine)


def test_driver_fails_loudly_without_a_gpu():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(d.TriskError):
        run.main(["hexagon", "2"])


def test_galewsky_case():
    """The jet: the balanced height has mean depth 1 and balances the jet up to a truncation
    error that falls with resolution (its tendency against that of the same jet over a flat
    surface: 9 % at level 4, less than half that at level 5); half a day with
    the oracle conserves mass, energy and enstrophy as the scheme does, reported in days."""
    from dmplex_b200.cases import Galewsky
    case = Galewsky(days=0.5, perturbed=False)
    phi = np.linspace(-np.pi / 2, np.pi / 2, 2001)
    h = case.balanced_height(phi)
    assert abs(np.trapezoid(h * np.cos(phi), phi) / 2 - 1) < 1e-6
    assert case.jet(np.array([0.0, np.pi / 4, 1.2]))[0] == 0 and case.jet(np.array([np.pi / 4]))[0] > 0.7 * case.u_max

    def imbalance(level):
        g = d.TRiSKGrid(d.create_hexagon_mesh(level))
        o = Oracle(d.model_tables(g, gravity=case.gravity, omega=1.0))
        y = run.edge_and_cell_state(g, case)
        flat = y.copy()
        flat[g.ne:] = 1.0
        return np.linalg.norm(o.tendency(y)) / np.linalg.norm(o.tendency(flat)), g, y
    r4, g, y = imbalance(4)
    r5, _, _ = imbalance(5)
    assert r4 < 0.15 and r5 < r4 / 2                 # balanced up to a truncation error that converges
    perturbed = run.edge_and_cell_state(g, Galewsky(days=0.5))
    assert 0 < np.abs(perturbed - y).max() <= 120 / 1e4
    last = run.main(["--case=galewsky", "hexagon", "3", "0.5", "--kinetic=vertex"], engine=OracleEngine)
    assert last["day"] == pytest.approx(0.5) and abs(last["mass"]) < 1e-14
    assert abs(last["energy"]) < 1e-5 and abs(last["enstrophy"]) < 1e-2


@pytest.mark.gpu
@pytest.mark.parametrize("args", [["hexagon", "3", "--gassmann", "--kinetic=vertex"], ["triangle", "3", "--icon"],
                                  ["--case=galewsky", "hexagon", "4", "0.5"],
                                  ["--case=galewsky", "triangle", "4", "0.5", "--icon", "--centered-k"]])
def test_driver_on_the_gpu(require_gpu, tmp_path, args):
    last = run.main(args + [f"--log={tmp_path / 'run.jsonl'}", f"--checkpoint={tmp_path / 'end.bin'}",
                            f"--vtkhdf={tmp_path / 'out.vtkhdf'}"])
    assert abs(last["mass"]) < 1e-13
    if "--case=galewsky" not in args:
        # the examples' report rule: every nsteps // 4 steps, plus the last step when that is
        # not a multiple of it (5 records for the 51 steps of triangle 3)
        records = read_run_log(str(tmp_path / "run.jsonl"))
        assert last["h_l2"] < 2e-3
        assert [r["step"] for r in records] == sorted(run.CASES["williamson2"]().reports(last["step"]))
    else:
        assert len(read_run_log(str(tmp_path / "run.jsonl"))) == 1 and last["day"] == pytest.approx(0.5)
    read_hdf5(str(tmp_path / "out.vtkhdf"))
