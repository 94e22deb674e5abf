"""The Williamson-2 driver (the counterpart of the reference's examples/trisk_shallow_water.jl):
its flags, a whole run with the CPU oracle standing in for the GPU model (diagnostics, run
log, checkpoints, VTKHDF output), a resumed run equal to the uninterrupted one bit for bit,
and on the GPU the same run through the library's models."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import run
from dmplex_b200.checkpoint import load_state, read_run_log, save_state
from oracle.oracle import Oracle

from hdf5_spec_reader import read_hdf5


class OracleEngine:
    """The CPU oracle behind the driver's engine interface (test infrastructure)."""

    def __init__(self, grid, cfg):
        self.grid = grid
        self.o = Oracle(d.model_tables(grid, pv_flux=cfg["pv_flux"], kinetic_energy=cfg["kinetic_energy"]))

    def initial_state(self):
        g = self.grid
        u = np.einsum("ij,ij->i", run.velocity(g.edge_points), g.edge_normals)
        return np.ascontiguousarray(np.concatenate([u, run.height(g.centers)]))

    def step(self, y, dt, n):
        self.o.rk4_step(y, dt, n)

    def diagnostics(self, y):
        return {"mass": self.o.total_mass(y), "energy": self.o.total_energy(y),
                "enstrophy": self.o.potential_enstrophy(y)}

    def cell_field(self, y, y0):
        from dmplex_b200.vtkhdf import cell_vorticity
        return "vorticity", cell_vorticity(self.grid, y)


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
    with pytest.raises(ValueError):
        run.parse(["--bogus"])
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
    g = d.TRiSKGrid(run.load_mesh(cfg))
    eng = OracleEngine(g, cfg)
    y = eng.initial_state()
    dt = min(0.2 * np.sqrt(4 * np.pi / g.nc), 0.4 * float(g.dual_lengths.min()))
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


@pytest.mark.gpu
@pytest.mark.parametrize("args", [["hexagon", "3", "--gassmann", "--kinetic=vertex"], ["triangle", "3", "--icon"]])
def test_driver_on_the_gpu(require_gpu, tmp_path, args):
    last = run.main(args + [f"--log={tmp_path / 'run.jsonl'}", f"--checkpoint={tmp_path / 'end.bin'}",
                            f"--vtkhdf={tmp_path / 'out.vtkhdf'}"])
    assert abs(last["mass"]) < 1e-13 and last["h_l2"] < 2e-3
    assert len(read_run_log(str(tmp_path / "run.jsonl"))) == 4
    read_hdf5(str(tmp_path / "out.vtkhdf"))
