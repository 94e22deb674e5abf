"""Checkpoint and resume (the reference has none; its state is the flat vector y): a run
stopped, written, read back and continued equals the uninterrupted run bit for bit — with the
CPU oracle here, with the library's model on the GPU — and damaged, foreign or truncated
files are refused. Also the JSON-lines run log."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import checkpoint as ck
from dmplex_b200 import workloads as w
from oracle.oracle import Oracle

from conftest import trisk_grid


def test_resume_is_bitwise_cpu(tmp_path):
    g = trisk_grid(3, True)
    si = w.si_parameters()
    o = Oracle(d.model_tables(g, pv_flux="gassmann", kinetic_energy="vertex", **si))
    y0 = w.synthetic_state(g, seed=7)
    straight = o.rk4_step(y0.copy(), 300.0, 6)
    y = o.rk4_step(y0.copy(), 300.0, 3)
    path = str(tmp_path / "state.bin")
    ck.save_state(path, y, g, step=3, time=900.0, meta={"dt": 300.0})
    z, h = ck.load_state(path, g)
    assert (h["step"], h["time"], h["meta"]["dt"], h["members"]) == (3, 900.0, 300.0, 1)
    assert np.array_equal(z, y)
    resumed = o.rk4_step(z, 300.0, 3)
    assert np.array_equal(resumed, straight)


def test_ensemble_state_and_refusals(tmp_path):
    g = trisk_grid(2, False)
    rng = np.random.default_rng(0)
    Y = rng.standard_normal((4, g.ne + g.nc))
    path = str(tmp_path / "ens.bin")
    ck.save_state(path, Y, g, step=10, kind="ensemble")
    Z, h = ck.load_state(path, g)
    assert Z.shape == (4, g.ne + g.nc) and np.array_equal(Z, Y) and h["kind"] == "ensemble"
    # another mesh, a renumbered mesh
    with pytest.raises(ValueError, match="different mesh"):
        ck.load_state(path, trisk_grid(3, False))
    with pytest.raises(ValueError, match="different mesh"):
        ck.load_state(path, d.TRiSKGrid(d.hilbert_order(d.create_hexagon_mesh(2))))
    raw = bytearray(open(path, "rb").read())
    bad = tmp_path / "bad.bin"
    flipped = bytearray(raw)
    flipped[-20] ^= 0x01                       # a payload bit
    bad.write_bytes(bytes(flipped))
    with pytest.raises(ValueError, match="CRC"):
        ck.load_state(str(bad))
    bad.write_bytes(bytes(raw[:-100]))
    with pytest.raises(ValueError, match="truncated"):
        ck.load_state(str(bad))
    bad.write_bytes(b"not a checkpoint at all")
    with pytest.raises(ValueError, match="not a state checkpoint"):
        ck.load_state(str(bad))
    with pytest.raises(ValueError):
        ck.save_state(path, Y[:, :-1], g)        # wrong state size for a TRiSK state
    with pytest.raises(ValueError):
        ck.save_state(path, Y.astype(np.float32), g, kind="ensemble")
    # nothing but the final file is left behind
    assert sorted(p.name for p in tmp_path.iterdir()) == ["bad.bin", "ens.bin"]


def test_run_log(tmp_path):
    path = str(tmp_path / "run.jsonl")
    with ck.RunLog(path, level=5, pv_flux="trisk") as log:
        log.write(day=0.5, mass=np.float64(1e-16), ms_per_step=0.12)
        log.write(day=1.0, mass=2e-16, ms_per_step=0.11, gbs=6900.0)
    recs = ck.read_run_log(path)
    assert [r["day"] for r in recs] == [0.5, 1.0]
    assert recs[0]["level"] == 5 and recs[1]["gbs"] == 6900.0


@pytest.mark.gpu
def test_resume_is_bitwise_gpu(require_gpu, tmp_path):
    """The library's model: 3 steps, checkpoint, read back into a fresh model, 3 steps ==
    6 steps straight through."""
    g = trisk_grid(4, True)
    si = w.si_parameters()
    y0 = w.synthetic_state(g, seed=8)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    straight = y0.copy()
    d.rk4_step(straight, 300.0, d.tendency, d.RK4Cache(straight), m, nsteps=6)
    y = y0.copy()
    d.rk4_step(y, 300.0, d.tendency, d.RK4Cache(y), m, nsteps=3)
    path = str(tmp_path / "state.bin")
    ck.save_state(path, y, g, step=3)
    del m
    z, _ = ck.load_state(path, g)
    m2 = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    d.rk4_step(z, 300.0, d.tendency, d.RK4Cache(z), m2, nsteps=3)
    assert np.array_equal(z, straight)
