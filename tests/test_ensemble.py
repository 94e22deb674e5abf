"""Batched ensembles: every member of every group follows the single-model RK4 step (and so
the oracle) bit for bit, groups stop at their own step counts, and the graph advances all
groups with one set of launches."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import workloads as w
from conftest import tables, trisk_grid

pytestmark = pytest.mark.gpu


def member_states(g, count, seed):
    return w.ensemble_members(g, count, seed, degree=6)


@pytest.mark.parametrize("pv,ke", [("trisk", "cell"), ("gassmann", "vertex"), ("gassmann_mean", "mixed")])
def test_ensemble_matches_single_models(require_gpu, pv, ke):
    si = w.si_parameters()
    levels, members, nsteps = (3, 4, 5), (5, 3, 2), (7, 5, 3)
    grids = [trisk_grid(n, True) for n in levels]
    models = [d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si) for g in grids]
    dts = [w.courant_dt(g) for g in grids]
    ens = d.Ensemble([(m, k, dt, s) for m, k, dt, s in zip(models, members, dts, nsteps)])
    states = [member_states(g, k, seed) for g, k, seed in zip(grids, members, (1, 2, 3))]
    for gi, group in enumerate(states):
        for k, y in enumerate(group):
            ens.set_member(gi, k, y)
    for gi, group in enumerate(states):  # set/get round trip before stepping
        for k, y in enumerate(group):
            assert np.array_equal(ens.get_member(gi, k), y)
    ens.run(max(nsteps) + 2)
    assert ens.steps_taken() == list(nsteps)
    for gi, group in enumerate(states):
        for k, y in enumerate(group):
            ref = y.copy()
            d.rk4_step(ref, dts[gi], d.tendency, d.RK4Cache(ref), models[gi], nsteps=nsteps[gi])
            assert np.array_equal(ens.get_member(gi, k), ref), (gi, k)


def test_ensemble_oracle_parity(require_gpu):
    """One group against the CPU oracle directly (1e-12 relative, and bitwise)."""
    from oracle.oracle import Oracle
    si = w.si_parameters()
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si)
    o = Oracle(tables(4, "gassmann", "vertex", True, None, **si))
    dt = w.courant_dt(g)
    ens = d.Ensemble([(m, 4, dt, 6)])
    states = member_states(g, 4, 9)
    for k, y in enumerate(states):
        ens.set_member(0, k, y)
    ens.run(6)
    for k, y in enumerate(states):
        ref = y.copy()
        o.rk4_step(ref, dt, 6)
        got = ens.get_member(0, k)
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)
        assert np.array_equal(got, ref)


def test_ensemble_reset_and_launches(require_gpu):
    g = trisk_grid(3, True)
    m = d.TRiSKShallowWater(g)
    ens = d.Ensemble([(m, 3, 0.001, 2)])
    for k, y in enumerate(member_states(g, 3, 4)):
        ens.set_member(0, k, y)
    ens.run(1)  # captures the graph
    before = ens.launch_count()
    ens.run(3)
    assert ens.launch_count() - before == 3 * 13
    assert ens.steps_taken() == [2]
    ens.reset()
    assert ens.steps_taken() == [0]


def test_ensemble_member_copies_ordered_after_default_stream(require_gpu):
    import torch
    g = trisk_grid(3, True)
    m = d.TRiSKShallowWater(g)
    ens = d.Ensemble([(m, 2, 0.001, 1)])
    states = member_states(g, 2, 5)
    src = torch.from_numpy(states[1]).cuda()
    col = torch.zeros_like(src)
    torch.cuda.synchronize()
    torch.cuda._sleep(20_000_000)
    col.copy_(src)
    ens.set_member(0, 1, col)                  # reads col after the copy
    assert np.array_equal(ens.get_member(0, 1), states[1])
    ens.set_member(0, 0, states[0])
    out = torch.full_like(src, 3.0)
    torch.cuda._sleep(20_000_000)
    seen = out * 1.0                           # queued read of the old contents
    ens.get_member(0, 0, out)                  # overwrites out after that read
    assert bool((seen == 3.0).all())
    assert np.array_equal(out.cpu().numpy(), states[0])


def test_ensemble_nonfinite_member(require_gpu):
    g = trisk_grid(3, True)
    m = d.TRiSKShallowWater(g)
    ens = d.Ensemble([(m, 2, 0.001, 2)])
    ys = member_states(g, 2, 5)
    ys[1][3] = np.inf
    ens.set_member(0, 0, ys[0])
    ens.set_member(0, 1, ys[1])
    with pytest.raises(d.TriskError) as e:
        ens.run(2)
    assert e.value.status == 4
    ref = ys[0].copy()
    d.rk4_step(ref, 0.001, d.tendency, d.RK4Cache(ref), m, nsteps=2)
    assert np.array_equal(ens.get_member(0, 0), ref)  # the other member is unaffected
