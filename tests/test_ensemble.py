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


@pytest.mark.parametrize("pv,ke,slices", [("trisk", "cell", None), ("gassmann", "vertex", None),
                                          ("gassmann_mean", "mixed", None), ("trisk", "cell", [2, 1, 2]),
                                          ("gassmann", "vertex", [3, 2, 1])])
def test_ensemble_matches_single_models(require_gpu, pv, ke, slices):
    """Every member of three groups of uneven meshes and step counts equals the single-model
    RK4 step bit for bit, with the default slicing and with groups split into slices of one to
    three members (launch sets of several slices, odd and even slice sizes)."""
    si = w.si_parameters()
    levels, members, nsteps = (3, 4, 5), (5, 3, 2), (7, 5, 3)
    grids = [trisk_grid(n, True) for n in levels]
    models = [d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si) for g in grids]
    dts = [w.courant_dt(g) for g in grids]
    ens = d.Ensemble([(m, k, dt, s) for m, k, dt, s in zip(models, members, dts, nsteps)])
    if slices:
        ens.set_slices(slices)
        assert ens.slices() == slices
    states = [member_states(g, k, seed) for g, k, seed in zip(grids, members, (1, 2, 3))]
    for gi, group in enumerate(states):
        for k, y in enumerate(group):
            ens.set_member(gi, k, y)
    for gi, group in enumerate(states):  # set/get round trip before stepping
        for k, y in enumerate(group):
            assert np.array_equal(ens.get_member(gi, k), y)
    ens.run(2)
    if slices:  # re-slicing in the middle of a run keeps every member's state
        ens.set_slices([1, 3, 1])
    ens.run(max(nsteps))
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
    ens.run(3)  # one step is left: one replay of 12 phase launches and the counter update
    assert ens.launch_count() - before == 13
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


@pytest.mark.parametrize("pv,ke", [("trisk", "cell"), ("gassmann", "vertex")])
def test_fp32_state_ensemble(require_gpu, pv, ke):
    """FP32 storage of state and work vectors (FP64 arithmetic and tables): set/get round to
    float exactly, 20 steps stay within float rounding of the FP64 ensemble, mass is
    conserved to float rounding, and a non-finite member is still reported."""
    si = w.si_parameters()
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si)
    dt = w.courant_dt(g)
    states = member_states(g, 3, 11)
    e64 = d.Ensemble([(m, 3, dt, 20)])
    e32 = d.Ensemble([(m, 3, dt, 20)], state_bits=32)
    for k, y in enumerate(states):
        e64.set_member(0, k, y)
        e32.set_member(0, k, y)
        assert np.array_equal(e32.get_member(0, k), y.astype(np.float32).astype(np.float64))
    e64.run(20)
    e32.run(20)
    ne = g.ne
    for k in range(3):
        a, b = e64.get_member(0, k), e32.get_member(0, k)
        assert np.isfinite(b).all()
        assert np.linalg.norm(b[ne:] - a[ne:]) <= 1e-6 * np.linalg.norm(a[ne:])
        assert np.linalg.norm(b[:ne] - a[:ne]) <= 1e-4 * np.linalg.norm(a[:ne])
        mass_a, mass_b = g.cell_areas @ a[ne:], g.cell_areas @ b[ne:]
        assert abs(mass_b - mass_a) <= 1e-7 * abs(mass_a)
    energy = e32.energy(0)
    assert np.all(np.abs(energy - e64.energy(0)) <= 1e-5 * np.abs(energy))
    bad = states[0].copy()
    bad[5] = np.nan
    e32.reset()
    e32.set_member(0, 2, bad)
    with pytest.raises(d.TriskError) as err:
        e32.run(1)
    assert err.value.status == 4


@pytest.mark.parametrize("state_bits", [64, 32])
def test_closure_two_members_per_thread(require_gpu, state_bits):
    """The closure path with two and four members per thread (an even member count) against one
    member per thread (an odd count): the network is row-wise, so every member is
    bit-identical."""
    from dmplex_b200.closure import ClosureMLP
    from dmplex_b200.coarsen import edge_geometry
    si = w.si_parameters()
    g = trisk_grid(3, True)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    states = member_states(g, 5, 13)
    net = ClosureMLP(seed=3)
    u = np.abs(states[0][:g.ne]).mean()
    norm = np.concatenate([np.zeros(24), np.ones(24), [1e-3 * u, 1e-3 * u / 3600]])
    out = {}
    for M, mpt in ((4, 2), (4, 4), (5, 2)):
        ens = d.Ensemble([(m, M, 150.0, 6)], state_bits=state_bits)
        ens.set_members_per_thread(mpt)
        for k in range(M):
            ens.set_member(0, k, states[k])
        ens.set_closure(0, net, edge_geometry(g), norm)
        ens.run(6)
        ens.closure_check()
        out[M, mpt] = [ens.get_member(0, k) for k in range(4)]
    plain = d.Ensemble([(m, 4, 150.0, 6)], state_bits=state_bits)
    for k in range(4):
        plain.set_member(0, k, states[k])
    plain.run(6)
    for k in range(4):
        assert np.array_equal(out[4, 2][k], out[5, 2][k]), k
        assert np.array_equal(out[4, 4][k], out[5, 2][k]), k
        assert not np.array_equal(out[4, 2][k], plain.get_member(0, k))


def test_ensemble_autotune_keeps_results(require_gpu):
    """The batched path's autotuner times block-size combinations on the members' own states
    and restores them (states, step counters, step counts): the run afterwards is bit for
    bit the run without it, and other block sizes give the same numbers too."""
    si = w.si_parameters()
    grids = [trisk_grid(n, True) for n in (3, 4)]
    models = [d.TRiSKShallowWater(g, pv_flux="gassmann", kinetic_energy="vertex", **si) for g in grids]
    dts = [w.courant_dt(g) for g in grids]
    states = [member_states(g, k, s) for g, k, s in zip(grids, (4, 3), (21, 22))]

    def fresh():
        ens = d.Ensemble([(m, k, dt, 4) for m, k, dt in zip(models, (4, 3), dts)])
        for gi, group in enumerate(states):
            for k, y in enumerate(group):
                ens.set_member(gi, k, y)
        return ens

    ref = fresh()
    ref.run(2)
    tuned = fresh()
    tuned.run(2)
    ms = tuned.autotune(3)
    assert ms > 0 and all(b in (64, 128, 256) for b in tuned.block())
    assert tuned.steps_taken() == [2, 2]
    ref.run(3)
    tuned.run(3)
    assert tuned.steps_taken() == [4, 4]
    for gi, group in enumerate(states):
        for k in range(len(group)):
            assert np.array_equal(tuned.get_member(gi, k), ref.get_member(gi, k)), (gi, k)
    other = fresh()
    other.set_block([64, 256, 96])
    other.run(4)
    for gi, group in enumerate(states):
        for k in range(len(group)):
            assert np.array_equal(other.get_member(gi, k), ref.get_member(gi, k)), (gi, k)
    with pytest.raises(d.TriskError):
        other.set_block([32, 128, 128])


@pytest.mark.parametrize("work_free", [False, True])
def test_closure_energy_monitor_is_deterministic(require_gpu, work_free):
    """The per-member energies that drive the closure's fallback, and the work-free projection's
    per-member sums, are reduced in a fixed order (per-block partials, then one fixed-order
    sum per member): two runs of the same closure ensemble give bit-identical energies after
    every check, the same fallback decisions and bit-identical states."""
    from dmplex_b200.closure import ClosureMLP
    from dmplex_b200.coarsen import edge_geometry
    si = w.si_parameters()
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    M = 6
    states = member_states(g, M, 31)
    net = ClosureMLP(seed=5)
    u = np.abs(states[0][:g.ne]).mean()
    norm = np.concatenate([np.zeros(24), np.ones(24), [1e-2 * u, 1e-2 * u / 3600]])

    def run():
        ens = d.Ensemble([(m, M, 150.0, 40)])
        for k in range(M):
            ens.set_member(0, k, states[k])
        ens.set_closure(0, net, edge_geometry(g), norm, work_free=work_free)
        on = np.ones(M, dtype=np.float32)
        e0 = ens.energy(0)
        energies, masks = [e0], []
        for check in range(4):
            ens.run(10)
            e = ens.energy(0)
            energies.append(e)
            if check == 0:  # the members drifting more than the median fall back to the plain step
                drift = np.abs(e - e0) / np.abs(e0)
                on[drift > np.median(drift)] = 0.0
                ens.closure_mask(0, on)
            masks.append(on.copy())
        ens.closure_check()
        return energies, masks, [ens.get_member(0, k) for k in range(M)]

    e1, m1, y1 = run()
    e2, m2, y2 = run()
    for a, b in zip(e1, e2):
        assert np.array_equal(a, b)
    for a, b in zip(m1, m2):
        assert np.array_equal(a, b)
    assert 0 < m1[-1].sum() < M
    for a, b in zip(y1, y2):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("state_bits", [64, 32])
def test_fused_closure_kernel_equals_three_launches(require_gpu, state_bits):
    """The fused closure kernel (features built in shared memory, the network on the tensor
    cores, the corrections written from registers) against features, network and corrections
    as three launches through device memory: every member bit for bit after several steps, at
    one network call per step and at every stage."""
    from dmplex_b200.closure import ClosureMLP
    from dmplex_b200.coarsen import edge_geometry
    si = w.si_parameters()
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    M = 6
    states = member_states(g, M, 41)
    net = ClosureMLP(seed=8)
    u = np.abs(states[0][:g.ne]).mean()
    norm = np.concatenate([np.zeros(24), np.ones(24), [1e-3 * u, 1e-3 * u / 3600]])
    for every_stage in (False, True):
        out = []
        for fused in (True, False):
            ens = d.Ensemble([(m, M, 150.0, 5)], state_bits=state_bits)
            for k, y in enumerate(states):
                ens.set_member(0, k, y)
            ens.set_closure(0, net, edge_geometry(g), norm, every_stage=every_stage, fused=fused)
            ens.run(5)
            ens.closure_check()
            out.append([ens.get_member(0, k) for k in range(M)])
        for a, b in zip(*out):
            assert np.array_equal(a, b)


def test_closure_network_interval(require_gpu):
    """The network every n steps with its corrections kept between: a network of constant
    output gives the every-step run bit for bit; a real network gives the every-step run on the
    first step and a different one after; a member turned off loses its kept corrections at
    once and then follows the plain step bit for bit; the interval needs the one-kernel form at
    stage 1."""
    from oracle import closure_oracle as co
    from dmplex_b200.closure import ClosureMLP
    from dmplex_b200.coarsen import edge_geometry
    si = w.si_parameters()
    g = trisk_grid(4, True)
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", **si)
    M = 4
    states = member_states(g, M, 51)
    u = np.abs(states[0][:g.ne]).mean()
    norm = np.concatenate([np.zeros(24), np.ones(24), [1e-3 * u, 1e-3 * u / 3600]])

    def run(net, every, steps, off_after=None):
        ens = d.Ensemble([(m, M, 150.0, 50)], state_bits=64)
        for k, y in enumerate(states):
            ens.set_member(0, k, y)
        ens.set_closure(0, net, edge_geometry(g), norm, every=every)
        if off_after is None:
            ens.run(steps)
        else:
            ens.run(off_after)
            ens.closure_mask(0, np.array([0, 1, 1, 1], dtype=np.float32))
            mid = ens.get_member(0, 0)
            ens.run(steps - off_after)
            return [ens.get_member(0, k) for k in range(M)], mid
        ens.closure_check()
        return [ens.get_member(0, k) for k in range(M)]

    p = co.init_params(3)
    blocks = {}
    k = 0
    for name, shape in co.SHAPES:
        n = int(np.prod(shape))
        blocks[name] = slice(k, k + n)
        k += n
    const = p.copy()
    const[blocks["W3"]] = 0.0
    const[blocks["b3"]] = [0.7, -0.4]
    const_net = ClosureMLP(const.astype(np.float32))
    for a, b in zip(run(const_net, 1, 5), run(const_net, 3, 5)):
        assert np.array_equal(a, b)
    net = ClosureMLP(seed=9)
    one, three = run(net, 1, 1), run(net, 3, 1)
    for a, b in zip(one, three):
        assert np.array_equal(a, b)
    one, three = run(net, 1, 4), run(net, 3, 4)
    assert not all(np.array_equal(a, b) for a, b in zip(one, three))
    after, mid = run(net, 4, 3, off_after=1)  # member 0 off after the first (network) step
    ref = mid.copy()
    d.rk4_step(ref, 150.0, d.tendency, d.RK4Cache(ref), m, nsteps=2)
    assert np.array_equal(after[0], ref)
    # new states mid-interval: the network runs on the next step (as on a fresh ensemble's first)
    fresh = member_states(g, M, 52)
    ens = d.Ensemble([(m, M, 150.0, 50)], state_bits=64)
    for k, y in enumerate(states):
        ens.set_member(0, k, y)
    ens.set_closure(0, net, edge_geometry(g), norm, every=4)
    ens.run(2)
    for k, y in enumerate(fresh):
        ens.set_member(0, k, y)
    ens.run(1)
    ref = d.Ensemble([(m, M, 150.0, 50)], state_bits=64)
    for k, y in enumerate(fresh):
        ref.set_member(0, k, y)
    ref.set_closure(0, net, edge_geometry(g), norm, every=4)
    ref.run(1)
    for k in range(M):
        assert np.array_equal(ens.get_member(0, k), ref.get_member(0, k)), k
    ens = d.Ensemble([(m, M, 150.0, 5)])
    with pytest.raises(d.TriskError) as e:
        ens.set_closure(0, net, edge_geometry(g), norm, every=2, fused=False)
    assert e.value.status == 6
    with pytest.raises(d.TriskError) as e:
        ens.set_closure(0, net, edge_geometry(g), norm, every=2, every_stage=True)
    assert e.value.status == 6


@pytest.mark.parametrize("pv,ke,state_bits", [("trisk", "cell", 32), ("gassmann", "vertex", 64),
                                              ("gassmann_mean", "mixed", 32), ("trisk", "vertex", 64)])
def test_four_members_per_thread_bitwise(require_gpu, pv, ke, state_bits):
    """Four members per thread (16-byte FP32 or two 16-byte FP64 vectors per gathered value)
    against the default two: every member bit for bit, with a closure-free group of 8 and one of
    12 members in sliced and whole form; refused while a slice's member count is not a multiple
    of four, and dropped back to two by a slicing that breaks it."""
    si = w.si_parameters()
    levels, members, nsteps = (3, 4), (8, 12), (6, 4)
    grids = [trisk_grid(n, True) for n in levels]
    models = [d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, **si) for g in grids]
    dts = [w.courant_dt(g) for g in grids]
    states = [member_states(g, k, seed) for g, k, seed in zip(grids, members, (7, 8))]
    out = []
    for mpt, slices in ((2, None), (4, None), (4, [4, 8])):
        ens = d.Ensemble([(m, k, dt, s) for m, k, dt, s in zip(models, members, dts, nsteps)],
                         state_bits=state_bits)
        if slices:
            ens.set_slices(slices)
        ens.set_members_per_thread(mpt)
        assert ens.members_per_thread == mpt
        for gi, group in enumerate(states):
            for k, y in enumerate(group):
                ens.set_member(gi, k, y)
        ens.run(max(nsteps))
        assert ens.steps_taken() == list(nsteps)
        out.append([[ens.get_member(gi, k) for k in range(len(group))] for gi, group in enumerate(states)])
        if slices:
            ens.set_slices([2, 6])  # 2 is not a multiple of four: back to two per thread
            assert ens.members_per_thread == 2
    for other in out[1:]:
        for ga, gb in zip(out[0], other):
            for a, b in zip(ga, gb):
                assert np.array_equal(a, b)
    odd = d.Ensemble([(models[0], 6, dts[0], 2)])
    with pytest.raises(d.TriskError) as e:
        odd.set_members_per_thread(4)
    assert e.value.status == 6
    # the default: four per thread for FP32 state where the groups allow it, else two
    assert d.Ensemble([(models[0], 8, dts[0], 2)], state_bits=32).members_per_thread == 4
    assert d.Ensemble([(models[0], 8, dts[0], 2)], state_bits=64).members_per_thread == 2
    assert d.Ensemble([(models[0], 6, dts[0], 2)], state_bits=32).members_per_thread == 2
