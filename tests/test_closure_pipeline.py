"""The learned closure end to end on small meshes: fine runs coarse-grained, residual
targets with a mass-conserving flux part, tensor-core training, and coarse ensembles with
the closure that conserve mass to round-off; the trained network explains part of the
held-out residual variance (its gain over the method without it)."""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200 import closure_pipeline as cp
from dmplex_b200 import workloads as w
from dmplex_b200.coarsen import divergence_matrix

@pytest.mark.gpu
@pytest.mark.parametrize("tendency_targets", [True, False])
def test_closure_pipeline_small(require_gpu, tendency_targets):
    import torch
    gf, gc = cp._grid(5), cp._grid(3)
    Y0, Y1, delta, _, _ = cp.fine_snapshots(gf, gc, [1, 2, 3, 4, 5, 6], 0.5, 24, dt_fine=60.0, pair_steps=4,
                                            tendency_targets=tendency_targets)
    assert Y0.shape == (gc.ne + gc.nc, Y0.shape[1]) and Y0.shape[1] >= 100
    assert (delta == 0) == tendency_targets
    dF, dQ, mc, ens = cp.residual_targets(gc, Y0, Y1, delta)
    # the flux part reproduces the height residual: -D dF = r_h minus its null-space part
    D = divergence_matrix(d.model_tables(gc, pv_flux="trisk", kinetic_energy="cell", **w.si_parameters()))
    r_h = -(D @ dF.cpu().numpy())
    assert np.isfinite(r_h).all() and np.abs(gc.cell_areas @ r_h).max() < 1e-12 * np.abs(r_h).max() * gc.nc
    X, T, norm = cp.build_dataset(gc, Y0, dF, dQ, ens)
    assert X.shape == (gc.ne * Y0.shape[1], 24) and T.shape == (X.shape[0], 2)
    mlp = cp.ClosureMLP(seed=0)
    history, held, zero = cp.train(mlp, X, T, epochs=4, batch=4096, lr=2e-3)
    # the network explains part of the held-out residual the coarse model leaves
    assert history[-1] < history[0] and held < 0.95 * zero
    # coarse runs with the closure conserve mass to round-off
    init = Y0[:, :3].contiguous()
    m = d.TRiSKShallowWater(gc, pv_flux="trisk", kinetic_energy="cell", **w.si_parameters())
    e = d.Ensemble([(m, 3, 150.0, 40)])
    col = torch.empty(m.state_size, dtype=torch.float64, device=init.device)
    for k in range(3):
        col.copy_(init[:, k])
        e.set_member(0, k, col)
    from dmplex_b200.coarsen import edge_geometry
    e.set_closure(0, mlp, edge_geometry(gc), norm)
    mass0 = [gc.cell_areas @ e.get_member(0, k)[gc.ne:] for k in range(3)]
    e.run(40)
    e.closure_check()
    for k in range(3):
        y = e.get_member(0, k)
        assert np.isfinite(y).all()
        assert abs(gc.cell_areas @ y[gc.ne:] - mass0[k]) <= 1e-13 * abs(mass0[k])
    # and the closure changes the result (it is applied), while a zero mask restores the plain step
    plain = d.Ensemble([(m, 3, 150.0, 40)])
    for k in range(3):
        col.copy_(init[:, k])
        plain.set_member(0, k, col)
    plain.run(40)
    assert not np.array_equal(plain.get_member(0, 0), e.get_member(0, 0))
    masked = d.Ensemble([(m, 3, 150.0, 40)])
    for k in range(3):
        col.copy_(init[:, k])
        masked.set_member(0, k, col)
    masked.set_closure(0, mlp, edge_geometry(gc), norm)
    masked.closure_mask(0, np.zeros(3))
    masked.run(40)
    assert np.array_equal(plain.get_member(0, 1), masked.get_member(0, 1))
    # the work-free option removes the correction's power: over one short step (1 s, so the
    # first-order change dominates) the energy changes far less than with the same
    # (amplified, momentum-only) correction without it
    strong = np.array(norm, dtype=np.float64)
    strong[48], strong[49] = 0.0, 10.0 * strong[49]
    de = {}
    for wf in (False, True, None):
        one = d.Ensemble([(m, 3, 1.0, 1)])
        for k in range(3):
            col.copy_(init[:, k])
            one.set_member(0, k, col)
        if wf is not None:
            one.set_closure(0, mlp, edge_geometry(gc), strong, work_free=wf)
        one.run(1)
        de[wf] = one.energy(0)
    power_free = np.abs(de[True] - de[None])
    power = np.abs(de[False] - de[None])
    assert np.all(power > 0) and np.all(power_free <= 0.05 * power), (power_free, power)


@pytest.mark.gpu
def test_run_coarse_reports_errors(require_gpu):
    gf, gc = cp._grid(4), cp._grid(3)
    _, _, _, daily, secs = cp.fine_snapshots(gf, gc, [7, 8], 2, 0, dt_fine=60.0, spinup_days=0.0, record_days=True)
    assert len(daily) == 3 and secs > 0
    res = cp.run_coarse(gc, daily[0], 2, 300.0, daily)
    assert len(res["h_l2"]) == 2 and all(np.isfinite(res["h_l2"][-1]))
    assert res["h_l2"][1][0] > 0


def test_equal_error_cost_interpolates_log_linearly():
    """The plain method's cost at a target error, log-linear in (error, cost) between two levels:
    exact at the levels, and one level's factor per halving of the error between them."""
    errors, costs = {6: 20.0, 7: 5.0}, {6: 1.0, 7: 8.0}
    assert cp.equal_error_cost(errors, costs, 20.0) == pytest.approx(1.0)
    assert cp.equal_error_cost(errors, costs, 5.0) == pytest.approx(8.0)
    assert cp.equal_error_cost(errors, costs, 10.0) == pytest.approx(8.0 ** 0.5)
    assert np.isnan(cp.equal_error_cost({6: 1.0, 7: 1.0}, costs, 1.0))


@pytest.mark.gpu
def test_plain_level_errors_and_costs(require_gpu):
    """An intermediate level judged on the coarse mesh: its errors against the coarse-grained
    fine run are finite and below the coarse level's, and the cost of a member-day is positive
    and grows with the level."""
    gf, gm, gc = cp._grid(5), cp._grid(4), cp._grid(3)
    _, _, _, daily, _ = cp.fine_snapshots(gf, gc, [7, 8], 1, 0, dt_fine=60.0, spinup_days=0.0, record_days=True)
    coarse = cp.run_coarse(gc, daily[0], 1, 300.0, daily)
    inter = cp.plain_level_errors(gf, gc, gm, [7, 8], 1, 150.0, daily)
    assert np.isfinite(inter["h_l2"]).all() and np.mean(inter["h_l2"][0]) < np.mean(coarse["h_l2"][0])
    c3 = cp.member_day_cost(gc, 8, 300.0, steps=8)
    c4 = cp.member_day_cost(gm, 8, 150.0, steps=8)
    assert 0 < c3 < c4
