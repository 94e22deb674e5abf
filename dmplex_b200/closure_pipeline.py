"""Learned flux closure: training data, training and evaluation (no reference counterpart).

1. Fine runs. Plain TRiSK runs on a fine hexagon mesh (a batched ensemble, one member per
   seed) are coarse-grained (coarsen.CoarseGrainer) to the coarse mesh at snapshot times t
   (with their tendencies, or also at t + delta).
2. Targets. The coarse model's missing tendency at the coarse-grained state, r =
   C(f_fine(y)) - f_coarse(C(y)) (C: the linear coarse-graining; the default), or, over a
   window, r = (Y_c(t + delta) - Y_hat) / delta with Y_hat the coarse run over delta from
   Y_c(t). It splits into
     - the momentum correction dQ_e = r_u (edges), and
     - a mass-flux correction dF with -D dF = r_h (D: the coarse divergence), the minimum-
       norm solution dF = D^T psi, (D D^T) psi = -r_h, by batched conjugate gradients. The
       continuity equation stays in flux form, so the corrected model conserves mass to
       round-off.
3. Training: the edge-local MLP (closure.ClosureMLP, tensor cores) on normalized features
   and targets, Adam, batches of 65536 edges; then the momentum output's scale is chosen
   a posteriori by 2-day coarse runs from separate validation seeds (calibrate).
4. Evaluation: coarse ensembles with and without the closure, started from the coarse-
   grained fine state, against the coarse-grained fine run; h and relative-vorticity L2
   errors per day; the closure is switched off for a member whose energy drifts by more
   than a threshold per day (the plain FP64 step is the fallback).
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import workloads as w
from .closure import ClosureMLP
from .coarsen import CoarseGrainer, divergence_matrix, edge_geometry, relative_vorticity_matrix
from .ensemble import Ensemble
from .mesh import TRiSKGrid, create_hexagon_mesh
from .model import TRiSKShallowWater, model_tables

PV, KE = "trisk", "cell"
NFEAT = 24


def _grid(level):
    return TRiSKGrid(create_hexagon_mesh(level, centroidal=True))


def _torch_sparse(m, device):
    import torch
    m = m.tocsr()
    return torch.sparse_csr_tensor(torch.from_numpy(m.indptr), torch.from_numpy(m.indices),
                                   torch.from_numpy(m.data), size=m.shape, dtype=torch.float64, device=device)


def fine_snapshots(gf, gc, seeds, days, snapshots_per_member, dt_fine=20.0, pair_steps=8, spinup_days=0.25,
                   device=0, record_days=False, tendency_targets=False):
    """Coarse-grained pairs (Y0 at t, Y1 at t + pair_steps dt_fine) of fine runs, as CUDA
    float64 tensors (state x snapshots); with tendency_targets, Y1 is instead the coarse-
    grained fine tendency at t (the coarse-graining is linear, so this is the tendency of
    the coarse-grained fine state) and delta is 0. With record_days also the coarse state at
    every whole day (days + 1 states per seed). Returns (Y0, Y1, delta, daily, seconds)."""
    import torch
    from .model import tendency
    si = w.si_parameters()
    mf = TRiSKShallowWater(gf, pv_flux=PV, kinetic_energy=KE, device=device, **si)
    total = int(round(days * 86400 / dt_fine))
    ens = Ensemble([(mf, len(seeds), dt_fine, total)])
    for k, seed in enumerate(seeds):
        ens.set_member(0, k, w.synthetic_state(gf, seed=seed))
    cg = CoarseGrainer(gf, gc)
    dev = f"cuda:{device}"
    buf = torch.empty((mf.state_size, len(seeds)), dtype=torch.float64, device=dev)
    col = torch.empty(mf.state_size, dtype=torch.float64, device=dev)

    def coarse_now():
        for k in range(len(seeds)):
            ens.get_member(0, k, col)
            buf[:, k] = col
        torch.cuda.synchronize()
        return cg.torch_apply(buf)

    dcol = torch.empty_like(col)

    def coarse_tendency_now():
        for k in range(len(seeds)):
            ens.get_member(0, k, col)
            tendency(dcol, col, mf)
            buf[:, k] = dcol
        torch.cuda.synchronize()
        return cg.torch_apply(buf)

    spinup = int(round(spinup_days * 86400 / dt_fine))
    span = max(total - spinup - pair_steps, 1)
    every = max(span // max(snapshots_per_member, 1), pair_steps + 1)
    marks = set(range(spinup, total - pair_steps, every)) if snapshots_per_member else set()
    day_steps = int(round(86400 / dt_fine))
    Y0, Y1, daily = [], [], []
    step, seconds = 0, 0.0
    if record_days:
        daily.append(coarse_now())
    while step < total:
        nxt = [s for s in sorted(marks) if s > step]
        targets = [total] + ([nxt[0]] if nxt else []) + ([(step // day_steps + 1) * day_steps] if record_days else [])
        stop = min(targets)
        t0 = time.perf_counter()
        ens.run(stop - step)
        seconds += time.perf_counter() - t0
        step = stop
        if step in marks and tendency_targets:
            Y0.append(coarse_now())
            Y1.append(coarse_tendency_now())
        elif step in marks:
            Y0.append(coarse_now())
            t0 = time.perf_counter()
            ens.run(pair_steps)
            seconds += time.perf_counter() - t0
            step += pair_steps
            Y1.append(coarse_now())
        if record_days and step % day_steps == 0:
            daily.append(coarse_now())
    cat = (lambda a: torch.cat(a, dim=1)) if Y0 else (lambda a: None)
    return cat(Y0), cat(Y1), 0.0 if tendency_targets else pair_steps * dt_fine, daily, seconds


def cg_solve(DDt, rhs, null, iters=500, rtol=1e-9):
    """Solve (D D^T) x = rhs column by column (batched CG), rhs projected orthogonal to the
    null vector `null` first."""
    import torch
    rhs = rhs - null[:, None] * (null @ rhs)[None, :] / (null @ null)
    x = torch.zeros_like(rhs)
    r = rhs.clone()
    p = r.clone()
    rs = (r * r).sum(0)
    rs0 = rs.clone().clamp_min(1e-300)
    for _ in range(iters):
        Ap = DDt(p)
        alpha = rs / (p * Ap).sum(0).clamp_min(1e-300)
        x += alpha * p
        r -= alpha * Ap
        rs_new = (r * r).sum(0)
        if float((rs_new / rs0).max().sqrt()) < rtol:
            break
        p = r + (rs_new / rs.clamp_min(1e-300)) * p
        rs = rs_new
    return x


def residual_targets(gc, Y0, Y1, delta, device=0, coarse_steps=1):
    """(dF, dQ): edges x snapshots (CUDA float64). delta > 0: the coarse model covers delta
    in `coarse_steps` RK4 steps from Y0 and the residual is the mean missing tendency over
    the window, (Y1 - Y_coarse(delta)) / delta. delta = 0: Y1 holds the coarse-grained fine
    tendency at Y0 and the residual is Y1 - f_coarse(Y0), the coarse model's missing
    tendency at the same state."""
    import torch
    from .model import tendency
    si = w.si_parameters()
    mc = TRiSKShallowWater(gc, pv_flux=PV, kinetic_energy=KE, device=device, **si)
    S = Y0.shape[1]
    ens = Ensemble([(mc, S, max(delta, 1.0) / coarse_steps, coarse_steps)])
    col = torch.empty(mc.state_size, dtype=torch.float64, device=Y0.device)
    if delta > 0:
        for k in range(S):
            col.copy_(Y0[:, k])
            ens.set_member(0, k, col)
        ens.run(coarse_steps)
        ens.reset()
        Yh = torch.empty_like(Y0)
        for k in range(S):
            ens.get_member(0, k, col)
            Yh[:, k] = col
        r = (Y1 - Yh) / delta
    else:
        r = torch.empty_like(Y0)
        dcol = torch.empty_like(col)
        for k in range(S):
            col.copy_(Y0[:, k])
            tendency(dcol, col, mc)
            r[:, k] = Y1[:, k] - dcol
        torch.cuda.synchronize()
    for k in range(S):  # the features are those of the state at t
        col.copy_(Y0[:, k])
        ens.set_member(0, k, col)
    ne = gc.ne
    coeffs = model_tables(gc, pv_flux=PV, kinetic_energy=KE, **si)
    D = _torch_sparse(divergence_matrix(coeffs), Y0.device)
    Dt = _torch_sparse(divergence_matrix(coeffs).T.tocsr(), Y0.device)
    A = torch.from_numpy(gc.cell_areas).to(Y0.device)
    psi = cg_solve(lambda p: D @ (Dt @ p), -r[ne:], A)
    dF = Dt @ psi
    return dF, r[:ne].clone(), mc, ens


def features(ens, group, gc, norm, device=0):
    import torch
    rows = gc.ne * ens.groups[group][1]
    X = torch.empty((rows, NFEAT), dtype=torch.bfloat16, device=f"cuda:{device}")
    return ens.features(group, X, norm, edge_geometry(gc))


def build_dataset(gc, Y0, dF, dQ, ens, device=0, sample=2_000_000):
    """Normalized (X, T) over all (edge, snapshot) rows in file edge order e * S + s, the
    feature normalization and the target scales."""
    import torch
    S = Y0.shape[1]
    raw_norm = np.concatenate([np.zeros(NFEAT), np.ones(NFEAT), [1.0, 1.0]])
    Xraw = features(ens, 0, gc, raw_norm, device)
    idx = torch.randint(0, Xraw.shape[0], (min(sample, Xraw.shape[0]),), device=Xraw.device)
    xs = Xraw[idx].double()
    mean = xs.mean(0).cpu().numpy()
    std = xs.std(0).cpu().numpy()
    std[std == 0] = 1.0
    del Xraw
    T = torch.stack([dF.reshape(-1), dQ.reshape(-1)], dim=1)  # rows e * S + s
    tstd = T.std(0).cpu().numpy()
    tstd[tstd == 0] = 1.0
    norm = np.concatenate([mean, 1.0 / std, tstd])
    X = features(ens, 0, gc, norm, device)
    Tn = (T / torch.from_numpy(tstd).to(T.device)).float().contiguous()
    return X, Tn, norm


def train(mlp: ClosureMLP, X, T, epochs=3, batch=65536, lr=1e-3, holdout=0.05, seed=0, input_noise=0.0):
    """Adam on random batches; returns per-epoch mean losses, the held-out loss and the
    held-out loss of predicting zero (the coarse model without the closure). input_noise > 0
    adds Gaussian noise of that standard deviation to the normalized training inputs (not to
    the held-out rows): a regularization towards states the coarse run visits but the
    coarse-grained fine run does not."""
    import torch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    n = X.shape[0]
    perm = torch.randperm(n, device=X.device, generator=g)
    nh = int(n * holdout)
    hold, tr = perm[:nh], perm[nh:]
    history = []
    steps = max(1, (len(tr) // batch))
    total = epochs * steps
    k = 0
    for ep in range(epochs):
        order = tr[torch.randperm(len(tr), device=X.device, generator=g)]
        losses = []
        for b in range(steps):
            idx = order[b * batch:(b + 1) * batch]
            rate = lr * 0.5 * (1 + np.cos(np.pi * k / total))  # cosine schedule
            xb = X[idx]
            if input_noise > 0:
                noise = torch.randn(xb.shape, device=X.device, generator=g, dtype=torch.float32)
                xb = (xb.float() + input_noise * noise).to(torch.bfloat16)
            losses.append(mlp.train_step(xb.contiguous(), T[idx].contiguous(), rate))
            k += 1
        history.append(float(np.mean(losses)))
    held = []
    for b in range(0, nh, batch):
        idx = hold[b:b + batch]
        _, l = mlp.gradients(X[idx].contiguous(), T[idx].contiguous())
        held.append(l * len(idx))
    zero = float((T[hold].double() ** 2).sum(1).mean()) if nh else float("nan")
    return history, float(np.sum(held) / max(nh, 1)), zero


def output_skill(mlp: ClosureMLP, X, T, rows=2_000_000, seed=1):
    """Per output: 1 - MSE / mean square of the target on a random sample (1: perfect, 0:
    no better than the coarse model without the closure)."""
    import torch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    idx = torch.randint(0, X.shape[0], (min(rows, X.shape[0]),), device=X.device, generator=g)
    Y = mlp.forward(X[idx].contiguous()).double()
    Tt = T[idx].double()
    return (1 - ((Y - Tt) ** 2).mean(0) / (Tt ** 2).mean(0)).cpu().numpy().tolist()


def l2_errors(gc, Vc, Y, Yt):
    """h and relative-vorticity area-weighted L2 errors (columns = members)."""
    ne = gc.ne
    dh = Y[ne:] - Yt[ne:]
    eh = np.sqrt((gc.cell_areas[:, None] * dh ** 2).sum(0) / (4 * np.pi))
    dz = Vc @ (Y[:ne] - Yt[:ne])
    ez = np.sqrt((gc.vertex_areas[:, None] * dz ** 2).sum(0) / (4 * np.pi))
    return eh, ez


def run_coarse(gc, Y_init, days, dt, daily_truth, mlp=None, norm=None, drift_per_day=1e-6, device=0,
               every_stage=False, momentum_scale=1.0, state_bits=64, checks_per_day=8, work_free=False, every=1):
    """Coarse ensemble (members = columns of Y_init) for `days` days; h and vorticity errors
    against the daily truth, GPU seconds, and the members that fell back to the plain step
    (energy drift per elapsed day above drift_per_day, checked checks_per_day times a day).
    momentum_scale multiplies the closure's momentum correction (0 keeps only the mass-flux
    correction); state_bits 32 stores the members' states as float; every: the network runs
    on every `every`-th step, its corrections kept in between."""
    if norm is not None:
        norm = np.array(norm, dtype=np.float64)
        norm[2 * NFEAT + 1] *= momentum_scale
    import torch
    si = w.si_parameters()
    mc = TRiSKShallowWater(gc, pv_flux=PV, kinetic_energy=KE, device=device, **si)
    S = Y_init.shape[1]
    steps_day = int(round(86400 / dt))
    ens = Ensemble([(mc, S, 86400 / steps_day, steps_day * days)], state_bits=state_bits)
    col = torch.empty(mc.state_size, dtype=torch.float64, device=Y_init.device)
    for k in range(S):
        col.copy_(Y_init[:, k])
        ens.set_member(0, k, col)
    if mlp is not None:
        ens.set_closure(0, mlp, edge_geometry(gc), norm, every_stage, work_free, every=every)
    on = np.ones(S, dtype=np.float32)
    e0 = ens.energy(0)
    Vc = relative_vorticity_matrix(model_tables(gc, pv_flux=PV, kinetic_energy=KE, **si))
    stream = torch.cuda.ExternalStream(ens.stream(), device=Y_init.device)
    from ._lib import TriskError
    errs_h, errs_z, drifts, gpu_ms = [], [], [], 0.0
    diverged = None
    checks = max(1, min(int(checks_per_day), steps_day))
    bounds = [round(steps_day * c / checks) for c in range(checks + 1)]
    for day in range(1, days + 1):
        for c in range(checks):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ens.run_async(bounds[c + 1] - bounds[c])
            b.record(stream)
            try:
                ens.synchronize()
            except TriskError as err:
                if err.status != 4:
                    raise
                diverged = day  # a member's state became non-finite during this day
                break
            gpu_ms += a.elapsed_time(b)
            elapsed = day - 1 + (c + 1) / checks
            drift = np.abs(ens.energy(0) - e0) / np.abs(e0) / elapsed
            if mlp is not None:
                ens.closure_check()
                newly = (drift > drift_per_day) & (on > 0)
                if newly.any():
                    on[newly] = 0.0
                    ens.closure_mask(0, on)
        if diverged:
            break
        drifts.append(float(drift.max()))
        Y = np.stack([ens.get_member(0, k) for k in range(S)], axis=1)
        eh, ez = l2_errors(gc, Vc, Y, daily_truth[day].cpu().numpy())
        errs_h.append(eh.tolist())
        errs_z.append(ez.tolist())
    done = len(errs_h)
    return {"h_l2": errs_h, "zeta_l2": errs_z, "max_energy_drift_per_day": drifts, "diverged_on_day": diverged,
            "gpu_seconds": gpu_ms / 1e3, "gpu_seconds_per_member_day": gpu_ms / 1e3 / (S * max(done, 1)),
            "fallback_members": int((on == 0).sum()) if mlp is not None else None, "members": S,
            "state_bits": state_bits}


def plain_level_errors(gf, gc, gm, seeds, days, dt, daily_truth, device=0, state_bits=64):
    """Plain runs on an intermediate mesh gm (between the coarse gc and the fine gf) from the
    fine initial states coarse-grained to gm, judged like the coarse runs: every day the gm
    state is coarse-grained to gc and compared with the coarse-grained fine run (daily_truth,
    on gc). Returns h and vorticity L2 errors per day (members as columns) and the GPU seconds
    per member-day of the gm runs."""
    import torch
    si = w.si_parameters()
    mm = TRiSKShallowWater(gm, pv_flux=PV, kinetic_energy=KE, device=device, **si)
    to_m, m_to_c = CoarseGrainer(gf, gm), CoarseGrainer(gm, gc)
    steps_day = int(round(86400 / dt))
    S = len(seeds)
    ens = Ensemble([(mm, S, 86400 / steps_day, steps_day * days)], state_bits=state_bits)
    for k, seed in enumerate(seeds):
        ens.set_member(0, k, np.ascontiguousarray(to_m(w.synthetic_state(gf, seed=seed))))
    Vc = relative_vorticity_matrix(model_tables(gc, pv_flux=PV, kinetic_energy=KE, **si))
    stream = torch.cuda.ExternalStream(ens.stream(), device=device)
    errs_h, errs_z, gpu_ms = [], [], 0.0
    for day in range(1, days + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ens.run_async(steps_day)
        b.record(stream)
        ens.synchronize()
        gpu_ms += a.elapsed_time(b)
        Y = np.stack([m_to_c(ens.get_member(0, k)) for k in range(S)], axis=1)
        eh, ez = l2_errors(gc, Vc, Y, daily_truth[day].cpu().numpy())
        errs_h.append(eh.tolist())
        errs_z.append(ez.tolist())
    return {"h_l2": errs_h, "zeta_l2": errs_z, "gpu_seconds_per_member_day": gpu_ms / 1e3 / (S * days),
            "cells": int(gm.nc), "dt": 86400 / steps_day, "members": S, "state_bits": state_bits}


def member_day_cost(g, members, dt, state_bits=64, mlp=None, norm=None, steps=96, device=0, seed=3,
                    every=1) -> float:
    """GPU seconds per member and simulated day of a `members`-member ensemble on grid g at
    time step dt (with the closure if mlp is given, its network every `every` steps), from
    `steps` timed steps after a warm-up."""
    import torch
    si = w.si_parameters()
    m = TRiSKShallowWater(g, pv_flux=PV, kinetic_energy=KE, device=device, **si)
    ens = Ensemble([(m, members, dt, steps + 2)], state_bits=state_bits)
    for k, y in enumerate(w.ensemble_members(g, members, seed=seed, degree=8, rms_range=(100.0, 100.0))):
        ens.set_member(0, k, y)
    if mlp is not None:
        ens.set_closure(0, mlp, edge_geometry(g), norm, every=every)
    ens.run(2)
    stream = torch.cuda.ExternalStream(ens.stream(), device=device)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ens.run_async(steps)
    b.record(stream)
    ens.synchronize()
    return a.elapsed_time(b) / 1e3 / steps * (86400 / dt) / members


def equal_error_cost(errors: dict, costs: dict, target: float) -> float:
    """GPU seconds per member-day the plain method needs to reach the h error `target`:
    log-linear interpolation (or extrapolation) of cost against error between the two plain
    levels, errors = {level: h error}, costs = {level: GPU seconds per member-day}."""
    (l1, e1), (l2, e2) = sorted(errors.items())
    if e1 <= 0 or e2 <= 0 or e1 == e2 or target <= 0:
        return float("nan")
    slope = np.log(costs[l2] / costs[l1]) / np.log(e2 / e1)
    return float(costs[l1] * (target / e1) ** slope)


def calibrate(gf, gc, mlp, norm, seeds=(501, 502), days=2, coarse_dt=150.0, fine_dt=20.0,
              scales=(0.0, 0.05, 0.1, 0.2, 0.4, 1.0), device=0, log=print, work_free=False, daily=None, every=1):
    """A-posteriori choice of the momentum correction's scale: coarse runs with the closure
    (no fallback, mass-flux part unscaled) from validation seeds, none of them a training or
    evaluation seed, against their coarse-grained fine runs (daily: those, if already made);
    the scale with the smallest mean h error over the days wins (a run that turns non-finite
    loses). Returns (scale, table)."""
    if daily is None:
        _, _, _, daily, _ = fine_snapshots(gf, gc, list(seeds), days, 0, dt_fine=fine_dt, device=device,
                                           spinup_days=0.0, record_days=True)
    table = {}
    for sc in scales:
        r = run_coarse(gc, daily[0], days, coarse_dt, daily, mlp, norm, drift_per_day=np.inf, device=device,
                       momentum_scale=sc, state_bits=32, work_free=work_free, every=every)
        err = float(np.mean(r["h_l2"])) if r["diverged_on_day"] is None else float("inf")
        table[str(sc)] = err
        log(f"calibration: momentum scale {sc}: mean h L2 over {days} days {err:.3f} m")
    best = min(scales, key=lambda sc: table[str(sc)])
    return best, table


def pipeline(fine_level=8, coarse_level=6, train_seeds=32, train_days=10, snapshots=2000, eval_seeds=4,
             eval_days=10, coarse_dt=150.0, window=1800.0, fine_dt=20.0, epochs=3, device=0, out_params=None,
             target="tendency", log=print, input_noise=(0.0,), calibrate_days=4,
             scales=(0.0, 0.05, 0.1, 0.15, 0.2, 0.25, 0.3), every=1):
    """The whole closure experiment; returns a JSON-able summary. target "tendency": the
    residual is the coarse model's missing tendency at the coarse-grained state; "window":
    the mean missing tendency over `window` seconds (window / fine_dt fine steps, window /
    coarse_dt coarse steps). One network is trained, calibrated and evaluated per value of
    input_noise on the same data; the first is the summary's, the others follow under
    "variants" (out_params gets the first)."""
    import torch
    if target not in ("tendency", "window"):
        raise ValueError("target must be 'tendency' or 'window'")
    t_start = time.perf_counter()
    gf, gc = _grid(fine_level), _grid(coarse_level)
    log(f"meshes: fine {gf.nc} cells, coarse {gc.nc} cells ({time.perf_counter() - t_start:.1f} s)")
    per_member = max(1, snapshots // max(train_seeds, 1))
    pair_steps = max(1, int(round(window / fine_dt)))
    coarse_steps = max(1, int(round(window / coarse_dt)))
    Y0, Y1, delta, _, fine_train_s = fine_snapshots(gf, gc, list(range(1, train_seeds + 1)), train_days,
                                                    per_member, dt_fine=fine_dt, pair_steps=pair_steps,
                                                    device=device, tendency_targets=target == "tendency")
    log(f"training snapshots: {Y0.shape[1]} ({target} targets), fine GPU {fine_train_s:.1f} s")
    dF, dQ, mc, ens = residual_targets(gc, Y0, Y1, delta, device, coarse_steps=coarse_steps)
    X, T, norm = build_dataset(gc, Y0, dF, dQ, ens, device)
    del ens, Y1
    torch.cuda.empty_cache()
    log(f"dataset: {X.shape[0]} rows")
    _, _, _, cal_daily, _ = fine_snapshots(gf, gc, [501, 502], calibrate_days, 0, dt_fine=fine_dt,
                                           device=device, spinup_days=0.0, record_days=True)
    eval_list = list(range(1001, 1001 + eval_seeds))
    _, _, _, eval_daily, fine_eval_s = fine_snapshots(gf, gc, eval_list, eval_days, 0, dt_fine=fine_dt,
                                                      device=device, spinup_days=0.0, record_days=True)
    results = []
    for noise in input_noise:
        mlp = ClosureMLP(device=device, seed=0)
        history, held, zero = train(mlp, X, T, epochs=epochs, input_noise=noise)
        skill = output_skill(mlp, X, T)
        log(f"input noise {noise}: training loss per epoch {history}, held-out {held:.4f} (without the closure "
            f"{zero:.4f}), skill (mass flux, momentum) {skill}")
        scale, table = calibrate(gf, gc, mlp, norm, days=calibrate_days, coarse_dt=coarse_dt, fine_dt=fine_dt,
                                 scales=scales, device=device, log=log, daily=cal_daily, every=every)
        vnorm = np.array(norm, dtype=np.float64)
        vnorm[2 * NFEAT + 1] *= scale  # the calibrated momentum scale is part of the saved closure
        if out_params and not results:
            np.savez(out_params, params=mlp.params(), norm=vnorm, fine_level=fine_level, coarse_level=coarse_level,
                     window=window if target == "window" else 0.0, target=target, momentum_scale=scale,
                     input_noise=noise, closure_every=every)
        r = {"input_noise": noise, "train_loss": history, "heldout_loss": held, "heldout_loss_without_closure": zero,
             "output_skill": skill, "calibrated_momentum_scale": scale, "calibration_mean_h_l2": table,
             "calibration_days": calibrate_days}
        r.update(evaluate(gf, gc, mlp, vnorm, eval_seeds, eval_days, coarse_dt, fine_dt, device, log,
                          daily=eval_daily, fine_eval_seconds=fine_eval_s, every=every))
        results.append(r)
    del X, T
    torch.cuda.empty_cache()
    summary = {
        "fine_level": fine_level, "coarse_level": coarse_level, "train_seeds": train_seeds,
        "train_days": train_days, "training_snapshots": int(Y0.shape[1]), "target": target,
        "window_seconds": delta if target == "window" else None,
        "coarse_steps_per_window": coarse_steps if target == "window" else None, "epochs": epochs,
        "fine_training_gpu_seconds": fine_train_s, "gelu": "tanh form (Hendrycks and Gimpel 2016)",
    }
    summary.update(results[0])
    if len(results) > 1:
        summary["variants"] = results[1:]
    summary["wall_seconds"] = time.perf_counter() - t_start
    return summary


def evaluate(gf, gc, mlp, norm, eval_seeds=4, eval_days=10, coarse_dt=150.0, fine_dt=20.0, device=0, log=print,
             work_free=False, daily=None, fine_eval_seconds=None, every=1):
    """Coarse runs from the coarse-grained state of held-out seeds against the coarse-grained
    fine run (daily: that run's daily coarse-grained states, if already made): plain (FP64 and
    FP32 state), and with FP32 state the closure with the energy-drift fallback, without it,
    evaluated at every RK4 stage, and the mass-flux correction alone; then the equal-error
    table. every: the closure runs its network every `every` steps (not in the every-stage
    variant)."""
    eval_list = list(range(1001, 1001 + eval_seeds))
    fine_eval_s = fine_eval_seconds
    if daily is None:
        _, _, _, daily, fine_eval_s = fine_snapshots(gf, gc, eval_list, eval_days, 0, dt_fine=fine_dt,
                                                     device=device, spinup_days=0.0, record_days=True)
    out = {"eval_seeds": eval_seeds, "eval_days": eval_days, "coarse_dt": coarse_dt, "fine_dt": fine_dt,
           "fine_gpu_seconds_per_member_day": fine_eval_s / (eval_seeds * eval_days)}
    init = daily[0]
    f32 = {"state_bits": 32}
    out["work_free_momentum_correction"] = bool(work_free)
    out["closure_every"] = int(every)
    variants = {"plain_coarse": {},
                "plain_coarse_fp32": dict(f32),
                "closure_coarse": {"mlp": mlp, "norm": norm, **f32},
                "closure_coarse_no_fallback": {"mlp": mlp, "norm": norm, "drift_per_day": np.inf, **f32},
                "closure_every_stage_no_fallback": {"mlp": mlp, "norm": norm, "drift_per_day": np.inf,
                                                    "every_stage": True, **f32},
                "closure_mass_flux_only_no_fallback": {"mlp": mlp, "norm": norm, "drift_per_day": np.inf,
                                                       "momentum_scale": 0.0, **f32}}
    for name, kw in variants.items():
        if "mlp" in kw:
            kw["work_free"] = work_free
            if not kw.get("every_stage"):
                kw["every"] = every
        r = run_coarse(gc, init, eval_days, coarse_dt, daily, device=device, **kw)
        out[name] = r
        log(f"{name}: h L2 per day {[round(float(np.mean(x)), 2) for x in r['h_l2']]}, vorticity "
            f"{[float('%.3g' % np.mean(x)) for x in r['zeta_l2']]}, fallback {r['fallback_members']}, "
            f"diverged on day {r['diverged_on_day']}")
    out.update(equal_error_table(gf, gc, mlp, norm, eval_list, eval_days, coarse_dt, daily, out, device, log,
                                 every=every))
    return out


def equal_error_table(gf, gc, mlp, norm, seeds, days, coarse_dt, daily, runs, device=0, log=print, every=1):
    """The comparison at equal h L2 error: plain FP64 runs one level finer than
    the coarse mesh (dt halved) judged on the coarse mesh like the others, the GPU seconds per
    member-day of large ensembles (128 coarse members, 32 finer ones; the closure with FP32
    state), and per day the plain cost at the closure's error (log-linear between the two plain
    levels) against the closure's cost."""
    level = int(round(np.log2((gc.nc - 2) / 10) / 2))
    gm = _grid(level + 1)
    inter = plain_level_errors(gf, gc, gm, seeds, days, coarse_dt / 2, daily, device=device)
    costs = {"plain_coarse_fp64": member_day_cost(gc, 128, coarse_dt, 64, device=device),
             "plain_finer_fp64": member_day_cost(gm, 32, coarse_dt / 2, 64, device=device),
             "closure_coarse_fp32": member_day_cost(gc, 128, coarse_dt, 32, mlp, norm, device=device, every=every)}
    table = []
    closure = runs.get("closure_coarse", {}).get("h_l2", [])
    for d in range(min(days, len(closure))):
        e6, e7 = float(np.mean(runs["plain_coarse"]["h_l2"][d])), float(np.mean(inter["h_l2"][d]))
        ec = float(np.mean(closure[d]))
        plain_at = equal_error_cost({level: e6, level + 1: e7},
                                    {level: costs["plain_coarse_fp64"], level + 1: costs["plain_finer_fp64"]}, ec)
        table.append({"day": d + 1, "h_plain_coarse": e6, "h_plain_finer": e7, "h_closure": ec,
                      "plain_gpu_s_per_member_day_at_closure_error": plain_at,
                      "plain_over_closure": plain_at / costs["closure_coarse_fp32"]})
    log(f"plain hexagon {level + 1}: h L2 per day {[round(float(np.mean(x)), 2) for x in inter['h_l2']]}; "
        f"costs (GPU s per member-day) {costs}")
    for row in table:
        log(f"day {row['day']}: h plain {row['h_plain_coarse']:.2f} / {row['h_plain_finer']:.2f}, closure "
            f"{row['h_closure']:.2f}; plain at the closure's error {row['plain_gpu_s_per_member_day_at_closure_error']:.4g}"
            f" GPU s per member-day, {row['plain_over_closure']:.3g} x the closure's")
    return {"plain_finer": inter, "finer_level": level + 1, "gpu_seconds_per_member_day": costs,
            "equal_error": table}


def main():
    import argparse
    p = argparse.ArgumentParser(description=__doc__)
    p.add_argument("--fine", type=int, default=8)
    p.add_argument("--coarse", type=int, default=6)
    p.add_argument("--train-seeds", type=int, default=32)
    p.add_argument("--train-days", type=float, default=10)
    p.add_argument("--snapshots", type=int, default=2000)
    p.add_argument("--eval-seeds", type=int, default=4)
    p.add_argument("--eval-days", type=int, default=10)
    p.add_argument("--coarse-dt", type=float, default=150.0)
    p.add_argument("--fine-dt", type=float, default=20.0)
    p.add_argument("--window", type=float, default=1800.0)
    p.add_argument("--target", default="tendency", choices=["tendency", "window"])
    p.add_argument("--epochs", type=int, default=3)
    p.add_argument("--out", default="closure_summary.json")
    p.add_argument("--params", default=None, help="where to save the trained network")
    p.add_argument("--evaluate", default=None, help="skip training: evaluate this saved network (.npz)")
    p.add_argument("--training-summary", default=None, help="JSON of the training run to merge (with --evaluate)")
    p.add_argument("--momentum-scale", type=float, default=None,
                   help="with --evaluate: the scale the saved closure's momentum output had at training "
                        "(when the file does not record it); the closure is then re-calibrated")
    p.add_argument("--calibrate-days", type=int, default=4)
    p.add_argument("--work-free", action="store_true",
                   help="with --evaluate: the momentum correction does no work on each member's flow")
    p.add_argument("--scales", default="0,0.05,0.1,0.15,0.2,0.25,0.3", help="momentum scales the calibration tries")
    p.add_argument("--input-noise", default="0", help="comma-separated: one network per training-input noise level")
    p.add_argument("--closure-every", type=int, default=1,
                   help="run the network every N steps and keep its corrections in between")
    a = p.parse_args()
    scales = tuple(float(x) for x in a.scales.split(","))
    if a.evaluate:
        z = np.load(a.evaluate)
        gf, gc = _grid(int(z["fine_level"])), _grid(int(z["coarse_level"]))
        s = {}
        if a.training_summary:
            with open(a.training_summary) as f:
                s.update(json.load(f))
        mlp, norm = ClosureMLP(z["params"]), np.array(z["norm"], dtype=np.float64)
        old = float(z["momentum_scale"]) if "momentum_scale" in z.files else a.momentum_scale
        if old is not None:  # back to the trained output scale, then calibrate again
            if old <= 0:
                raise SystemExit("the saved closure's momentum output is off; nothing to re-calibrate")
            norm[2 * NFEAT + 1] /= old
            scale, table = calibrate(gf, gc, mlp, norm, days=a.calibrate_days, coarse_dt=a.coarse_dt,
                                     fine_dt=a.fine_dt, scales=scales, work_free=a.work_free, every=a.closure_every)
            norm[2 * NFEAT + 1] *= scale
            s.update({"calibrated_momentum_scale": scale, "calibration_mean_h_l2": table,
                      "calibration_days": a.calibrate_days})
            if a.params:
                np.savez(a.params, **{k: z[k] for k in z.files
                                      if k not in ("norm", "momentum_scale", "work_free", "closure_every")},
                         norm=norm, momentum_scale=scale, work_free=a.work_free, closure_every=a.closure_every)
        s.update(evaluate(gf, gc, mlp, norm, a.eval_seeds, a.eval_days, a.coarse_dt, a.fine_dt,
                          work_free=a.work_free, every=a.closure_every))
    else:
        s = pipeline(a.fine, a.coarse, a.train_seeds, a.train_days, a.snapshots, a.eval_seeds, a.eval_days,
                     a.coarse_dt, a.window, a.fine_dt, a.epochs, out_params=a.params, target=a.target,
                     input_noise=tuple(float(x) for x in a.input_noise.split(",")),
                     calibrate_days=a.calibrate_days, scales=scales, every=a.closure_every)
    s["command"] = "python -m dmplex_b200.closure_pipeline " + " ".join(__import__("sys").argv[1:])
    with open(a.out, "w") as f:
        json.dump(s, f, indent=1)
    print(json.dumps({k: v for k, v in s.items() if not isinstance(v, dict)}))


if __name__ == "__main__":
    main()
