#!/usr/bin/env python
"""Benchmark of the TRiSK shallow-water RK4 step on B200.

Workload (one "step" = one classical RK4 step = 4 tendencies): create_hexagon_mesh(7;
centroidal=true) (163842 cells, 491520 edges, 327680 vertices), Gassmann PV flux, vertex
kinetic energy, FP64, dt = 75 s, a seeded synthetic height/wind state on the Earth.

  value  device-resident throughput in cell-steps/s (state and tables in HBM, one
         trisk_rk4_step_async call of K steps, CUDA events on the model's stream).
  e2e    the same metric through the public C ABI (trisk_rk4_step) with the state in
         pinned host memory: every step copies the state in and reads it back.
  roofline  the dominant kernel (k_tend: PV flux + gradient + continuity + RK4 update),
         its algorithmic bytes per launch over its CUDA-event duration, against the
         measured HBM copy bandwidth.
  cpu_baseline  the CPU oracle (a C restatement of the reference kernels, not Julia) on
         all host cores, over a bounded sample of the same workload.
  ensemble  64 x hexagon 5 + 32 x hexagon 6 + 8 x hexagon 7 in one persistent CUDA-graph
         launch per phase, one simulated day each (FP64, and FP32 state).
  closure  128 x hexagon 6 with the learned closure (FP32 state) for one simulated day, the
         same without it, one plain hexagon-8 member, and the committed closure errors.
  hexagon5  the reference's CPU-runnable case: CPU restatement and B200, 100 steps.
  icon   the ICON triangle model (level 8: 1.31 M triangles), ms per RK4 step.

--impl reference times that CPU restatement alone (the reference itself is Julia, which
is not installed). With N > 1 GPUs (torchrun) every rank runs an independent replica.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s on 1 B200: plain FP64 vs batched+closure at equal h L2 error"
LEVEL, PV, KE, DT = 7, "gassmann", "vertex", 75.0
WORKLOAD = "hexagon7-gassmann-vertex-fp64-rk4"
REPEATS = 5  # timed windows of --steps steps each; the headline is their median


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="bounded CPU-baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    p.add_argument("--no-closure", action="store_true", help="skip the learned-closure leg")
    p.add_argument("--no-hexagon5", action="store_true", help="skip the hexagon-5 CPU/GPU leg")
    p.add_argument("--ensemble-days", type=float, default=1.0, help="simulated days of the ensemble leg")
    p.add_argument("--ensemble-groups", default=None,
                   help="groups of the ensemble leg as level x members, e.g. 7x8,6x32 (default: 5x64,6x32,7x8)")
    p.add_argument("--ensemble-scheme", default=f"{PV}/{KE}",
                   help="PV flux / kinetic energy of the ensemble leg, e.g. trisk/cell (default: gassmann/vertex)")
    p.add_argument("--ensemble-state", default="both", choices=["both", "64", "32"],
                   help="state precision of the ensemble leg: FP64 and FP32 (both), or one of them")
    p.add_argument("--ensemble-no-autotune", action="store_true",
                   help="ensemble leg at the default block sizes and slices, without the autotuner")
    p.add_argument("--no-icon", action="store_true", help="skip the ICON triangle-model leg")
    p.add_argument("--icon-level", type=int, default=8, help="triangle level of the ICON leg (8: 1.31 M cells)")
    p.add_argument("--icon-steps", type=int, default=100, help="timed RK4 steps of the ICON leg")
    p.add_argument("--no-mpas", action="store_true", help="skip the 3-D MPAS-Gassmann operators leg")
    p.add_argument("--mpas-level", type=int, default=7, help="hexagon level of the MPAS leg")
    p.add_argument("--mpas-calls", type=int, default=50, help="timed calls of the MPAS leg")
    p.add_argument("--no-galewsky", action="store_true", help="skip the Galewsky-jet leg (hexagon 8, 6 days)")
    p.add_argument("--level", type=int, default=LEVEL, help="mesh level (7 is the benchmark workload)")
    p.add_argument("--block", default=None,
                   help="fixed block sizes of the three phases, e.g. 128,128,64 (skips the autotuner)")
    p.add_argument("--l2-keep-mb", type=int, default=0,
                   help="with --block: L2-resident table prefix in MB (the autotuner's other choice)")
    args = p.parse_args()
    return args


def rank_barrier(world, cuda=True):
    """All ranks meet here (after their GPU work has finished, with cuda)."""
    import torch
    if cuda:
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks_of(x, world, device=None):
    """The largest x over all ranks (device None: a CPU tensor, for gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, cells, steps, ms):
    """cell-steps/s of the whole job: every rank advances its own replica of `cells` cells
    by `steps` RK4 steps; ms is the slowest rank's time."""
    return world * cells * steps / (ms * 1e-3)


def build_workload(seed, level=LEVEL):
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    g = d.TRiSKGrid(d.create_hexagon_mesh(level, centroidal=True))
    y = w.synthetic_state(g, seed=seed)
    return g, y


def config_dict(g, n, level=LEVEL):
    workload = WORKLOAD if level == LEVEL else WORKLOAD.replace(f"hexagon{LEVEL}", f"hexagon{level}")
    return {"workload": workload, "mesh": f"create_hexagon_mesh({level}; centroidal=true)", "cells": int(g.nc),
            "edges": int(g.ne), "vertices": int(g.nv), "pv_flux": PV, "kinetic_energy": KE, "dt_s": DT,
            "state": "seeded spherical harmonics deg<=8, 100 m rms, geostrophic u max 40 m/s",
            "l2": "inputs larger than L2: the scheme's tables are 181 MB (L2 126 MB)",
            "parallelism": "replicas" if n > 1 else "single"}


def oracle_baseline(g, y, seconds, threads):
    """CPU restatement of the reference kernels on `threads` host threads: bounded sample."""
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    o = Oracle(d.model_tables(g, pv_flux=PV, kinetic_energy=KE, **w.si_parameters()), threads=threads)
    z = y.copy()
    o.rk4_step(z, DT, 1)  # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        o.rk4_step(z, DT, 1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds or steps >= 1000:
            break
    return g.nc * steps / el, steps, el


def run_hexagon5_leg(local_rank, threads, cpu=True):
    """The reference's CPU-runnable case: hexagon 5, TRiSK PV flux, cell K, dt 300 s, 100 RK4
    steps from a seeded degree-8, 100 m rms state. The CPU restatement on `threads` host
    threads (median of 5 repeats) and the B200 path (device-resident state)."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    si = w.si_parameters()
    g = d.TRiSKGrid(d.create_hexagon_mesh(5, centroidal=True))
    y = w.synthetic_state(g, seed=0)
    out = {"workload": "hexagon5-trisk-cell-fp64-rk4, dt 300 s, 100 steps", "cells": g.nc}
    if cpu:
        o = Oracle(d.model_tables(g, pv_flux="trisk", kinetic_energy="cell", **si), threads=threads)
        times = []
        for _ in range(5):
            z = y.copy()
            o.rk4_step(z, 300.0, 1)
            t0 = time.perf_counter()
            o.rk4_step(z, 300.0, 100)
            times.append(time.perf_counter() - t0)
        out["cpu_cell_steps_per_s"] = g.nc * 100 / float(np.median(times))
        out["cpu_cores"] = threads
        out["cpu_kind"] = "CPU restatement of the reference kernels in C with OpenMP (not Julia)"
    m = d.TRiSKShallowWater(g, pv_flux="trisk", kinetic_energy="cell", device=local_rank, **si)
    yd = torch.from_numpy(y).to(f"cuda:{local_rank}")
    m.autotune(yd, 300.0, 20)
    stream = torch.cuda.ExternalStream(m.stream(), device=local_rank)
    m.rk4_async(yd, 300.0, 10)
    m.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    m.rk4_async(yd, 300.0, 1000)
    b.record(stream)
    m.synchronize()
    sec = a.elapsed_time(b) / 1e3
    out["gpu_cell_steps_per_s"] = g.nc * 1000 / sec
    out["gpu_us_per_step"] = sec / 1000 * 1e6
    out["gpu_step_bytes"] = m.algorithmic_bytes()["rk4_step"]
    out["gpu_step_gbs"] = out["gpu_step_bytes"] / (sec / 1000) / 1e9
    out["note"] = "tables and state (39 MB per step) stay in the 126 MB L2"
    return out


def optional_leg(fn, *args, **kwargs):
    """Run an auxiliary leg (no collectives inside); a failure is reported in the JSON line
    as {"error": ...} and on stderr instead of taking the headline measurement with it."""
    import traceback
    try:
        return fn(*args, **kwargs)
    except Exception as exc:  # noqa: BLE001 - reported, not hidden
        traceback.print_exc()
        return {"error": f"{type(exc).__name__}: {exc}"}


def run_icon_leg(local_rank, level=8, steps=100, hilbert=True, cpu_steps=3):
    """ICON triangle shallow water (the reference's ICONShallowWater) on create_triangle_mesh
    (level), plain bisection — 20 * 4^level triangles, the size of the ICON grid R02B(level - 1): Williamson
    test case 2 on the unit sphere, dt = 0.2 min d_e, `steps` RK4 steps on a device-resident
    state, timed around the synchronous call (12 launches per step). The mesh is renumbered
    along the Hilbert curve (hilbert_order), as ICON's own grid files are spatially ordered."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200.icon import ICONShallowWater
    mesh = d.create_triangle_mesh(level)
    g = d.TRiSKGrid(d.hilbert_order(mesh) if hilbert else mesh)
    m = ICONShallowWater(g, device=local_rank)
    u0 = 0.2
    x = g.edge_points
    u = u0 * (-x[:, 1] * g.edge_normals[:, 0] + x[:, 0] * g.edge_normals[:, 1])
    h = 1 - (u0 + u0 ** 2 / 2) * g.centers[:, 2] ** 2
    y_host = np.concatenate([u, h])
    yd = torch.from_numpy(y_host).to(f"cuda:{local_rank}")
    dt = 0.2 * float(g.dual_lengths.min())
    m.rk4_step(yd, dt, 5)  # warm-up, and the capture of the step's CUDA graph
    torch.cuda.synchronize(local_rank)
    launches0 = m.launch_count()
    t0 = time.perf_counter()
    m.rk4_step(yd, dt, steps)
    torch.cuda.synchronize(local_rank)
    ms = (time.perf_counter() - t0) * 1e3 / steps
    launches = m.launch_count() - launches0
    nbytes = m.algorithmic_bytes()
    peak = measured_peak()[0]
    # CPU baseline: the oracle's C port on all host cores, a few steps of the same workload
    from oracle.icon_oracle import IconOracleC
    threads = os.cpu_count() or 1
    o = IconOracleC(m.tables, threads=threads)
    yc = y_host.copy()
    o.rk4_step(yc, dt, 1)
    t0 = time.perf_counter()
    o.rk4_step(yc, dt, cpu_steps)
    cpu_ms = (time.perf_counter() - t0) * 1e3 / cpu_steps
    return {"workload": f"ICON triangle shallow water, create_triangle_mesh({level})"
                        f"{' Hilbert-ordered' if hilbert else ''}, TC2, FP64",
            "cells": g.nc, "edges": g.ne, "ms_per_step": ms, "cell_steps_per_s": g.nc / (ms * 1e-3),
            "launches_per_step": launches / steps, "step_bytes": nbytes["rk4_step"],
            "gbs": nbytes["rk4_step"] / (ms * 1e-3) / 1e9, "frac": nbytes["rk4_step"] / (ms * 1e-3) / 1e9 / peak,
            "timing": "wall clock around one synchronous rk4_step call of all steps (one CUDA-graph replay per "
                      "step; the state copies in and out of the call are included)",
            "cpu_baseline": {"ms_per_step": cpu_ms, "cell_steps_per_s": g.nc / (cpu_ms * 1e-3), "cores": threads,
                             "kind": "port", "sample": f"{cpu_steps} RK4 steps, the oracle's C restatement with "
                                                       "OpenMP (not Julia)"},
            "published_a100_ms_per_step_same_size": {7: 1.5, 8: 2.4, 9: 7.8}.get(level),
            "note": "the reference's A100 figure is on the ICON grid file of this size (R02B06/07/08 for "
                    "levels 7/8/9); this mesh is the icosahedral bisection of the same size"}


def run_galewsky_leg(local_rank, level=8, days=6.0, schemes=("trisk", "gassmann"), icon=True):
    """The Galewsky jet of the reference's examples/trisk_galewsky.jl through the public API:
    create_hexagon_mesh(level) with its generators as centers, the example's nondimensional
    gravity, balanced height and bump, dt rule and `days` days, FP64, device-resident state,
    the wall time of all RK4 steps (one synchronous rk4_step call after a 2-step warm-up on a
    copy), and the outcome the reference reports beside it: potential enstrophy change and the
    largest relative vorticity. The reference: 28 s (TRiSK), 58 s (gassmann) and 43 s
    (gassmann_mean) for hexagon 8 over 6 days on 4 x A100, and on hexagon 7 |zeta| <= 1.6e-4 1/s
    and +0.4 % enstrophy for TRiSK, 5e-4 and +51 % for gassmann (docs/STATUS.md:29-34)."""
    import dmplex_b200 as d
    from dmplex_b200.cases import OMEGA, Galewsky
    case = Galewsky(days)
    g = d.TRiSKGrid(d.create_hexagon_mesh(level))
    dt, nsteps = case.steps(g)
    dev = f"cuda:{local_rank}"
    out = {"workload": f"Galewsky jet, create_hexagon_mesh({level}), {days:g} days, FP64", "cells": g.nc,
           "steps": nsteps, "dt_seconds": dt / OMEGA}
    published = {"trisk": 28.0, "gassmann": 58.0, "gassmann_mean": 43.0}
    published_outcome = {"trisk": "hexagon 7: |zeta| <= 1.6e-4 1/s, potential enstrophy +0.4 %",
                         "gassmann_mean": "hexagon 7: |zeta| <= 1.6e-4 1/s, potential enstrophy +0.4 %",
                         "gassmann": "hexagon 7: |zeta| 5e-4 1/s, potential enstrophy +51 %"}
    for pv in schemes:
        out[pv] = optional_leg(_galewsky_trisk, d, g, case, pv, dt, nsteps, dev, local_rank,
                               published.get(pv), published_outcome.get(pv))
    if icon:
        out["icon_centered"] = optional_leg(_galewsky_icon, d, case, level, dev, local_rank)
    return out


def _galewsky_trisk(d, g, case, pv, dt, nsteps, dev, local_rank, published_seconds, published_outcome):
    """One PV flux of the Galewsky leg (its own error, if any, stays in its own entry)."""
    import torch
    from dmplex_b200.cases import OMEGA
    from dmplex_b200.vtkhdf import cell_vorticity
    m = d.TRiSKShallowWater(g, gravity=case.gravity, omega=1.0, pv_flux=pv, device=local_rank)
    y = torch.from_numpy(d.initial_state(m, case.velocity, case.height)).to(dev)
    warm = y.clone()
    d.rk4_step(warm, dt, d.tendency, d.RK4Cache(warm), m, nsteps=2)
    mass0, energy0, ens0 = d.total_mass(m, y), d.total_energy(m, y), d.potential_enstrophy(m, y)
    torch.cuda.synchronize(local_rank)
    t0 = time.perf_counter()
    d.rk4_step(y, dt, d.tendency, d.RK4Cache(y), m, nsteps=nsteps)
    torch.cuda.synchronize(local_rank)
    wall = time.perf_counter() - t0
    zeta = OMEGA * cell_vorticity(g, y.cpu().numpy())
    return {"seconds": wall, "ms_per_step": 1e3 * wall / nsteps,
            "mass_change": (d.total_mass(m, y) - mass0) / mass0,
            "energy_change": (d.total_energy(m, y) - energy0) / energy0,
            "enstrophy_change": (d.potential_enstrophy(m, y) - ens0) / ens0,
            "max_abs_vorticity_per_s": float(np.abs(zeta).max()),
            "published_4xa100_seconds": published_seconds, "published_outcome": published_outcome}


def _galewsky_icon(d, case, level, dev, local_rank):
    """ICON triangles of the same level (plain bisection, Hilbert-ordered) with ICON's
    divergence damping and the centered kinetic-energy gradient, which the reference prescribes
    for irregular triangles (ICON's own form blows up on bisection meshes)."""
    import torch
    from dmplex_b200.cases import OMEGA
    from dmplex_b200.vtkhdf import cell_vorticity
    from dmplex_b200.icon import ICONShallowWater
    gt = d.TRiSKGrid(d.hilbert_order(d.create_triangle_mesh(level)))
    dti, ni = case.steps(gt)
    m = ICONShallowWater(gt, gravity=case.gravity, divergence_damping=case.icon_damping(gt, dti),
                         kinetic_gradient="centered", device=local_rank)
    u = np.einsum("ij,ij->i", case.velocity(gt.edge_points), gt.edge_normals)
    y = torch.from_numpy(np.concatenate([u, case.height(gt.centers)])).to(dev)
    warm = y.clone()
    m.rk4_step(warm, dti, 2)
    mass0 = m.total_mass(y.cpu().numpy())
    torch.cuda.synchronize(local_rank)
    t0 = time.perf_counter()
    m.rk4_step(y, dti, ni)
    torch.cuda.synchronize(local_rank)
    wall = time.perf_counter() - t0
    yh = y.cpu().numpy()
    return {"cells": gt.nc, "steps": ni, "seconds": wall, "ms_per_step": 1e3 * wall / ni,
            "mass_change": (m.total_mass(yh) - mass0) / mass0, "finite": bool(np.isfinite(yh).all()),
            "max_abs_vorticity_per_s": float(np.abs(OMEGA * cell_vorticity(gt, yh)).max()),
            "published": "ICON model on the ICON grid R02B07 (the same number of triangles), "
                         "4 x A100: 40406 steps in 60 s, |zeta| <= 1.7e-4 1/s (docs/STATUS.md:104-105)"}


def run_mpas_leg(local_rank, level=7, nlev=30, calls=50, cpu_level=None, hilbert=True, lpt=0, cpu_calls=3):
    """The horizontal operators of the 3-D MPAS-Gassmann dycore (slow_tendencies!, flat ground,
    the reference's ICON-IAP defaults) on create_hexagon_mesh(level) x nlev equidistant layers
    up to 30 km — the grid of the reference's baroclinic wave, Hilbert-ordered as its
    example orders it (hilbert_order) — on a perturbed stratified state, device-resident:
    `calls` calls timed with CUDA events on the library's stream, against the algorithmic
    bytes of the five phases. The CPU baseline is the oracle's C port (OpenMP on all host
    cores) on the same workload (or on create_hexagon_mesh(cpu_level)), `cpu_calls` calls."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200 import mpas
    from dmplex_b200.gridfiles import hilbert_order
    from oracle.mpas_oracle import MpasOracleC

    def case(n):
        mesh = d.create_hexagon_mesh(n)
        g = d.TRiSKGrid(hilbert_order(mesh) if hilbert else mesh)
        v = mpas.vertical_grid(nlev, 30000.0)
        t = mpas.mpas_tables(g, v)
        rng = np.random.default_rng(11)
        z = v["z_full"]
        rho = np.repeat((1.2 * np.exp(-z / 8000.0))[:, None], g.nc, axis=1) * (1 + 1e-3 * rng.standard_normal((nlev, g.nc)))
        theta = np.repeat((290.0 * np.exp(z / 30000.0))[:, None], g.nc, axis=1)
        vn = 10 * rng.standard_normal((nlev, g.ne))
        w = np.zeros((nlev + 1, g.nc))
        w[1:nlev] = 0.1 * rng.standard_normal((nlev - 1, g.nc))
        return g, t, (vn, w, rho, rho * theta)

    g, t, state = case(level)
    ops = mpas.MPASOperators(t, device=local_rank, levels_per_thread=lpt)
    dev = f"cuda:{local_rank}"
    ys = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in state]
    out = ops.work(torch.device(dev))
    f = ops.fields(*ys, out=out)
    sp = C.c_void_p()
    from dmplex_b200._lib import check, lib
    check(lib.trisk_mpas_stream(ops._h, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value, device=dev)
    for _ in range(5):
        check(lib.trisk_mpas_slow_tendencies_async(ops._h, C.byref(f), 1.0))
    check(lib.trisk_mpas_synchronize(ops._h))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(calls):
        check(lib.trisk_mpas_slow_tendencies_async(ops._h, C.byref(f), 1.0))
    e1.record(stream)
    check(lib.trisk_mpas_synchronize(ops._h))
    ms = e0.elapsed_time(e1) / calls
    nbytes = mpas.algorithmic_bytes(t)
    peak = measured_peak()[0]
    gc, tc, sc = (g, t, state) if cpu_level in (None, level) else case(cpu_level)
    threads = os.cpu_count() or 1
    o = MpasOracleC(tc, threads=threads)
    o.slow_tendencies(*sc)
    t0 = time.perf_counter()
    for _ in range(cpu_calls):
        o.slow_tendencies(*sc)
    cpu_s = (time.perf_counter() - t0) / cpu_calls
    return {"workload": f"MPAS-Gassmann slow_tendencies!, create_hexagon_mesh({level})"
                        f"{' Hilbert-ordered' if hilbert else ''} x {nlev} layers, flat, ICON-IAP defaults, FP64",
            "levels_per_thread": ops.levels_per_thread, "cells": g.nc, "edges": g.ne, "layers": nlev,
            "ms_per_call": ms, "cell_levels_per_s": g.nc * nlev / (ms * 1e-3), "launches_per_call": 5,
            "algorithmic_bytes": nbytes, "gbs": nbytes / (ms * 1e-3) / 1e9, "frac": nbytes / (ms * 1e-3) / 1e9 / peak,
            "cpu_baseline": {"cells": gc.nc, "seconds_per_call": cpu_s, "cell_levels_per_s": gc.nc * nlev / cpu_s,
                             "cores": threads, "kind": "port",
                             "sample": f"{cpu_calls} calls, the oracle's C restatement with OpenMP (not Julia)"},
            "published_a100_context": "hexagon 7, 30 layers: vn_tendency alone 4.5 ms per time step (two stages)"}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [s.strip() for s in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        loaded = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                return float(parts[1])
    return None


ENSEMBLE_GROUPS = ((5, 64), (6, 32), (7, 8))  # (mesh level, members), one simulated day, FP64


def run_ensemble_leg(local_rank, seed, days=1.0, state_bits=64, groups_spec=ENSEMBLE_GROUPS, pv=PV, ke=KE,
                     autotune=True):
    """Batched ensemble of three mesh levels in one persistent CUDA-graph launch per phase:
    every member has its own seed, harmonic degree <= 12 and height rms in 50-300 m; each
    level has its own dt (Courant 0.5) and runs `days` simulated days (state_bits 32: the
    states and work vectors are stored as float, the arithmetic stays FP64). groups_spec:
    (level, members) of each group, 64 x hexagon 5, 32 x hexagon 6 and 8 x hexagon 7 by default;
    pv/ke: the scheme (Gassmann PV flux and vertex kinetic energy by default); autotune: let
    the autotuner pick block sizes and slices first."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    si = w.si_parameters()
    groups, info = [], []
    for level, members in groups_spec:
        g = d.TRiSKGrid(d.create_hexagon_mesh(level, centroidal=True))
        m = d.TRiSKShallowWater(g, pv_flux=pv, kinetic_energy=ke, device=local_rank, **si)
        nsteps, dt = w.day_steps(g)
        nsteps = max(1, int(round(nsteps * days)))
        groups.append((m, members, dt, nsteps))
        info.append((g, m, members, nsteps, dt))
    ens = d.Ensemble(groups, state_bits=state_bits)
    for gi, (g, m, members, nsteps, dt) in enumerate(info):
        for k, y in enumerate(w.ensemble_members(g, members, seed=seed + gi)):
            ens.set_member(gi, k, y)
    tuned_ms = ens.autotune(5) if autotune else None  # block sizes and slices; the states are kept
    stream = torch.cuda.ExternalStream(ens.stream(), device=local_rank)
    longest = max(x[3] for x in info)
    ens.run(3)  # warm-up (graph capture)
    ens.reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ens.launch_count()
    e0.record(stream)
    ens.run_async(longest)
    e1.record(stream)
    ens.synchronize()
    ms = e0.elapsed_time(e1)
    taken = ens.steps_taken()
    cell_steps = sum(g.nc * members * s for (g, m, members, _, _), s in zip(info, taken))
    nbytes = 0.0
    for (g, m, members, _, _), s in zip(info, taken):
        n_b = 8.0 * m.state_size
        T = (m.algorithmic_bytes()["rk4_step"] - 23 * n_b) / 4
        n_b *= state_bits / 64  # the state in its storage precision
        nbytes += s * (4 * (T + 2 * members * n_b) + 15 * members * n_b)
    peak, _ = measured_peak()
    return {"workload": "ensemble " + " + ".join(f"{k}x hexagon{l}" for l, k in groups_spec) +
                        f", {pv}/{ke}, {'FP64' if state_bits == 64 else 'FP32 state, FP64 arithmetic'}, "
                        f"{days:g} simulated day each",
            "value": cell_steps / (ms * 1e-3), "unit": "cell-steps/s",
            "gpu_seconds_per_simulated_day": ms * 1e-3 / days,
            "steps": taken, "dt_s": [round(x[4], 3) for x in info], "members": [x[2] for x in info],
            "gpu_launches": ens.launch_count() - launches0, "gbs": nbytes / (ms * 1e-3) / 1e9,
            "block": ens.block(), "members_per_slice": ens.slices(), "autotune_ms_per_step": tuned_ms,
            "frac": nbytes / (ms * 1e-3) / 1e9 / peak}


CLOSURE_WEIGHTS = os.path.join(ROOT, "dmplex_b200", "data", "closure_hexagon6.npz")
CLOSURE_SUMMARY = os.path.join(ROOT, "dmplex_b200", "data", "closure_hexagon6.json")


def run_closure_leg(local_rank, members=128, seed=7):
    """GPU seconds per simulated day: hexagon 6 x `members` with the learned closure (dt 150
    s, TRiSK, FP32 state with FP64 arithmetic and energy sums), the same ensemble without it
    (FP32 and FP64 state), and one plain hexagon-8 member (dt 20 s); plus the errors of the
    committed closure experiment, when present."""
    import torch
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from dmplex_b200.closure import ClosureMLP
    from dmplex_b200.coarsen import edge_geometry
    from dmplex_b200._lib import TriskError
    si = w.si_parameters()
    out = {"workload": f"hexagon6 x {members} members, TRiSK/cell, dt 150 s, FP32 state (FP64 arithmetic and "
                       f"sums), 1 simulated day",
           "members": members}
    g6 = d.TRiSKGrid(d.create_hexagon_mesh(6, centroidal=True))
    m6 = d.TRiSKShallowWater(g6, pv_flux="trisk", kinetic_energy="cell", device=local_rank, **si)
    states = w.ensemble_members(g6, members, seed=seed, degree=8, rms_range=(100.0, 100.0))
    steps = 576
    net, norm, every = None, None, 1
    if os.path.exists(CLOSURE_WEIGHTS):
        z = np.load(CLOSURE_WEIGHTS)
        net, norm = ClosureMLP(z["params"], device=local_rank), z["norm"]
        every = int(z["closure_every"]) if "closure_every" in z.files else 1
        out["weights"] = "trained (dmplex_b200/data/closure_hexagon6.npz)"
    else:
        net = ClosureMLP(device=local_rank, seed=0)
        norm = np.concatenate([np.zeros(24), np.ones(24), [0.0, 0.0]])
        out["weights"] = "untrained, zero output scales (timing only)"

    def timed(with_closure, state_bits=32):
        ens = d.Ensemble([(m6, members, 150.0, steps)], state_bits=state_bits)
        for k, y in enumerate(states):
            ens.set_member(0, k, y)
        if with_closure:
            ens.set_closure(0, net, edge_geometry(g6), norm, every=every)
        e0 = ens.energy(0)
        ens.run(2)
        ens.reset()
        for k, y in enumerate(states):
            ens.set_member(0, k, y)
        stream = torch.cuda.ExternalStream(ens.stream(), device=local_rank)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = ens.launch_count()
        a.record(stream)
        ens.run_async(steps)
        b.record(stream)
        try:
            ens.synchronize()
        except TriskError as err:  # a member blew up: the day was still computed and timed
            if err.status != 4:
                raise
            torch.cuda.synchronize(local_rank)
            return a.elapsed_time(b) / 1e3, ens.launch_count() - launches0, "non-finite state"
        if with_closure:
            ens.closure_check()
        drift = np.abs(ens.energy(0) - e0) / np.abs(e0)
        return a.elapsed_time(b) / 1e3, ens.launch_count() - launches0, float(drift.max())

    out["closure_gpu_seconds_per_simulated_day"], out["closure_gpu_launches"], out["closure_max_energy_drift_day"] = \
        timed(True)
    out["plain_gpu_seconds_per_simulated_day"], _, out["plain_max_energy_drift_day"] = timed(False)
    out["plain_fp64_gpu_seconds_per_simulated_day"], _, out["plain_fp64_max_energy_drift_day"] = timed(False, 64)
    out["closure_cell_steps_per_s"] = members * g6.nc * steps / out["closure_gpu_seconds_per_simulated_day"]
    # one plain hexagon-8 member at dt = 20 s: time 40 steps, scale to a day
    g8 = d.TRiSKGrid(d.create_hexagon_mesh(8, centroidal=True))
    m8 = d.TRiSKShallowWater(g8, pv_flux="trisk", kinetic_energy="cell", device=local_rank, **si)
    y8 = torch.from_numpy(w.synthetic_state(g8, seed=seed)).to(f"cuda:{local_rank}")
    s8 = torch.cuda.ExternalStream(m8.stream(), device=local_rank)
    m8.rk4_async(y8, 20.0, 5)
    m8.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s8)
    m8.rk4_async(y8, 20.0, 40)
    b.record(s8)
    m8.synchronize()
    per_day8 = a.elapsed_time(b) / 1e3 / 40 * 4320
    out["plain_hexagon8_gpu_seconds_per_member_day"] = per_day8
    per_member = out["closure_gpu_seconds_per_simulated_day"] / members
    out["closure_gpu_seconds_per_member_day"] = per_member
    out["gpu_seconds_ratio_hexagon8_over_closure_hexagon6"] = per_day8 / per_member
    # plain FP64 hexagon 7 (dt 75 s), 32 members: the second plain level of the equal-error figure
    g7 = d.TRiSKGrid(d.create_hexagon_mesh(7, centroidal=True))
    m7 = d.TRiSKShallowWater(g7, pv_flux="trisk", kinetic_energy="cell", device=local_rank, **si)
    e7 = d.Ensemble([(m7, 32, 75.0, 1152)])
    for k, y in enumerate(w.ensemble_members(g7, 32, seed=seed, degree=8, rms_range=(100.0, 100.0))):
        e7.set_member(0, k, y)
    e7.run(2)
    e7.reset()
    s7 = torch.cuda.ExternalStream(e7.stream(), device=local_rank)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s7)
    e7.run_async(96)
    b.record(s7)
    e7.synchronize()
    out["plain_hexagon7_fp64_gpu_seconds_per_member_day"] = a.elapsed_time(b) / 1e3 / 96 * 1152 / 32
    del e7
    out["network_every_steps"] = every
    out["measured_errors"] = optional_leg(closure_errors, local_rank, g6, g7, g8, net, norm, out, every=every)
    if os.path.exists(CLOSURE_SUMMARY):
        with open(CLOSURE_SUMMARY) as f:
            s = json.load(f)
        out["errors_vs_coarse_grained_hexagon8"] = {
            k: {"h_l2_per_day_m": [round(float(np.mean(x)), 3) for x in s[k]["h_l2"]],
                "zeta_l2_last_day": float(np.mean(s[k]["zeta_l2"][-1])),
                "fallback_members": s[k].get("fallback_members"), "diverged_on_day": s[k].get("diverged_on_day"),
                "state_bits": s[k].get("state_bits", 64)}
            for k in ("plain_coarse", "plain_coarse_fp32", "closure_coarse", "closure_coarse_no_fallback",
                      "closure_every_stage_no_fallback", "closure_mass_flux_only_no_fallback") if k in s}
        out["errors_source"] = ("errors_vs_coarse_grained_hexagon8: the committed 10-day experiment "
                                "(dmplex_b200/data/closure_hexagon6.json, python -m dmplex_b200.closure_pipeline); "
                                "measured_errors: computed in this run")
    return out


def closure_errors(local_rank, g6, g7, g8, net, norm, costs, seeds=(2001, 2002), days=2, every=1):
    """The closure's comparison measured here: fine hexagon-8 runs (dt 20 s) from held-out
    seeds, coarse-grained to hexagon 6 every day, judge plain FP64 hexagon 6 (dt 150 s) and 7
    (dt 75 s, coarse-grained to hexagon 6 for the comparison) and the closure on hexagon 6 (FP32
    state, energy-drift fallback); then the GPU seconds per member-day the plain method needs
    at the closure's h error, interpolated log-linearly between the two plain levels, against
    the closure's own (costs: the large-ensemble timings of the closure leg)."""
    from dmplex_b200 import closure_pipeline as cp
    _, _, _, daily, fine_s = cp.fine_snapshots(g8, g6, list(seeds), days, 0, dt_fine=20.0, device=local_rank,
                                               spinup_days=0.0, record_days=True)
    init = daily[0]
    runs = {"plain_hexagon6_fp64": cp.run_coarse(g6, init, days, 150.0, daily, device=local_rank),
            "closure_hexagon6": cp.run_coarse(g6, init, days, 150.0, daily, net, norm, device=local_rank,
                                              state_bits=32, every=every),
            "plain_hexagon7_fp64": cp.plain_level_errors(g8, g6, g7, list(seeds), days, 75.0, daily,
                                                         device=local_rank)}
    err = {k: [float(np.mean(x)) for x in r["h_l2"]] for k, r in runs.items()}
    zeta = {k: [float(np.mean(x)) for x in r["zeta_l2"]] for k, r in runs.items()}
    c6 = costs["plain_fp64_gpu_seconds_per_simulated_day"] / costs["members"]
    c7 = costs["plain_hexagon7_fp64_gpu_seconds_per_member_day"]
    cc = costs["closure_gpu_seconds_per_member_day"]
    last = days - 1
    plain_at = cp.equal_error_cost({6: err["plain_hexagon6_fp64"][last], 7: err["plain_hexagon7_fp64"][last]},
                                   {6: c6, 7: c7}, err["closure_hexagon6"][last])
    return {"seeds": list(seeds), "days": days, "h_l2_per_day_m": err, "zeta_l2_per_day": zeta,
            "fallback_members": runs["closure_hexagon6"]["fallback_members"],
            "diverged_on_day": runs["closure_hexagon6"]["diverged_on_day"],
            "gpu_seconds_per_member_day": {"plain_hexagon6_fp64": c6, "plain_hexagon7_fp64": c7, "closure_hexagon6": cc},
            "summary": {"day": days, "h_plain6": err["plain_hexagon6_fp64"][last],
                        "h_plain7": err["plain_hexagon7_fp64"][last], "h_closure": err["closure_hexagon6"][last],
                        "plain_gpu_s_per_member_day_at_closure_error": plain_at,
                        "closure_gpu_s_per_member_day": cc,
                        "plain_over_closure_at_equal_error": plain_at / cc if cc > 0 else None},
            "fine_gpu_seconds": fine_s}


def _pick(d, *keys, digits=4):
    """The entries `keys` of the leg result d that exist, rounded to `digits` significant digits."""
    if not isinstance(d, dict):
        return None
    if "error" in d:
        return {"error": d["error"][:120]}
    out = {}
    for k in keys:
        v = d
        for part in k.split("."):
            v = v.get(part) if isinstance(v, dict) else None
        if isinstance(v, float):
            v = float(f"{v:.{digits}g}")
        if v is not None:
            out[k.replace(".", "_")] = v
    return out


def leg_summary(line):
    """Compact key figures of the headline and of every leg (a few hundred bytes)."""
    r = line["roofline"]
    return {
        "headline": {"cell_steps_per_s": float(f"{line['value']:.4g}"), "ms_per_step": round(line["ms_per_step"], 5),
                     "spread": round(line["timing"]["spread"], 4), "k_tend_frac": round(r["frac"], 3),
                     "k_tend_frac_on_implementation_bytes": round(r["frac_on_implementation_bytes"], 3),
                     "step_frac": round(r["step_frac"], 3),
                     "e2e_cell_steps_per_s": float(f"{line['e2e']['value']:.4g}")},
        "ensemble": _pick(line.get("ensemble"), "value", "gpu_seconds_per_simulated_day", "frac",
                          "fp32_state.gpu_seconds_per_simulated_day", "fp32_state.frac"),
        "closure": _pick(line.get("closure"), "closure_gpu_seconds_per_member_day",
                         "plain_hexagon8_gpu_seconds_per_member_day", "gpu_seconds_ratio_hexagon8_over_closure_hexagon6",
                         "closure_cell_steps_per_s", "measured_errors.summary"),
        "icon": _pick(line.get("icon"), "ms_per_step", "frac", "gbs"),
        "mpas": _pick(line.get("mpas"), "ms_per_call", "frac"),
        "hexagon5": _pick(line.get("hexagon5"), "gpu_us_per_step", "gpu_cell_steps_per_s", "cpu_cell_steps_per_s"),
        "galewsky": _pick(line.get("galewsky"), "trisk.seconds", "gassmann.seconds", "icon_centered.seconds"),
    }


def run_reference(args, rank, world):
    if rank != 0:
        return
    g, y = build_workload(seed=0, level=args.level)
    threads = os.cpu_count() or 1
    budget = max(5.0, min(args.cpu_seconds * 4, 150.0))
    value, steps, el = oracle_baseline(g, y, budget, threads)
    kind = "port"
    line = {"metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(g, 1, args.level), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": threads, "kind": kind,
                             "sample": f"{steps} RK4 steps of the workload ({el:.1f} s); CPU restatement of "
                                       f"the reference kernels in C (Julia is not installed)"},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w

    torch.cuda.set_device(local_rank)
    if world > 1:
        os.environ.setdefault("OMP_NUM_THREADS", str(max(1, (os.cpu_count() or 8) // world)))
    g, y_host = build_workload(seed=rank, level=args.level)
    m = d.TRiSKShallowWater(g, pv_flux=PV, kinetic_energy=KE, device=local_rank, **w.si_parameters())
    stream = torch.cuda.ExternalStream(m.stream(), device=local_rank)
    yd = torch.from_numpy(y_host).to(f"cuda:{local_rank}")

    dev = f"cuda:{local_rank}"

    def barrier():
        rank_barrier(world, cuda=True)

    def max_over_ranks(x):
        return max_over_ranks_of(x, world, dev)

    # block shapes from the autotuner (or given), then warm-up (also captures the CUDA graph)
    if args.block:
        m.set_block([int(b) for b in args.block.split(",")])
        m.set_l2_residency(args.l2_keep_mb << 20)
        tuned_ms = None
    else:
        tuned_ms = m.autotune(yd, DT, 20)
    m.rk4_async(yd, DT, max(args.warmup, 3))
    m.synchronize()
    barrier()
    # REPEATS windows of exactly K steps each, every one bracketed by a barrier and a device
    # synchronization; the headline is the median window (max over ranks), the others are
    # reported beside it
    windows, launches = [], 0
    with ClockSampler(local_rank) as clocks:
        for _ in range(REPEATS):
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            launches0 = m.launch_count()
            barrier()
            start.record(stream)
            m.rk4_async(yd, DT, args.steps)
            end.record(stream)
            m.synchronize()
            barrier()
            launches = m.launch_count() - launches0
            windows.append(max_over_ranks(start.elapsed_time(end)))
    ms = statistics.median(windows)
    value = whole_job_value(world, g.nc, args.steps, ms)

    # e2e: the public synchronous call with a pinned host state, one step per call
    pinned = torch.from_numpy(y_host.copy()).pin_memory()
    ya = pinned.numpy()
    nbytes = ya.nbytes
    d.rk4_step(ya, DT, d.tendency, d.RK4Cache(ya), m)
    barrier()
    e_steps = max(1, min(args.steps, 200))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    cache = d.RK4Cache(ya)
    for _ in range(e_steps):
        d.rk4_step(ya, DT, d.tendency, cache, m)
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e = {"value": whole_job_value(world, g.nc, e_steps, e_ms), "unit": "cell-steps/s", "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "steps": e_steps}

    # roofline of the dominant kernel: a second, instrumented pass with events around
    # every launch of the same workload
    prof_steps = max(1, min(args.steps, 50))
    phases = m.profile_phases(yd, DT, prof_steps)
    nbytes_phase = m.algorithmic_bytes()
    peak, peak_kind = measured_peak()
    achieved = nbytes_phase["tend"] / (phases["tend"] * 1e-3) / 1e9
    step_gbs = nbytes_phase["rk4_step"] / (ms / args.steps * 1e-3) / 1e9
    info = m.info()
    moved = nbytes_phase["tend"] - info["derived_pv_bytes_saved"]
    roofline = {"bound": "hbm", "kernel": "k_tend<gassmann,stage>", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": ncu_traffic("k_tend"), "algorithmic_bytes_per_launch": nbytes_phase["tend"],
                "implementation_bytes_per_launch": moved,
                "frac_on_implementation_bytes": moved / (phases["tend"] * 1e-3) / 1e9 / peak,
                "frac_note": "frac counts every table of the scheme (the canonical byte model); with the "
                             "Gassmann PV derived from the rhombus PV (pv_mode 3) the kernel never reads the "
                             "12 PV-edge indices per edge, so frac_on_implementation_bytes, on the bytes it "
                             "does read, is the bandwidth it sustains",
                "pv_mode": info["pv_mode"], "block": info["block"],
                "l2_resident_table_bytes": info["l2_resident_table_bytes"], "autotune_ms_per_step": tuned_ms,
                "launch_ms": phases["tend"], "phase_ms": phases,
                "phase_bytes": {k: nbytes_phase[k] for k in ("vertex", "flux", "tend")},
                "step_bytes": nbytes_phase["rk4_step"], "step_gbs": step_gbs, "step_frac": step_gbs / peak}

    ensemble = None
    if not args.no_ensemble:
        spec = ENSEMBLE_GROUPS if not args.ensemble_groups else \
            tuple(tuple(int(v) for v in gr.split("x")) for gr in args.ensemble_groups.split(","))
        pv, ke = args.ensemble_scheme.split("/")
        leg = dict(seed=1000 * (rank + 1), days=args.ensemble_days, groups_spec=spec, pv=pv, ke=ke,
                   autotune=not args.ensemble_no_autotune)
        ensemble = f32 = None
        if args.ensemble_state in ("both", "64"):
            ensemble = optional_leg(run_ensemble_leg, local_rank, **leg)
        if args.ensemble_state in ("both", "32"):
            f32 = optional_leg(run_ensemble_leg, local_rank, state_bits=32, **leg)
        if ensemble is None:
            ensemble = f32
        elif f32 is not None and "error" not in ensemble and "error" not in f32:
            ensemble["fp32_state"] = {k: f32[k] for k in ("value", "gpu_seconds_per_simulated_day", "gbs", "frac")}
        if world > 1 and "error" not in ensemble:
            ensemble["value_all_ranks"] = world * ensemble["value"]
    closure = None
    if not args.no_closure:
        closure = optional_leg(run_closure_leg, local_rank)
    icon_leg = None
    if not args.no_icon:
        icon_leg = optional_leg(run_icon_leg, local_rank, level=args.icon_level, steps=args.icon_steps)
    mpas_leg = None
    if not args.no_mpas:
        mpas_leg = optional_leg(run_mpas_leg, local_rank, level=args.mpas_level, calls=args.mpas_calls,
                                cpu_calls=1 if args.no_cpu_baseline else 3)
    galewsky = None
    if world == 1 and not args.no_galewsky:   # an end-to-end run, not a per-GPU rate: at N = 1 only
        galewsky = optional_leg(run_galewsky_leg, local_rank)
    hexagon5 = None
    if rank == 0 and not args.no_hexagon5:
        hexagon5 = optional_leg(run_hexagon5_leg, local_rank, os.cpu_count() or 1,
                                cpu=world == 1 and not args.no_cpu_baseline)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, steps, el = oracle_baseline(g, y_host, args.cpu_seconds, threads)
        cpu = {"value": v, "unit": "cell-steps/s", "cores": threads, "kind": "port",
               "sample": f"{steps} RK4 steps of the workload ({el:.1f} s); CPU restatement of the reference "
                         f"kernels in C with OpenMP (not Julia)"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config_dict(g, world, args.level), "clocks": clocks.summary(), "e2e": e2e,
                "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu,
                "timing": {"windows_ms": windows, "median_ms": ms, "min_ms": min(windows), "max_ms": max(windows),
                           "spread": (max(windows) - min(windows)) / ms, "steps_per_window": args.steps,
                           "gpu_launches_per_window": int(launches)},
                "ensemble": ensemble, "closure": closure, "hexagon5": hexagon5, "icon": icon_leg, "mpas": mpas_leg,
                "galewsky": galewsky}
        # the key figures of every leg last, so that they stay in a short tail of the output
        line["summary"] = leg_summary(line)
        print(json.dumps(line), flush=True)
    del m


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
