"""The shallow-water examples of the reference on the GPU: Williamson test case 2 (steady
geostrophic solid-body rotation, examples/trisk_shallow_water.jl) and the Galewsky jet
(examples/trisk_galewsky.jl):

    python -m dmplex_b200.run [mesh] [resolution] [flags]                              # case 2
    python -m dmplex_b200.run --case=galewsky [mesh] [resolution] [days] [perturbed] [flags]

mesh: hexagon (the Voronoi dual of the icosahedral mesh, its generators as centers), triangle
(the icosahedral mesh; the ICON model, --icon), or an ICON or MPAS grid file (classic NetCDF:
TRiSK on its Voronoi cells, the ICON model with --icon on its triangles). The cases, their
units, time steps and report times are those of the examples (dmplex_b200.cases). Flags as
there: --gassmann, --gassmann-mean, --kinetic=cell|mixed|vertex|alpha, --spring[=beta], --scvt,
--icon, --centered-k. Further:

    --log=FILE        JSON-lines record of the diagnostics (RunLog)
    --checkpoint=FILE state written at the end (and every --every=N steps)
    --resume=FILE     continue from a checkpoint of the same mesh and configuration
    --vtkhdf=FILE     cell vorticity (TRiSK; 1/s for the Galewsky jet) or height change (ICON)

The diagnostics (mass change, relative energy and enstrophy change, |h - h0|_2 and max, ms per
step) are printed at the examples' report steps. Runs on the GPU only.
"""
from __future__ import annotations

import json
import math
import sys
import time

import numpy as np

from .cases import CASES


def parse(argv: list) -> dict:
    """The examples' arguments (trisk_shallow_water.jl:29-41, 79-82; trisk_galewsky.jl:39-51,
    126-131) plus this driver's own."""
    flags = [a for a in argv if a.startswith("--")]
    pos = [a for a in argv if not a.startswith("--")]
    value = {a.split("=", 1)[0]: a.split("=", 1)[1] for a in flags if "=" in a}
    known = {"--icon", "--gassmann", "--gassmann-mean", "--scvt", "--centered-k", "--spring", "--kinetic", "--log",
             "--checkpoint", "--resume", "--vtkhdf", "--every", "--device", "--case"}
    for a in flags:
        if a.split("=", 1)[0] not in known:
            raise ValueError(f"unknown flag {a}")
    case = value.get("--case", "williamson2")
    if case not in CASES:
        raise ValueError(f"unknown case {case} (one of {', '.join(CASES)})")
    icon = "--icon" in flags
    spring = [a for a in flags if a.startswith("--spring")]
    kin = value.get("--kinetic", "cell")
    galewsky = case == "galewsky"
    if len(pos) > (4 if galewsky else 2):
        raise ValueError("too many arguments")
    perturbed = True
    if galewsky and len(pos) > 3:
        if pos[3].lower() not in ("true", "false"):
            raise ValueError("perturbed must be true or false")
        perturbed = pos[3].lower() == "true"
    return {
        "case": case,
        "mesh": pos[0] if pos else ("triangle" if icon else "hexagon"),
        "resolution": int(pos[1]) if len(pos) > 1 else (6 if galewsky else 5),
        "days": float(pos[2]) if galewsky and len(pos) > 2 else (6.0 if galewsky else None),
        "perturbed": perturbed,
        "icon": icon,
        "pv_flux": "gassmann_mean" if "--gassmann-mean" in flags else "gassmann" if "--gassmann" in flags else "trisk",
        "kinetic_energy": kin if kin in ("cell", "mixed", "vertex") else float(kin),
        "spring_beta": (1.2 if spring[0] == "--spring" else float(spring[0].split("=", 1)[1])) if spring else None,
        "centroidal": "--scvt" in flags,
        "kinetic_gradient": "centered" if "--centered-k" in flags else "icon",
        "log": value.get("--log"), "checkpoint": value.get("--checkpoint"), "resume": value.get("--resume"),
        "vtkhdf": value.get("--vtkhdf"), "every": int(value.get("--every", 0)),
        "device": int(value.get("--device", 0)),
    }


def make_case(cfg: dict):
    return CASES[cfg["case"]](cfg["days"], cfg["perturbed"])


def config_meta(cfg: dict) -> dict:
    """What a checkpoint records of the run's configuration (a resume must match it)."""
    keys = ("case", "mesh", "resolution", "days", "perturbed", "icon", "pv_flux", "kinetic_energy", "spring_beta",
            "centroidal", "kinetic_gradient")
    return json.loads(json.dumps({k: cfg[k] for k in keys}))


def load_mesh(cfg: dict):
    """The mesh with the centers its grid uses (load_mesh, trisk_shallow_water.jl:48-66)."""
    import os
    import dmplex_b200 as d
    mesh = cfg["mesh"]
    if mesh == "triangle":
        return d.create_triangle_mesh(cfg["resolution"], cfg["centroidal"], cfg["spring_beta"])
    if mesh == "hexagon":
        return d.create_hexagon_mesh(cfg["resolution"], cfg["centroidal"], cfg["spring_beta"])
    if not os.path.isfile(mesh):
        raise ValueError(f"unknown mesh {mesh}")
    from .gridfiles import _Dataset
    with _Dataset(mesh) as ds:
        icon_file = "vertex_of_cell" in ds
    # TRiSK on ICON grids: the hexagonal dual; the ICON model on MPAS grids: the Delaunay triangles
    return d.read_grid(mesh, dual=(not cfg["icon"]) if icon_file else cfg["icon"])


def edge_and_cell_state(grid, case) -> np.ndarray:
    """[u; h]: the normal wind at the edge points, the height at the cell centers."""
    u = np.einsum("ij,ij->i", case.velocity(grid.edge_points), grid.edge_normals)
    return np.ascontiguousarray(np.concatenate([u, case.height(grid.centers)]))


class _TriskEngine:
    """TRiSKShallowWater on the GPU with the examples' diagnostics."""

    def __init__(self, grid, cfg, case, dt):
        import dmplex_b200 as d
        self.d, self.grid, self.case = d, grid, case
        self.m = d.TRiSKShallowWater(grid, gravity=case.gravity, omega=1.0, pv_flux=cfg["pv_flux"],
                                     kinetic_energy=cfg["kinetic_energy"], device=cfg["device"])
        self.cache = None

    def initial_state(self):
        return self.d.initial_state(self.m, self.case.velocity, self.case.height)

    def step(self, y, dt, n):
        if self.cache is None:
            self.cache = self.d.RK4Cache(y)
        self.d.rk4_step(y, dt, self.d.tendency, self.cache, self.m, nsteps=n)

    def diagnostics(self, y):
        d = self.d
        return {"mass": d.total_mass(self.m, y), "energy": d.total_energy(self.m, y),
                "enstrophy": d.potential_enstrophy(self.m, y)}

    def cell_field(self, y, y0):
        from .vtkhdf import cell_vorticity
        return "vorticity", self.case.vorticity_scale * cell_vorticity(self.grid, y)


class _IconEngine:
    """ICONShallowWater on the GPU (mass only among the invariants, as the model offers), with
    the case's divergence damping."""

    def __init__(self, grid, cfg, case, dt):
        from .icon import ICONShallowWater
        self.grid, self.case = grid, case
        self.m = ICONShallowWater(grid, gravity=case.gravity, divergence_damping=case.icon_damping(grid, dt),
                                  kinetic_gradient=cfg["kinetic_gradient"], device=cfg["device"])

    def initial_state(self):
        return edge_and_cell_state(self.grid, self.case)

    def step(self, y, dt, n):
        self.m.rk4_step(y, dt, n)

    def diagnostics(self, y):
        return {"mass": self.m.total_mass(y)}

    def cell_field(self, y, y0):
        return "height_change", (y - y0)[self.grid.ne:]


def main(argv: list | None = None, engine=None) -> dict:
    """Run the case; returns the last diagnostics record. ``engine(grid, cfg, case, dt)``
    replaces the GPU model (used by the tests with the CPU oracle)."""
    import dmplex_b200 as d
    from .checkpoint import RunLog, load_state, save_state
    cfg = parse(sys.argv[1:] if argv is None else argv)
    case = make_case(cfg)
    mesh = load_mesh(cfg)
    g = d.TRiSKGrid(mesh)
    dt, nsteps = case.steps(g)
    if engine is None:
        engine = _IconEngine if cfg["icon"] else _TriskEngine
    model = engine(g, cfg, case, dt)
    print(f"{g.nc} cells, {g.ne} edges, {g.nv} vertices; {case.name}, "
          f"{'ICON' if cfg['icon'] else cfg['pv_flux']} model; {nsteps} RK4 steps", flush=True)
    y0 = model.initial_state()
    y = y0.copy()
    h0 = y0[g.ne:].copy()
    start = 0
    meta = config_meta(cfg)
    if cfg["resume"]:
        y, header = load_state(cfg["resume"], g)
        if header["meta"].get("config") != meta:
            raise ValueError("the checkpoint was written by a run of another configuration")
        start = header["step"]
    inv0 = model.diagnostics(y0)
    reports = case.reports(nsteps)
    stops = sorted(reports | ({s for s in range(cfg["every"], nsteps + 1, cfg["every"])} if cfg["every"] else set()))
    log = RunLog(cfg["log"], **meta) if cfg["log"] else None
    elapsed, last = 0.0, {}
    step = start
    try:
        for stop in stops:
            if stop <= step:
                continue
            t0 = time.perf_counter()
            model.step(y, dt, stop - step)
            elapsed += time.perf_counter() - t0
            step = stop
            if cfg["checkpoint"] and cfg["every"] and step % cfg["every"] == 0:
                save_state(cfg["checkpoint"], y, g, step=step, time=step * dt, meta={"config": meta})
            if step in reports:
                inv = model.diagnostics(y)
                dh = y[g.ne:] - h0
                last = {"step": step, case.time_label: step * dt / case.time_unit,
                        "h_l2": float(np.sqrt(np.sum(g.cell_areas * dh ** 2) / (4 * np.pi))),
                        "h_max": float(np.abs(dh).max()), "mass": (inv["mass"] - inv0["mass"]) / inv0["mass"],
                        "ms_per_step": 1e3 * elapsed / max(step - start, 1)}
                for k in ("energy", "enstrophy"):
                    if k in inv:
                        last[k] = (inv[k] - inv0[k]) / inv0[k]
                print(f"{case.time_label} = {last[case.time_label]:.3f}  |h - h0|_2 = {last['h_l2']:.3e}  "
                      f"max = {last['h_max']:.3e}  mass: {last['mass']:.2e}"
                      + "".join(f"  {k}: {last[k]:.2e}" for k in ("energy", "enstrophy") if k in last), flush=True)
                if log:
                    log.write(**last)
    finally:
        if log:
            log.close()
    if cfg["checkpoint"]:
        save_state(cfg["checkpoint"], y, g, step=step, time=step * dt, meta={"config": meta})
    if cfg["vtkhdf"]:
        from .vtkhdf import write_vtkhdf
        name, field = model.cell_field(y, y0)
        write_vtkhdf(cfg["vtkhdf"], mesh, **{name: field})
    print(f"{elapsed:.2f} s in {step - start} time steps, {1e3 * elapsed / max(step - start, 1):.2f} ms per step",
          flush=True)
    return last


if __name__ == "__main__":
    main()
