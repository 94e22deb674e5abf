"""Writes the golden fixtures of the TRiSK shallow-water path (tests/golden/*.npz).

The reference (dmplex.jl) ships no golden vectors and cannot run here (Julia is not
installed), so these fixtures are outputs of the CPU oracle (oracle/trisk_oracle.c, the C
restatement of TRiSKShallowWater.jl's kernels and RungeKutta.jl's rk4_step!), whose
correctness is pinned by the reference's own test assertions (tests/test_oracle.py). They
freeze, for hexagon 3 (642 cells), each scheme's mesh summary, a seeded state, its tendency
and one RK4 step, so that the oracle and the CUDA path are both checked against committed
numbers rather than only against each other.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CASES = (("trisk", "cell", 300.0), ("gassmann", "vertex", 300.0), ("gassmann_mean", "mixed", 300.0))
LEVEL, SEED = 3, 21


def case_data(pv, ke, dt):
    import dmplex_b200 as d
    from dmplex_b200 import workloads as w
    from oracle.oracle import Oracle
    g = d.TRiSKGrid(d.create_hexagon_mesh(LEVEL, centroidal=True))
    si = w.si_parameters()
    o = Oracle(d.model_tables(g, pv_flux=pv, kinetic_energy=ke, **si))
    y = w.synthetic_state(g, seed=SEED)
    dy = o.tendency(y)
    y1 = y.copy()
    o.rk4_step(y1, dt, 1)
    mesh = np.array([g.nc, g.ne, g.nv, g.cell_areas.sum(), g.primal_lengths.sum(), g.dual_lengths.sum()])
    return {"mesh": mesh, "y": y, "dy": dy, "y1": y1, "dt": np.array(dt)}


def path(pv, ke):
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), f"hexagon{LEVEL}_{pv}_{ke}.npz")


if __name__ == "__main__":
    for pv, ke, dt in CASES:
        np.savez_compressed(path(pv, ke), **case_data(pv, ke, dt))
        print("wrote", path(pv, ke))
