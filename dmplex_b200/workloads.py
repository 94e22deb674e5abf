"""Seeded synthetic shallow-water states on the Earth, in the reference's unit-sphere units.

The reference's runs use analytic test cases (Williamson TC2, Galewsky). The workloads of
this package use seeded random fields with the same character instead:

  h = 10000 m + a real spherical-harmonic field of degree <= L, rescaled to a given
      area-weighted rms (100 m by default);
  u = the geostrophic wind of that field with the constant f0 = 2 Omega sin 45 deg,
      u_e = -(psi_v2 - psi_v1) / l_e with psi = g h' / f0 at the vertices: a discrete skew
      gradient, so the initial flow has zero discrete divergence (the identity
      test/finite_volumes.jl:57-58 checks); then scaled to max |u| = 40 m/s.

Units: the mesh is the unit sphere as in the reference (TRiSKGrid.jl:2), so with
R = 6.371e6 m the SI system maps exactly onto the model with gravity = g / R^2,
coriolis(x) = 2 Omega x[3], u stored as u_SI / R (rad/s), h in m and t in s.
"""
from __future__ import annotations

import numpy as np

EARTH_RADIUS = 6.371e6
GRAVITY = 9.80616
OMEGA = 7.292e-5
MEAN_DEPTH = 1.0e4


def legendre_normalized(z: np.ndarray, degree: int) -> dict:
    """Fully normalized associated Legendre functions P_l^m(z), 0 <= m <= l <= degree, by the
    standard three-term recurrences in l (4 pi normalization)."""
    s = np.sqrt(np.maximum(0.0, 1 - z * z))
    P = {(0, 0): np.ones_like(z)}
    for m in range(1, degree + 1):
        f = np.sqrt(3.0) if m == 1 else np.sqrt((2 * m + 1) / (2 * m))
        P[(m, m)] = f * s * P[(m - 1, m - 1)]
    for m in range(0, degree):
        P[(m + 1, m)] = np.sqrt(2 * m + 3) * z * P[(m, m)]
    for m in range(0, degree + 1):
        for l in range(m + 2, degree + 1):
            a = np.sqrt((4 * l * l - 1) / (l * l - m * m))
            b = np.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
            P[(l, m)] = a * (z * P[(l - 1, m)] - b * P[(l - 2, m)])
    return P


class HarmonicField:
    """sum_{l=1..L} sum_m c_lm P_l^m(z) (cos m lambda | sin m lambda), c_lm ~ N(0, 1)."""

    def __init__(self, degree: int, seed: int):
        rng = np.random.default_rng(seed)
        self.degree = degree
        self.coeffs = [(l, m, rng.standard_normal(), rng.standard_normal() if m > 0 else 0.0)
                       for l in range(1, degree + 1) for m in range(0, l + 1)]

    def __call__(self, x: np.ndarray) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        z = np.clip(x[:, 2], -1.0, 1.0)
        lam = np.arctan2(x[:, 1], x[:, 0])
        P = legendre_normalized(z, self.degree)
        out = np.zeros(len(x))
        for l, m, a, b in self.coeffs:
            out += P[(l, m)] * (a * np.cos(m * lam) + (b * np.sin(m * lam) if m else 0.0))
        return out


def synthetic_state(grid, seed: int, degree: int = 8, rms: float = 100.0, umax: float = 40.0,
                    mean_depth: float = MEAN_DEPTH) -> np.ndarray:
    """y = [u (rad/s); h (m)] in file numbering for a TRiSKGrid of the unit sphere."""
    field = HarmonicField(degree, seed)
    hc = field(grid.centers)
    scale = rms / np.sqrt((grid.cell_areas * hc ** 2).sum() / grid.cell_areas.sum())
    hv = field(grid.vertices) * scale
    f0 = 2 * OMEGA * np.sin(np.pi / 4)
    psi = GRAVITY * hv / f0
    ev = grid.edge_vertices - 1
    u_si = -(psi[ev[:, 1]] - psi[ev[:, 0]]) / (grid.primal_lengths * EARTH_RADIUS)
    u_si *= umax / np.abs(u_si).max()
    return np.ascontiguousarray(np.concatenate([u_si / EARTH_RADIUS, mean_depth + hc * scale]))


def si_parameters() -> dict:
    """gravity and omega of the model for the Earth in SI units on the unit-sphere mesh."""
    return {"gravity": GRAVITY / EARTH_RADIUS ** 2, "omega": OMEGA}


def courant_dt(grid, courant: float = 0.5, umax: float = 40.0) -> float:
    """dt = C min d_e / (sqrt(g H 1.1) + U_max), the reference's formula
    (examples/trisk_galewsky.jl:139) in seconds."""
    c = np.sqrt(GRAVITY * MEAN_DEPTH * 1.1) + umax
    return courant * grid.dual_lengths.min() * EARTH_RADIUS / c


def day_steps(grid, days: float = 1.0, courant: float = 0.5):
    """(nsteps, dt) covering `days` simulated days at the Courant-number time step, with dt
    shortened to divide the span exactly (examples/trisk_galewsky.jl:139-141)."""
    span = 86400.0 * days
    n = int(np.ceil(span / courant_dt(grid, courant)))
    return n, span / n


def ensemble_members(grid, count: int, seed: int, degree: int = 12, rms_range=(50.0, 300.0)):
    """`count` member states with their own seeds, harmonic degree <= `degree` and rms drawn
    uniformly from rms_range."""
    rng = np.random.default_rng(seed)
    states = []
    for k in range(count):
        rms = rng.uniform(*rms_range)
        states.append(synthetic_state(grid, seed=seed * 100003 + k, degree=degree, rms=rms))
    return states


# Named workloads (sizes and schemes of the benchmark configurations).
CONFIGS = {
    "L5-trisk-cell": {"level": 5, "pv_flux": "trisk", "kinetic_energy": "cell", "dt": 300.0, "steps": 100},
    "L7-gassmann-vertex": {"level": 7, "pv_flux": "gassmann", "kinetic_energy": "vertex", "dt": 75.0,
                           "steps": 1000},
}
