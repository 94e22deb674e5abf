"""The shallow-water test cases of the reference's examples, on the unit sphere (a = Omega = 1):

    Williamson et al. (1992) case 2, steady geostrophic solid-body rotation
        examples/trisk_shallow_water.jl:79-108 (g = 1, u0 = 0.2, one time unit)
    Galewsky et al. (2004) barotropically unstable mid-latitude jet
        examples/trisk_galewsky.jl:49-83, 126-160 (g = g H / (a Omega)^2 with H = 10 km,
        heights in units of H, the 120 m bump at 45 N, dt = 0.5 min d_e / (sqrt(1.1 g) + u_max))

Each case gives the gravity, the velocity and height fields (functions of (n, 3) unit vectors),
the time step and step count for a grid, the steps at which the example reports, and, for the
ICON model, the example's fourth-order divergence damping.
"""
from __future__ import annotations

import math

import numpy as np

EARTH_RADIUS = 6.37122e6
OMEGA = 7.292e-5
GRAVITY = 9.80616


class Williamson2:
    """Steady solid-body rotation, u0 = 0.2, h = 1 - (u0 + u0^2/2) z^2, one time unit."""

    name = "williamson2"
    gravity = 1.0
    time_unit = 1.0          # report times in model time units
    time_label = "t"
    vorticity_scale = 1.0

    def __init__(self, days: float | None = None, perturbed: bool = True):
        self.u0 = 0.2
        self.duration = 1.0

    def velocity(self, x):
        return self.u0 * np.stack([-x[:, 1], x[:, 0], np.zeros(len(x))], axis=1)

    def height(self, x):
        return 1 - (self.u0 + self.u0 ** 2 / 2) * x[:, 2] ** 2

    def steps(self, grid):
        """(dt, nsteps): dt = min(0.2 sqrt(4 pi / nc), 0.4 min d_e) (locally refined meshes)."""
        dt = min(0.2 * math.sqrt(4 * math.pi / grid.nc), 0.4 * float(grid.dual_lengths.min()))
        return dt, math.ceil(self.duration / dt)

    def reports(self, nsteps: int) -> set:
        every = max(1, nsteps // 4)
        return {s for s in range(1, nsteps + 1) if s % every == 0 or s == nsteps}

    def icon_damping(self, grid, dt):
        return 0.0


class Galewsky:
    """The Galewsky jet with (or without) its height perturbation, `days` days."""

    name = "galewsky"
    mean_depth = 1.0e4
    gravity = GRAVITY * mean_depth / (EARTH_RADIUS * OMEGA) ** 2
    day = 86400 * OMEGA
    time_unit = day          # report times in days
    time_label = "day"
    vorticity_scale = OMEGA  # relative vorticity in 1/s
    u_max = 80 / (EARTH_RADIUS * OMEGA)
    phi0, phi1 = math.pi / 7, math.pi / 2 - math.pi / 7

    def __init__(self, days: float | None = 6.0, perturbed: bool = True):
        self.duration = (6.0 if days is None else float(days)) * self.day
        self.perturbed = bool(perturbed)
        self.en = math.exp(-4 / (self.phi1 - self.phi0) ** 2)
        self._profile()

    def jet(self, phi):
        phi = np.asarray(phi, dtype=np.float64)
        inside = (phi > self.phi0) & (phi < self.phi1)
        safe = np.where(inside, phi, (self.phi0 + self.phi1) / 2)
        return np.where(inside, self.u_max / self.en * np.exp(1 / ((safe - self.phi0) * (safe - self.phi1))), 0.0)

    def _profile(self):
        """g h(phi) = g h0 - integral of u (f + tan(phi') u) dphi' by the trapezoid rule on 40001
        latitudes, h0 such that the mean depth is 1 (trisk_galewsky.jl:67-81)."""
        phi = np.linspace(-math.pi / 2, math.pi / 2, 40001)
        step = phi[1] - phi[0]
        u = self.jet(phi)
        with np.errstate(invalid="ignore", over="ignore"):
            integrand = u * (2 * np.sin(phi) + np.tan(phi) * u)
        integrand[[0, -1]] = 0.0
        cumulative = np.concatenate([[0.0], np.cumsum((integrand[:-1] + integrand[1:]) / 2 * step)])
        profile = -cumulative / self.gravity
        mean = np.sum((profile[:-1] + profile[1:]) / 2 * (np.cos(phi[:-1]) + np.cos(phi[1:])) / 2 * step) / 2
        self._phi, self._step, self._prof, self._h0 = phi, step, profile, 1 - mean

    def balanced_height(self, phi):
        s = (np.asarray(phi) + math.pi / 2) / self._step
        i = np.clip(np.floor(s).astype(np.int64), 0, len(self._prof) - 2)
        return self._h0 + self._prof[i] + (s - i) * (self._prof[i + 1] - self._prof[i])

    @staticmethod
    def _lonlat(x):
        return np.arctan2(x[:, 1], x[:, 0]), np.arcsin(np.clip(x[:, 2], -1, 1))

    def velocity(self, x):
        r = np.hypot(x[:, 0], x[:, 1])
        ok = r >= 1e-14
        rs = np.where(ok, r, 1.0)
        u = np.where(ok, self.jet(self._lonlat(x)[1]), 0.0)
        return np.stack([-u * x[:, 1] / rs, u * x[:, 0] / rs, np.zeros(len(x))], axis=1)

    def perturbation(self, x):
        lam, phi = self._lonlat(x)
        return 120 / self.mean_depth * np.cos(phi) * np.exp(-(3 * lam) ** 2) * np.exp(-(15 * (math.pi / 4 - phi)) ** 2)

    def height(self, x):
        h = self.balanced_height(self._lonlat(x)[1])
        return h + self.perturbation(x) if self.perturbed else h

    def steps(self, grid):
        dt = 0.5 * float(grid.dual_lengths.min()) / (math.sqrt(self.gravity * 1.1) + self.u_max)
        nsteps = math.ceil(self.duration / dt)
        return self.duration / nsteps, nsteps

    def reports(self, nsteps: int) -> set:
        """Every half day (trisk_galewsky.jl:165)."""
        count = round(2 * self.duration / self.day)
        return {int(v) for v in np.round(np.linspace(0, nsteps, count + 1)[1:])}

    def icon_damping(self, grid, dt):
        """ICON's fourth-order divergence damping, divdamp_fac = 0.0025 per time step with the
        local cell area (trisk_galewsky.jl:141-145)."""
        local_area = (grid.cell_areas[grid.edge_cells[:, 0] - 1] + grid.cell_areas[grid.edge_cells[:, 1] - 1]) / 2
        return 0.0025 * local_area ** 2 / dt


CASES = {"williamson2": Williamson2, "galewsky": Galewsky}
