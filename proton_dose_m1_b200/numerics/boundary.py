"""Gaussian pencil-beam inflow at the z-min face
(proton_solver/numerics/boundary.py:11-114).

The transverse profile is the exact cell average of a Gaussian (erf
differences), cut at ``cutoff_sigma`` on the cell-centre radius and
renormalised to unit discrete mass; the spectrum is Gaussian in energy.
Profiles are computed on the host once per beam; the GPU evaluates the
spectrum factor per energy.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any

import numpy as np


def gaussian_cell_average(centers, spacing, mean, sigma):
    scale = math.sqrt(2.0) * sigma
    lower = (centers - 0.5 * spacing - mean) / scale
    upper = (centers + 0.5 * spacing - mean) / scale
    mass = np.fromiter((0.5 * (math.erf(b) - math.erf(a)) for a, b in zip(lower, upper)),
                       dtype=float, count=len(centers))
    return mass / spacing


def transverse_profile(beam, grid):
    x = np.asarray(grid.x)
    y = np.asarray(grid.y)
    gx = gaussian_cell_average(x, grid.dx, beam.center[0], beam.sigma[0])
    gy = gaussian_cell_average(y, grid.dy, beam.center[1], beam.sigma[1])
    profile = gx[:, None] * gy[None, :]
    r2 = (((x[:, None] - beam.center[0]) / beam.sigma[0]) ** 2
          + ((y[None, :] - beam.center[1]) / beam.sigma[1]) ** 2)
    profile = np.where(r2 <= beam.cutoff_sigma ** 2, profile, 0.0)
    mass = profile.sum() * grid.dx * grid.dy
    if not math.isfinite(mass) or mass <= 0:
        raise ValueError("Beam profile has zero or non-finite mass on the domain.")
    return profile / mass


def energy_density(beam, energy: float) -> float:
    """Gaussian spectrum value at ``energy`` [1/MeV]."""
    if beam.energy_spread == 0:
        raise ValueError("Zero energy spread is not supported by the Gaussian inflow.")
    return (math.exp(-(energy - beam.energy) ** 2 / (2.0 * beam.energy_spread ** 2))
            / (math.sqrt(2.0 * math.pi) * beam.energy_spread))


@dataclass(frozen=True)
class BeamInflow:
    beam: Any
    spatial: Any       # (nx, ny) host float64, n_protons * normalised profile

    @classmethod
    def from_beam(cls, beam, grid, xp=np):
        return cls(beam=beam, spatial=beam.n_protons * transverse_profile(beam, grid))

    def state(self, energy: float, xp=np):
        """The M1 inflow state (4, nx, ny) at ``energy``."""
        phi = np.asarray(self.spatial) * energy_density(self.beam, energy)
        U = np.empty((4, *phi.shape), dtype=phi.dtype)
        U[0] = phi
        U[1] = 0.0
        U[2] = 0.0
        U[3] = math.exp(-self.beam.angular_spread ** 2) * phi
        return U
