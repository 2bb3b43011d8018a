"""Cell-centred grid (proton_solver/numerics/grid.py:7-61).

x and y are centred on the beam axis, z starts at the entrance plane.
Coordinates are host NumPy arrays; the march only needs the spacings.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np


@dataclass(frozen=True)
class Grid:
    x: Any
    y: Any
    z: Any
    dx: float
    dy: float
    dz: float
    shape: tuple[int, int, int]

    @classmethod
    def from_geometry(cls, geometry, xp=np):
        nx, ny, nz = geometry.resolution
        lx, ly, lz = geometry.size
        dx, dy, dz = lx / nx, ly / ny, lz / nz
        x = (np.arange(nx) + 0.5) * dx - 0.5 * lx
        y = (np.arange(ny) + 0.5) * dy - 0.5 * ly
        z = (np.arange(nz) + 0.5) * dz
        return cls(x=x, y=y, z=z, dx=dx, dy=dy, dz=dz, shape=(nx, ny, nz))

    nx = property(lambda self: self.shape[0])
    ny = property(lambda self: self.shape[1])
    nz = property(lambda self: self.shape[2])
    spacing = property(lambda self: (self.dx, self.dy, self.dz))
    cell_volume = property(lambda self: self.dx * self.dy * self.dz)
