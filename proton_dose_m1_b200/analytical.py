"""Analytical CSDA + straight-streaming dose on the GPU
(proton_solver/analytical.py:173-338): the reference's reduced-model
verifier and its default comparison solution (``Reference.ANALYTICAL``),
through ``pdm1_analytical_csda_dose``."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

RANGE_TABLE_POINTS = 200_000          # analytical.py:13
ENERGY_QUADRATURE_POINTS = 128_000    # analytical.py:22


def analytical_available(config) -> bool:
    """Straight streaming applies: no scattering, no nuclear removal, no
    angular spread (analytical.py:329-338)."""
    return (config.physics.scattering.name == "OFF" and not config.physics.nuclear
            and config.beam.angular_spread == 0.0)


def analytical_csda_dose(config, material_map, grid, inflow,
                         num_energy_points: int = ENERGY_QUADRATURE_POINTS):
    """The analytical dose (nx, ny, nz), host NumPy."""
    import torch
    from .numerics.energy import _problem_struct
    if not analytical_available(config):
        raise ValueError("Analytical reference is not available for this configuration.")
    p, keep, _ = _problem_struct(config, material_map, grid, inflow.spatial)
    dose = torch.empty(tuple(int(n) for n in grid.shape), dtype=torch.float64, device="cuda")
    _native.check(_native.lib().pdm1_analytical_csda_dose(
        C.byref(p), int(num_energy_points), RANGE_TABLE_POINTS, C.c_void_p(dose.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return dose.cpu().numpy()


__all__ = ["analytical_available", "analytical_csda_dose", "RANGE_TABLE_POINTS", "ENERGY_QUADRATURE_POINTS"]
