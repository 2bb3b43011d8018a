"""``Solver(config).solve()`` (proton_solver/solver.py:29-218) on the GPU.

Builds the grid, the material map and the beam inflow, runs the M1 energy
march (``numerics.energy.energy_march``, on the current CUDA device) and
returns a ``Result``; with ``config.output.save_results`` the run directory
is written as the reference writes it.  Of the reference's comparison
solutions, the analytical CSDA dose (the default ``Reference.ANALYTICAL``)
runs on the GPU too (``analytical.py``); the Monte Carlo references (BFP-MC,
TOPAS) are not part of this library and raise ``NotImplementedError`` naming
them, so a caller sets ``References(reference=Reference.NONE)`` or scores
against doses it holds (``Result.compare``).
"""

from __future__ import annotations

import time

import numpy as np

from .config import SolverConfig
from .enums import Backend, Reference
from .numerics.boundary import BeamInflow
from .numerics.energy import energy_march
from .numerics.grid import Grid
from .persistence import save_result
from .physics.materials import MaterialMap
from .result import Result


class Solver:
    def __init__(self, config: SolverConfig):
        self.config = config

    def solve(self, snapshot_energies: tuple[float, ...] = ()) -> Result:
        """Solve the configured pencil-beam problem."""
        from .analytical import analytical_available, analytical_csda_dose
        cfg = self.config
        requested = [r for r in (cfg.references.reference, *cfg.references.additional_references)
                     if r is not Reference.NONE]
        outside = [r for r in requested if r is not Reference.ANALYTICAL]
        if outside:
            names = ", ".join(r.name for r in outside)
            raise NotImplementedError(
                f"reference solution(s) {names} are outside this library (the M1 march and the "
                "analytical CSDA dose only); use References(reference=Reference.NONE)")
        if Reference.ANALYTICAL in requested and not analytical_available(cfg):
            raise ValueError("Analytical reference is not available for this configuration.")
        grid = Grid.from_geometry(cfg.geometry)
        material_map = MaterialMap.from_geometry(cfg.geometry, grid)
        inflow = BeamInflow.from_beam(cfg.beam, grid)
        phi = J = dose = energies = None
        snapshots = {}
        runtime = None
        if cfg.solve_deterministic:
            U = None if cfg.numerics.moving_active_domain else np.zeros((4, *grid.shape))
            start = time.perf_counter()
            U, dose, energies, snapshots = energy_march(U, material_map, grid, inflow, cfg, np,
                                                        snapshot_energies=snapshot_energies)
            runtime = time.perf_counter() - start
            if U is not None:
                phi, J = U[0], U[1:4]
        analytical_dose = (analytical_csda_dose(cfg, material_map, grid, inflow)
                           if Reference.ANALYTICAL in requested else None)
        result = Result(phi=phi, J=J, dose=dose, grid=grid, energies=energies, snapshots=snapshots,
                        analytical_dose=analytical_dose, runtime=runtime, backend=Backend.GPU)
        if cfg.output.save_results:
            result.run_directory = save_result(result, cfg)
        return result


__all__ = ["Solver"]
