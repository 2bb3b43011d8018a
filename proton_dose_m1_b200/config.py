"""Configuration dataclasses (proton_solver/config.py:16-209).

``Physics``, ``Numerics``, ``References``, ``OutputConfig`` and
``SolverConfig`` keep the reference's fields, defaults and ``ValueError``
checks so a reference configuration is accepted unchanged.  ``Accel`` holds
the knobs that only the GPU march has (precision, tile override, box
proposer); its defaults give the plain FP64 method.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

from .beam import Beam
from .enums import (Backend, CoefficientInterpolation, EnergyScheme, Precision, Reference,
                    Scattering, SpatialScheme, WaveSpeeds)
from .geometry import Geometry


@dataclass(frozen=True)
class Physics:
    scattering: Scattering = Scattering.OFF
    nuclear: bool = False
    coefficient_interpolation: CoefficientInterpolation = CoefficientInterpolation.LINEAR


@dataclass(frozen=True)
class Numerics:
    spatial_scheme: SpatialScheme = SpatialScheme.WENO_Z
    energy_scheme: EnergyScheme = EnergyScheme.SSPRK3
    wave_speeds: WaveSpeeds = WaveSpeeds.EXACT
    max_energy_step: float = 0.25
    cfl: float = 0.99
    energy_min: float = 1e-4
    energy_window_sigma: float = 5.0
    active_domain: bool = False
    active_relative_tolerance: float = 1.0e-14
    moving_active_domain: bool = False
    vacuum_aware_cfl: bool = False
    active_truncation_sigma: float = 5.0
    active_guard_cells: int = 9

    def __post_init__(self):
        if not all(math.isfinite(x) for x in (
                self.max_energy_step, self.cfl, self.energy_min, self.energy_window_sigma,
                self.active_relative_tolerance, self.active_truncation_sigma)):
            raise ValueError("Numerical parameters must be finite.")
        if self.max_energy_step <= 0:
            raise ValueError("max_energy_step must be positive.")
        if not 0 < self.cfl <= 1:
            raise ValueError("cfl must lie in (0, 1].")
        if self.energy_min < 0:
            raise ValueError("energy_min cannot be negative.")
        if self.energy_window_sigma <= 0:
            raise ValueError("energy_window_sigma must be positive.")
        if self.active_relative_tolerance < 0:
            raise ValueError("active_relative_tolerance cannot be negative.")
        if self.active_truncation_sigma <= 0:
            raise ValueError("active_truncation_sigma must be positive.")
        if type(self.vacuum_aware_cfl) is not bool:
            raise ValueError("vacuum_aware_cfl must be a bool.")
        if type(self.active_guard_cells) is not int or self.active_guard_cells < 4:
            raise ValueError("active_guard_cells must be an integer >= 4.")


@dataclass(frozen=True)
class References:
    reference: Reference = Reference.ANALYTICAL
    additional_references: tuple[Reference, ...] = ()
    topas_histories: int = 1_000_000
    topas_seed: int = 1
    topas_force_rerun: bool = False
    bfp_mc_histories: int = 1_000_000
    bfp_mc_seed: int = 137
    bfp_mc_force_rerun: bool = False
    bfp_mc_threads: int = 12
    bfp_mc_max_step_mm: float = 0.25
    bfp_mc_max_energy_loss_mev: float = 0.25
    bfp_mc_max_scattering_optical_depth: float = 0.02
    bfp_mc_stop_energy_mev: float = 1.0

    def __post_init__(self):
        if type(self.topas_histories) is not int or self.topas_histories <= 0:
            raise ValueError("topas_histories must be a positive integer.")
        if type(self.topas_seed) is not int or self.topas_seed < 0:
            raise ValueError("topas_seed must be a non-negative integer.")
        if type(self.bfp_mc_histories) is not int or self.bfp_mc_histories <= 0:
            raise ValueError("bfp_mc_histories must be a positive integer.")
        if type(self.bfp_mc_seed) is not int or self.bfp_mc_seed < 0:
            raise ValueError("bfp_mc_seed must be a non-negative integer.")
        if type(self.bfp_mc_force_rerun) is not bool:
            raise ValueError("bfp_mc_force_rerun must be a bool.")
        if type(self.bfp_mc_threads) is not int or self.bfp_mc_threads <= 0:
            raise ValueError("bfp_mc_threads must be a positive integer.")
        if not all(math.isfinite(x) and x > 0.0 for x in (
                self.bfp_mc_max_step_mm, self.bfp_mc_max_energy_loss_mev,
                self.bfp_mc_max_scattering_optical_depth, self.bfp_mc_stop_energy_mev)):
            raise ValueError("BFP Monte Carlo step controls must be finite and positive.")


@dataclass(frozen=True)
class OutputConfig:
    save_results: bool = False
    results_directory: str = "results"
    store_final_state: bool = True


TILE_SHAPES = ((4, 8, 8), (8, 8, 4), (2, 8, 16))


@dataclass(frozen=True)
class Accel:
    """GPU-only knobs.  The defaults reproduce the plain FP64 method."""

    precision: Precision = Precision.FP64
    # Steps recorded per CUDA graph replay of the march (host syncs once per chunk).
    graph_chunk_steps: int = 32
    # Tile shape of the stage kernels: None = 4x8x8, a shape (x, y, z) among
    # TILE_SHAPES, or "auto" = the fastest shape measured on the plan's problem
    # by the autotuner (cached per precision, grid and beam count).
    tile: tuple[int, int, int] | str | None = None
    # Learned moving box (learned_box.BoxModel); None = the fixed heuristic box.
    # Needs numerics.moving_active_domain.
    box_model: object | None = None
    # Moving box: bound every energy step by the vacuum speed in the phantom's
    # material of least stopping power, as the full-domain march does (its
    # cells outside the beam hold no fluence), so the moving box follows the
    # plain method's step sequence.  False = the reference's rule (the bound
    # over the box only).
    phantom_cfl: bool = False

    def __post_init__(self):
        if not isinstance(self.precision, Precision):
            raise ValueError("precision must be a Precision value.")
        if type(self.graph_chunk_steps) is not int or self.graph_chunk_steps <= 0:
            raise ValueError("graph_chunk_steps must be a positive integer.")
        if not (self.tile is None or self.tile == "auto" or tuple(self.tile) in TILE_SHAPES):
            raise ValueError(f"tile must be None, 'auto' or one of {TILE_SHAPES}.")


@dataclass
class SolverConfig:
    geometry: Geometry
    beam: Beam
    physics: Physics = field(default_factory=Physics)
    numerics: Numerics = field(default_factory=Numerics)
    backend: Backend = Backend.AUTO
    solve_deterministic: bool = True
    references: References = field(default_factory=References)
    output: OutputConfig = field(default_factory=OutputConfig)
    accel: Accel = field(default_factory=Accel)

    def __post_init__(self):
        x0, y0 = self.beam.center
        lx, ly, _ = self.geometry.size
        if not -lx / 2 <= x0 < lx / 2:
            raise ValueError("Beam center lies outside the x-domain.")
        if not -ly / 2 <= y0 < ly / 2:
            raise ValueError("Beam center lies outside the y-domain.")
        if self.numerics.energy_min >= self.beam.energy:
            raise ValueError("energy_min must be smaller than the initial beam energy.")
