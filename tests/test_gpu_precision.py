"""The FP32-stencil / FP64-dose form against the plain FP64 GPU path.

The gate of the north star: gamma(1%/1 mm) >= 99.5% and |max dose difference|
<= 0.5% against the FP64 full-domain march, on the reference's golden cases
and at full size, with and without the moving box.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from dataclasses import replace

from proton_dose_m1_b200 import Accel, Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200 import metrics
from proton_dose_m1_b200.enums import EnergyScheme, Material, Precision, Scattering
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap
from tests import cases

pytestmark = pytest.mark.gpu

GAMMA_MIN = 99.5          # percent, 1%/1 mm
MAX_DOSE_REL = 0.005


def march(cfg):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    _, dose, E, _ = plan.march(None)
    return dose, E, grid


def accelerated(cfg, moving):
    num = replace(cfg.numerics, moving_active_domain=moving)
    return SolverConfig(geometry=cfg.geometry, beam=cfg.beam, physics=cfg.physics, numerics=num,
                        accel=Accel(precision=Precision.FP32_FP64))


def check_gate(cfg, moving):
    ref, E_ref, grid = march(cfg)
    dose, E, _ = march(accelerated(cfg, moving))
    score = metrics.compare(dose, ref, grid)
    assert score["gamma_1pct_1mm_pass_percent"] >= GAMMA_MIN, score
    assert abs(score["maximum_dose_relative_difference"]) <= MAX_DOSE_REL, score
    return score


@pytest.mark.parametrize("name", ["kat2mm_reduced_water", "kat2mm_extended_transversal", "hetero_snapshots"])
@pytest.mark.parametrize("moving", [False, True])
def test_fp32_gate_on_golden_cases(name, moving):
    check_gate(cases.march_config(cases.march_specs()[name]), moving)


@pytest.mark.parametrize("moving", [False, True])
def test_fp32_gate_full_size_slab(moving):
    """80x80x200 @0.5 mm, 2 cm bone slab at 4 cm, Wentzel + nuclear (a shortened
    copy of the bench workload that keeps the test quick)."""
    geo = Geometry(size=(0.04, 0.04, 0.1), resolution=(80, 80, 200),
                   objects=[Box(-0.02, 0.02, -0.02, 0.02, 0.04, 0.06, Material.BONE_COMPACT)])
    cfg = SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=100.0, energy_spread=1.0,
                                               sigma=(0.003, 0.003)),
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
    score = check_gate(cfg, moving)
    assert abs(score["range"]["r80_difference_mm"]) < 0.1


@pytest.mark.parametrize("n_protons", [1e6, 1e12])
def test_fp32_gate_holds_at_high_fluence(n_protons):
    """WENO-Z's smoothness ratio tau5 / (beta + 1e-12) grows with the square
    of the fluence (beta ~ phi^2 against an absolute epsilon): with 1e12
    protons it leaves the float range.  The FP32 form holds it at 1e30 and
    keeps the gate against the FP64 march of the same beam."""
    geo = Geometry(size=(0.03, 0.03, 0.06), resolution=(30, 30, 60),
                   objects=[Box(-0.015, 0.0, -0.015, 0.015, 0.02, 0.03, Material.BONE_COMPACT)])
    cfg = SolverConfig(geometry=geo,
                       beam=Beam(n_protons=n_protons, energy=60.0, energy_spread=1.0, sigma=(0.003, 0.003)),
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
    check_gate(cfg, True)
