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


def _staging_marches(plan_march, handles):
    """The same march with bulk row copies and with cell-by-cell loads."""
    from proton_dose_m1_b200 import _native
    out = []
    for bulk in (1, 0):
        for h in handles():
            _native.check(_native.lib().pdm1_plan_set_staging(h, bulk))
        out.append(plan_march())
    return out


def test_bulk_staging_equals_cell_loads_static():
    """Stages B and C of the FP32 form copy their float4 source tile row by
    row with cp.async.bulk (the TMA engine) onto an mbarrier; with staging 0
    they load it cell by cell.  A grid whose sides are not multiples of the
    tile (11 x 9 x 43) and a beam that leaves through z-max exercise the
    clamped rows and the z-max ghost patch: the marches agree bit for bit."""
    geo = Geometry(size=(0.022, 0.018, 0.043), resolution=(11, 9, 43),
                   objects=[Box(-0.011, 0.0, -0.009, 0.009, 0.01, 0.02, Material.BONE_COMPACT)])
    cfg = SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=80.0, energy_spread=1.0,
                                               sigma=(0.003, 0.002), center=(0.001, 0.0)),
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5),
                       accel=Accel(precision=Precision.FP32_FP64))
    grid = Grid.from_geometry(geo)
    mm = MaterialMap.from_geometry(geo, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))

    def run():
        U, dose, E, _ = plan.march(np.zeros((4, *grid.shape)))
        return U.cpu().numpy(), dose.cpu().numpy(), E

    (U1, d1, E1), (U0, d0, E0) = _staging_marches(run, lambda: [plan._h])
    plan.close()
    np.testing.assert_array_equal(E1, E0)
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(U1, U0)
    assert d1.max() > 0


def test_bulk_staging_equals_cell_loads_field():
    """The same on a batched field of moving boxes (boxes of every size, rows
    clipped at the box faces)."""
    from proton_dose_m1_b200.numerics.energy import FieldPlan
    geo = Geometry(size=(0.032, 0.032, 0.06), resolution=(32, 32, 60),
                   objects=[Box(-0.016, 0.0, -0.016, 0.016, 0.02, 0.03, Material.BONE_COMPACT),
                            Box(0.004, 0.016, -0.016, 0.0, 0.035, 0.05, Material.LUNG)])
    cfg = SolverConfig(geometry=geo, beam=Beam(energy=60.0),
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                         moving_active_domain=True),
                       accel=Accel(precision=Precision.FP32_FP64))
    beams = [Beam(n_protons=1e6, energy=55.0, energy_spread=1.0, sigma=(0.003, 0.003), center=(-0.006, -0.004)),
             Beam(n_protons=2e6, energy=62.0, energy_spread=0.8, sigma=(0.002, 0.004), center=(0.005, 0.003)),
             Beam(n_protons=1e6, energy=70.0, energy_spread=1.2, sigma=(0.004, 0.002), center=(0.0, 0.008))]
    grid = Grid.from_geometry(geo)
    mm = MaterialMap.from_geometry(geo, grid)
    fp = FieldPlan(cfg, mm, grid, beams)

    def run():
        dose, steps = fp.march()
        return dose.cpu().numpy(), steps

    (d1, s1), (d0, s0) = _staging_marches(run, lambda: list(fp._plans.values()))
    fp.close()
    assert s1 == s0
    # the field dose sums the beams with FP64 atomics, whose order is not fixed
    assert np.abs(d1 - d0).max() <= 1e-12 * d0.max()
