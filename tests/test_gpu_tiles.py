"""Tile shapes of the stage kernels and the autotuner.

Every face flux, divergence and stage update is the same arithmetic whatever
tile the cell sits in, so the FP64 march must give the same energies and dose
bit for bit with every tile shape (the dose is one atomic add per cell and
step, the CFL bound and slab maxima are maxima).  The FP32 form is compared
within the FP32 gate."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from proton_dose_m1_b200 import _native, metrics
from proton_dose_m1_b200 import Accel, Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200.config import TILE_SHAPES
from proton_dose_m1_b200.enums import EnergyScheme, Material, Precision, Scattering
from proton_dose_m1_b200.numerics import energy as en
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import FieldPlan, M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap

pytestmark = pytest.mark.gpu


def _cfg(moving, precision=Precision.FP64, tile=None, shape=(22, 26, 60)):
    geo = Geometry(size=(shape[0] * 1e-3, shape[1] * 1e-3, shape[2] * 1e-3), resolution=shape,
                   objects=[Box(-0.004, shape[0] * 5e-4, -shape[1] * 5e-4, shape[1] * 5e-4, 0.02, 0.03,
                                Material.BONE_COMPACT)])
    return SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=55.0, energy_spread=1.0,
                                                sigma=(0.003, 0.0025), center=(0.001, -0.002)),
                        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                          moving_active_domain=moving),
                        accel=Accel(precision=precision, tile=tile))


def _march(cfg):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    U = None if cfg.numerics.moving_active_domain else torch.zeros((4, *grid.shape), dtype=torch.float64,
                                                                   device="cuda")
    _, dose, E, _ = plan.march(U)
    plan.close()
    return dose.cpu().numpy(), E, grid


@pytest.mark.parametrize("moving", [False, True])
def test_every_tile_shape_gives_the_same_fp64_march(moving):
    ref_d, ref_E, _ = _march(_cfg(moving))
    for shape in TILE_SHAPES[1:]:
        d, E, _ = _march(_cfg(moving, tile=shape))
        np.testing.assert_array_equal(E, ref_E)
        np.testing.assert_array_equal(d, ref_d)


def test_every_tile_shape_passes_the_fp32_gate():
    full, _, grid = _march(_cfg(False))
    for shape in TILE_SHAPES:
        d, _, _ = _march(_cfg(True, Precision.FP32_FP64, tile=shape))
        sc = metrics.compare(d, full, grid)
        assert sc["gamma_1pct_1mm_pass_percent"] >= 99.5, (shape, sc)
        assert abs(sc["maximum_dose_relative_difference"]) <= 0.005, (shape, sc)


def test_autotuner_measures_every_shape_and_keeps_the_fastest():
    cfg = _cfg(True)
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    best = C.c_int(-1)
    ns = (C.c_double * _native.NUM_TILES)()
    _native.check(_native.lib().pdm1_plan_autotune(plan._h, 40, C.byref(best), ns,
                                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    times = list(ns)
    assert 0 <= best.value < _native.NUM_TILES
    assert all(t > 0 for t in times) and times[best.value] == min(times)
    # the tuned plan marches exactly like the default tile
    _, dose, E, _ = plan.march(None)
    plan.close()
    ref_d, ref_E, _ = _march(cfg)
    np.testing.assert_array_equal(E, ref_E)
    np.testing.assert_array_equal(dose.cpu().numpy(), ref_d)


def test_auto_tile_field_equals_default_field():
    beams = [Beam(n_protons=1e6, energy=50.0 + 4 * k, energy_spread=1.0, sigma=(0.002 + 0.0005 * k,) * 2,
                  center=(-0.004 + 0.003 * k, 0.002)) for k in range(3)]
    doses = []
    for tile in (None, "auto"):
        cfg = _cfg(True, tile=tile)
        grid = Grid.from_geometry(cfg.geometry)
        fp = FieldPlan(cfg, MaterialMap.from_geometry(cfg.geometry, grid), grid, beams,
                       box_capacity_cells=int(np.prod(grid.shape)))
        d, steps = fp.march()
        fp.close()
        doses.append((d.cpu().numpy(), steps))
    assert doses[0][1] == doses[1][1]
    np.testing.assert_allclose(doses[1][0], doses[0][0], rtol=0, atol=1e-12 * doses[0][0].max())
    assert any(k[2] == "field" for k in en.autotuned_tiles())
