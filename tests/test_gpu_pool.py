"""The plans' caching allocator: a destroyed plan's buffers are reused by the
next plan of the same sizes, marches on recycled (non-zero) memory equal
marches on fresh memory, and pdm1_pool_release returns the cache."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from proton_dose_m1_b200 import _native
from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan, energy_march
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap

pytestmark = pytest.mark.gpu


def _problem(n=24):
    geo = Geometry(size=(0.024, 0.024, 0.05), resolution=(n, n, 50 * n // 24),
                   objects=[Box(-0.012, 0.0, -0.012, 0.012, 0.02, 0.03, Material.BONE_COMPACT)])
    cfg = SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=55.0, energy_spread=1.0, sigma=(0.003, 0.003)),
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                         moving_active_domain=True))
    grid = Grid.from_geometry(geo)
    return cfg, MaterialMap.from_geometry(geo, grid), grid, BeamInflow.from_beam(cfg.beam, grid)


def test_pool_reuses_buffers_and_releases_them():
    L = _native.lib()
    cfg, mm, grid, inflow = _problem()
    _native.check(L.pdm1_pool_release())
    assert L.pdm1_pool_cached_bytes() == 0
    plan = M1Plan(cfg, mm, grid, inflow)
    _, d0, E0, _ = plan.march(None)
    d0 = d0.cpu().numpy()
    plan.close()
    cached = L.pdm1_pool_cached_bytes()
    assert cached > 0
    plan = M1Plan(cfg, mm, grid, inflow)
    assert L.pdm1_pool_cached_bytes() < cached
    plan.close()
    # recycled blocks hold the previous march's data: a march must not read
    # memory it did not write
    for _ in range(2):
        plan = M1Plan(cfg, mm, grid, inflow)
        _, d1, E1, _ = plan.march(None)
        plan.close()
        np.testing.assert_array_equal(E1, E0)
        np.testing.assert_array_equal(d1.cpu().numpy(), d0)
        assert L.pdm1_pool_cached_bytes() == cached
    _native.check(L.pdm1_pool_release())
    assert L.pdm1_pool_cached_bytes() == 0


def test_host_outputs_equal_device_outputs():
    cfg, mm, grid, inflow = _problem(48)   # U of 7.4 MB: the staged copy; dose of 1.8 MB: the plain one
    U = np.zeros((4, *grid.shape))
    Uh, dh, Eh, _ = energy_march(U, mm, grid, inflow, cfg, np)
    Ud, dd, Ed, _ = energy_march(torch.zeros((4, *grid.shape), dtype=torch.float64, device="cuda"),
                                 mm, grid, inflow, cfg, np)
    assert isinstance(dh, np.ndarray) and dh.dtype == np.float64 and dh.shape == grid.shape
    np.testing.assert_array_equal(Eh, Ed)
    np.testing.assert_array_equal(dh, dd.cpu().numpy())
    np.testing.assert_array_equal(Uh, Ud.cpu().numpy())
