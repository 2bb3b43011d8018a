"""The allocation-free march, pdm1_march_noalloc, through the C ABI.

It exists for callers that cannot call cudaMalloc (an application that owns
the device memory through its own pool, a host that forbids device
allocation in plugins, a path that must not take an allocation's implicit
synchronisation): its scratch is a fixed 16 MiB device array inside the
library.  It must give the same dose, energies and final state as the
planned march (pdm1_plan_create + pdm1_march), bit for bit, and keep doing so
on back-to-back calls that reuse the shared array.  This file is collected
last so that a stop at the first failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from proton_dose_m1_b200 import _native
from proton_dose_m1_b200 import Beam, Geometry, Numerics, SolverConfig
from proton_dose_m1_b200.enums import EnergyScheme, SpatialScheme
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap
from proton_dose_m1_b200.physics.tables import material_tables
from tests import cases

pytestmark = pytest.mark.gpu

_SCATTER = {"OFF": 0, "ROSSI": 1, "WENTZEL": 2}
_SCHEME = {"FORWARD_EULER": 0, "SSPRK3": 1, "IF_SSPRK3": 2}
_SPATIAL = {"WENO_Z": 0, "FIRST_ORDER": 1, "MUSCL": 2, "WENO3": 3}


def problem_struct(cfg):
    """A pdm1_problem for `cfg`, plus the host arrays it points into."""
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    inflow = BeamInflow.from_beam(cfg.beam, grid)
    ids = np.ascontiguousarray(mm.ids, dtype=np.int32)
    spatial = np.ascontiguousarray(inflow.spatial, dtype=np.float64)
    keep = [ids, spatial]
    mats = (_native.Material * len(mm.materials))()
    dp = C.POINTER(C.c_double)
    for k, m in enumerate(mm.materials):
        t = material_tables(m.value)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (t.sp_energy, t.sp_value, t.tr_energy, t.tr_value, t.nuc_energy, t.nuc_value)]
        keep += arrs
        ptr = [a.ctypes.data_as(dp) for a in arrs]
        mats[k] = _native.Material(_native.Table(len(arrs[0]), ptr[0], ptr[1]),
                                   _native.Table(len(arrs[2]), ptr[2], ptr[3]),
                                   _native.Table(len(arrs[4]), ptr[4], ptr[5]),
                                   t.density, t.radiation_length)
    keep.append(mats)
    num, phys, beam = cfg.numerics, cfg.physics, cfg.beam
    p = _native.Problem()
    p.nx, p.ny, p.nz = grid.shape
    p.dx, p.dy, p.dz = grid.dx, grid.dy, grid.dz
    p.n_materials = len(mm.materials)
    p.materials = mats
    p.ids = ids.ctypes.data_as(C.POINTER(C.c_int32))
    p.inflow_spatial = spatial.ctypes.data_as(dp)
    p.beam_energy, p.energy_spread, p.angular_spread = beam.energy, beam.energy_spread, beam.angular_spread
    p.scattering = _SCATTER[phys.scattering.name]
    p.nuclear = int(phys.nuclear)
    p.interpolation = 0 if phys.coefficient_interpolation.name == "LINEAR" else 1
    p.energy_scheme = _SCHEME[num.energy_scheme.name]
    p.wave_speeds = 0 if num.wave_speeds.name == "EXACT" else 1
    p.max_energy_step, p.cfl = num.max_energy_step, num.cfl
    p.energy_min, p.energy_window_sigma = num.energy_min, num.energy_window_sigma
    p.active_guard_cells = num.active_guard_cells
    p.precision = 0
    p.spatial_scheme = _SPATIAL[num.spatial_scheme.name]
    return p, keep, (mm, grid, inflow)


def noalloc_march(lib, p, shape, max_steps=100_000):
    U = torch.zeros((4, *shape), dtype=torch.float64, device="cuda")
    dose = torch.full(shape, float("nan"), dtype=torch.float64, device="cuda")
    energies = torch.empty(max_steps + 1, dtype=torch.float64, device="cuda")
    info = _native.MarchInfo()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.pdm1_march_noalloc(C.byref(p), C.c_void_p(U.data_ptr()), C.c_void_p(dose.data_ptr()),
                                C.c_void_p(energies.data_ptr()), max_steps, C.byref(info), stream)
    _native.check(rc)
    return U.cpu().numpy(), dose.cpu().numpy(), energies[: info.n_steps + 1].cpu().numpy()


@pytest.fixture(scope="module")
def lib():
    L = _native.lib()
    L.pdm1_march_noalloc.argtypes = [C.POINTER(_native.Problem), C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_int, C.POINTER(_native.MarchInfo), C.c_void_p]
    return L


@pytest.mark.parametrize("name", ["kat2mm_extended_transversal", "hetero_snapshots"])
def test_noalloc_matches_planned_march_twice(lib, name):
    cfg = cases.march_config(cases.march_specs()[name])
    p, keep, (mm, grid, inflow) = problem_struct(cfg)
    plan = M1Plan(cfg, mm, grid, inflow)
    U_ref, dose_ref, E_ref, _ = plan.march(None)
    U_ref, dose_ref = U_ref.cpu().numpy(), dose_ref.cpu().numpy()
    for _ in range(2):   # back-to-back calls share the scratch array
        U, dose, E = noalloc_march(lib, p, grid.shape)
        np.testing.assert_array_equal(E, E_ref)
        np.testing.assert_array_equal(dose, dose_ref)
        np.testing.assert_array_equal(U, U_ref)


def _variant(name, **numerics):
    from dataclasses import replace
    cfg = cases.march_config(cases.march_specs()[name])
    return replace(cfg, numerics=replace(cfg.numerics, **numerics))


# the integrators and reconstructions besides IF-SSPRK3 + WENO-Z: forward Euler
# (its own stage and finishing kernel), SSPRK3 with the Strang-split sources,
# and the narrower reconstructions with their own inflow ghosts
VARIANTS = {
    "forward_euler": dict(energy_scheme=EnergyScheme.FORWARD_EULER),
    "ssprk3_strang": dict(energy_scheme=EnergyScheme.SSPRK3),
    "muscl": dict(spatial_scheme=SpatialScheme.MUSCL),
    "weno3_euler": dict(spatial_scheme=SpatialScheme.WENO3, energy_scheme=EnergyScheme.FORWARD_EULER),
}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_noalloc_matches_planned_march_other_schemes(lib, variant):
    cfg = _variant("hetero_snapshots", **VARIANTS[variant])
    p, keep, (mm, grid, inflow) = problem_struct(cfg)
    plan = M1Plan(cfg, mm, grid, inflow)
    U_ref, dose_ref, E_ref, _ = plan.march(None)
    U_ref, dose_ref = U_ref.cpu().numpy(), dose_ref.cpu().numpy()
    plan.close()
    for _ in range(2):
        U, dose, E = noalloc_march(lib, p, grid.shape)
        np.testing.assert_array_equal(E, E_ref)
        np.testing.assert_array_equal(dose, dose_ref)
        np.testing.assert_array_equal(U, U_ref)


def test_noalloc_rejects_the_fp32_form(lib):
    cfg = cases.march_config(cases.march_specs()["hetero_snapshots"])
    p, keep, (_, grid, _) = problem_struct(cfg)
    p.precision = 1
    with pytest.raises(NotImplementedError, match="FP64"):
        noalloc_march(lib, p, grid.shape, max_steps=10)


def test_noalloc_alternating_sizes(lib):
    """A smaller problem after a larger one: stale scratch contents do not leak."""
    small = cases.march_config(cases.march_specs()["hetero_snapshots"])
    large = cases.march_config(cases.march_specs()["kat2mm_reduced_water"])
    ps, ks, (_, gs, _) = problem_struct(small)
    pl, kl, (_, gl, _) = problem_struct(large)
    _, d_small_1, _ = noalloc_march(lib, ps, gs.shape)
    _, d_large, _ = noalloc_march(lib, pl, gl.shape)
    _, d_small_2, _ = noalloc_march(lib, ps, gs.shape)
    np.testing.assert_array_equal(d_small_1, d_small_2)
    assert np.isfinite(d_large).all()


def test_noalloc_rejects_problems_beyond_the_scratch(lib):
    cfg = SolverConfig(geometry=Geometry(size=(0.1, 0.1, 0.1), resolution=(100, 100, 100)),
                       beam=Beam(energy=50.0, sigma=(0.005, 0.005)),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3))
    p, keep, (_, grid, _) = problem_struct(cfg)
    with pytest.raises(ValueError, match="scratch"):
        noalloc_march(lib, p, grid.shape, max_steps=10)
