"""Seeded synthetic phantoms, spot fields and field planning (host side)."""

import numpy as np
import pytest

from proton_dose_m1_b200 import Numerics, SolverConfig, phantoms
from proton_dose_m1_b200.enums import Material
from proton_dose_m1_b200.numerics.energy import estimate_box_cells, field_waves
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap
from proton_dose_m1_b200.physics.tables import material_tables


def test_ellipsoid_phantom_is_seeded():
    a, ia = phantoms.ellipsoid_phantom(7, shape=(32, 32, 64), spacing=(4e-3, 4e-3, 4e-3))
    b, ib = phantoms.ellipsoid_phantom(7, shape=(32, 32, 64), spacing=(4e-3, 4e-3, 4e-3))
    c, _ = phantoms.ellipsoid_phantom(8, shape=(32, 32, 64), spacing=(4e-3, 4e-3, 4e-3))
    np.testing.assert_array_equal(a.voxel_ids, b.voxel_ids)
    assert ia == ib
    assert not np.array_equal(a.voxel_ids, c.voxel_ids)
    assert 6 <= len(ia["ellipsoids"]) <= 12
    assert a.voxel_ids.dtype == np.int32 and a.voxel_ids.shape == (32, 32, 64)
    assert set(a.voxel_materials) <= set(phantoms.ELLIPSOID_MATERIALS)
    assert Material.AIR not in a.voxel_materials
    assert a.voxel_materials[0] == Material.WATER and (a.voxel_ids == 0).mean() > 0.5


def test_ellipsoid_voxelisation_of_a_sphere():
    """With an identity rotation the voxelisation is the cell-centre test."""
    geo, info = phantoms.ellipsoid_phantom(3, shape=(40, 40, 40), spacing=(1e-3, 1e-3, 1e-3),
                                           n_ellipsoids=(6, 6), semi_axis_mm=(8.0, 8.0),
                                           materials=(Material.BONE_COMPACT,))
    grid = Grid.from_geometry(geo)
    X, Y, Z = np.meshgrid(grid.x, grid.y, grid.z, indexing="ij")
    inside = np.zeros(grid.shape, bool)
    for e in info["ellipsoids"]:
        c, r = np.array(e["centre_m"]), e["semi_axes_m"][0]
        inside |= (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r ** 2 * (1 - 1e-12)
    bone = geo.voxel_materials.index(Material.BONE_COMPACT)
    # spheres are rotation invariant: the map is the union of the balls
    # (cells within rounding of a sphere surface may go either way)
    edge = np.zeros(grid.shape, bool)
    for e in info["ellipsoids"]:
        c, r = np.array(e["centre_m"]), e["semi_axes_m"][0]
        d = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2)
        edge |= np.abs(d - r) < 1e-9
    assert np.array_equal((geo.voxel_ids == bone)[~edge], inside[~edge])


def test_pelvis_phantom_layers():
    geo, info = phantoms.pelvis_phantom(5, shape=(64, 16, 80), spacing=(4e-3, 4e-3, 4e-3))
    ids = geo.voxel_ids
    mats = geo.voxel_materials
    assert mats == (Material.WATER, Material.ADIPOSE_SYNTH, Material.MUSCLE_SKELETAL, Material.BONE_COMPACT)
    frac = np.bincount(ids.ravel(), minlength=4) / ids.size
    assert (frac > 0).all()
    # entrance plane and domain corners are outside the body: water
    assert (ids[:, :, 0] == 0).all() and ids[0, 0, 40] == 0
    # along the central axis the beam meets the adipose shell before muscle
    axis = ids[32, 8, :]
    first = {m: int(np.argmax(axis == m)) for m in (1, 2)}
    assert 0 < first[1] < first[2]


def test_spot_grid():
    beams = phantoms.spot_grid(4, 16, 5e-3)
    assert len(beams) == 256
    xs = sorted({b.center[0] for b in beams})
    assert len(xs) == 16 and np.allclose(np.diff(xs), 5e-3) and abs(sum(xs)) < 1e-12
    E = np.array([b.energy for b in beams])
    s = np.array([b.sigma[0] for b in beams])
    assert E.min() >= 70 and E.max() <= 220 and s.min() >= 2e-3 and s.max() <= 6e-3
    assert all(b.sigma[0] == b.sigma[1] and b.n_protons == 1e6 for b in beams)
    assert phantoms.spot_grid(4, 16, 5e-3) == beams


def test_adipose_is_density_scaled_water():
    w, a = material_tables(Material.WATER), material_tables(Material.ADIPOSE_SYNTH)
    assert a.density == 950.0
    f = 950.0 / w.density
    np.testing.assert_array_equal(a.sp_energy, w.sp_energy)
    np.testing.assert_allclose(a.sp_value, w.sp_value * f, rtol=1e-15)
    np.testing.assert_allclose(a.tr_value, w.tr_value * f, rtol=1e-15)
    np.testing.assert_allclose(a.nuc_value, w.nuc_value * f, rtol=1e-15)
    assert a.radiation_length == pytest.approx(w.radiation_length / f, rel=1e-15)


def test_adipose_range_scales_with_density():
    """Same mass stopping power: the depth of the Bragg peak scales 1/0.95."""
    from oracle.oracle import OracleProblem
    from proton_dose_m1_b200 import Beam, Geometry
    from proton_dose_m1_b200.enums import EnergyScheme
    peaks = {}
    for m in (Material.WATER, Material.ADIPOSE_SYNTH):
        geo = Geometry(size=(0.012, 0.012, 0.06), resolution=(6, 6, 120), background_material=m)
        cfg = SolverConfig(geometry=geo, beam=Beam(energy=60.0, sigma=(0.004, 0.004)),
                           numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, max_energy_step=0.5))
        _, dose, _, _ = OracleProblem(cfg).march(np.zeros((4, 6, 6, 120)))
        idd = dose.sum(axis=(0, 1))
        k = int(np.argmax(idd))
        peaks[m] = (k + 0.5) * 0.5e-3
    assert peaks[Material.ADIPOSE_SYNTH] / peaks[Material.WATER] == pytest.approx(1 / 0.95, abs=0.02)


def test_box_estimate_and_waves():
    geo, _ = phantoms.ellipsoid_phantom(4)
    grid = Grid.from_geometry(geo)
    beams = phantoms.spot_grid(4, 4, 5e-3)
    cfg = SolverConfig(geometry=geo, beam=beams[0], numerics=Numerics(moving_active_domain=True))
    est = [estimate_box_cells(cfg, grid, b) for b in beams]
    N = int(np.prod(grid.shape))
    assert all(0 < e <= N for e in est)
    # wider, more energetic beams need larger boxes
    lo = min(beams, key=lambda b: b.energy * b.sigma[0])
    hi = max(beams, key=lambda b: b.energy * b.sigma[0])
    assert estimate_box_cells(cfg, grid, hi) > estimate_box_cells(cfg, grid, lo)
    E = [b.energy for b in beams]
    waves = field_waves(E, 100, 450)
    assert [len(w) for w in waves] == [4, 4, 4, 4]
    assert sorted(sum(waves, [])) == list(range(16))
    flat = [E[k] for k in sum(waves, [])]
    assert flat == sorted(E, reverse=True)
    assert field_waves(E, 100, 10) == [[k] for k in sum(waves, [])]
    assert field_waves(E, 100, 10**9) == [sum(waves, [])]
