"""The benchmark's reference arm: the unmodified reference, installed under
baseline/_ref by baseline/install_reference.sh, given this library's inputs.

Its own moving-box march (numerics/energy.py:1262-1494) of a small phantom with
water, compact bone and skeletal muscle is compared with the oracle's march of
the same inputs: the same energy steps and the dose within the parity bar.
This checks the conversion bench.py makes (material map by Geant4 name, beam,
physics, numerics) on the path its timing runs.  Skipped where the reference
is not installed.
"""

from __future__ import annotations

import numpy as np
import pytest

import bench
from tests.cases import reference_rtol

pytestmark = pytest.mark.skipif(not bench.reference_installed(),
                                reason="reference not installed under baseline/_ref")


def _phantom():
    from proton_dose_m1_b200 import Beam, Geometry, Numerics, Physics, SolverConfig
    from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
    ids = np.zeros((16, 14, 40), dtype=np.int32)
    ids[:, :, 12:16] = 1                  # compact-bone slab across the beam
    ids[9:, :, 20:] = 2                   # muscle block beside the axis, deeper
    geo = Geometry.from_ids((0.016, 0.014, 0.04), ids,
                            (Material.WATER, Material.BONE_COMPACT, Material.MUSCLE_SKELETAL))
    cfg = SolverConfig(
        geometry=geo,
        beam=Beam(n_protons=1e6, energy=40.0, energy_spread=1.0, sigma=(0.002, 0.0025), center=(0.001, -0.0005)),
        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                          moving_active_domain=True))
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    return cfg, MaterialMap.from_geometry(geo, Grid.from_geometry(geo))


def test_reference_material_map_keys_tables_by_geant4_name():
    bench.import_installed_reference()
    cfg, mm = _phantom()
    rmm = bench.reference_material_map(cfg, mm)
    assert [m.value for m in rmm.materials] == ["G4_WATER", "G4_BONE_COMPACT_ICRU", "G4_MUSCLE_SKELETAL_ICRP"]
    assert np.array_equal(rmm.ids, mm.ids)


def test_reference_march_of_converted_inputs_matches_the_oracle():
    from oracle.oracle import OracleProblem
    ps = bench.import_installed_reference()
    from proton_solver.numerics.energy import energy_march as reference_march
    cfg, mm = _phantom()
    rcfg, grid, inflow = bench.reference_spot(ps, cfg)
    _, dose_r, energies_r, _ = reference_march(None, bench.reference_material_map(cfg, mm), grid, inflow, rcfg, np)
    _, dose_o, energies_o, _ = OracleProblem(cfg, mm).march(None)
    energies_r = np.asarray(energies_r)
    assert len(energies_r) == len(energies_o)
    assert np.allclose(energies_r, energies_o, rtol=0.0, atol=1e-12)
    scale = float(np.max(dose_r))
    assert scale > 0.0
    assert float(np.max(np.abs(np.asarray(dose_o) - dose_r))) <= reference_rtol(cfg) * scale
