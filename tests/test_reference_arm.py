"""The benchmark's reference arm: the unmodified reference, installed under
baseline/_ref by baseline/install_reference.sh, given this library's inputs.

Its own moving-box march (numerics/energy.py:1262-1494) of a small phantom of
water, compact bone, skeletal muscle and synthetic adipose is compared with the
oracle's march of the same inputs: the same energy steps and the dose within
the parity bar.  This checks the conversion bench.py makes (material map by
table name, beam, physics, numerics, the synthetic adipose tables) on the path
its timing runs.  Skipped where the reference is not installed.
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
    ids[:, :, :3] = 3                     # adipose entrance layer (this library's synthetic table)
    geo = Geometry.from_ids((0.016, 0.014, 0.04), ids,
                            (Material.WATER, Material.BONE_COMPACT, Material.MUSCLE_SKELETAL,
                             Material.ADIPOSE_SYNTH))
    cfg = SolverConfig(
        geometry=geo,
        beam=Beam(n_protons=1e6, energy=40.0, energy_spread=1.0, sigma=(0.002, 0.0025), center=(0.001, -0.0005)),
        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                          moving_active_domain=True))
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    return cfg, MaterialMap.from_geometry(geo, Grid.from_geometry(geo))


def test_reference_material_map_keys_tables_by_name():
    bench.import_installed_reference()
    cfg, mm = _phantom()
    rmm = bench.reference_material_map(cfg, mm)
    assert [m.value for m in rmm.materials] == ["G4_WATER", "G4_BONE_COMPACT_ICRU", "G4_MUSCLE_SKELETAL_ICRP",
                                                "ADIPOSE_SYNTH"]
    assert np.array_equal(rmm.ids, mm.ids)


def test_synthetic_tables_read_back_exactly():
    """The reference's own loaders read the ADIPOSE_SYNTH tables back as the
    same doubles this library marches with."""
    bench.import_installed_reference()
    from proton_solver.physics.materials import density, radiation_length
    from proton_solver.physics.nuclear import _load_nuclear_table
    from proton_solver.physics.scattering import _load_transport_table
    from proton_solver.physics.stopping_power import load_stopping_power_table
    from proton_dose_m1_b200.physics.tables import material_tables
    cfg, mm = _phantom()
    adipose = bench.reference_material_map(cfg, mm).materials[3]
    t = material_tables("ADIPOSE_SYNTH")
    sp = load_stopping_power_table(adipose)
    assert np.array_equal(sp["energy_mev"], t.sp_energy)
    assert np.array_equal(sp["electronic_stopping_power_mev_per_m"], t.sp_value)
    e, v = _load_transport_table(adipose)
    assert np.array_equal(e, t.tr_energy) and np.array_equal(v, t.tr_value)
    e, v = _load_nuclear_table(adipose)[:2]
    assert np.array_equal(e, t.nuc_energy) and np.array_equal(v, t.nuc_value)
    assert density(adipose) == t.density and radiation_length(adipose) == t.radiation_length


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


def test_reference_arm_waits_for_the_last_spots(monkeypatch, capsys):
    """Three spots on two workers, polled every half second: one worker runs
    out of spots and exits while the other still marches; the arm waits for
    it and prints one line with every spot."""
    import argparse
    import json
    import os
    if len(os.sched_getaffinity(0)) < 2 * bench.REF_THREADS_PER_WORKER:
        pytest.skip("needs two reference workers")
    monkeypatch.setattr(bench, "REF_POLL_S", 0.5)
    args = argparse.Namespace(workload="water40", steps=3, warmup=1)
    bench.run_reference_numba(args, 1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["cpu_baseline"]["kind"] == "reference"
    assert line["value"] > 0.0 and line["steps"] == 3
    # three marches of the same spot on the same thread count; the count itself
    # (458 here) may move by a step with the host CPU's evaluation order
    import re
    steps = json.loads(re.search(r"(\[[0-9, ]+\]) energy steps", line["cpu_baseline"]["sample"]).group(1))
    assert len(steps) == 3 and len(set(steps)) == 1 and 440 <= steps[0] <= 480


@pytest.mark.parametrize("workload", ["pelvis1024", "field256"])
def test_field_spot_through_the_reference_energies(workload):
    """A spot of a benchmark field (the pelvis: 256x256x320 at 1 mm with the
    synthetic adipose shell on its written tables; field256: 128x128x256 at
    1 mm with ellipsoids of water, lung, bone and muscle), the lowest of four
    energy quantiles, marched by the reference on its moving box and by the
    oracle through the reference's own energies: the dose within the
    full-size bar (the floor of equally valid evaluation orders at these grid
    sizes; measured 1.4e-11 of the maximum on the pelvis spot, 9.2e-10 on the
    field256 spot, whose ellipsoids put material interfaces across the beam).
    With the CFL rule the two step sequences can part by ~1e-11 MeV after a few
    steps: the bound's sensitivity to evaluation order."""
    from tests.cases import FULL_SIZE_DOSE_RTOL
    from oracle.oracle import OracleProblem
    ps = bench.import_installed_reference()
    from proton_solver.numerics.energy import energy_march as reference_march
    cfg, mm, _ = bench.reference_sample(workload, 4)[0]
    rcfg, grid, inflow = bench.reference_spot(ps, cfg)
    _, dose_r, energies_r, _ = reference_march(None, bench.reference_material_map(cfg, mm), grid, inflow, rcfg, np)
    energies_r = np.asarray(energies_r)
    prob = OracleProblem(cfg, mm)
    prob.set_schedule(energies_r)
    _, dose_o, energies_o, _ = prob.march(None)
    assert np.array_equal(np.asarray(energies_o), energies_r)
    scale = float(np.max(dose_r))
    assert scale > 0.0
    assert float(np.max(np.abs(np.asarray(dose_o) - dose_r))) <= FULL_SIZE_DOSE_RTOL * scale
    assert abs(float(np.max(dose_o)) - scale) <= FULL_SIZE_DOSE_RTOL * scale
