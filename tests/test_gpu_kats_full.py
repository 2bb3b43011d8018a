"""The published deterministic results of the reference at full size.

The reference publishes, for its WENO-Z runs (thesis_results/**/weno_z/
metrics.json), the maximum dose, R80 and the distal falloff width of each
deterministic march; tests/golden/published_kats_full.json collects them
for four grids: 24x24x200 (1 mm cubes), 50x50x200, and 100x100x400
(0.24 x 0.24 x 0.5 mm) both on the full domain and on the reference's moving
active box (numerics/moving_active_domain.py).  tests/golden/
published_schedules.npz holds, for the cases the unmodified reference was
run on here, its own energy steps (and it reproduces the published maximum
to the last digit).

Two comparisons per case, on the plain FP64 path (or its moving box):

* with the reference's own energy steps (the fixed-schedule mode,
  pdm1_plan_set_schedule): the maximum dose to cases.FULL_SIZE_DOSE_RTOL
  (1e-7; the measured distances are 4e-10 .. 3.4e-8, and two builds of the
  oracle that differ only in FMA contraction differ by 6.5e-9 at this size) --
  the arithmetic of every step at full size;
* with the CFL rule: the step sequence follows the reference's while the
  CFL bound is set by cells that hold real fluence, but on several of these
  grids it is set, at some step, by a cell of the lateral boundary whose
  fluence is ~1e-18 of the peak: its value is rounding noise (it differs by
  1e-5 relative between two correct FP64 evaluation orders), and so is the
  bound it sets (e.g. coarse_grid_1mm reduced water: step 18 differs by
  6e-7 MeV, 626 against 628 steps, maximum dose 6.5e-4 apart; the two oracle
  builds themselves part at step 8 and end 3.4e-7 apart).  Where the step
  sequence equals the reference's the bar is the same as above; where it does
  not, the maximum dose must agree to 2e-3 and R80 to 0.05 mm.
"""

import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from proton_dose_m1_b200 import metrics
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap
from tests import cases

pytestmark = pytest.mark.gpu

KATS = json.loads((cases.GOLDEN / "published_kats_full.json").read_text())
_SCHED_FILE = cases.GOLDEN / "published_schedules.npz"
SCHEDULES = dict(np.load(_SCHED_FILE)) if _SCHED_FILE.exists() else {}
R80_TOL_MM = 1e-6
NOISE_DOSE_RTOL = 2e-3
NOISE_R80_MM = 0.05


def _march(cfg, schedule=None):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    try:
        if schedule is not None:
            plan.set_schedule(schedule)
        _, dose, energies, _ = plan.march(None)
    finally:
        plan.close()
    return dose.cpu().numpy(), energies, grid


def _range(kat, dose, grid):
    if kat["peak_search_from_mm"] is None:
        return None, None
    r80, dfw = metrics.range_metrics(grid.z, dose, kat["peak_search_from_mm"] / 1000.0)
    return 1000.0 * r80, 1000.0 * dfw


@pytest.mark.parametrize("case", sorted(KATS))
def test_published_full_size_cfl_rule(case):
    kat = KATS[case]
    cfg = cases.published_config(kat)
    dose, energies, grid = _march(cfg)
    assert np.all(np.diff(energies) < 0)
    ref = kat["maximum_dose_Gy"]
    rel = (float(dose.max()) - ref) / ref
    r80, dfw = _range(kat, dose, grid)
    sched = SCHEDULES.get(f"{case}/energies")
    same_steps = (sched is not None and len(sched) == len(energies) and np.array_equal(sched, energies)
                  and float(SCHEDULES[f"{case}/max_dose"]) == ref)
    if same_steps:
        assert abs(rel) <= cases.FULL_SIZE_DOSE_RTOL, rel
        if r80 is not None:
            assert abs(r80 - kat["r80_mm"]) <= R80_TOL_MM and abs(dfw - kat["dfw_mm"]) <= R80_TOL_MM
    else:
        assert abs(rel) <= NOISE_DOSE_RTOL, rel
        if r80 is not None:
            assert abs(r80 - kat["r80_mm"]) <= NOISE_R80_MM


@pytest.mark.parametrize("case", sorted(k.rsplit("/", 1)[0] for k in SCHEDULES if k.endswith("/energies")))
def test_published_full_size_reference_steps(case):
    """The march through the reference's own energies reproduces the maximum
    dose of the reference run here (the unmodified current reference) and,
    where that run reproduces the published value (the 1 mm grids; the
    50x50x200 and 100x100x400 results were published from an earlier version
    of the reference, git 3ef7a4d / e7b79c3, and differ from the current
    code's by up to 1.2e-4), the published maximum, R80 and DFW."""
    kat = KATS[case]
    cfg = cases.published_config(kat)
    sched = SCHEDULES[f"{case}/energies"]
    dose, energies, grid = _march(cfg, sched)
    np.testing.assert_array_equal(energies, sched)
    ref = float(SCHEDULES[f"{case}/max_dose"])
    rel = (float(dose.max()) - ref) / ref
    assert abs(rel) <= cases.FULL_SIZE_DOSE_RTOL, rel
    if ref == kat["maximum_dose_Gy"]:
        r80, dfw = _range(kat, dose, grid)
        if r80 is not None:
            assert abs(r80 - kat["r80_mm"]) <= R80_TOL_MM
            assert abs(dfw - kat["dfw_mm"]) <= R80_TOL_MM
