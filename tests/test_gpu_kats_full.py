"""The published deterministic results of the reference at full size.

The reference publishes, for its WENO-Z runs (thesis_results/**/weno_z/
metrics.json), the maximum dose, R80 and the distal falloff width of each
deterministic march; tests/golden/published_kats_full.json collects them
for four grids: 24x24x200 (1 mm cubes), 50x50x200, and 100x100x400
(0.24 x 0.24 x 0.5 mm) both on the full domain and on the reference's moving
active box (numerics/moving_active_domain.py).  Each case marches the plain
FP64 path (or its moving box) on the GPU, exactly as the reference's config
asks, and compares:

* the maximum dose, to cases.reference_rtol of itself (1e-10 with scattering;
  2e-9 near free streaming, the rounding floor between this FP64 arithmetic
  and the reference's Numba fastmath build);
* R80 and DFW (ResultMetrics.range_comparison, metrics.py:427-460, with the
  published peak-search depth), to 1e-6 mm.
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
R80_TOL_MM = 1e-6


@pytest.mark.parametrize("case", sorted(KATS))
def test_published_full_size(case):
    kat = KATS[case]
    cfg = cases.published_config(kat)
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    try:
        _, dose, energies, _ = plan.march(None)
    finally:
        plan.close()
    dmax = float(dose.max())
    ref = kat["maximum_dose_Gy"]
    assert abs(dmax - ref) <= cases.reference_rtol(cfg) * ref, (dmax, ref, (dmax - ref) / ref)
    if kat["peak_search_from_mm"] is not None:
        d = dose.cpu().numpy()
        r80, dfw = metrics.range_metrics(grid.z, d, kat["peak_search_from_mm"] / 1000.0)
        assert abs(1000.0 * r80 - kat["r80_mm"]) <= R80_TOL_MM
        assert abs(1000.0 * dfw - kat["dfw_mm"]) <= R80_TOL_MM
    assert np.all(np.diff(energies) < 0)
