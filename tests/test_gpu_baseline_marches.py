"""The first three benchmark configurations against the reference's own marches.

tests/golden/baseline_marches.npz holds, for cfg1 (40x40x200 @1 mm water,
CSDA only, full domain), cfg2 (80x80x400 @0.5 mm with a 2 cm bone slab, full
physics, moving box) and cfg3 (80x80x400 @0.5 mm, bone for x > 0, full
physics, moving box), the energies, maximum dose and depth-dose curve of the
unmodified reference run here (tests/golden/make_golden.py baseline).  The
plain FP64 path (its moving box where the case asks for it) marches each
case at full size:

* through the reference's own energies (fixed-schedule mode): maximum dose
  and depth-dose curve to cases.FULL_SIZE_DOSE_RTOL of the maximum (cfg3's
  depth-dose curve, across a material interface parallel to the beam, to
  cases.LATERAL_INTERFACE_DEPTH_DOSE_RTOL: the rounding floor measured there);
* with the CFL rule: the step sequence and the maximum dose as far as the
  rounding floor of the CFL bound allows (see tests/test_gpu_kats_full.py):
  the step count within 2% and the maximum dose within 2e-3.
"""

import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap
from tests import cases

pytestmark = pytest.mark.gpu

_FILE, _SPEC = cases.GOLDEN / "baseline_marches.npz", cases.GOLDEN / "baseline_marches.json"
MARCHES = dict(np.load(_FILE)) if _FILE.exists() and _SPEC.exists() else {}
SPECS = json.loads(_SPEC.read_text()) if MARCHES else {}
NAMES = sorted(k.rsplit("/", 1)[0] for k in MARCHES if k.endswith("/energies"))


def _config(spec):
    objects = [Box(*o[:6], Material[o[6]]) for o in spec["objects"]]
    phys = Physics(**{k: (Scattering[v] if k == "scattering" else v) for k, v in spec["physics"].items()})
    return SolverConfig(geometry=Geometry(size=tuple(spec["size"]), resolution=tuple(spec["resolution"]),
                                          objects=objects),
                        beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)),
                        physics=phys,
                        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                          moving_active_domain=spec["moving"]))


def _lateral_interface(spec):
    """An object whose x or y faces lie inside the grid: a material interface
    parallel to the beam."""
    hx, hy = spec["size"][0] / 2, spec["size"][1] / 2
    return any(-hx < o[0] or o[1] < hx or -hy < o[2] or o[3] < hy for o in spec["objects"])


def _march(cfg, schedule=None):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    try:
        if schedule is not None:
            plan.set_schedule(schedule)
        U0 = None if cfg.numerics.moving_active_domain else np.zeros((4, *grid.shape))
        _, dose, energies, _ = plan.march(U0)
    finally:
        plan.close()
    return dose.cpu().numpy(), energies


@pytest.mark.parametrize("name", NAMES)
def test_reference_steps_reproduce_the_reference_march(name):
    cfg = _config(SPECS[name])
    sched = MARCHES[f"{name}/energies"]
    dose, energies = _march(cfg, sched)
    np.testing.assert_array_equal(energies, sched)
    ref_max = float(MARCHES[f"{name}/max_dose"])
    assert abs(float(dose.max()) - ref_max) <= cases.FULL_SIZE_DOSE_RTOL * ref_max
    idd, ref_idd = dose.sum(axis=(0, 1)), MARCHES[f"{name}/depth_dose"]
    bar = cases.LATERAL_INTERFACE_DEPTH_DOSE_RTOL if _lateral_interface(SPECS[name]) else cases.FULL_SIZE_DOSE_RTOL
    assert np.abs(idd - ref_idd).max() <= bar * ref_idd.max()


@pytest.mark.parametrize("name", NAMES)
def test_cfl_rule_follows_the_reference_march(name):
    cfg = _config(SPECS[name])
    sched = MARCHES[f"{name}/energies"]
    dose, energies = _march(cfg)
    assert abs(len(energies) - len(sched)) <= 0.02 * len(sched)
    ref_max = float(MARCHES[f"{name}/max_dose"])
    assert abs(float(dose.max()) - ref_max) <= 2e-3 * ref_max
