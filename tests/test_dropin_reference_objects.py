"""The drop-in contract on the host side: ``energy_march`` accepts the
reference's own configuration, grid, material map and beam inflow
(proton_solver/solver.py:57-112 builds them) in place of this package's
mirrors.  The C problem this library builds from the reference's objects
must equal, field by field and array by array, the one it builds from its own
objects for the same configuration.  No GPU is needed: the problem is built on
the host before the plan is created.  Skipped where the reference is not
installed under baseline/_ref.
"""

from __future__ import annotations

import numpy as np
import pytest

import bench

pytestmark = pytest.mark.skipif(not bench.reference_installed(),
                                reason="reference not installed under baseline/_ref")

_SCALARS = ("nx", "ny", "nz", "dx", "dy", "dz", "n_materials", "beam_energy", "energy_spread",
            "angular_spread", "scattering", "nuclear", "interpolation", "energy_scheme", "wave_speeds",
            "max_energy_step", "cfl", "energy_min", "energy_window_sigma", "moving_active_domain",
            "vacuum_aware_cfl", "active_guard_cells", "active_relative_tolerance", "precision",
            "spatial_scheme", "phantom_cfl_floor")


def _array(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


def _problem_dump(p):
    out = {f: getattr(p, f) for f in _SCALARS}
    n = p.nx * p.ny * p.nz
    out["ids"] = _array(p.ids, n)
    out["inflow"] = _array(p.inflow_spatial, p.nx * p.ny)
    for k in range(p.n_materials):
        m = p.materials[k]
        for name in ("stopping_power", "transport", "nuclear"):
            t = getattr(m, name)
            out[f"m{k}/{name}/energy"] = _array(t.energy, t.n_nodes)
            out[f"m{k}/{name}/value"] = _array(t.value, t.n_nodes)
        out[f"m{k}/density"] = m.density
        out[f"m{k}/radiation_length"] = m.radiation_length
    return out


def _ours(cfg):
    from proton_dose_m1_b200.numerics.boundary import BeamInflow
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    grid = Grid.from_geometry(cfg.geometry)
    return cfg, MaterialMap.from_geometry(cfg.geometry, grid), grid, BeamInflow.from_beam(cfg.beam, grid)


def _theirs(ps, cfg_kwargs):
    """The reference's objects, built by its own constructors as Solver.solve does."""
    from proton_solver.numerics.boundary import BeamInflow
    from proton_solver.numerics.grid import Grid
    from proton_solver.physics.materials import MaterialMap
    cfg = ps.SolverConfig(**cfg_kwargs, backend=ps.Backend.CPU, references=ps.References(reference=ps.Reference.NONE))
    grid = Grid.from_geometry(cfg.geometry, np)
    return cfg, MaterialMap.from_geometry(cfg.geometry, grid, np), grid, BeamInflow.from_beam(cfg.beam, grid, np)


def _case(lib, enums, name, tmp_path):
    """One configuration in the types of ``lib`` (this package or the
    reference) and its ``enums`` module."""
    beam = dict(n_protons=2e6, energy=95.0, energy_spread=0.8, sigma=(0.0021, 0.0017), center=(0.0012, -0.0008))
    phys = dict(nuclear=True)
    num = dict(cfl=0.8, max_energy_step=0.3, moving_active_domain=name != "slab")
    if name == "slab":
        geo = dict(size=(0.02, 0.018, 0.06), resolution=(20, 18, 60),
                   objects=[lib.Box(-0.01, 0.01, -0.009, 0.009, 0.02, 0.03, enums.Material.BONE_COMPACT)])
    elif name == "lateral":
        geo = dict(size=(0.024, 0.024, 0.05), resolution=(24, 24, 100),
                   objects=[lib.Box(-0.012, 0.0, -0.012, 0.012, 0.0, 0.05, enums.Material.BONE_COMPACT),
                            lib.Box(0.004, 0.012, -0.012, 0.012, 0.01, 0.02, enums.Material.LUNG)])
    else:   # CT: HU classes lung / water / bone on the solver grid, a body mask
        rng = np.random.default_rng(7)
        hu = rng.choice([-700.0, 0.0, 40.0, 900.0], size=(16, 12, 40))
        mask = np.ones(hu.shape, bool)
        mask[:2] = False
        path = tmp_path / "ct.npz"
        np.savez(path, HU=hu, body_mask=mask)
        geo = dict(size=(0.016, 0.012, 0.04), resolution=(16, 12, 40),
                   ct_scan=lib.CTScan(path, (1e-3, 1e-3, 1e-3)), hu_partition=lib.HUPartition())
    return dict(geometry=lib.Geometry(**geo), beam=lib.Beam(**beam),
                physics=lib.Physics(scattering=enums.Scattering.WENTZEL, **phys),
                numerics=lib.Numerics(energy_scheme=enums.EnergyScheme.IF_SSPRK3, **num))


@pytest.mark.parametrize("name", ["slab", "lateral", "ct"])
def test_problem_from_reference_objects_equals_problem_from_ours(name, tmp_path):
    import proton_dose_m1_b200 as ours
    from proton_dose_m1_b200 import enums as our_enums
    from proton_dose_m1_b200.numerics.energy import _problem_struct
    ps = bench.import_installed_reference()
    from proton_solver import enums as their_enums
    mine = _ours(ours.SolverConfig(**_case(ours, our_enums, name, tmp_path)))
    theirs = _theirs(ps, _case(ps, their_enums, name, tmp_path))
    a = _problem_dump(_problem_struct(mine[0], mine[1], mine[2], mine[3].spatial)[0])
    b = _problem_dump(_problem_struct(theirs[0], theirs[1], theirs[2], theirs[3].spatial)[0])
    assert a.keys() == b.keys()
    for key in a:
        if isinstance(a[key], np.ndarray):
            assert a[key].dtype == b[key].dtype and np.array_equal(a[key], b[key]), key
        else:
            assert a[key] == b[key], key
    assert a["n_materials"] >= 2 and a["ids"].max() == a["n_materials"] - 1
