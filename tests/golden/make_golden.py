"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the unmodified reference ``proton_solver`` (imported from its source
tree, FP64 NumPy/Numba CPU path) on seeded inputs and stores inputs and
outputs as small ``.npz`` files; also collects the deterministic maxima the
reference publishes for its 2 mm coarse-grid runs.  Only this script reads
the reference; the tests read the fixtures.

Usage:  NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py <reference root> [part]

The reference imports plotting and gamma modules at import time that are not
on the energy-march path (matplotlib, pymedphys); they are replaced by empty
stub modules here.
"""

from __future__ import annotations

import json
import os
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def import_reference(root: Path):
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
    for name in ["matplotlib", "matplotlib.pyplot", "matplotlib.lines", "matplotlib.patches",
                 "mpl_toolkits", "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.art3d", "pymedphys"]:
        sys.modules[name] = types.ModuleType(name)
    sys.modules["matplotlib.lines"].Line2D = object
    sys.modules["matplotlib.patches"].Patch = object
    sys.modules["mpl_toolkits.mplot3d.art3d"].Poly3DCollection = object
    sys.path.insert(0, str(root / "src"))
    import proton_solver  # noqa: F401
    return proton_solver


def unit_vectors(ps, rng):
    from proton_solver.numerics.reconstruction_methods.weno_z import _weno_z_left_scalar
    from proton_solver.numerics.realizability import project_realizable
    from proton_solver.numerics.wave_speeds import eigenvalues
    from proton_solver.numerics.flux import hll_flux
    from proton_solver.enums import WaveSpeeds, Material, CoefficientInterpolation as CI
    from proton_solver.physics.stopping_power import stopping_power
    from proton_solver.physics.scattering import first_transport_coefficient, rossi_transport_coefficient
    from proton_solver.physics.nuclear import nuclear_removal_coefficient

    out = {}
    n = 600
    # WENO-Z stencils: smooth, steps, zeros, huge and tiny magnitudes
    smooth = np.cumsum(rng.normal(size=(n, 5)), axis=1)
    steps = np.where(rng.random((n, 5)) < 0.5, 0.0, 1.0) * rng.lognormal(0, 3, size=(n, 1))
    scale = 10.0 ** rng.uniform(-12, 12, size=(n, 1))
    w = np.concatenate([smooth, steps, smooth * scale, np.zeros((4, 5)), np.ones((4, 5))])
    out["weno_in"] = w
    out["weno_out"] = np.array([_weno_z_left_scalar(*row) for row in w])

    def states(m):
        phi = 10.0 ** rng.uniform(-6, 12, size=m)
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1)[:, None]
        f = rng.choice([0.0, 1e-12, 0.3, 0.9, 0.999999, 1.0 - 1e-10, 1.2], size=m)
        J = d * (f * phi)[:, None]
        s = np.column_stack([phi, J])
        s[: m // 20, 0] *= -1.0          # negative densities
        s[m // 20: m // 10] = 0.0        # vacuum
        return s

    P = states(n)
    out["proj_in"] = P
    out["proj_out"] = project_realizable(P.T.reshape(4, n, 1, 1).copy(), np).reshape(4, n).T
    R = out["proj_out"]
    eig = np.zeros((n, 3, 2))
    for ax in range(3):
        lo, hi = eigenvalues(R.T.reshape(4, n, 1, 1).copy(), ax, np)
        eig[:, ax, 0], eig[:, ax, 1] = lo.ravel(), hi.ravel()
    out["eig_in"], out["eig_out"] = R, eig
    L = project_realizable(states(n).T.reshape(4, n, 1, 1).copy(), np).reshape(4, n).T
    Rr = project_realizable(states(n).T.reshape(4, n, 1, 1).copy(), np).reshape(4, n).T
    hll = np.zeros((n, 3, 4))
    hllu = np.zeros((n, 3, 4))
    for ax in range(3):
        a = L.T.reshape(4, n, 1, 1).copy()
        b = Rr.T.reshape(4, n, 1, 1).copy()
        hll[:, ax] = hll_flux(a, b, ax, WaveSpeeds.EXACT, np).reshape(4, n).T
        hllu[:, ax] = hll_flux(a, b, ax, WaveSpeeds.UNIT, np).reshape(4, n).T
    out["hll_left"], out["hll_right"], out["hll_exact"], out["hll_unit"] = L, Rr, hll, hllu

    class M(__import__("enum").Enum):   # all five data/ materials by Geant4 name
        WATER = "G4_WATER"
        BONE_COMPACT = "G4_BONE_COMPACT_ICRU"
        LUNG = "G4_LUNG_ICRP"
        AIR = "G4_AIR"
        MUSCLE_SKELETAL = "G4_MUSCLE_SKELETAL_ICRP"
    mats = list(M)
    E = np.concatenate([10.0 ** rng.uniform(-4, np.log10(300.0), size=300),
                        [1e-4, 300.0, 150.0, 70.0, 1.0]])
    out["coef_energy"] = E
    out["coef_materials"] = np.array([m.value for m in mats])
    out["sp"] = np.array([[stopping_power(m, e) for e in E] for m in mats])
    out["tr_linear"] = np.array([[first_transport_coefficient(m, e, CI.LINEAR) for e in E] for m in mats])
    out["tr_pchip"] = np.array([[first_transport_coefficient(m, e, CI.PCHIP) for e in E] for m in mats])
    out["nuc_linear"] = np.array([[nuclear_removal_coefficient(m, e, CI.LINEAR) for e in E] for m in mats])
    out["nuc_pchip"] = np.array([[nuclear_removal_coefficient(m, e, CI.PCHIP) for e in E] for m in mats])
    out["rossi"] = np.array([[rossi_transport_coefficient(m, e) for e in E] for m in mats])
    np.savez_compressed(OUT / "unit_vectors.npz", **out)


def _config(ps, *, size, resolution, objects=(), beam=None, physics=None, numerics=None):
    from proton_solver import (Geometry, Box, Beam, SolverConfig, Physics, Numerics, References,
                               Reference, Backend)
    geo = Geometry(size=size, resolution=resolution, objects=list(objects))
    return SolverConfig(geometry=geo, beam=beam or Beam(), physics=physics or Physics(),
                        numerics=numerics or Numerics(), backend=Backend.CPU,
                        references=References(reference=Reference.NONE))


def operators(ps, rng):
    """Operator-level fixtures on a small heterogeneous grid."""
    from proton_solver import (Box, Beam, Material, Physics, Numerics, Scattering, EnergyScheme,
                               CoefficientInterpolation as CI, WaveSpeeds, SpatialScheme)
    from proton_solver.numerics.grid import Grid
    from proton_solver.numerics.boundary import BeamInflow
    from proton_solver.physics.materials import MaterialMap
    from proton_solver.numerics.spatial import spatial_operator
    from proton_solver.numerics import energy as en

    size, res = (0.018, 0.02, 0.024), (9, 10, 12)
    objects = [Box(-0.009, 0.0, -0.01, 0.01, 0.008, 0.016, Material.BONE_COMPACT),
               Box(0.002, 0.009, -0.01, 0.0, 0.0, 0.024, Material.LUNG)]
    beam = Beam(n_protons=1e6, energy=100.0, energy_spread=1.5, sigma=(0.003, 0.0025),
                center=(0.001, -0.0005), angular_spread=0.05)
    cases = {
        "if_full": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.IF_SSPRK3),
        "if_rossi_pchip": (Physics(scattering=Scattering.ROSSI, nuclear=True,
                                   coefficient_interpolation=CI.PCHIP), EnergyScheme.IF_SSPRK3),
        "if_nuclear_only": (Physics(nuclear=True), EnergyScheme.IF_SSPRK3),
        "ssprk3_csda": (Physics(), EnergyScheme.SSPRK3),
        "strang_ssprk3": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.SSPRK3),
        "strang_euler": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.FORWARD_EULER),
        "euler_csda": (Physics(), EnergyScheme.FORWARD_EULER),
    }
    # random realizable state: smooth bump plus noise, some vacuum
    x = np.linspace(-1, 1, res[0])[:, None, None]
    y = np.linspace(-1, 1, res[1])[None, :, None]
    z = np.linspace(0, 1, res[2])[None, None, :]
    phi = 1e9 * np.exp(-3 * (x ** 2 + y ** 2) - 5 * (z - 0.4) ** 2) * (1 + 0.3 * rng.random(res))
    phi[:, :, -2:] = 0.0
    d = rng.normal(size=(3, *res)) * 0.15
    d[2] += 1.0
    d /= np.linalg.norm(d, axis=0)
    f = rng.uniform(0.2, 1.0 - 1e-10, size=res)
    U = np.concatenate([phi[None], d * (f * phi)[None]], axis=0)
    bc_custom = np.abs(rng.normal(size=(4, res[0], res[1]))) * 1e8
    bc_custom[1:3] *= 0.1
    out = {"U": U, "size": np.array(size), "res": np.array(res), "bc_custom": bc_custom}
    E, dE = 90.0, 0.21
    out["E"], out["dE"] = E, dE
    base = _config(ps, size=size, resolution=res, objects=objects, beam=beam,
                   numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.8, max_energy_step=0.5))
    grid = Grid.from_geometry(base.geometry, np)
    mm = MaterialMap.from_geometry(base.geometry, grid, np)
    inflow = BeamInflow.from_beam(beam, grid, np)
    out["ids"] = np.asarray(mm.ids)
    out["material_names"] = np.array([m.value for m in mm.materials])
    out["inflow_spatial"] = inflow.spatial
    out["inflow_state"] = inflow.state(E, np)
    out["rhs"] = spatial_operator(U.copy(), E, grid, inflow, SpatialScheme.WENO_Z, WaveSpeeds.EXACT, np)
    out["rhs_bc"] = spatial_operator(U.copy(), E, grid, inflow, SpatialScheme.WENO_Z,
                                     WaveSpeeds.EXACT, np, boundary_state=bc_custom)
    out["rhs_unit"] = spatial_operator(U.copy(), E, grid, inflow, SpatialScheme.WENO_Z, WaveSpeeds.UNIT, np)
    out["dE_exact"] = en.compute_energy_step(U.copy(), E, mm, grid, inflow, base, np)
    unit_cfg = _config(ps, size=size, resolution=res, objects=objects, beam=beam,
                       numerics=Numerics(wave_speeds=WaveSpeeds.UNIT, cfl=0.8, max_energy_step=0.5))
    out["dE_unit"] = en.compute_energy_step(U.copy(), E, mm, grid, inflow, unit_cfg, np)
    for name, (phys, scheme) in cases.items():
        cfg = _config(ps, size=size, resolution=res, objects=objects, beam=beam, physics=phys,
                      numerics=Numerics(energy_scheme=scheme, cfl=0.8, max_energy_step=0.5))
        if scheme is EnergyScheme.IF_SSPRK3:
            Un, ed = en.if_ssprk3(U.copy(), E, dE, mm, grid, inflow, cfg, np)
        elif phys.scattering is not Scattering.OFF or phys.nuclear:
            Un, ed = en.strang_energy_step(U.copy(), E, dE, mm, grid, inflow, cfg, np)
        else:
            Un, ed = en.advance_energy_step(U.copy(), E, dE, mm, grid, inflow, cfg, np)
        out[f"step_{name}_U"], out[f"step_{name}_edep"] = Un, ed
    np.savez_compressed(OUT / "operators.npz", **out)


MARCHES = {
    # name: (size, resolution, objects, beam kwargs, physics kwargs, numerics kwargs, snapshots)
    "kat2mm_reduced_water": ((0.024, 0.024, 0.2), (12, 12, 100), [], {}, {}, {}, ()),
    "kat2mm_extended_transversal": ((0.024, 0.024, 0.2), (12, 12, 100),
                                    [(-0.012, 0.0, -0.012, 0.012, 0.0, 0.2, "BONE_COMPACT")], {},
                                    {"scattering": "WENTZEL", "nuclear": True}, {}, ()),
    "hetero_snapshots": ((0.02, 0.016, 0.06), (10, 8, 30),
                         [(-0.01, 0.01, -0.008, 0.008, 0.02, 0.03, "BONE_COMPACT"),
                          (0.0, 0.01, -0.008, 0.0, 0.035, 0.06, "LUNG")],
                         {"energy": 60.0, "energy_spread": 0.8, "sigma": (0.003, 0.002),
                          "center": (0.0015, 0.0), "angular_spread": 0.02},
                         {"scattering": "WENTZEL", "nuclear": True}, {"max_energy_step": 0.5},
                         (55.0, 30.0, 10.0)),
    "moving_box_extended": ((0.032, 0.032, 0.16), (16, 16, 64),
                            [(0.0, 0.016, -0.016, 0.016, 0.0, 0.16, "BONE_COMPACT")],
                            {"energy": 120.0, "sigma": (0.003, 0.003)},
                            {"scattering": "WENTZEL", "nuclear": True},
                            {"moving_active_domain": True, "max_energy_step": 0.5}, (60.0,)),
    "moving_box_vacuum_cfl": ((0.04, 0.04, 0.1), (20, 20, 50), [],
                              {"energy": 80.0, "sigma": (0.003, 0.003)}, {},
                              {"moving_active_domain": True, "vacuum_aware_cfl": True,
                               "max_energy_step": 0.5}, ()),
}

# the other reconstructions of reconstruction_methods/ (ghost widths 1 and 2)
_HETERO = MARCHES["hetero_snapshots"]
SCHEME_MARCHES = {
    f"scheme_{s.lower()}": (*_HETERO[:5], {**_HETERO[5], "spatial_scheme": s}, _HETERO[6])
    for s in ("FIRST_ORDER", "MUSCL", "WENO3")
}
SCHEME_MARCHES["scheme_muscl_moving_vacuum"] = (
    *MARCHES["moving_box_vacuum_cfl"][:5],
    {**MARCHES["moving_box_vacuum_cfl"][5], "spatial_scheme": "MUSCL"}, ())


def marches(ps, table=None, spec_file="marches.json"):
    from proton_solver import (Box, Beam, Material, Physics, Numerics, Scattering, EnergyScheme,
                               Solver, SpatialScheme)
    table = MARCHES if table is None else table
    for name, (size, res, objs, bk, pk, nk, snaps) in table.items():
        objects = [Box(*o[:6], Material[o[6]]) for o in objs]
        beam = Beam(**{"n_protons": 1e6, "energy": 150.0, "energy_spread": 1.0,
                       "sigma": (0.002, 0.002), **bk})
        phys = Physics(**{k: (Scattering[v] if k == "scattering" else v) for k, v in pk.items()})
        nk = {k: (SpatialScheme[v] if k == "spatial_scheme" else v) for k, v in nk.items()}
        num = Numerics(**{"energy_scheme": EnergyScheme.IF_SSPRK3, "cfl": 0.9,
                          "max_energy_step": 0.25, **nk})
        cfg = _config(ps, size=size, resolution=res, objects=objects, beam=beam, physics=phys,
                      numerics=num)
        r = Solver(cfg).solve(snapshot_energies=snaps)
        out = {"dose": r.dose, "energies": r.energies}
        if r.dose.size <= 5000:          # final states only for the smallest grid
            out["phi"], out["J"] = r.phi, r.J
        for k, (e, s) in enumerate(sorted(r.snapshots.items(), reverse=True)):
            out[f"snap{k}_energy"] = e
            out[f"snap{k}"] = s
        np.savez_compressed(OUT / f"march_{name}.npz", **out)
    spec = {n: {"size": v[0], "resolution": v[1], "objects": v[2], "beam": v[3], "physics": v[4],
                "numerics": v[5], "snapshots": v[6]} for n, v in table.items()}
    (OUT / spec_file).write_text(json.dumps(spec, indent=1))


def analytical(ps):
    """The reference's analytical CSDA dose on a small slab phantom (analytical.npz)."""
    from proton_solver import Box, Beam, Material, Numerics, EnergyScheme
    from proton_solver.numerics.grid import Grid
    from proton_solver.numerics.boundary import BeamInflow
    from proton_solver.physics.materials import MaterialMap
    from proton_solver.analytical import analytical_csda_dose
    spec = ANALYTICAL_CASE
    objects = [Box(*o[:6], Material[o[6]]) for o in spec["objects"]]
    cfg = _config(ps, size=spec["size"], resolution=spec["resolution"], objects=objects,
                  beam=Beam(**spec["beam"]),
                  numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, max_energy_step=0.5))
    grid = Grid.from_geometry(cfg.geometry, np)
    mm = MaterialMap.from_geometry(cfg.geometry, grid, np)
    dose = analytical_csda_dose(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid, np))
    np.savez_compressed(OUT / "analytical.npz", dose=dose, spec=json.dumps(spec))


ANALYTICAL_CASE = {"size": (0.02, 0.016, 0.06), "resolution": (10, 8, 60),
                   "objects": [(-0.01, 0.0, -0.008, 0.008, 0.02, 0.03, "BONE_COMPACT"),
                               (0.0, 0.01, -0.008, 0.0, 0.035, 0.05, "LUNG")],
                   "beam": {"n_protons": 1e6, "energy": 60.0, "energy_spread": 0.8, "sigma": (0.003, 0.002),
                            "center": (0.0015, 0.0)}}


def schemes(ps):
    """First-order, MUSCL and WENO3 operators on the state of operators.npz,
    and marches (scheme_marches.json)."""
    from proton_solver import Physics, Numerics, Scattering, EnergyScheme, WaveSpeeds, SpatialScheme
    from proton_solver.numerics.grid import Grid
    from proton_solver.numerics.boundary import BeamInflow
    from proton_solver.physics.materials import MaterialMap
    from proton_solver.numerics.spatial import spatial_operator
    from proton_solver.numerics import energy as en
    from proton_solver import Box, Beam, Material
    g = np.load(OUT / "operators.npz")
    U, E, dE, bc = g["U"], float(g["E"]), float(g["dE"]), g["bc_custom"]
    size, res = tuple(g["size"]), tuple(int(n) for n in g["res"])
    objects = [Box(-0.009, 0.0, -0.01, 0.01, 0.008, 0.016, Material.BONE_COMPACT),
               Box(0.002, 0.009, -0.01, 0.0, 0.0, 0.024, Material.LUNG)]
    beam = Beam(n_protons=1e6, energy=100.0, energy_spread=1.5, sigma=(0.003, 0.0025),
                center=(0.001, -0.0005), angular_spread=0.05)
    out = {}
    for s in (SpatialScheme.FIRST_ORDER, SpatialScheme.MUSCL, SpatialScheme.WENO3):
        cfg = _config(ps, size=size, resolution=res, objects=objects, beam=beam,
                      physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                      numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.8, max_energy_step=0.5,
                                        spatial_scheme=s))
        grid = Grid.from_geometry(cfg.geometry, np)
        mm = MaterialMap.from_geometry(cfg.geometry, grid, np)
        inflow = BeamInflow.from_beam(beam, grid, np)
        key = s.name.lower()
        out[f"rhs_{key}"] = spatial_operator(U.copy(), E, grid, inflow, s, WaveSpeeds.EXACT, np)
        out[f"rhs_bc_{key}"] = spatial_operator(U.copy(), E, grid, inflow, s, WaveSpeeds.EXACT, np,
                                                boundary_state=bc)
        Un, ed = en.if_ssprk3(U.copy(), E, dE, mm, grid, inflow, cfg, np)
        out[f"step_{key}_U"], out[f"step_{key}_edep"] = Un, ed
    np.savez_compressed(OUT / "schemes.npz", **out)
    marches(ps, SCHEME_MARCHES, "scheme_marches.json")


def published(root: Path):
    """Deterministic maxima/R80 the reference publishes for the 2 mm grids."""
    base = root / "thesis_results" / "robustness" / "coarse_grid_2mm"
    cases = {}
    for model in ("reduced_physics", "scattering_nuclear"):
        for case in ("homogeneous_water", "longitudinal_slabs", "transversal_slabs"):
            d = base / model / case / "weno_z"
            cfg = json.loads((d / "config.json").read_text())
            met = json.loads((d / "metrics.json").read_text())
            cases[f"{model}/{case}"] = {
                "source": f"thesis_results/robustness/coarse_grid_2mm/{model}/{case}/weno_z",
                "config": {k: cfg[k] for k in ("beam", "geometry", "numerics", "physics")},
                "maximum_dose_Gy": met["maximum_dose"]["deterministic_Gy"],
                "r80_mm": met["range"]["deterministic_r80_mm"],
                "dfw_mm": met["range"]["deterministic_dfw_mm"],
                "peak_search_from_mm": met["range"]["peak_search_from_mm"],
            }
    (OUT / "published_kats.json").write_text(json.dumps(cases, indent=1))


# Groups of published WENO-Z runs at full size (a GPU march each; the CPU
# oracle is pinned on the 2 mm grids of published()):
#   coarse_grid_1mm  24x24x200, 1 mm cubes;   coarse_grid  50x50x200;
#   full             100x100x400 (0.24 x 0.24 x 0.5 mm), static full domain;
#   moving           the same grids on the reference's moving active box.
FULL_GROUPS = {
    "coarse_grid_1mm": "thesis_results/robustness/coarse_grid_1mm/{model}/{case}/weno_z",
    "coarse_grid": "thesis_results/robustness/coarse_grid/{model}/{case}/weno_z",
    "full": "thesis_results/{model}/{case}/weno_z",
    "moving": "thesis_results/robustness/moving_active_domain/{model}/{case}/weno_z",
}


def published_full(root: Path):
    """Deterministic maxima, R80 and DFW the reference publishes for its
    WENO-Z runs on finer grids (published_kats_full.json)."""
    cases = {}
    for group, pattern in FULL_GROUPS.items():
        for model in ("reduced_physics", "scattering_nuclear"):
            for case in ("homogeneous_water", "longitudinal_slabs", "transversal_slabs"):
                rel = pattern.format(model=model, case=case)
                d = root / rel
                cfg = json.loads((d / "config.json").read_text())
                met = json.loads((d / "metrics.json").read_text())
                cases[f"{group}/{model}/{case}"] = {
                    "source": rel,
                    "config": {k: cfg[k] for k in ("beam", "geometry", "numerics", "physics")},
                    "maximum_dose_Gy": met["maximum_dose"]["deterministic_Gy"],
                    "r80_mm": met["range"]["deterministic_r80_mm"],
                    "dfw_mm": met["range"]["deterministic_dfw_mm"],
                    "peak_search_from_mm": met["range"].get("peak_search_from_mm"),
                    "runtime_s": met["performance"]["deterministic_runtime_seconds"],
                }
    (OUT / "published_kats_full.json").write_text(json.dumps(cases, indent=1))


def _reference_config(ps, c):
    """The reference's SolverConfig for a published config dict (no reference solve)."""
    g, b, n, ph = c["geometry"], c["beam"], c["numerics"], c["physics"]
    objects = [ps.Box(o["x_min"], o["x_max"], o["y_min"], o["y_max"], o["z_min"], o["z_max"],
                      ps.Material[o["material"]]) for o in g["objects"]]
    geo = ps.Geometry(size=tuple(g["size"]), resolution=tuple(g["resolution"]),
                      background_material=ps.Material[g["background_material"]], objects=objects)
    beam = ps.Beam(n_protons=b["n_protons"], energy=b["energy"], energy_spread=b["energy_spread"],
                   sigma=tuple(b["sigma"]), center=tuple(b["center"]), angular_spread=b["angular_spread"],
                   cutoff_sigma=b["cutoff_sigma"])
    phys = ps.Physics(scattering=ps.Scattering[ph["scattering"]], nuclear=ph["nuclear"])
    num = ps.Numerics(spatial_scheme=ps.SpatialScheme[n["spatial_scheme"]],
                      energy_scheme=ps.EnergyScheme[n["energy_scheme"]], wave_speeds=ps.WaveSpeeds[n["wave_speeds"]],
                      max_energy_step=n["max_energy_step"], cfl=n["cfl"], energy_min=n["energy_min"],
                      energy_window_sigma=n["energy_window_sigma"], moving_active_domain=n["moving_active_domain"],
                      vacuum_aware_cfl=n["vacuum_aware_cfl"], active_truncation_sigma=n["active_truncation_sigma"],
                      active_guard_cells=n["active_guard_cells"])
    return ps.SolverConfig(geometry=geo, beam=beam, physics=phys, numerics=num, backend=ps.Backend.CPU,
                           references=ps.References(reference=ps.Reference.NONE))


def published_schedules(ps, groups):
    """The reference's own energy steps (and maximum dose) for the full-size
    published cases of ``groups``, run here with the unmodified reference:
    published_schedules.npz, keys '<case>/energies' and '<case>/max_dose'.
    Cases already in the file are kept."""
    kats = json.loads((OUT / "published_kats_full.json").read_text())
    out_file = OUT / "published_schedules.npz"
    out = dict(np.load(out_file)) if out_file.exists() else {}
    for name, kat in kats.items():
        if name.split("/")[0] not in groups or f"{name}/energies" in out:
            continue
        r = ps.Solver(_reference_config(ps, kat["config"])).solve()
        out[f"{name}/energies"] = np.asarray(r.energies, dtype=np.float64)
        out[f"{name}/max_dose"] = np.float64(r.dose.max())
        print(name, len(r.energies) - 1, float(r.dose.max()), r.runtime, flush=True)
        np.savez_compressed(out_file, **out)


# The first three benchmark configurations, run with the unmodified reference:
#   cfg1  40x40x200 @1 mm water, 150 MeV, sigma 3 mm, CSDA only, full domain;
#   cfg2  80x80x400 @0.5 mm water + 2 cm bone slab at 8 cm, full physics, moving box;
#   cfg3  80x80x400 @0.5 mm, bone for x > 0, full physics, moving box.
# (sigma_E 1 MeV: the reference rejects 0; IF-SSPRK3, cfl 0.9, max dE 0.5.)
BASELINE_CASES = {
    "cfg1_static": dict(size=(0.04, 0.04, 0.2), resolution=(40, 40, 200), objects=[], physics={},
                        moving=False),
    "cfg2_moving": dict(size=(0.04, 0.04, 0.2), resolution=(80, 80, 400),
                        objects=[(-0.02, 0.02, -0.02, 0.02, 0.08, 0.10, "BONE_COMPACT")],
                        physics={"scattering": "WENTZEL", "nuclear": True}, moving=True),
    "cfg3_moving": dict(size=(0.04, 0.04, 0.2), resolution=(80, 80, 400),
                        objects=[(0.0, 0.02, -0.02, 0.02, 0.0, 0.2, "BONE_COMPACT")],
                        physics={"scattering": "WENTZEL", "nuclear": True}, moving=True),
}


def baseline_marches(ps):
    """Energies, maximum dose and depth-dose curve of the reference's own march of
    the BASELINE_CASES (baseline_marches.npz + baseline_marches.json).  Cases
    already in the file are kept."""
    (OUT / "baseline_marches.json").write_text(json.dumps(
        {k: {**v, "objects": [list(o) for o in v["objects"]]} for k, v in BASELINE_CASES.items()}, indent=1))
    out_file = OUT / "baseline_marches.npz"
    out = dict(np.load(out_file)) if out_file.exists() else {}
    for name, c in BASELINE_CASES.items():
        if f"{name}/energies" in out:
            continue
        objects = [ps.Box(*o[:6], ps.Material[o[6]]) for o in c["objects"]]
        phys = ps.Physics(**{k: (ps.Scattering[v] if k == "scattering" else v) for k, v in c["physics"].items()})
        cfg = ps.SolverConfig(
            geometry=ps.Geometry(size=c["size"], resolution=c["resolution"], objects=objects),
            beam=ps.Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)),
            physics=phys,
            numerics=ps.Numerics(energy_scheme=ps.EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                                 moving_active_domain=c["moving"]),
            backend=ps.Backend.CPU, references=ps.References(reference=ps.Reference.NONE))
        r = ps.Solver(cfg).solve()
        out[f"{name}/energies"] = np.asarray(r.energies, dtype=np.float64)
        out[f"{name}/max_dose"] = np.float64(r.dose.max())
        out[f"{name}/depth_dose"] = np.asarray(r.dose.sum(axis=(0, 1)), dtype=np.float64)
        out[f"{name}/runtime_s"] = np.float64(r.runtime)
        print(name, len(r.energies) - 1, float(r.dose.max()), r.runtime, flush=True)
        np.savez_compressed(out_file, **out)


def published_configs(root: Path):
    """The canonical configurations and their hashes from the reference's own
    run directories (config.json, metadata.json of thesis_results/)."""
    out = []
    for meta in sorted((root / "thesis_results").rglob("metadata.json")):
        d = meta.parent
        out.append({"source": str(d.relative_to(root)),
                    "config": json.loads((d / "config.json").read_text()),
                    "config_hash": json.loads(meta.read_text())["config_hash"]})
    (OUT / "published_configs.json").write_text(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference root> [configs|published|schedules [groups]|baseline|schemes|analytical]")
    root = Path(sys.argv[1])
    if len(sys.argv) > 2 and sys.argv[2] == "configs":
        published_configs(root)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "published":
        published(root)
        published_full(root)
        sys.exit(0)
    ps = import_reference(root)
    if len(sys.argv) > 2 and sys.argv[2] == "baseline":
        baseline_marches(ps)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "schedules":
        published_schedules(ps, sys.argv[3].split(",") if len(sys.argv) > 3 else ["coarse_grid_1mm"])
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "schemes":
        schemes(ps)
        sys.exit(0)
    if len(sys.argv) > 2 and sys.argv[2] == "analytical":
        analytical(ps)
        sys.exit(0)
    rng = np.random.default_rng(20261203)
    published(root)
    published_full(root)
    published_configs(root)
    unit_vectors(ps, rng)
    operators(ps, rng)
    marches(ps)
    schemes(ps)
    analytical(ps)
