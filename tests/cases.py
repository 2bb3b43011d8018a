"""Shared construction of the golden cases from the committed fixture specs."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200.enums import (CoefficientInterpolation, EnergyScheme, Material,
                                       Scattering, SpatialScheme, WaveSpeeds)

GOLDEN = Path(__file__).resolve().parent / "golden"

# Dose parity bars against the reference's own fixtures, relative to the
# maximum dose.  With scattering (Wentzel-VI) the oracle lands within 1e-10 of
# every reference fixture (measured: <= 9.4e-12 on the marches, <= 4.2e-12 on
# the published 2 mm maxima), so the bar is 1e-10.  Without scattering the
# fluence streams almost freely: the M1 closure's isotropic part
# 0.5*(1-chi) falls to ~1e-10 and one-ulp differences in chi move the
# transverse fluxes at 1e-6 relative.  There the distance is a rounding floor,
# not a defect: 1.9e-10 .. 1.4e-9 on the published 2 mm reduced-physics maxima,
# 6.2e-10 on kat2mm_reduced_water; builds of the oracle with FMA contraction
# (5.6e-10) or with fast-math reassociation (1.8e-9) do not get closer, and the
# reference itself evaluates its HLL loop under Numba fastmath.  The bar there
# is 2e-9.
REFERENCE_DOSE_RTOL = 1e-10
FREE_STREAMING_DOSE_RTOL = 2e-9


# At full size (24x24x200 .. 100x100x400) the same rounding floor grows: with the
# reference's own energy steps the oracle (and this library, bit for bit) lands
# 4e-10 .. 3.4e-8 from the reference run, and three builds of the oracle
# (contraction off, FMA, fast-math reassociation) spread over 4.4e-8 on
# coarse_grid/reduced_physics/transversal_slabs.  The full-size bar is 1e-7.
FULL_SIZE_DOSE_RTOL = 1e-7

# A material interface parallel to the beam (bone for x > 0 in 80x80x400 at
# 0.5 mm) makes the fluence at a given energy jump across the beam, where
# WENO-Z's nonlinear weights amplify rounding: through the same 853 energies,
# two oracle builds differing only in FMA contraction end 6.0e-4 of the
# maximum apart in some voxel and 3.4e-6 of its maximum apart in the
# depth-dose curve (the reference run is 4.9e-4 / 2.4e-6 from the committed
# build), while the maximum dose agrees to 2e-8.  On a z slab of the same
# size the spread stays at the 1e-10 floor.  The depth-dose bar there is 1e-5.
LATERAL_INTERFACE_DEPTH_DOSE_RTOL = 1e-5


def reference_rtol(cfg) -> float:
    """The parity bar against the reference for configuration ``cfg``."""
    return REFERENCE_DOSE_RTOL if cfg.physics.scattering.name != "OFF" else FREE_STREAMING_DOSE_RTOL


def load(name: str):
    return np.load(GOLDEN / name)


def march_specs() -> dict:
    return json.loads((GOLDEN / "marches.json").read_text())


def scheme_march_specs() -> dict:
    """Marches with the first-order, MUSCL and WENO3 reconstructions."""
    return json.loads((GOLDEN / "scheme_marches.json").read_text())


SCHEMES = (SpatialScheme.FIRST_ORDER, SpatialScheme.MUSCL, SpatialScheme.WENO3)


def march_config(spec: dict) -> SolverConfig:
    objects = [Box(*o[:6], Material[o[6]]) for o in spec["objects"]]
    beam_kw = {"n_protons": 1e6, "energy": 150.0, "energy_spread": 1.0, "sigma": (0.002, 0.002)}
    beam_kw.update({k: tuple(v) if isinstance(v, list) else v for k, v in spec["beam"].items()})
    phys = Physics(**{k: Scattering[v] if k == "scattering" else v for k, v in spec["physics"].items()})
    num_kw = {"energy_scheme": EnergyScheme.IF_SSPRK3, "cfl": 0.9, "max_energy_step": 0.25}
    num_kw.update({k: SpatialScheme[v] if k == "spatial_scheme" else v for k, v in spec["numerics"].items()})
    geo = Geometry(size=tuple(spec["size"]), resolution=tuple(spec["resolution"]), objects=objects)
    return SolverConfig(geometry=geo, beam=Beam(**beam_kw), physics=phys, numerics=Numerics(**num_kw))


def published_kats() -> dict:
    return json.loads((GOLDEN / "published_kats.json").read_text())


def published_config(case: dict) -> SolverConfig:
    c = case["config"]
    g, b, n, p = c["geometry"], c["beam"], c["numerics"], c["physics"]
    objects = [Box(o["x_min"], o["x_max"], o["y_min"], o["y_max"], o["z_min"], o["z_max"],
                   Material[o["material"]]) for o in g["objects"]]
    geo = Geometry(size=tuple(g["size"]), resolution=tuple(g["resolution"]),
                   background_material=Material[g["background_material"]], objects=objects)
    beam = Beam(n_protons=b["n_protons"], energy=b["energy"], energy_spread=b["energy_spread"],
                sigma=tuple(b["sigma"]), center=tuple(b["center"]),
                angular_spread=b["angular_spread"], cutoff_sigma=b["cutoff_sigma"])
    phys = Physics(scattering=Scattering[p["scattering"]], nuclear=p["nuclear"],
                   coefficient_interpolation=CoefficientInterpolation[p.get("coefficient_interpolation", "LINEAR")])
    num = Numerics(spatial_scheme=SpatialScheme[n["spatial_scheme"]],
                   energy_scheme=EnergyScheme[n["energy_scheme"]],
                   wave_speeds=WaveSpeeds[n["wave_speeds"]], max_energy_step=n["max_energy_step"],
                   cfl=n["cfl"], energy_min=n["energy_min"],
                   energy_window_sigma=n["energy_window_sigma"],
                   moving_active_domain=n["moving_active_domain"],
                   vacuum_aware_cfl=n["vacuum_aware_cfl"],
                   active_truncation_sigma=n["active_truncation_sigma"],
                   active_guard_cells=n["active_guard_cells"])
    return SolverConfig(geometry=geo, beam=beam, physics=phys, numerics=num)


OPERATOR_CASES = {
    "if_full": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.IF_SSPRK3),
    "if_rossi_pchip": (Physics(scattering=Scattering.ROSSI, nuclear=True,
                               coefficient_interpolation=CoefficientInterpolation.PCHIP),
                       EnergyScheme.IF_SSPRK3),
    "if_nuclear_only": (Physics(nuclear=True), EnergyScheme.IF_SSPRK3),
    "ssprk3_csda": (Physics(), EnergyScheme.SSPRK3),
    "strang_ssprk3": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.SSPRK3),
    "strang_euler": (Physics(scattering=Scattering.WENTZEL, nuclear=True), EnergyScheme.FORWARD_EULER),
    "euler_csda": (Physics(), EnergyScheme.FORWARD_EULER),
}


def operator_geometry():
    g = load("operators.npz")
    mats = tuple(next(m for m in Material if m.value == n) for n in g["material_names"])
    geo = Geometry.from_ids(tuple(float(s) for s in g["size"]), g["ids"], mats)
    beam = Beam(n_protons=1e6, energy=100.0, energy_spread=1.5, sigma=(0.003, 0.0025),
                center=(0.001, -0.0005), angular_spread=0.05)
    return g, geo, beam


def operator_config(name: str | None = None, **numerics) -> SolverConfig:
    _, geo, beam = operator_geometry()
    phys, scheme = OPERATOR_CASES[name] if name else (Physics(), EnergyScheme.IF_SSPRK3)
    num = Numerics(**{"energy_scheme": scheme, "cfl": 0.8, "max_energy_step": 0.5, **numerics})
    return SolverConfig(geometry=geo, beam=beam, physics=phys, numerics=num)
