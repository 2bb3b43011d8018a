"""Material coefficient tables and properties.

The tables are the reference's Geant4 exports (data/stopping_power,
data/wentzel_transport, data/nuclear_attenuation, data/materials.csv),
packed into ``data/material_tables.npz`` by ``data/pack_tables.py``.
Each table is 6000 log-spaced nodes from 1e-4 to 300 MeV.

``ADIPOSE_SYNTH`` has no Geant4 export: it is water scaled to 950 kg/m^3.
Every coefficient here is per unit length and proportional to density for a
fixed composition, so S, Sigma_tr and Sigma_r are the water values x 0.95 and
the radiation length (in metres) is water's / 0.95.  It stands in for the
adipose shell of synthetic pelvis phantoms.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache
from pathlib import Path

import numpy as np

from ..enums import Material

TABLE_FILE = Path(__file__).resolve().parents[1] / "data" / "material_tables.npz"


@dataclass(frozen=True)
class MaterialTables:
    name: str
    sp_energy: np.ndarray      # MeV
    sp_value: np.ndarray       # electronic stopping power, MeV/m
    tr_energy: np.ndarray
    tr_value: np.ndarray       # Wentzel-VI first transport coefficient, 1/m
    nuc_energy: np.ndarray
    nuc_value: np.ndarray      # nuclear removal coefficient, 1/m
    density: float             # kg/m^3
    radiation_length: float    # m


@lru_cache
def _archive():
    with np.load(TABLE_FILE) as z:
        return {k: z[k] for k in z.files}


SYNTHETIC_SCALED = {"ADIPOSE_SYNTH": ("G4_WATER", 950.0)}


@lru_cache
def material_tables(material: Material | str) -> MaterialTables:
    name = material.value if isinstance(material, Material) else str(material)
    if name in SYNTHETIC_SCALED:
        base_name, rho = SYNTHETIC_SCALED[name]
        base = material_tables(base_name)
        f = rho / base.density
        return MaterialTables(name=name, sp_energy=base.sp_energy, sp_value=base.sp_value * f,
                              tr_energy=base.tr_energy, tr_value=base.tr_value * f,
                              nuc_energy=base.nuc_energy, nuc_value=base.nuc_value * f,
                              density=rho, radiation_length=base.radiation_length / f)
    a = _archive()
    if f"{name}/sp_energy" not in a:
        raise FileNotFoundError(f"No stopping-power data found for {name}.")
    tables = MaterialTables(
        name=name,
        sp_energy=a[f"{name}/sp_energy"], sp_value=a[f"{name}/sp_value"],
        tr_energy=a[f"{name}/tr_energy"], tr_value=a[f"{name}/tr_value"],
        nuc_energy=a[f"{name}/nuc_energy"], nuc_value=a[f"{name}/nuc_value"],
        density=float(a[f"{name}/density"]),
        radiation_length=float(a[f"{name}/radiation_length"]),
    )
    _validate(tables)
    return tables


def _validate(t: MaterialTables) -> None:
    """The table checks of physics/stopping_power.py:73-91 and nuclear.py:60-79."""
    for energy, label in ((t.sp_energy, "Stopping-power"), (t.tr_energy, "Wentzel"),
                          (t.nuc_energy, "Nuclear-attenuation")):
        if len(energy) < 2:
            raise ValueError(f"{label} table for {t.name} must contain at least two points.")
        if not np.all(np.diff(energy) > 0.0):
            raise ValueError(f"{label} energies for {t.name} must be strictly increasing.")
    if not np.all(np.isfinite(t.sp_value)) or not np.all(t.sp_value > 0.0):
        raise ValueError(f"Stopping-power values for {t.name} must be finite and positive.")
    if not np.all(np.isfinite(t.nuc_value)) or np.any(t.nuc_value < 0.0):
        raise ValueError(f"Nuclear-removal coefficients for {t.name} must be finite and non-negative.")
    if not np.isfinite(t.radiation_length) or t.radiation_length <= 0.0:
        raise ValueError(f"Invalid radiation length for {t.name}: {t.radiation_length}")


def density(material: Material) -> float:
    """Material density in kg/m^3 (physics/materials.py:29-38)."""
    return material_tables(material).density


def radiation_length(material: Material) -> float:
    """Radiation length in metres (physics/materials.py:40-63)."""
    return material_tables(material).radiation_length
