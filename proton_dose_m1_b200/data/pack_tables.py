"""Pack the material data tables into one binary file for the package.

The proton_solver data directory ships one CSV per material and per table
(electronic stopping power, Wentzel-VI first transport coefficient, nuclear
removal coefficient) plus ``materials.csv`` (density, radiation length).
They are the inputs of the energy march, not code.  This script parses them
with the same reader the reference uses (``numpy.genfromtxt`` with a header
row, so every value is the same IEEE double) and writes
``material_tables.npz`` next to this file, which is what the package loads
at run time.

Usage:  python proton_dose_m1_b200/data/pack_tables.py <proton_solver data dir>
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

MATERIALS = (
    "G4_WATER",
    "G4_BONE_COMPACT_ICRU",
    "G4_LUNG_ICRP",
    "G4_AIR",
    "G4_MUSCLE_SKELETAL_ICRP",
)


def pack(data_dir: Path, out: Path) -> None:
    arrays: dict[str, np.ndarray] = {}
    props = np.genfromtxt(
        data_dir / "materials.csv", delimiter=",", names=True,
        dtype=None, encoding="utf-8",
    )
    for name in MATERIALS:
        sp = np.genfromtxt(data_dir / "stopping_power" / f"{name}.csv",
                           delimiter=",", names=True)
        tr = np.genfromtxt(data_dir / "wentzel_transport" / f"{name}.csv",
                           delimiter=",", names=True, dtype=float)
        nu = np.genfromtxt(data_dir / "nuclear_attenuation" / f"{name}.csv",
                           delimiter=",", names=True, dtype=float)
        row = props[props["material"] == name]
        arrays[f"{name}/sp_energy"] = np.asarray(sp["energy_mev"], float)
        arrays[f"{name}/sp_value"] = np.asarray(
            sp["electronic_stopping_power_mev_per_m"], float)
        arrays[f"{name}/tr_energy"] = np.asarray(tr["energy_mev"], float)
        arrays[f"{name}/tr_value"] = np.asarray(
            tr["first_transport_coefficient_per_m"], float)
        arrays[f"{name}/nuc_energy"] = np.asarray(nu["energy_mev"], float)
        arrays[f"{name}/nuc_value"] = np.asarray(
            nu["nuclear_removal_coefficient_per_m"], float)
        arrays[f"{name}/density"] = np.asarray(
            float(row["density_kg_m3"][0]))
        arrays[f"{name}/radiation_length"] = np.asarray(
            float(row["radiation_length_m"][0]))
    np.savez_compressed(out, **arrays)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    pack(Path(sys.argv[1]), Path(__file__).with_name("material_tables.npz"))
