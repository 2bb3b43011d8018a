"""Write this library's synthetic material tables into the installed
reference's data directory, in the reference's own table formats, so that the
reference marches the same phantoms.

``ADIPOSE_SYNTH`` (water scaled to 950 kg/m^3: stopping power, Wentzel-VI
transport and nuclear removal x 0.95, radiation length / 0.95) has no Geant4
export.  The reference finds a material's tables by its name
(physics/stopping_power.py:14-30, scattering.py:23-52, nuclear.py:30-60, and
the density and radiation length in materials.csv, materials.py:16-60), so one
CSV per table directory and one materials.csv row make it a material the
reference can march.  Every value is written with the shortest decimal that
parses back to the same double, so the reference reads exactly the numbers
this library and its oracle use.

Usage:  python baseline/synth_tables.py <installed reference data directory>
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from proton_dose_m1_b200.physics.tables import SYNTHETIC_SCALED, material_tables  # noqa: E402


def _write_csv(path: Path, header: str, columns) -> None:
    rows = np.column_stack(columns)
    with open(path, "w") as f:
        f.write(header + "\n")
        for row in rows:
            f.write(",".join(repr(float(v)) for v in row) + "\n")


def write_tables(data_dir: Path) -> list[str]:
    written = []
    for name in SYNTHETIC_SCALED:
        t = material_tables(name)
        _write_csv(data_dir / "stopping_power" / f"{name}.csv",
                   "energy_mev,electronic_stopping_power_mev_per_m", (t.sp_energy, t.sp_value))
        with np.errstate(divide="ignore"):
            mfp = np.where(t.tr_value > 0, 1.0 / t.tr_value, np.inf)
        _write_csv(data_dir / "wentzel_transport" / f"{name}.csv",
                   "energy_mev,first_transport_coefficient_per_m,first_transport_mean_free_path_m",
                   (t.tr_energy, t.tr_value, mfp))
        _write_csv(data_dir / "nuclear_attenuation" / f"{name}.csv",
                   "energy_mev,nuclear_removal_coefficient_per_m", (t.nuc_energy, t.nuc_value))
        table = data_dir / "materials.csv"
        lines = table.read_text().splitlines()
        lines = [ln for ln in lines if not ln.startswith(name + ",")]
        lines.append(f"{name},{float(t.density)!r},{float(t.radiation_length)!r}")
        table.write_text("\n".join(lines) + "\n")
        written.append(name)
    return written


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: synth_tables.py <installed reference data directory>")
    print("synthetic tables:", ", ".join(write_tables(Path(sys.argv[1]))))
