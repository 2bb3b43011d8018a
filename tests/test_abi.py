"""The C ABI: libpdm1.so loads and exports every function include/pdm1.h declares;
host-side argument checks raise the reference's exception types."""

import re
from pathlib import Path

import numpy as np
import pytest

from proton_dose_m1_b200 import _native
from proton_dose_m1_b200 import Beam, Geometry, Numerics, SolverConfig
from proton_dose_m1_b200.enums import EnergyScheme, SpatialScheme

HEADER = Path(__file__).resolve().parents[1] / "include" / "pdm1.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(pdm1_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _native.lib()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), f"{name} missing from libpdm1.so"
    assert set(_native.EXPORTED_SYMBOLS) <= set(names)
    assert L.pdm1_version().startswith(b"pdm1")


def _cfg(**num):
    return SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)),
                        beam=Beam(energy=50.0), numerics=Numerics(**num))


def test_energy_march_argument_errors():
    from proton_dose_m1_b200.numerics.energy import energy_march, _check_supported
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.numerics.boundary import BeamInflow
    from proton_dose_m1_b200.physics.materials import MaterialMap
    cfg = _cfg()
    grid = Grid.from_geometry(cfg.geometry)
    with pytest.raises(ValueError, match="full-grid initial state"):
        energy_march(None, MaterialMap.from_geometry(cfg.geometry, grid), grid,
                     BeamInflow.from_beam(cfg.beam, grid), cfg, np)
    for scheme in SpatialScheme:   # every reconstruction of the reference has a GPU kernel
        _check_supported(_cfg(spatial_scheme=scheme))
    with pytest.raises(NotImplementedError, match="has not been migrated"):
        _check_supported(_cfg(energy_scheme=EnergyScheme.TRAPEZOIDAL))
    with pytest.raises(NotImplementedError):
        _check_supported(_cfg(active_domain=True))
    with pytest.raises(ValueError, match="Zero energy spread"):
        _check_supported(SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)),
                                      beam=Beam(energy=50.0, energy_spread=0.0)))


def test_config_validation_matches_reference():
    with pytest.raises(ValueError, match="cfl must lie"):
        Numerics(cfl=0.0)
    with pytest.raises(ValueError, match="active_guard_cells"):
        Numerics(active_guard_cells=3)
    with pytest.raises(ValueError, match="Beam center lies outside the x-domain"):
        SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)),
                     beam=Beam(energy=50.0, center=(0.02, 0.0)))
    with pytest.raises(ValueError, match="energy_min must be smaller"):
        SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)),
                     beam=Beam(energy=50.0), numerics=Numerics(energy_min=60.0))
