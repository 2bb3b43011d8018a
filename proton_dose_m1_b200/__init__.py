"""B200-native M1 proton dose march behind the proton_solver API.

The energy march (WENO-Z + HLL + IF-SSPRK3 + realizability + CSDA dose) runs
as hand-written sm_100a CUDA in ``libpdm1.so`` (``csrc/``), called through a
plain C ABI (``include/pdm1.h``).  The Python layer mirrors the reference
package's configuration objects and its ``energy_march`` entry point.
"""

from .beam import Beam
from .config import Accel, Numerics, OutputConfig, Physics, References, SolverConfig
from .enums import (Backend, CoefficientInterpolation, EnergyScheme, Material, Precision,
                    Reference, Scattering, SpatialScheme, WaveSpeeds)
from .geometry import Box, CTScan, Geometry, HUPartition

__all__ = [
    "Beam", "Accel", "Numerics", "OutputConfig", "Physics", "References", "SolverConfig",
    "Backend", "CoefficientInterpolation", "EnergyScheme", "Material", "Precision",
    "Reference", "Scattering", "SpatialScheme", "WaveSpeeds",
    "Box", "CTScan", "Geometry", "HUPartition", "Result", "Solver",
]


def __getattr__(name):
    # Solver and Result pull in the march shim; import them on first use
    if name == "Solver":
        from .solver import Solver
        return Solver
    if name == "Result":
        from .result import Result
        return Result
    raise AttributeError(name)
