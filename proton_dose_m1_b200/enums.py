"""Enumerations of the proton_solver public API (proton_solver/enums.py:1-50).

Member names and ``Material`` values match the reference so configurations
written for it work unchanged.  ``Material`` additionally lists the two
materials whose tables ship with the reference data but which its enum
omits (AIR, MUSCLE_SKELETAL); the table loaders only use ``.value``.
ADIPOSE_SYNTH is a density-scaled water (950 kg/m^3) for phantoms with an
adipose layer, for which the reference data has no table.
"""

from enum import Enum, auto


class Backend(Enum):
    AUTO = auto()
    CPU = auto()
    GPU = auto()


class Material(Enum):
    WATER = "G4_WATER"
    BONE_COMPACT = "G4_BONE_COMPACT_ICRU"
    LUNG = "G4_LUNG_ICRP"
    AIR = "G4_AIR"
    MUSCLE_SKELETAL = "G4_MUSCLE_SKELETAL_ICRP"
    ADIPOSE_SYNTH = "ADIPOSE_SYNTH"


class SpatialScheme(Enum):
    FIRST_ORDER = auto()
    MUSCL = auto()
    WENO3 = auto()
    WENO_Z = auto()


class EnergyScheme(Enum):
    FORWARD_EULER = auto()
    BACKWARD_EULER = auto()
    TRAPEZOIDAL = auto()
    SSPRK2 = auto()
    SSPRK3 = auto()
    IF_SSPRK3 = auto()


class WaveSpeeds(Enum):
    EXACT = auto()
    UNIT = auto()


class Reference(Enum):
    NONE = auto()
    ANALYTICAL = auto()
    TOPAS = auto()
    BFP_MC = auto()
    SELF = auto()


class CoefficientInterpolation(Enum):
    LINEAR = auto()
    PCHIP = auto()


class Scattering(Enum):
    OFF = auto()
    ROSSI = auto()
    WENTZEL = auto()


class Precision(Enum):
    """Arithmetic of the transport stencil on the GPU.

    FP64: every operation in double precision (the parity path).
    FP32_FP64: WENO-Z, HLL and the stage update in single precision, with the
    realizability projection and the dose accumulation kept in double.
    """

    FP64 = auto()
    FP32_FP64 = auto()
