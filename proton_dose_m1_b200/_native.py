"""ctypes binding of libpdm1.so (the C ABI in include/pdm1.h).

The library is the only compute path: importing this module on a machine
without the built library, or calling into it without a CUDA device, raises
instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpdm1.so"

PDM1_OK = 0
ERR_ARGUMENT, ERR_RANGE, ERR_CUDA, ERR_MAX_STEPS, ERR_NO_BEAM, ERR_UNSUPPORTED, ERR_NONFINITE, ERR_TIMEOUT = range(1, 9)

_dp = C.POINTER(C.c_double)
_vp = C.c_void_p


class Table(C.Structure):
    _fields_ = [("n_nodes", C.c_int), ("energy", _dp), ("value", _dp)]


class Material(C.Structure):
    _fields_ = [("stopping_power", Table), ("transport", Table), ("nuclear", Table),
                ("density", C.c_double), ("radiation_length", C.c_double)]


class Problem(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("n_materials", C.c_int), ("materials", C.POINTER(Material)),
                ("ids", C.POINTER(C.c_int32)), ("inflow_spatial", _dp),
                ("beam_energy", C.c_double), ("energy_spread", C.c_double),
                ("angular_spread", C.c_double),
                ("scattering", C.c_int), ("nuclear", C.c_int), ("interpolation", C.c_int),
                ("energy_scheme", C.c_int), ("wave_speeds", C.c_int),
                ("max_energy_step", C.c_double), ("cfl", C.c_double),
                ("energy_min", C.c_double), ("energy_window_sigma", C.c_double),
                ("moving_active_domain", C.c_int), ("vacuum_aware_cfl", C.c_int),
                ("active_guard_cells", C.c_int), ("active_relative_tolerance", C.c_double),
                ("precision", C.c_int), ("spatial_scheme", C.c_int), ("phantom_cfl_floor", C.c_int)]


class BeamDesc(C.Structure):
    _fields_ = [("energy", C.c_double), ("energy_spread", C.c_double),
                ("angular_spread", C.c_double), ("inflow_spatial", _dp)]


class MarchInfo(C.Structure):
    _fields_ = [("n_steps", C.c_int), ("n_snapshots", C.c_int), ("final_state_valid", C.c_int),
                ("graph_replays", C.c_int), ("kernel_launches", C.c_int),
                ("stage_launches", C.c_int), ("stage_ms", C.c_double),
                ("cell_steps", C.c_double), ("max_box_cells", C.c_double),
                ("box_grow_events", C.c_int), ("box_fallbacks", C.c_int)]


BOX_FEATURES, BOX_OUTPUTS, BOX_PARAMS, RECORD_WIDTH = 16, 6, 5638, 40


class BoxModel(C.Structure):
    _fields_ = [("params", C.POINTER(C.c_float)),
                ("x_mean", C.c_float * BOX_FEATURES), ("x_inv_std", C.c_float * BOX_FEATURES),
                ("y_scale", C.c_float * BOX_OUTPUTS), ("y_offset", C.c_float * BOX_OUTPUTS),
                ("margin_min", C.c_int), ("margin_max", C.c_int),
                ("grow_cells", C.c_int), ("extra_max", C.c_int),
                ("leak_tolerance", C.c_double)]


_lib = None


def lib():
    """Load libpdm1.so once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is not built; run `python -m proton_dose_m1_b200.build` "
                "(the M1 march has no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        L.pdm1_last_error.restype = C.c_char_p
        L.pdm1_version.restype = C.c_char_p
        L.pdm1_plan_create.argtypes = [C.POINTER(Problem), C.POINTER(_vp)]
        L.pdm1_plan_destroy.argtypes = [_vp]
        L.pdm1_plan_workspace_bytes.argtypes = [_vp]
        L.pdm1_plan_workspace_bytes.restype = C.c_size_t
        L.pdm1_pool_cached_bytes.argtypes = []
        L.pdm1_pool_cached_bytes.restype = C.c_size_t
        L.pdm1_pool_release.argtypes = []
        L.pdm1_pool_release.restype = C.c_int
        L.pdm1_plan_set_staging.argtypes = [_vp, C.c_int]
        L.pdm1_plan_set_schedule.argtypes = [_vp, _dp, C.c_int]
        L.pdm1_march.argtypes = [_vp, _vp, _vp, _vp, C.c_int, _dp, C.c_int, _vp, _dp,
                                 C.POINTER(MarchInfo), _vp]
        L.pdm1_field_plan_create.argtypes = [C.POINTER(Problem), C.POINTER(BeamDesc), C.c_int,
                                             C.c_size_t, C.POINTER(_vp)]
        L.pdm1_field_march.argtypes = [_vp, _vp, C.c_int, C.POINTER(C.c_int), C.POINTER(MarchInfo), _vp]
        L.pdm1_march_steps.argtypes = [_vp, _vp, _vp, _vp, C.c_int, C.c_int,
                                       C.POINTER(MarchInfo), _vp]
        L.pdm1_spatial_operator.argtypes = [_vp, _vp, C.c_double, _vp, _vp, _vp]
        L.pdm1_energy_step.argtypes = [_vp, _vp, C.c_double, _dp, _vp]
        L.pdm1_advance.argtypes = [_vp, _vp, C.c_double, C.c_double, _vp, _vp]
        L.pdm1_coefficients.argtypes = [_vp, _dp, C.c_int, _dp]
        L.pdm1_weno_batch.argtypes = [_vp, _vp, C.c_int, _vp]
        L.pdm1_project_batch.argtypes = [_vp, C.c_int, _vp]
        L.pdm1_eigen_batch.argtypes = [_vp, C.c_int, _vp, C.c_int, _vp]
        L.pdm1_hll_batch.argtypes = [_vp, _vp, C.c_int, C.c_int, _vp, C.c_int, _vp]
        L.pdm1_exp_batch.argtypes = [_vp, _vp, C.c_int, _vp]
        L.pdm1_plan_set_box_model.argtypes = [_vp, C.POINTER(BoxModel)]
        L.pdm1_tile_shape.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.pdm1_plan_set_tile.argtypes = [_vp, C.c_int]
        L.pdm1_plan_autotune.argtypes = [_vp, C.c_int, C.POINTER(C.c_int), _dp, _vp]
        L.pdm1_plan_set_recorder.argtypes = [_vp, _vp, C.c_int, C.c_double, C.c_double]
        L.pdm1_mlp_train.argtypes = [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                     C.c_uint, C.POINTER(C.c_float), _vp]
        L.pdm1_mlp_gradients.argtypes = [_vp, _vp, _vp, C.c_int, C.c_float, _vp, _vp, _vp]
        L.pdm1_mlp_forward.argtypes = [_vp, _vp, C.c_int, _vp, _vp]
        L.pdm1_box_model_infer.argtypes = [C.POINTER(BoxModel), _vp, C.c_int, _vp, _vp]
        L.pdm1_analytical_csda_dose.argtypes = [C.POINTER(Problem), C.c_int, C.c_int, _vp, _vp]
        L.pdm1_gamma.argtypes = [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                 C.c_double, C.c_double, _vp, _dp, _vp]
        _lib = L
    return _lib


def check(rc: int) -> None:
    """Translate a status into the reference's exception types."""
    if rc == PDM1_OK:
        return
    msg = lib().pdm1_last_error().decode()
    if rc in (ERR_ARGUMENT, ERR_RANGE, ERR_NO_BEAM):
        raise ValueError(msg)
    if rc == ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(f"pdm1 status {rc}: {msg}")


EXPORTED_SYMBOLS = (
    "pdm1_plan_create", "pdm1_plan_destroy", "pdm1_plan_workspace_bytes", "pdm1_march",
    "pdm1_march_steps", "pdm1_field_plan_create", "pdm1_field_march",
    "pdm1_spatial_operator", "pdm1_energy_step", "pdm1_advance", "pdm1_coefficients",
    "pdm1_weno_batch", "pdm1_project_batch", "pdm1_eigen_batch", "pdm1_hll_batch",
    "pdm1_exp_batch", "pdm1_gamma", "pdm1_last_error", "pdm1_version",
    "pdm1_march_noalloc", "pdm1_plan_set_box_model", "pdm1_plan_set_recorder", "pdm1_mlp_train",
    "pdm1_mlp_gradients", "pdm1_mlp_forward", "pdm1_box_model_infer",
    "pdm1_tile_shape", "pdm1_plan_set_tile", "pdm1_plan_autotune", "pdm1_analytical_csda_dose",
    "pdm1_pool_cached_bytes", "pdm1_pool_release", "pdm1_plan_set_staging",
    "pdm1_plan_set_schedule",
)
NUM_TILES = 3
