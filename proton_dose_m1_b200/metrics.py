"""Dose comparison metrics: gamma index (GPU), maximum dose, R80, distal falloff.

The range metrics restate proton_solver/metrics.py:371-460 (integrated depth
dose, deepest-peak search, R80/R20 by linear interpolation on the distal
side, search window RANGE_SEARCH_UPSTREAM upstream of the reference's deepest
peak).  The gamma index runs in libpdm1.so (``pdm1_gamma``) with the
parameters the reference passes to pymedphys.gamma (metrics.py:581-594).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native

RANGE_SEARCH_UPSTREAM = 0.02   # m, metrics.py:405


def _np(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def gamma(dose_eval, dose_ref, spacing_mm, dose_percent=1.0, distance_mm=1.0,
          lower_percent_dose_cutoff=10.0, interp_fraction=10, max_gamma=1.1,
          global_normalisation=None):
    """Return (pass_rate_percent, gamma) of ``dose_eval`` against ``dose_ref``.

    Both are (nx, ny, nz) doses on the same grid; CUDA tensors are used in
    place, NumPy arrays are copied to the current device.
    """
    import torch
    ref = torch.as_tensor(dose_ref, dtype=torch.float64).cuda().contiguous()
    ev = torch.as_tensor(dose_eval, dtype=torch.float64).cuda().contiguous()
    if ref.shape != ev.shape or ref.dim() != 3:
        raise ValueError("gamma needs two 3-D doses of the same shape")
    norm = float(ref.max()) if global_normalisation is None else float(global_normalisation)
    out = torch.empty_like(ref)
    rate = C.c_double()
    nx, ny, nz = ref.shape
    rc = _native.lib().pdm1_gamma(
        C.c_void_p(ref.data_ptr()), C.c_void_p(ev.data_ptr()), nx, ny, nz,
        float(spacing_mm[0]), float(spacing_mm[1]), float(spacing_mm[2]),
        float(dose_percent), float(distance_mm), float(lower_percent_dose_cutoff),
        int(interp_fraction), float(max_gamma), norm, C.c_void_p(out.data_ptr()),
        C.byref(rate), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc != 0:
        raise ValueError(f"pdm1_gamma failed with status {rc}")
    return rate.value, out


def integrated_depth_dose(dose):
    """Laterally integrated depth dose I(z), up to the constant dx*dy (metrics.py:346-350)."""
    return np.asarray(_np(dose), dtype=float).sum(axis=(0, 1))


def distal_peak_index(curve, window=10, min_fraction=0.3):
    """Deepest peak of a depth-dose curve (metrics.py:352-369)."""
    curve = np.asarray(curve, dtype=float)
    threshold = min_fraction * float(np.max(curve))
    n = len(curve)
    for i in range(n - 1, -1, -1):
        if curve[i] < threshold:
            continue
        lo, hi = max(0, i - window), min(n, i + window + 1)
        if curve[i] >= float(np.max(curve[lo:hi])):
            return i
    return int(np.argmax(curve))


def distal_depth(z, curve, level, z_from=None):
    """Depth where the curve falls to level * peak on the distal side (metrics.py:371-398)."""
    z = np.asarray(z, dtype=float)
    curve = np.asarray(curve, dtype=float)
    i_start = 0 if z_from is None else int(np.searchsorted(z, z_from))
    i_start = min(max(i_start, 0), len(curve) - 1)
    i_peak = i_start + int(np.argmax(curve[i_start:]))
    target = level * float(curve[i_peak])
    for i in range(i_peak, len(curve) - 1):
        if curve[i] >= target > curve[i + 1]:
            return float(z[i] + (target - curve[i]) * (z[i + 1] - z[i]) / (curve[i + 1] - curve[i]))
    return None


def range_metrics(z, dose, z_from=None):
    """(R80, DFW = R20 - R80) in metres (metrics.py:407-425)."""
    idd = integrated_depth_dose(dose)
    r80 = distal_depth(z, idd, 0.8, z_from)
    r20 = distal_depth(z, idd, 0.2, z_from)
    if r80 is None or r20 is None:
        return r80, None
    return r80, r20 - r80


def range_comparison(z, dose, reference):
    """R80 and DFW of ``dose`` against ``reference`` in mm (metrics.py:427-460)."""
    z = np.asarray(z, dtype=float)
    idd_ref = integrated_depth_dose(reference)
    z_from = float(z[distal_peak_index(idd_ref)]) - RANGE_SEARCH_UPSTREAM
    r80, dfw = range_metrics(z, dose, z_from)
    r80_ref, dfw_ref = range_metrics(z, reference, z_from)
    mm = lambda v: None if v is None else 1000.0 * v
    diff = lambda a, b: None if a is None or b is None else 1000.0 * (a - b)
    return {"r80_mm": mm(r80), "reference_r80_mm": mm(r80_ref), "r80_difference_mm": diff(r80, r80_ref),
            "dfw_mm": mm(dfw), "reference_dfw_mm": mm(dfw_ref), "dfw_difference_mm": diff(dfw, dfw_ref),
            "peak_search_from_mm": 1000.0 * z_from}


def compare(dose, reference, grid, gamma_cases=((1.0, 1.0),)):
    """Score a dose against a reference dose the way the reference's thesis scripts do."""
    d, r = _np(dose), _np(reference)
    rmax = float(r.max())
    out = {"maximum_dose_Gy": float(d.max()), "reference_maximum_dose_Gy": rmax,
           "maximum_dose_relative_difference": (float(d.max()) - rmax) / rmax,
           "max_abs_difference_over_max": float(np.abs(d - r).max()) / rmax}
    spacing = (grid.dx * 1000.0, grid.dy * 1000.0, grid.dz * 1000.0)
    for dd, dta in gamma_cases:
        rate, _ = gamma(dose, reference, spacing, dd, dta)
        out[f"gamma_{dd:g}pct_{dta:g}mm_pass_percent"] = rate
    out["range"] = range_comparison(grid.z, d, r)
    return out
