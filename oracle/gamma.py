"""Brute-force NumPy gamma index (test infrastructure only).

Same definition as the GPU kernel (Low et al. 1998, global, lower dose cutoff,
search lattice of spacing DTA/interp_fraction inside max_gamma*DTA, trilinear
interpolation of the evaluated dose, candidates outside the grid skipped);
used to check pdm1_gamma on small grids.
"""

from __future__ import annotations

import numpy as np


def _trilinear(D, fi, fj, fk):
    nx, ny, nz = D.shape
    def split(f, n):
        i = np.clip(np.floor(f).astype(int), 0, max(n - 2, 0))
        t = f - i if n > 1 else np.zeros_like(f)
        i1 = i + 1 if n > 1 else i
        return i, i1, t
    i, i1, ti = split(fi, nx)
    j, j1, tj = split(fj, ny)
    k, k1, tk = split(fk, nz)
    c00 = D[i, j, k] * (1 - tk) + D[i, j, k1] * tk
    c01 = D[i, j1, k] * (1 - tk) + D[i, j1, k1] * tk
    c10 = D[i1, j, k] * (1 - tk) + D[i1, j, k1] * tk
    c11 = D[i1, j1, k] * (1 - tk) + D[i1, j1, k1] * tk
    c0 = c00 * (1 - tj) + c01 * tj
    c1 = c10 * (1 - tj) + c11 * tj
    return c0 * (1 - ti) + c1 * ti


def gamma(dose_eval, dose_ref, spacing_mm, dose_percent=1.0, distance_mm=1.0, cutoff_percent=10.0,
          interp_fraction=10, max_gamma=1.1):
    ref = np.asarray(dose_ref, float)
    ev = np.asarray(dose_eval, float)
    norm = ref.max()
    dD = dose_percent / 100.0 * norm
    h = distance_mm / interp_fraction
    R = max_gamma * distance_mm
    m = int(np.floor(R / h + 1e-9))
    a = np.arange(-m, m + 1) * h
    ox, oy, oz = np.meshgrid(a, a, a, indexing="ij")
    r2 = ox ** 2 + oy ** 2 + oz ** 2
    keep = r2 <= R * R * (1 + 1e-12)
    ox, oy, oz, d2 = ox[keep], oy[keep], oz[keep], r2[keep] / distance_mm ** 2
    nx, ny, nz = ref.shape
    g = np.full(ref.shape, np.nan)
    idx = np.argwhere(ref >= cutoff_percent / 100.0 * norm)
    for i, j, k in idx:
        fi = i + ox / spacing_mm[0]
        fj = j + oy / spacing_mm[1]
        fk = k + oz / spacing_mm[2]
        inside = (fi >= 0) & (fi <= nx - 1) & (fj >= 0) & (fj <= ny - 1) & (fk >= 0) & (fk <= nz - 1)
        de = _trilinear(ev, fi[inside], fj[inside], fk[inside]) - ref[i, j, k]
        g2 = d2[inside] + de * de / (dD * dD)
        v = np.sqrt(g2.min()) if g2.size else np.inf
        g[i, j, k] = v if v <= max_gamma else np.inf
    valid = ~np.isnan(g)
    return 100.0 * np.mean(g[valid] <= 1.0), g
