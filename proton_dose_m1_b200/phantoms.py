"""Seeded synthetic phantoms and spot-scanning fields.

The reference ships no phantoms beyond axis-aligned boxes and one CT; the
batched-field and learned-box workloads need voxelised heterogeneous
phantoms, so they are generated here from ``numpy.random.default_rng(seed)``
and voxelised at cell centres (the same convention as the Box voxelisation
of proton_solver/physics/materials.py:103-118: a cell belongs to a shape
when its centre does).  Every phantom is a ``Geometry`` with pre-voxelised
ids, so ``MaterialMap.from_geometry`` and the march take it unchanged.

* ``ellipsoid_phantom``: a water body with 6-12 randomly placed, sized and
  oriented ellipsoids of WATER, LUNG, BONE_COMPACT or MUSCLE_SKELETAL
  (128 x 128 x 256 at 1 mm by default).  AIR is left out: one air voxel in a
  box throttles the CFL step of every beam that reaches it by ~1000x.
* ``pelvis_phantom``: 256 x 256 x 320 at 1 mm; an elliptic body (axis along
  y, the beam enters through its anterior surface) of water and muscle
  under an ADIPOSE_SYNTH shell, a bone ring and two bone femoral heads;
  outside the body is WATER (the reference's CT convention,
  physics/materials.py:86-90).
* ``lateral_interface_phantom``: water with bone for x > offset (the mirror
  of the reference's transversal-slab benchmark,
  thesis_experiments/scattering_nuclear/transversal_slabs.py:37-46).
* ``spot_grid``: a square grid of pencil beams with seeded energies and
  widths.
"""

from __future__ import annotations

import numpy as np

from .beam import Beam
from .enums import Material
from .geometry import Box, Geometry

ELLIPSOID_MATERIALS = (Material.WATER, Material.LUNG, Material.BONE_COMPACT, Material.MUSCLE_SKELETAL)


def _centres(shape, spacing):
    """Cell-centre coordinates (m) with x, y centred on the axis and z from 0
    (numerics/grid.py:30-32)."""
    nx, ny, nz = shape
    dx, dy, dz = spacing
    x = (np.arange(nx) + 0.5) * dx - 0.5 * nx * dx
    y = (np.arange(ny) + 0.5) * dy - 0.5 * ny * dy
    z = (np.arange(nz) + 0.5) * dz
    return x, y, z


def _random_rotation(rng):
    """A uniformly distributed rotation matrix (QR of a Gaussian matrix)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def ellipsoid_phantom(seed: int, shape=(128, 128, 256), spacing=(1e-3, 1e-3, 1e-3),
                      n_ellipsoids=(6, 12), semi_axis_mm=(6.0, 30.0),
                      materials=ELLIPSOID_MATERIALS):
    """Water body with seeded random ellipsoids.  Returns (Geometry, info)."""
    rng = np.random.default_rng(seed)
    x, y, z = _centres(shape, spacing)
    lx, ly, lz = (n * d for n, d in zip(shape, spacing))
    mats = tuple(dict.fromkeys((Material.WATER, *materials)))
    ids = np.zeros(shape, dtype=np.int32)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij", sparse=True)
    n = int(rng.integers(n_ellipsoids[0], n_ellipsoids[1] + 1))
    shapes = []
    for _ in range(n):
        c = np.array([rng.uniform(-0.35 * lx, 0.35 * lx), rng.uniform(-0.35 * ly, 0.35 * ly),
                      rng.uniform(0.08 * lz, 0.92 * lz)])
        a = rng.uniform(*semi_axis_mm, size=3) * 1e-3
        R = _random_rotation(rng)
        m = materials[int(rng.integers(len(materials)))]
        # body-frame coordinates: R^T (p - c)
        px, py, pz = X - c[0], Y - c[1], Z - c[2]
        q = [R[0, k] * px + R[1, k] * py + R[2, k] * pz for k in range(3)]
        inside = (q[0] / a[0]) ** 2 + (q[1] / a[1]) ** 2 + (q[2] / a[2]) ** 2 <= 1.0
        ids[inside] = mats.index(m)
        shapes.append({"centre_m": c.tolist(), "semi_axes_m": a.tolist(), "material": m.name})
    geo = Geometry.from_ids((lx, ly, lz), ids, mats)
    return geo, {"seed": seed, "ellipsoids": shapes}


def pelvis_phantom(seed: int, shape=(256, 256, 320), spacing=(1e-3, 1e-3, 1e-3)):
    """Synthetic pelvis-like phantom (seeded jitter of every shape).
    Returns (Geometry, info)."""
    rng = np.random.default_rng(seed)
    x, y, z = _centres(shape, spacing)
    lx, ly, lz = (n * d for n, d in zip(shape, spacing))
    W, ADI, MUS, BONE = (Material.WATER, Material.ADIPOSE_SYNTH, Material.MUSCLE_SKELETAL,
                         Material.BONE_COMPACT)
    mats = (W, ADI, MUS, BONE)
    j = lambda s: rng.uniform(-s, s)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij", sparse=True)
    ids = np.zeros(shape, dtype=np.int32)
    # body: elliptic cylinder along y; (x, z) cross-section
    zc = 0.5 * lz + j(5e-3)
    ax, az = 0.46 * lx + j(4e-3), 0.44 * lz + j(4e-3)
    shell = 12e-3 + j(3e-3)
    body = (X / ax) ** 2 + ((Z - zc) / az) ** 2 <= 1.0
    inner = (X / (ax - shell)) ** 2 + ((Z - zc) / (az - shell)) ** 2 <= 1.0
    ids[np.broadcast_to(body, shape)] = mats.index(ADI)
    ids[np.broadcast_to(inner, shape)] = mats.index(W)
    # muscle: a thick layer inside the shell, water (organs) at the core
    mx, mz = ax - shell - 25e-3 + j(4e-3), az - shell - 30e-3 + j(4e-3)
    core = (X / mx) ** 2 + ((Z - zc) / mz) ** 2 <= 1.0
    ids[np.broadcast_to(inner & ~core, shape)] = mats.index(MUS)
    # bone ring (pelvic girdle): elliptic annulus in (x, z) over a band of y
    rc_z = zc + 15e-3 + j(5e-3)
    rx, rz, t = 75e-3 + j(5e-3), 55e-3 + j(5e-3), 8e-3 + j(2e-3)
    r_out = (X / rx) ** 2 + ((Z - rc_z) / rz) ** 2 <= 1.0
    r_in = (X / (rx - t)) ** 2 + ((Z - rc_z) / (rz - t)) ** 2 <= 1.0
    band = np.abs(Y - j(5e-3)) <= 45e-3 + j(5e-3)
    ids[r_out & ~r_in & band] = mats.index(BONE)
    # femoral heads: two bone ellipsoids, mirrored in x, in the acetabula of the ring
    fy, fz, fr = -15e-3 + j(5e-3), rc_z + 25e-3 + j(5e-3), 22e-3 + j(3e-3)
    heads = []
    for sx in (-1.0, 1.0):
        fx = sx * (52e-3 + j(4e-3))
        head = ((X - fx) ** 2 + (Y - fy) ** 2 / 1.1 ** 2 + (Z - fz) ** 2) <= fr ** 2
        ids[head] = mats.index(BONE)
        heads.append([fx, fy, fz, fr])
    geo = Geometry.from_ids((lx, ly, lz), ids, mats)
    return geo, {"seed": seed, "body_semi_axes_m": [ax, az], "shell_m": shell,
                 "ring": [rx, rz, t, rc_z], "femoral_heads": heads}


def lateral_interface_phantom(offset_m: float, shape=(80, 80, 400), spacing=(5e-4, 5e-4, 5e-4)):
    """Water with a bone half-space x > offset over the full depth."""
    lx, ly, lz = (n * d for n, d in zip(shape, spacing))
    off = min(max(offset_m, -0.5 * lx), 0.5 * lx)
    objs = [] if off >= 0.5 * lx else [Box(off, 0.5 * lx, -0.5 * ly, 0.5 * ly, 0.0, lz, Material.BONE_COMPACT)]
    return Geometry(size=(lx, ly, lz), resolution=tuple(shape), objects=objs)


def spot_grid(seed: int, n_side: int, pitch_m: float, energy_mev=(70.0, 220.0),
              sigma_mm=(2.0, 6.0), n_protons=1e6, energy_spread=1.0):
    """``n_side`` x ``n_side`` pencil beams centred on the axis at ``pitch_m``,
    with energies and (symmetric) widths drawn uniformly from the ranges."""
    rng = np.random.default_rng(seed)
    half = 0.5 * (n_side - 1)
    beams = []
    for i in range(n_side):
        for k in range(n_side):
            E = float(rng.uniform(*energy_mev))
            s = float(rng.uniform(*sigma_mm)) * 1e-3
            beams.append(Beam(n_protons=n_protons, energy=E, energy_spread=energy_spread,
                              sigma=(s, s), center=((i - half) * pitch_m, (k - half) * pitch_m)))
    return beams


def csda_range_m(material: Material, energy_mev: float) -> float:
    """CSDA range by the trapezoid rule on the stopping-power table (for
    sizing estimates only)."""
    from .physics.tables import material_tables
    t = material_tables(material)
    e = t.sp_energy[t.sp_energy <= energy_mev]
    inv = 1.0 / t.sp_value[: len(e)]
    return float(np.sum(0.5 * (inv[1:] + inv[:-1]) * np.diff(e)))


__all__ = ["ellipsoid_phantom", "pelvis_phantom", "lateral_interface_phantom", "spot_grid",
           "csda_range_m", "ELLIPSOID_MATERIALS"]
