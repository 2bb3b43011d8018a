"""Phantom geometry (proton_solver/geometry.py:10-271).

``Box`` objects on a background material, or a CT whose voxels coincide with
the grid.  Field names, half-open conventions and validation errors follow
the reference.  ``Geometry.from_ids`` is an addition: it wraps a
pre-voxelised material map (for synthetic ellipsoid phantoms).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .enums import Material


@dataclass(frozen=True)
class Box:
    """Axis-aligned box using half-open intervals [min, max)."""

    x_min: float
    x_max: float
    y_min: float
    y_max: float
    z_min: float
    z_max: float
    material: Material

    def __post_init__(self):
        coords = (self.x_min, self.x_max, self.y_min, self.y_max, self.z_min, self.z_max)
        if not all(math.isfinite(c) for c in coords):
            raise ValueError("Box coordinates must be finite.")
        if self.x_min >= self.x_max or self.y_min >= self.y_max or self.z_min >= self.z_max:
            raise ValueError("Box minima must be smaller than maxima.")


def _check_ct_orientation(spacing, axis_order, flip_axes) -> None:
    """A CT's voxel spacing (three positive metres), axis permutation and
    per-axis flips, as the reference validates them."""
    if len(spacing) != 3 or not all(math.isfinite(s) and s > 0 for s in spacing):
        raise ValueError("CT spacing must contain three positive finite metres.")
    if sorted(axis_order) != [0, 1, 2]:
        raise ValueError("axis_order must be a permutation of (0, 1, 2).")
    if len(flip_axes) != 3 or not all(type(f) is bool for f in flip_axes):
        raise ValueError("flip_axes must contain three booleans.")


def _read_ct_npz(path) -> tuple[np.ndarray, np.ndarray | None]:
    """(HU volume, body mask or None) of a CT stored as NPZ.

    The volume is the array named ``HU``, else ``hu``, else the only array of
    a file that holds one unnamed array (NumPy stores those as ``arr_0``); an
    optional boolean ``body_mask`` of the same shape marks the patient.  The
    volume must be numeric, three-dimensional and finite."""
    with np.load(path, allow_pickle=False) as npz:
        names = list(npz.files)
        key = next((k for k in ("HU", "hu") if k in names), "arr_0" if names == ["arr_0"] else None)
        if key is None:
            raise ValueError("CT NPZ needs a 'HU', 'hu', or single 'arr_0' array.")
        hu = np.asarray(npz[key])
        mask = np.asarray(npz["body_mask"]) if "body_mask" in names else None
    if hu.ndim != 3 or not np.issubdtype(hu.dtype, np.number):
        raise ValueError("CT HU must be a numeric 3D array.")
    if not np.isfinite(hu).all():
        raise ValueError("CT HU contains non-finite values.")
    if mask is not None and mask.shape != hu.shape:
        raise ValueError("body_mask shape must match the HU array.")
    return hu, mask


def _orient(volume: np.ndarray, axis_order, flip_axes) -> np.ndarray:
    """``volume`` with its axes taken in ``axis_order`` (solver axis i is
    source axis ``axis_order[i]``), then the solver axes marked in
    ``flip_axes`` reversed; one strided view, copied once to C order."""
    reverse = tuple(slice(None, None, -1) if f else slice(None) for f in flip_axes)
    return np.ascontiguousarray(volume.transpose(axis_order)[reverse])


@dataclass(frozen=True)
class HUPartition:
    """Map HU values to transport materials with half-open bins."""

    cutoffs: tuple[float, ...] = (-200.0, 150.0)
    materials: tuple[Material, ...] = (Material.LUNG, Material.WATER, Material.BONE_COMPACT)

    def __post_init__(self):
        if len(self.materials) != len(self.cutoffs) + 1:
            raise ValueError("HUPartition needs one more material than cutoffs.")
        if not all(isinstance(m, Material) for m in self.materials):
            raise ValueError("HUPartition materials must be Material values.")
        if not all(math.isfinite(c) for c in self.cutoffs):
            raise ValueError("HU cutoffs must be finite.")
        if any(a >= b for a, b in zip(self.cutoffs, self.cutoffs[1:])):
            raise ValueError("HU cutoffs must be strictly increasing.")

    def classify(self, hu: np.ndarray) -> np.ndarray:
        hu = np.asarray(hu)
        if hu.ndim != 3 or not np.issubdtype(hu.dtype, np.number):
            raise ValueError("CT HU must be a numeric 3D array.")
        if not np.all(np.isfinite(hu)):
            raise ValueError("CT HU contains non-finite values.")
        return np.searchsorted(self.cutoffs, hu, side="right").astype(np.int32)


@dataclass(frozen=True)
class CTScan:
    """A CT volume from an NPZ (``HU``/``hu``/``arr_0`` and optional ``body_mask``)."""

    path: str | Path
    source_spacing_m: tuple[float, float, float]
    axis_order: tuple[int, int, int] = (0, 1, 2)
    flip_axes: tuple[bool, bool, bool] = (False, False, False)

    hu: np.ndarray = field(init=False, repr=False, compare=False)
    body_mask: np.ndarray | None = field(init=False, repr=False, compare=False)
    spacing: tuple[float, float, float] = field(init=False)

    def __post_init__(self):
        # The orientation is checked before the file is opened, the volume
        # after it; the messages are the reference's, in its order
        # (proton_solver/geometry.py:91-130), so a bad configuration raises the
        # same error under either library.
        _check_ct_orientation(self.source_spacing_m, self.axis_order, self.flip_axes)
        hu, mask = _read_ct_npz(self.path)
        set_ = object.__setattr__
        set_(self, "hu", _orient(hu, self.axis_order, self.flip_axes))
        set_(self, "body_mask", None if mask is None else _orient(mask.astype(bool), self.axis_order, self.flip_axes))
        set_(self, "spacing", tuple(self.source_spacing_m[a] for a in self.axis_order))

    @property
    def shape(self) -> tuple[int, int, int]:
        return self.hu.shape


@dataclass
class Geometry:
    size: tuple[float, float, float]
    resolution: tuple[int, int, int]
    background_material: Material = Material.WATER
    objects: list[Box] = field(default_factory=list)
    view_geometry: bool = False
    ct_scan: CTScan | None = None
    hu_partition: HUPartition = field(default_factory=HUPartition)
    # Pre-voxelised phantom: (ids int32 (nx,ny,nz), materials tuple).
    voxel_ids: np.ndarray | None = field(default=None, repr=False, compare=False)
    voxel_materials: tuple[Material, ...] = ()

    def __post_init__(self):
        if len(self.size) != 3 or len(self.resolution) != 3:
            raise ValueError("size and resolution must contain exactly three values.")
        if not all(math.isfinite(x) and x > 0 for x in self.size):
            raise ValueError("Geometry dimensions must be finite and positive.")
        if not all(type(n) is int and n > 0 for n in self.resolution):
            raise ValueError("Geometry resolution must contain positive integers.")
        self._verify_objects()
        if self.ct_scan is not None:
            if self.objects:
                raise ValueError("CT and Box objects cannot be combined.")
            if self.resolution != self.ct_scan.shape:
                raise ValueError("Geometry resolution must match the CT array shape.")
            if not all(math.isclose(a, b, rel_tol=1e-9, abs_tol=1e-12)
                       for a, b in zip(self.spacing, self.ct_scan.spacing)):
                raise ValueError("Geometry cell spacing must match the CT spacing.")
            if self.view_geometry:
                raise ValueError("3D Box viewer does not support CT; set view_geometry=False.")
        if self.voxel_ids is not None:
            ids = np.asarray(self.voxel_ids)
            if ids.shape != tuple(self.resolution):
                raise ValueError("voxel_ids must have the geometry resolution as shape.")
            if ids.size and (ids.min() < 0 or ids.max() >= len(self.voxel_materials)):
                raise ValueError("voxel_ids must index voxel_materials.")
            if self.objects or self.ct_scan is not None:
                raise ValueError("voxel_ids cannot be combined with boxes or a CT.")

    @classmethod
    def from_ct_scan(cls, path, *, source_spacing_m, axis_order=(0, 1, 2),
                     flip_axes=(False, False, False), hu_partition=None,
                     background_material=Material.WATER) -> "Geometry":
        scan = CTScan(path=path, source_spacing_m=source_spacing_m,
                      axis_order=axis_order, flip_axes=flip_axes)
        return cls(size=tuple(n * dx for n, dx in zip(scan.shape, scan.spacing)),
                   resolution=scan.shape, background_material=background_material,
                   ct_scan=scan,
                   hu_partition=hu_partition if hu_partition is not None else HUPartition())

    @classmethod
    def from_ids(cls, size, ids, materials) -> "Geometry":
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        return cls(size=tuple(size), resolution=tuple(int(n) for n in ids.shape),
                   background_material=materials[0], voxel_ids=ids,
                   voxel_materials=tuple(materials))

    @staticmethod
    def _boxes_overlap(a: Box, b: Box) -> bool:
        return (a.x_min < b.x_max and b.x_min < a.x_max and a.y_min < b.y_max
                and b.y_min < a.y_max and a.z_min < b.z_max and b.z_min < a.z_max)

    def _verify_objects(self):
        lx, ly, lz = self.size
        for obj in self.objects:
            if not (-lx / 2 <= obj.x_min < obj.x_max <= lx / 2
                    and -ly / 2 <= obj.y_min < obj.y_max <= ly / 2
                    and 0.0 <= obj.z_min < obj.z_max <= lz):
                raise ValueError("Geometry object extends outside the domain.")
        for i, a in enumerate(self.objects):
            for b in self.objects[i + 1:]:
                if self._boxes_overlap(a, b):
                    raise ValueError("Geometry objects may not overlap.")

    nx = property(lambda self: self.resolution[0])
    ny = property(lambda self: self.resolution[1])
    nz = property(lambda self: self.resolution[2])
    lx = property(lambda self: self.size[0])
    ly = property(lambda self: self.size[1])
    lz = property(lambda self: self.size[2])
    dx = property(lambda self: self.lx / self.nx)
    dy = property(lambda self: self.ly / self.ny)
    dz = property(lambda self: self.lz / self.nz)
    spacing = property(lambda self: (self.dx, self.dy, self.dz))
    shape = property(lambda self: self.resolution)
