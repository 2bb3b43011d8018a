"""Voxelised material map (proton_solver/physics/materials.py:65-137)."""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

from ..enums import Material
from .tables import density


@dataclass(frozen=True)
class MaterialMap:
    ids: Any                          # int32 (nx, ny, nz)
    materials: tuple[Material, ...]

    @classmethod
    def from_geometry(cls, geometry, grid, xp=np):
        """Boxes on a background, an oriented CT, or pre-voxelised ids."""
        if getattr(geometry, "voxel_ids", None) is not None:
            return cls(ids=np.ascontiguousarray(geometry.voxel_ids, dtype=np.int32),
                       materials=tuple(geometry.voxel_materials))
        if geometry.ct_scan is not None:
            partition = geometry.hu_partition
            materials = tuple(dict.fromkeys((*partition.materials, geometry.background_material)))
            classes = partition.classify(geometry.ct_scan.hu)
            ids = np.asarray([materials.index(partition.materials[i])
                              for i in range(len(partition.materials))], dtype=np.int32)[classes]
            if geometry.ct_scan.body_mask is not None:
                ids = ids.copy()
                ids[~geometry.ct_scan.body_mask] = materials.index(geometry.background_material)
            return cls(ids=np.ascontiguousarray(ids, dtype=np.int32), materials=materials)
        materials = tuple(dict.fromkeys([geometry.background_material,
                                         *(obj.material for obj in geometry.objects)]))
        index = {m: i for i, m in enumerate(materials)}
        ids = np.full(grid.shape, index[geometry.background_material], dtype=np.int32)
        x, y, z = (np.asarray(a) for a in (grid.x, grid.y, grid.z))
        for box in geometry.objects:
            ix = np.where((x >= box.x_min) & (x < box.x_max))[0]
            iy = np.where((y >= box.y_min) & (y < box.y_max))[0]
            iz = np.where((z >= box.z_min) & (z < box.z_max))[0]
            ids[ix[:, None, None], iy[None, :, None], iz[None, None, :]] = index[box.material]
        return cls(ids=ids, materials=materials)

    def id_for(self, material: Material) -> int:
        return self.materials.index(material)


def density_field(material_map: MaterialMap, xp=np):
    values = np.asarray([density(m) for m in material_map.materials])
    return values[np.asarray(material_map.ids)]
