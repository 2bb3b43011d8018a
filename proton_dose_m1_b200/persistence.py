"""Run directories of solver results (proton_solver/persistence.py:1-369).

The layout is the reference's, so its tools read GPU runs unchanged:
``<results_directory>/<timestamp>__<nx>x<ny>x<nz>__<scheme>__<config hash[:8]>__<git hash[:8]>/``
with ``config.json`` (the canonical configuration), ``metadata.json``
(creation time, config hash, git provenance, runtimes, backend) and
``results.npz`` (x, y, z and the solution arrays present).

The canonical configuration leaves out what does not change the solution
(output settings, the geometry viewer flag) and, so that a configuration
written for the reference hashes the same here, this library's additions
when they hold their defaults (``accel``, pre-voxelised ids).
"""

from __future__ import annotations

import hashlib
import json
import subprocess
from dataclasses import fields, is_dataclass
from datetime import datetime
from enum import Enum
from pathlib import Path
from typing import Any

import numpy as np


def _plain(value: Any):
    """JSON form: enums by name, arrays by shape, dtype and content hash,
    dataclasses as dicts, tuples as lists."""
    if isinstance(value, Enum):
        return value.name
    if isinstance(value, np.ndarray):
        return {"shape": [int(n) for n in value.shape], "dtype": str(value.dtype),
                "sha256": hashlib.sha256(np.ascontiguousarray(value).tobytes()).hexdigest()}
    if isinstance(value, np.generic):
        return value.item()
    if isinstance(value, Path):
        return str(value)
    if is_dataclass(value) and not isinstance(value, type):
        return {f.name: _plain(getattr(value, f.name)) for f in fields(value)}
    if isinstance(value, dict):
        return {str(k): _plain(v) for k, v in value.items()}
    if isinstance(value, (list, tuple)):
        return [_plain(v) for v in value]
    return value


def config_dict(config) -> dict:
    """The canonical configuration (persistence.py:56-71)."""
    from .config import Accel
    data = _plain(config)
    data.pop("output", None)
    geometry = data.get("geometry", {})
    geometry.pop("view_geometry", None)
    if getattr(config.geometry, "voxel_ids", None) is None:
        geometry.pop("voxel_ids", None)
        geometry.pop("voxel_materials", None)
    accel = getattr(config, "accel", None)
    if accel is None or (accel.precision == Accel().precision and accel.box_model is None):
        data.pop("accel", None)
    elif "accel" in data:
        data["accel"] = {"precision": accel.precision.name, "learned_box": accel.box_model is not None}
    return data


def config_hash(config) -> str:
    """SHA-256 of the canonical configuration (sorted keys, compact separators)."""
    payload = json.dumps(config_dict(config), sort_keys=True, separators=(",", ":")).encode("utf-8")
    return hashlib.sha256(payload).hexdigest()


def config_from_dict(data: dict):
    """A ``SolverConfig`` from a canonical configuration (a run directory's
    ``config.json``).  Box geometries only (a CT is stored by content hash).
    Keys that older versions of the configuration did not write take their
    defaults; keys this version does not know are ignored."""
    from dataclasses import fields as dc_fields
    from . import enums

    def known(cls, d):
        names = {f.name for f in dc_fields(cls)}
        return {k: v for k, v in d.items() if k in names}
    from .beam import Beam
    from .config import Numerics, OutputConfig, Physics, References, SolverConfig
    from .geometry import Box, Geometry, HUPartition
    g = data["geometry"]
    if g.get("ct_scan") is not None:
        raise NotImplementedError("a CT geometry is stored by content hash and cannot be rebuilt")
    kw = {}
    if "hu_partition" in g:
        hp = g["hu_partition"]
        kw["hu_partition"] = HUPartition(cutoffs=tuple(hp["cutoffs"]),
                                         materials=tuple(enums.Material[m] for m in hp["materials"]))
    geo = Geometry(size=tuple(g["size"]), resolution=tuple(int(n) for n in g["resolution"]),
                   background_material=enums.Material[g["background_material"]],
                   objects=[Box(o["x_min"], o["x_max"], o["y_min"], o["y_max"], o["z_min"], o["z_max"],
                                enums.Material[o["material"]]) for o in g["objects"]], **kw)
    b = known(Beam, data["beam"])
    for key in ("sigma", "center"):
        if key in b:
            b[key] = tuple(b[key])
    beam = Beam(**b)
    p = known(Physics, data.get("physics", {}))
    for key, enum in (("scattering", enums.Scattering), ("coefficient_interpolation",
                                                          enums.CoefficientInterpolation)):
        if key in p:
            p[key] = enum[p[key]]
    n = known(Numerics, data.get("numerics", {}))
    for key, enum in (("spatial_scheme", enums.SpatialScheme), ("energy_scheme", enums.EnergyScheme),
                      ("wave_speeds", enums.WaveSpeeds)):
        if key in n:
            n[key] = enum[n[key]]
    r = known(References, data.get("references", {}))
    if "reference" in r:
        r["reference"] = enums.Reference[r["reference"]]
    if "additional_references" in r:
        r["additional_references"] = tuple(enums.Reference[x] for x in r["additional_references"])
    return SolverConfig(geometry=geo, beam=beam, physics=Physics(**p), numerics=Numerics(**n),
                        backend=enums.Backend[data.get("backend", "AUTO")],
                        solve_deterministic=data.get("solve_deterministic", True),
                        references=References(**r), output=OutputConfig())


def _git(*args):
    return subprocess.run(["git", *args], capture_output=True, check=True).stdout


def git_provenance() -> dict:
    """Commit, dirty flag and a hash of the working tree state (commit, diff,
    untracked files), or Nones outside a git checkout."""
    try:
        commit = _git("rev-parse", "HEAD").decode().strip()
        root = Path(_git("rev-parse", "--show-toplevel").decode().strip())
        diff = _git("diff", "HEAD", "--binary")
        untracked = _git("ls-files", "--others", "--exclude-standard").decode().splitlines()
        h = hashlib.sha256()
        h.update(commit.encode("utf-8"))
        h.update(diff)
        for rel in sorted(untracked):
            h.update(rel.encode("utf-8"))
            p = root / rel
            if p.is_file():
                h.update(p.read_bytes())
        return {"git_commit": commit, "git_dirty": bool(diff or untracked), "git_state_hash": h.hexdigest()}
    except (subprocess.CalledProcessError, FileNotFoundError):
        return {"git_commit": None, "git_dirty": None, "git_state_hash": None}


def _host(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _speedup(ours, theirs):
    if ours is None or theirs is None or ours <= 0.0 or theirs <= 0.0:
        return None
    return float(theirs / ours)


def save_result(result, config) -> Path:
    """Write the run directory of ``result`` and return its path."""
    root = Path(config.output.results_directory)
    root.mkdir(parents=True, exist_ok=True)
    digest = config_hash(config)
    git = git_provenance()
    git_digest = git["git_state_hash"][:8] if git["git_state_hash"] is not None else "nogit"
    nx, ny, nz = config.geometry.resolution
    name = (f"{datetime.now().strftime('%Y%m%d_%H%M%S')}__{nx}x{ny}x{nz}"
            f"__{config.numerics.spatial_scheme.name.lower()}__{digest[:8]}__{git_digest}")
    run = root / name
    run.mkdir()
    with (run / "config.json").open("w") as f:
        json.dump(config_dict(config), f, indent=2, sort_keys=True)
    metadata = {
        "created_at": datetime.now().astimezone().isoformat(),
        "config_hash": digest,
        **git,
        "runtime_seconds": result.runtime,
        "bfp_mc_runtime_seconds": result.bfp_mc_runtime,
        "topas_runtime_seconds": result.topas_runtime,
        "speedup_vs_bfp_mc_x": ("-" if result.reference_label != "BFP Monte Carlo"
                                else _speedup(result.runtime, result.bfp_mc_runtime)),
        "speedup_vs_topas_x": ("-" if result.reference_label != "TOPAS"
                               else _speedup(result.runtime, result.topas_runtime)),
        "backend": result.backend.name if result.backend is not None else None,
    }
    with (run / "metadata.json").open("w") as f:
        json.dump(metadata, f, indent=2)
    arrays = {"x": _host(result.x), "y": _host(result.y), "z": _host(result.z)}
    for key in ("phi", "J", "dose", "energies", "analytical_dose", "topas_dose", "bfp_mc_dose"):
        value = getattr(result, key)
        if value is not None:
            arrays[key] = _host(value)
    np.savez_compressed(run / "results.npz", **arrays)
    return run


__all__ = ["config_dict", "config_hash", "config_from_dict", "git_provenance", "save_result"]
