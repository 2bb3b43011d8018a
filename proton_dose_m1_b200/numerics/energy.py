"""The energy march: drop-in for proton_solver/numerics/energy.py:energy_march.

``energy_march(U, material_map, grid, inflow, config, xp, snapshot_energies)``
keeps the reference signature, argument meaning, exceptions and return
contract ``(U | None, dose, energies, snapshots)``.  The work runs in
libpdm1.so on the current CUDA device; PyTorch only provides device memory
and the stream.  NumPy inputs give NumPy outputs, CUDA tensors give CUDA
tensors, as the reference returns arrays of its ``xp``.
"""

from __future__ import annotations

import ctypes as C
import math
import os
import threading
from typing import Any

import numpy as np

from .. import _native
from ..physics.tables import material_tables

MEV_TO_JOULE = 1.602176634e-13

_SCATTER = {"OFF": 0, "ROSSI": 1, "WENTZEL": 2}
_INTERP = {"LINEAR": 0, "PCHIP": 1}
_SCHEME = {"FORWARD_EULER": 0, "SSPRK3": 1, "IF_SSPRK3": 2}
_SPEEDS = {"EXACT": 0, "UNIT": 1}
_PRECISION = {"FP64": 0, "FP32_FP64": 1}
_SPATIAL = {"WENO_Z": 0, "FIRST_ORDER": 1, "MUSCL": 2, "WENO3": 3}


def _to_numpy(a):
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    if hasattr(a, "get"):
        return a.get()
    return np.asarray(a)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the M1 march runs on a CUDA device; none is available")
    return torch


def _check_supported(config) -> None:
    num, phys = config.numerics, config.physics
    if num.spatial_scheme.name not in _SPATIAL:
        raise NotImplementedError(f"spatial scheme {num.spatial_scheme.name} has no GPU kernel")
    if getattr(num, "active_domain", False):
        raise NotImplementedError("the legacy per-operator active_domain crop has no GPU kernel")
    if num.energy_scheme.name not in _SCHEME:
        raise NotImplementedError(f"Energy scheme {num.energy_scheme} has not been migrated yet.")
    if config.beam.energy_spread == 0:
        raise ValueError("Zero energy spread is not supported by the Gaussian inflow.")


def _problem_struct(config, material_map, grid, spatial, precision=None):
    """The pdm1_problem of a configuration, and the host arrays it points into."""
    _check_supported(config)
    num, phys, beam = config.numerics, config.physics, config.beam
    shape = tuple(int(n) for n in grid.shape)
    ids = np.ascontiguousarray(_to_numpy(material_map.ids), dtype=np.int32)
    if ids.shape != shape:
        raise ValueError(f"material ids have shape {ids.shape}, expected {shape}")
    spatial = np.ascontiguousarray(_to_numpy(spatial), dtype=np.float64)
    materials = tuple(material_map.materials)
    keep = [ids, spatial]
    mats = (_native.Material * len(materials))()
    for k, m in enumerate(materials):
        t = material_tables(m.value)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (t.sp_energy, t.sp_value, t.tr_energy, t.tr_value, t.nuc_energy, t.nuc_value)]
        keep += arrs
        ptr = [a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs]
        mats[k] = _native.Material(_native.Table(len(arrs[0]), ptr[0], ptr[1]),
                                   _native.Table(len(arrs[2]), ptr[2], ptr[3]),
                                   _native.Table(len(arrs[4]), ptr[4], ptr[5]),
                                   t.density, t.radiation_length)
    keep.append(mats)
    if precision is None:
        accel = getattr(config, "accel", None)
        precision = accel.precision.name if accel is not None else "FP64"
    p = _native.Problem()
    p.nx, p.ny, p.nz = shape
    p.dx, p.dy, p.dz = float(grid.dx), float(grid.dy), float(grid.dz)
    p.n_materials = len(materials)
    p.materials = mats
    p.ids = ids.ctypes.data_as(C.POINTER(C.c_int32))
    p.inflow_spatial = spatial.ctypes.data_as(C.POINTER(C.c_double))
    p.beam_energy, p.energy_spread = beam.energy, beam.energy_spread
    p.angular_spread = beam.angular_spread
    p.scattering = _SCATTER[phys.scattering.name]
    p.nuclear = int(bool(phys.nuclear))
    p.interpolation = _INTERP[phys.coefficient_interpolation.name]
    p.energy_scheme = _SCHEME[num.energy_scheme.name]
    p.wave_speeds = _SPEEDS[num.wave_speeds.name]
    p.max_energy_step, p.cfl = num.max_energy_step, num.cfl
    p.energy_min, p.energy_window_sigma = num.energy_min, num.energy_window_sigma
    p.moving_active_domain = int(bool(num.moving_active_domain))
    p.vacuum_aware_cfl = int(bool(num.vacuum_aware_cfl))
    p.active_guard_cells = int(num.active_guard_cells)
    p.active_relative_tolerance = math.exp(-0.5 * num.active_truncation_sigma ** 2)
    p.precision = _PRECISION[precision]
    p.spatial_scheme = _SPATIAL[num.spatial_scheme.name]
    accel = getattr(config, "accel", None)
    p.phantom_cfl_floor = int(bool(getattr(accel, "phantom_cfl", False)))
    return p, keep, materials


_TILE_CACHE: dict = {}
AUTOTUNE_STEPS = 96


def _apply_tile(config, handle, shape, n_beams) -> None:
    """Set the plan's stage-kernel tile shape from ``config.accel.tile``."""
    from ..config import TILE_SHAPES
    tile = getattr(getattr(config, "accel", None), "tile", None)
    if tile is None:
        return
    if tile != "auto":
        _native.check(_native.lib().pdm1_plan_set_tile(handle, TILE_SHAPES.index(tuple(tile))))
        return
    # one choice per precision, grid and kind of plan (one beam, or a field of
    # any size: the waves of one field differ only in their beam counts)
    key = (config.accel.precision.name, tuple(shape), 1 if n_beams == 1 else "field",
           bool(config.numerics.moving_active_domain))
    if key not in _TILE_CACHE:
        torch = _torch()
        best = C.c_int()
        ns = (C.c_double * _native.NUM_TILES)()
        _native.check(_native.lib().pdm1_plan_autotune(handle, AUTOTUNE_STEPS, C.byref(best), ns,
                                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        _TILE_CACHE[key] = (int(best.value), [float(v) for v in ns])
    _native.check(_native.lib().pdm1_plan_set_tile(handle, _TILE_CACHE[key][0]))


def autotuned_tiles():
    """The autotuner's choices so far: {(precision, grid, 1 | "field", moving): (tile id, ns per cell-step)}."""
    return dict(_TILE_CACHE)


def _attach_box_model(config, handle) -> None:
    """Give a plan the configuration's learned box model, if any."""
    model = getattr(getattr(config, "accel", None), "box_model", None)
    if model is None:
        return
    if not config.numerics.moving_active_domain:
        raise ValueError("a learned box model needs numerics.moving_active_domain")
    model.attach(handle)


class M1Plan:
    """One beam on one phantom, resident on the GPU (a ``pdm1_plan``)."""

    def __init__(self, config, material_map, grid, inflow, precision: str | None = None):
        p, keep, materials = _problem_struct(config, material_map, grid, inflow.spatial, precision)
        num, beam = config.numerics, config.beam
        self.shape = tuple(int(n) for n in grid.shape)
        self.config = config
        self.materials = materials
        self.start_energy = beam.energy + num.energy_window_sigma * beam.energy_spread
        h = C.c_void_p()
        _native.check(_native.lib().pdm1_plan_create(C.byref(p), C.byref(h)))
        self._h = h
        self._keep = keep
        _attach_box_model(config, h)
        _apply_tile(config, h, self.shape, 1)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            _native.lib().pdm1_plan_destroy(h)
            self._h = None

    __del__ = close

    @property
    def workspace_bytes(self) -> int:
        return int(_native.lib().pdm1_plan_workspace_bytes(self._h))

    def set_schedule(self, energies=None) -> None:
        """March through the given energies (start energy first, decreasing)
        instead of the CFL steps; None restores the CFL rule."""
        E = np.ascontiguousarray([] if energies is None else energies, dtype=np.float64)
        _native.check(_native.lib().pdm1_plan_set_schedule(
            self._h, E.ctypes.data_as(C.POINTER(C.c_double)) if len(E) else None, len(E)))
        self._schedule = E

    @staticmethod
    def _stream():
        torch = _torch()
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def max_steps_bound(self) -> int:
        """A generous bound on the step count: dE >= cfl*S_min*d/(3*sqrt(3)) ... capped."""
        return 2_000_000

    def march_device(self, U, dose, energies, snapshot_energies=(), snap_out=None):
        """Run the march on device tensors; return (n_steps, snapshot energies)."""
        targets = np.ascontiguousarray(sorted({float(t) for t in snapshot_energies}), dtype=np.float64)
        ns = len(targets)
        snap_E = np.zeros(max(ns, 1))
        info = _native.MarchInfo()
        rc = _native.lib().pdm1_march(
            self._h, C.c_void_p(U.data_ptr()), C.c_void_p(dose.data_ptr()),
            C.c_void_p(energies.data_ptr()), int(energies.numel() - 1),
            targets.ctypes.data_as(C.POINTER(C.c_double)) if ns else None, ns,
            C.c_void_p(snap_out.data_ptr()) if snap_out is not None else None,
            snap_E.ctypes.data_as(C.POINTER(C.c_double)), C.byref(info), self._stream())
        _native.check(rc)
        self.last_info = info
        return info.n_steps, [float(snap_E[i]) for i in range(info.n_snapshots)]

    def march(self, U=None, snapshot_energies=(), max_steps=200_000):
        """(U, dose, energies, snapshots) with CUDA tensors for U/dose/snapshots."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        if U is None:
            Ud = torch.zeros((4, *self.shape), dtype=torch.float64, device=dev)
        else:
            Ud = torch.as_tensor(U, dtype=torch.float64).to(dev).contiguous().clone()
        dose = torch.empty(self.shape, dtype=torch.float64, device=dev)
        energies = torch.empty(max_steps + 1, dtype=torch.float64, device=dev)
        targets = sorted({float(t) for t in snapshot_energies})
        snap = (torch.empty((len(targets), 4, *self.shape), dtype=torch.float64, device=dev)
                if targets else None)
        n, snap_E = self.march_device(Ud, dose, energies, targets, snap)
        E = energies[: n + 1].cpu().numpy()
        snapshots = {e: snap[i].clone() for i, e in enumerate(snap_E)}
        return Ud, dose, E, snapshots

    def march_steps(self, steps, U=None, max_steps=200_000):
        """Run the first ``steps`` energy steps; return (U, dose, energies)."""
        torch = _torch()
        dev = torch.device("cuda", torch.cuda.current_device())
        Ud = (torch.zeros((4, *self.shape), dtype=torch.float64, device=dev) if U is None else
              torch.as_tensor(U, dtype=torch.float64).to(dev).contiguous().clone())
        dose = torch.empty(self.shape, dtype=torch.float64, device=dev)
        energies = torch.empty(max_steps + 1, dtype=torch.float64, device=dev)
        info = _native.MarchInfo()
        _native.check(_native.lib().pdm1_march_steps(
            self._h, C.c_void_p(Ud.data_ptr()), C.c_void_p(dose.data_ptr()),
            C.c_void_p(energies.data_ptr()), int(max_steps), int(steps), C.byref(info),
            self._stream()))
        self.last_info = info
        return Ud, dose, energies[: info.n_steps + 1].cpu().numpy()

    # -- building blocks (operator-level parity) --------------------------------
    def spatial_operator(self, U, energy, boundary_state=None):
        torch = _torch()
        Ud = torch.as_tensor(U, dtype=torch.float64).cuda().contiguous()
        bc = None if boundary_state is None else torch.as_tensor(
            boundary_state, dtype=torch.float64).cuda().contiguous()
        rhs = torch.empty_like(Ud)
        _native.check(_native.lib().pdm1_spatial_operator(
            self._h, C.c_void_p(Ud.data_ptr()), float(energy),
            C.c_void_p(bc.data_ptr()) if bc is not None else None,
            C.c_void_p(rhs.data_ptr()), self._stream()))
        return rhs

    def energy_step(self, U, energy):
        torch = _torch()
        Ud = torch.as_tensor(U, dtype=torch.float64).cuda().contiguous()
        out = C.c_double()
        _native.check(_native.lib().pdm1_energy_step(
            self._h, C.c_void_p(Ud.data_ptr()), float(energy), C.byref(out), self._stream()))
        return out.value

    def advance(self, U, energy, dE):
        torch = _torch()
        Ud = torch.as_tensor(U, dtype=torch.float64).cuda().contiguous().clone()
        edep = torch.empty(self.shape, dtype=torch.float64, device=Ud.device)
        _native.check(_native.lib().pdm1_advance(
            self._h, C.c_void_p(Ud.data_ptr()), float(energy), float(dE),
            C.c_void_p(edep.data_ptr()), self._stream()))
        return Ud, edep

    def coefficients(self, energies):
        E = np.ascontiguousarray(energies, dtype=np.float64)
        out = np.empty((len(E), len(self.materials), 3))
        _native.check(_native.lib().pdm1_coefficients(
            self._h, E.ctypes.data_as(C.POINTER(C.c_double)), len(E),
            out.ctypes.data_as(C.POINTER(C.c_double))))
        return out


# Device bytes per box cell of one beam in a field plan: U on the box (double
# buffered), the two stage states, V (4 components each, double), the dose
# quadrature part, and the activity mask byte.
FIELD_BYTES_PER_BOX_CELL = 21 * 8 + 1


def estimate_box_cells(config, grid, beam) -> int:
    """An upper estimate of the largest moving box (cells) of one beam.

    The box is the region where phi > exp(-s^2/2) max(phi) (s = the
    truncation sigma) plus ``active_guard_cells`` on every face
    (numerics/moving_active_domain.py:107-193).  Laterally the fluence is a
    Gaussian of width sqrt(sigma^2 + sigma_mcs^2) with multiple scattering
    bounded by 4% of the CSDA range; along z the band where protons carry
    energy E is the energy window 2 s sigma_E / S plus range straggling
    (bounded by 1.5% of the range on each side of s sigma).  The estimate is
    clipped to the phantom; a box that outgrows it stops the march with a
    capacity error and ``FieldPlan`` retries with more room.
    """
    from ..phantoms import csda_range_m
    from ..enums import Material
    num = config.numerics
    s = num.active_truncation_sigma
    g = int(num.active_guard_cells)
    nx, ny, nz = (int(n) for n in grid.shape)
    E0 = beam.energy + num.energy_window_sigma * beam.energy_spread
    R = min(csda_range_m(Material.WATER, E0), nz * grid.dz)
    sig = max(beam.sigma)
    lat = math.sqrt(sig ** 2 + (0.04 * R) ** 2)
    hx = int(math.ceil(s * lat / grid.dx)) + g + 3
    hy = int(math.ceil(s * lat / grid.dy)) + g + 3
    t = material_tables("G4_WATER")
    S_min = float(np.min(t.sp_value[(t.sp_energy >= 1.0) & (t.sp_energy <= E0)]))   # MeV/m
    window = 2.0 * s * beam.energy_spread / S_min + 2.0 * s * 0.015 * R
    wz = int(math.ceil(window / grid.dz)) + 2 * g + 8
    return int(min(2 * hx + 1, nx) * min(2 * hy + 1, ny) * min(wz, nz))


def field_waves(energies, bytes_per_beam: int, budget_bytes: int):
    """Split a field into waves whose beam buffers fit ``budget_bytes``.

    Beams are ordered by decreasing energy, so the beams of one wave take
    similar numbers of energy steps and finish together.  Returns lists of
    beam indices."""
    wave = max(1, int(budget_bytes // max(1, bytes_per_beam)))
    order = sorted(range(len(energies)), key=lambda k: (-energies[k], k))
    return [order[i:i + wave] for i in range(0, len(order), wave)]


class FieldPlan:
    """A spot-scanning field: many pencil beams on one phantom, batched.

    Every beam marches on its own moving active box with its own energy and
    CFL step (``pdm1_field_plan_create`` / ``pdm1_field_march``); the field
    dose is the sum of the beams' doses.  ``config`` gives the phantom,
    physics, numerics and precision; ``beams`` are ``Beam`` objects.

    ``profiles`` (optional) are the beams' inflow profiles, n_protons times
    ``transverse_profile`` (nx, ny), when the caller already holds them.

    Each beam's box buffers hold ``box_capacity_cells`` (0: the largest
    ``estimate_box_cells`` over the beams).  When all beams do not fit in
    ``max_workspace_bytes`` (0: 70% of the free device memory), the beams run
    in waves of similar energy, each wave one batched march, and the waves'
    doses are summed.
    """

    def __init__(self, config, material_map, grid, beams, box_capacity_cells: int = 0,
                 max_workspace_bytes: int = 0, profiles=None):
        from dataclasses import replace
        from .boundary import transverse_profile
        num = config.numerics
        if not num.moving_active_domain:
            config = type(config)(geometry=config.geometry, beam=config.beam, physics=config.physics,
                                  numerics=replace(num, moving_active_domain=True),
                                  accel=getattr(config, "accel", None) or type(config.accel)())
        beams = list(beams)
        if not beams:
            raise ValueError("a field needs at least one beam")
        for b in beams:
            if b.energy_spread == 0:
                raise ValueError("Zero energy spread is not supported by the Gaussian inflow.")
        self.beams = beams
        self.config = config
        self.material_map = material_map
        self.grid = grid
        self.shape = tuple(int(n) for n in grid.shape)
        self.n_beams = len(beams)
        self.auto_capacity = not box_capacity_cells
        self.capacity_retries = 0
        if profiles is None:
            profiles = [b.n_protons * transverse_profile(b, grid) for b in beams]
        elif len(profiles) != len(beams):
            raise ValueError("one inflow profile per beam is needed")
        self.profiles = [np.ascontiguousarray(q, dtype=np.float64) for q in profiles]
        self._budget = max_workspace_bytes
        self._plans = {}
        self._layout(int(box_capacity_cells or max(estimate_box_cells(config, grid, b) for b in beams)))

    def _layout(self, cap, members=None):
        """Set the box capacity and split the beams ``members`` (default: all)
        into waves; returns the waves.  With every beam in a single wave its
        plan is created once and kept."""
        self.close()
        N = int(np.prod(self.shape))
        nxy = self.shape[0] * self.shape[1]
        self.cap = int(min(N, cap))
        per_beam = self.cap * FIELD_BYTES_PER_BOX_CELL + nxy * 8 + 4096
        budget = self._budget
        if not budget:
            torch = _torch()
            torch.cuda.empty_cache()   # blocks the caching allocator holds are free for the plans
            free, _ = torch.cuda.mem_get_info()
            # blocks of destroyed plans that the plans' own pool keeps are free for these
            budget = int(0.7 * (free + int(_native.lib().pdm1_pool_cached_bytes())))
        idx = list(range(self.n_beams)) if members is None else list(members)
        order = field_waves([self.beams[i].energy for i in idx], per_beam, budget)
        waves = [[idx[k] for k in wave] for wave in order]
        if members is None:
            self.waves = waves
            if len(waves) == 1:
                self._plans[0] = self._create(waves[0])
        return waves

    def _create(self, members):
        """A native field plan for the beams ``members`` (indices into ``beams``)."""
        p, keep, _ = _problem_struct(self.config, self.material_map, self.grid, self.profiles[members[0]])
        descs = (_native.BeamDesc * len(members))()
        for k, i in enumerate(members):
            b = self.beams[i]
            descs[k] = _native.BeamDesc(b.energy, b.energy_spread, b.angular_spread,
                                        self.profiles[i].ctypes.data_as(C.POINTER(C.c_double)))
        h = C.c_void_p()
        _native.check(_native.lib().pdm1_field_plan_create(C.byref(p), descs, len(members),
                                                           int(self.cap), C.byref(h)))
        try:
            _attach_box_model(self.config, h)
        except Exception:
            _native.lib().pdm1_plan_destroy(h)
            raise
        return h

    def close(self):
        for h in getattr(self, "_plans", {}).values():
            if h:
                _native.lib().pdm1_plan_destroy(h)
        self._plans = {}

    __del__ = close

    @property
    def workspace_bytes(self) -> int:
        return sum(int(_native.lib().pdm1_plan_workspace_bytes(h)) for h in self._plans.values())

    def march_device(self, dose, max_steps=2_000_000):
        """Field dose into the device tensor ``dose``; returns steps per beam.

        ``last_info`` sums the march statistics over the waves.  With an
        estimated capacity, a box that outgrows it doubles the capacity: the
        beams of that wave and of the waves after it are split into new waves
        and marched at the new capacity; the waves already marched stand."""
        torch = _torch()
        N = int(np.prod(self.shape))
        steps_all = [0] * self.n_beams
        total = _native.MarchInfo()
        partial = None
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        waves = list(self.waves)
        regrown = False
        w = 0
        while w < len(waves):
            members = waves[w]
            if w > 0 and partial is None:
                partial = torch.empty_like(dose)
            out = dose if w == 0 else partial
            h = self._plans.get(w) if not regrown else None
            transient = h is None
            try:
                if transient:   # a beam's initial box beyond the capacity fails here
                    h = self._create(members)
                # tile shape (autotuned on the first march; a box that outgrows
                # the capacity there is retried like one in the march)
                _apply_tile(self.config, h, self.shape, len(members))
                steps = (C.c_int * len(members))()
                info = _native.MarchInfo()
                _native.check(_native.lib().pdm1_field_march(
                    h, C.c_void_p(out.data_ptr()), int(max_steps), steps, C.byref(info), stream))
            except ValueError as e:
                if not (self.auto_capacity and "capacity" in str(e) and self.cap < N):
                    raise
                if transient and h:
                    _native.lib().pdm1_plan_destroy(h)
                transient = False
                self.capacity_retries += 1
                rest = [i for wave in waves[w:] for i in wave]
                waves = waves[:w] + self._layout(2 * self.cap, rest)
                regrown = True
                continue
            finally:
                if transient and h:
                    _native.lib().pdm1_plan_destroy(h)
            if w > 0:
                dose.add_(partial)
            for k, i in enumerate(members):
                steps_all[i] = steps[k]
            total.n_steps = max(total.n_steps, info.n_steps)
            total.graph_replays += info.graph_replays
            total.kernel_launches += info.kernel_launches + (1 if w > 0 else 0)
            total.stage_launches += info.stage_launches
            total.stage_ms += info.stage_ms
            total.cell_steps += info.cell_steps
            total.max_box_cells = max(total.max_box_cells, info.max_box_cells)
            w += 1
        if regrown:   # the next march lays every beam out at the grown capacity
            self._layout(self.cap)
        self.last_info = total
        return steps_all

    def march(self, max_steps=2_000_000):
        torch = _torch()
        dose = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        steps = self.march_device(dose, max_steps)
        return dose, steps

    def march_steps(self, steps, max_steps=2_000_000):
        """The first ``steps`` energy steps of every beam (one wave only):
        the field dose of that prefix; ``last_info`` holds its statistics."""
        torch = _torch()
        if len(self.waves) != 1 or 0 not in self._plans:
            raise ValueError("march_steps needs a field that fits one wave")
        h = self._plans[0]
        _apply_tile(self.config, h, self.shape, len(self.waves[0]))
        dose = torch.empty(self.shape, dtype=torch.float64, device="cuda")
        info = _native.MarchInfo()
        _native.check(_native.lib().pdm1_march_steps(
            h, None, C.c_void_p(dose.data_ptr()), None, int(max_steps), int(steps), C.byref(info),
            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        self.last_info = info
        return dose


_STAGING: dict = {}          # device index -> page-locked uint8 tensor
_STAGING_LOCK = threading.Lock()
_COPY_THREADS = max(1, min(8, os.cpu_count() or 1))
_COPY_POOL = None


def _to_host(t):
    """Device tensor -> a new NumPy array.

    One device->host copy into a page-locked staging buffer that is kept
    across calls (page-locking fresh memory costs about 1 ms per MB, more
    than the copy), then a host copy into the returned array in parallel
    slices.  Small tensors take the plain path."""
    global _COPY_POOL
    torch = _torch()
    nbytes = t.numel() * t.element_size()
    if nbytes < (4 << 20):
        return t.cpu().numpy()
    src = t.contiguous().reshape(-1).view(torch.uint8)
    out = np.empty(tuple(t.shape), dtype=torch.empty(0, dtype=t.dtype).numpy().dtype)
    dst = out.reshape(-1).view(np.uint8)
    with _STAGING_LOCK:
        dev = t.device.index or 0
        buf = _STAGING.get(dev)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
            _STAGING[dev] = buf
        stage = buf[:nbytes]
        stage.copy_(src, non_blocking=True)
        torch.cuda.current_stream(t.device).synchronize()
        host = stage.numpy()
        if _COPY_POOL is None:
            from concurrent.futures import ThreadPoolExecutor
            _COPY_POOL = ThreadPoolExecutor(_COPY_THREADS)
        step = -(-nbytes // _COPY_THREADS)
        parts = [(a, min(a + step, nbytes)) for a in range(0, nbytes, step)]
        list(_COPY_POOL.map(lambda ab: np.copyto(dst[ab[0]:ab[1]], host[ab[0]:ab[1]]), parts))
    return out


def field_march(config, material_map, grid, beams, box_capacity_cells: int = 0,
                stats: dict | None = None):
    """Dose of a spot-scanning field (host NumPy in, host NumPy out).

    The field counterpart of ``energy_march``: the reference marches one beam
    per ``Solver.solve`` call (proton_solver/solver.py:34-218) and a field is
    the sum of its beams' doses.  Returns ``(dose, steps_per_beam)``.  A dict
    passed as ``stats`` receives the plan's layout (waves, box capacity,
    capacity retries) and the host seconds of planning, march and copy-back.
    """
    import time
    torch = _torch()
    t0 = time.perf_counter()
    plan = FieldPlan(config, material_map, grid, beams, box_capacity_cells)
    try:
        t1 = time.perf_counter()
        dose, steps = plan.march()
        torch.cuda.current_stream().synchronize()
        t2 = time.perf_counter()
        out = _to_host(dose)
        if stats is not None:
            stats.update(waves=len(plan.waves), box_capacity_cells=plan.cap,
                         capacity_retries=plan.capacity_retries, plan_s=t1 - t0, march_s=t2 - t1,
                         copy_s=time.perf_counter() - t2)
        return out, steps
    finally:
        plan.close()


def energy_march(U: Any, material_map, grid, inflow, config, xp=None,
                 snapshot_energies: tuple[float, ...] = ()):
    """March the M1 system from high to low kinetic energy on the GPU.

    Same contract as proton_solver/numerics/energy.py:1497-1643.
    """
    if not config.numerics.moving_active_domain and U is None:
        raise ValueError("A full-grid initial state is required when moving_active_domain "
                         "is disabled.")
    host = U is None or not hasattr(U, "is_cuda") or not U.is_cuda
    plan = M1Plan(config, material_map, grid, inflow)
    try:
        Ud, dose, energies, snaps = plan.march(U, snapshot_energies)
    finally:
        plan.close()
    store = getattr(getattr(config, "output", None), "store_final_state", True)
    if config.numerics.moving_active_domain and not store:
        Ud = None
    if host:
        conv = lambda t: None if t is None else _to_host(t)
        return conv(Ud), conv(dose), energies, {e: conv(s) for e, s in snaps.items()}
    return Ud, dose, energies, snaps
