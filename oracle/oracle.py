"""ctypes front end of the CPU oracle (liboracle.so, built from m1_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.

``OracleProblem(config, material_map)`` accepts this package's
``SolverConfig`` or the reference's (enums are matched by name, materials
by their Geant4 ``.value``) and exposes the march and its building blocks
with the reference's array layouts.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class _MatDesc(C.Structure):
    _fields_ = [("n_sp", C.c_int), ("sp_energy", _dp), ("sp_value", _dp),
                ("n_tr", C.c_int), ("tr_energy", _dp), ("tr_value", _dp),
                ("n_nuc", C.c_int), ("nuc_energy", _dp), ("nuc_value", _dp),
                ("density", C.c_double), ("radiation_length", C.c_double)]


class _ProbDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("n_materials", C.c_int), ("materials", C.POINTER(_MatDesc)), ("ids", _ip),
                ("n_protons", C.c_double), ("energy", C.c_double), ("energy_spread", C.c_double),
                ("sigma_x", C.c_double), ("sigma_y", C.c_double),
                ("center_x", C.c_double), ("center_y", C.c_double),
                ("angular_spread", C.c_double), ("cutoff_sigma", C.c_double),
                ("scattering", C.c_int), ("nuclear", C.c_int), ("interpolation", C.c_int),
                ("energy_scheme", C.c_int), ("wave_speeds", C.c_int),
                ("max_energy_step", C.c_double), ("cfl", C.c_double),
                ("energy_min", C.c_double), ("energy_window_sigma", C.c_double),
                ("moving_active_domain", C.c_int), ("vacuum_aware_cfl", C.c_int),
                ("active_guard_cells", C.c_int), ("active_truncation_sigma", C.c_double),
                ("store_final_state", C.c_int), ("spatial_scheme", C.c_int)]

_SPATIAL = {"WENO_Z": 0, "FIRST_ORDER": 1, "MUSCL": 2, "WENO3": 3}


def build(force: bool = False) -> Path:
    """Compile liboracle.so with the committed Makefile."""
    src = HERE / "m1_oracle.c"
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "liboracle.so"],
                       check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        L.orc_problem_create.argtypes = [C.POINTER(_ProbDesc), C.POINTER(C.c_void_p)]
        L.orc_problem_destroy.argtypes = [C.c_void_p]
        L.orc_last_error.restype = C.c_char_p
        L.orc_weno_left.argtypes = [_dp]
        L.orc_weno_left.restype = C.c_double
        L.orc_project.argtypes = [_dp]
        L.orc_eigenvalues.argtypes = [_dp, C.c_int, _dp, _dp]
        L.orc_hll_flux.argtypes = [_dp, _dp, C.c_int, C.c_int, _dp]
        for f in ("orc_stopping_power", "orc_transport_coefficient", "orc_nuclear_coefficient"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int, C.c_double, _dp]
        L.orc_optical_depths.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, _dp, _dp]
        L.orc_inflow_spatial.argtypes = [C.c_void_p, _dp]
        L.orc_inflow_state.argtypes = [C.c_void_p, C.c_double, _dp]
        L.orc_spatial_operator.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp]
        L.orc_energy_step.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.orc_advance.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double, _dp]
        L.orc_march.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int),
                                _dp, C.c_int, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_march_steps.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.POINTER(C.c_int)]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_schedule.argtypes = [C.c_void_p, _dp, C.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _check(rc):
    if rc != 0:
        msg = lib().orc_last_error().decode()
        if rc == 2 or rc == 5:
            raise ValueError(msg)
        raise RuntimeError(f"oracle error {rc}: {msg}")


def weno_left(v) -> float:
    v = np.ascontiguousarray(v, dtype=float)
    return lib().orc_weno_left(_ptr(v))


def project(u):
    u = np.array(u, dtype=float)
    lib().orc_project(_ptr(u))
    return u


def eigenvalues(u, axis):
    u = np.ascontiguousarray(u, dtype=float)
    lo, hi = C.c_double(), C.c_double()
    lib().orc_eigenvalues(_ptr(u), axis, C.byref(lo), C.byref(hi))
    return lo.value, hi.value


def hll_flux(left, right, axis, unit_speeds=False):
    L = np.ascontiguousarray(left, dtype=float)
    R = np.ascontiguousarray(right, dtype=float)
    F = np.empty(4)
    lib().orc_hll_flux(_ptr(L), _ptr(R), axis, 1 if unit_speeds else 0, _ptr(F))
    return F


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


_SCATTER = {"OFF": 0, "ROSSI": 1, "WENTZEL": 2}
_INTERP = {"LINEAR": 0, "PCHIP": 1}
_SCHEME = {"FORWARD_EULER": 0, "SSPRK3": 1, "IF_SSPRK3": 2}
_SPEEDS = {"EXACT": 0, "UNIT": 1}


class OracleProblem:
    """One beam on one phantom, held by the C oracle."""

    def __init__(self, config, material_map=None):
        from proton_dose_m1_b200.physics.tables import material_tables

        geo, beam, phys, num = config.geometry, config.beam, config.physics, config.numerics
        if num.spatial_scheme.name not in _SPATIAL:
            raise NotImplementedError(f"spatial scheme {num.spatial_scheme.name}")
        if num.energy_scheme.name not in _SCHEME:
            raise NotImplementedError(f"Energy scheme {num.energy_scheme} has not been migrated yet.")
        if material_map is None:
            from proton_dose_m1_b200.numerics.grid import Grid
            from proton_dose_m1_b200.physics.materials import MaterialMap
            material_map = MaterialMap.from_geometry(geo, Grid.from_geometry(geo))
        self.shape = tuple(int(n) for n in geo.resolution)
        self.materials = tuple(material_map.materials)
        self.ids = np.ascontiguousarray(np.asarray(material_map.ids), dtype=np.int32)
        self._keep = []
        mats = (_MatDesc * len(self.materials))()
        for k, m in enumerate(self.materials):
            t = material_tables(m.value)
            arrs = [np.ascontiguousarray(a, dtype=float) for a in
                    (t.sp_energy, t.sp_value, t.tr_energy, t.tr_value, t.nuc_energy, t.nuc_value)]
            self._keep += arrs
            mats[k] = _MatDesc(len(arrs[0]), _ptr(arrs[0]), _ptr(arrs[1]),
                               len(arrs[2]), _ptr(arrs[2]), _ptr(arrs[3]),
                               len(arrs[4]), _ptr(arrs[4]), _ptr(arrs[5]),
                               t.density, t.radiation_length)
        self._mats = mats
        d = _ProbDesc()
        d.nx, d.ny, d.nz = self.shape
        d.lx, d.ly, d.lz = (float(s) for s in geo.size)
        d.n_materials = len(self.materials)
        d.materials = mats
        d.ids = self.ids.ctypes.data_as(_ip)
        d.n_protons, d.energy, d.energy_spread = beam.n_protons, beam.energy, beam.energy_spread
        d.sigma_x, d.sigma_y = beam.sigma
        d.center_x, d.center_y = beam.center
        d.angular_spread, d.cutoff_sigma = beam.angular_spread, beam.cutoff_sigma
        d.scattering = _SCATTER[phys.scattering.name]
        d.nuclear = int(bool(phys.nuclear))
        d.interpolation = _INTERP[phys.coefficient_interpolation.name]
        d.energy_scheme = _SCHEME[num.energy_scheme.name]
        d.wave_speeds = _SPEEDS[num.wave_speeds.name]
        d.max_energy_step, d.cfl = num.max_energy_step, num.cfl
        d.energy_min, d.energy_window_sigma = num.energy_min, num.energy_window_sigma
        d.moving_active_domain = int(bool(num.moving_active_domain))
        d.vacuum_aware_cfl = int(bool(num.vacuum_aware_cfl))
        d.active_guard_cells = int(num.active_guard_cells)
        d.active_truncation_sigma = num.active_truncation_sigma
        d.store_final_state = int(bool(getattr(config.output, "store_final_state", True)))
        d.spatial_scheme = _SPATIAL[num.spatial_scheme.name]
        if beam.energy_spread == 0:
            raise ValueError("Zero energy spread is not supported by the Gaussian inflow.")
        self._desc = d
        h = C.c_void_p()
        _check(lib().orc_problem_create(C.byref(d), C.byref(h)))
        self._h = h
        self.config = config

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.orc_problem_destroy(h)
            self._h = None

    # -- building blocks ---------------------------------------------------
    def stopping_power(self, material_index, energy):
        out = C.c_double()
        _check(lib().orc_stopping_power(self._h, material_index, energy, C.byref(out)))
        return out.value

    def transport_coefficient(self, material_index, energy):
        out = C.c_double()
        _check(lib().orc_transport_coefficient(self._h, material_index, energy, C.byref(out)))
        return out.value

    def nuclear_coefficient(self, material_index, energy):
        out = C.c_double()
        _check(lib().orc_nuclear_coefficient(self._h, material_index, energy, C.byref(out)))
        return out.value

    def optical_depths(self, material_index, energy, dE):
        a, b = C.c_double(), C.c_double()
        _check(lib().orc_optical_depths(self._h, material_index, energy, dE, C.byref(a), C.byref(b)))
        return a.value, b.value

    def inflow_spatial(self):
        out = np.empty(self.shape[:2])
        lib().orc_inflow_spatial(self._h, _ptr(out))
        return out

    def inflow_state(self, energy):
        out = np.empty((4, *self.shape[:2]))
        lib().orc_inflow_state(self._h, energy, _ptr(out))
        return out

    def spatial_operator(self, U, energy, boundary_state=None):
        U = np.ascontiguousarray(U, dtype=float)
        bc = None if boundary_state is None else np.ascontiguousarray(boundary_state, dtype=float)
        rhs = np.empty_like(U)
        _check(lib().orc_spatial_operator(self._h, _ptr(U), energy, _ptr(bc), _ptr(rhs)))
        return rhs

    def energy_step(self, U, energy):
        U = np.ascontiguousarray(U, dtype=float)
        out = C.c_double()
        _check(lib().orc_energy_step(self._h, _ptr(U), energy, C.byref(out)))
        return out.value

    def advance(self, U, energy, dE):
        U = np.array(U, dtype=float, order="C")
        edep = np.empty(self.shape)
        _check(lib().orc_advance(self._h, _ptr(U), energy, dE, _ptr(edep)))
        return U, edep

    def set_schedule(self, energies=None):
        """March through the given energies instead of the CFL steps (None: CFL rule)."""
        E = np.ascontiguousarray([] if energies is None else energies, dtype=float)
        self._schedule = E
        _check(lib().orc_set_schedule(self._h, _ptr(E) if len(E) else None, len(E)))

    # -- the march ----------------------------------------------------------
    def march(self, U=None, snapshot_energies=(), max_steps=200000):
        """Return (U, dose, energies, snapshots) like numerics/energy.py:energy_march."""
        moving = bool(self._desc.moving_active_domain)
        if U is None and not moving:
            raise ValueError("A full-grid initial state is required when "
                             "moving_active_domain is disabled.")
        Ub = np.zeros((4, *self.shape)) if U is None else np.array(U, dtype=float, order="C")
        dose = np.empty(self.shape)
        energies = np.empty(max_steps + 1)
        n_steps = C.c_int()
        snaps = np.ascontiguousarray(sorted({float(t) for t in snapshot_energies}), dtype=float)
        ns = len(snaps)
        snap_out = np.empty((max(ns, 1), 4, *self.shape)) if ns else None
        snap_E = np.empty(max(ns, 1))
        taken, final = C.c_int(), C.c_int()
        _check(lib().orc_march(self._h, _ptr(Ub), _ptr(dose), _ptr(energies), max_steps,
                               C.byref(n_steps), _ptr(snaps) if ns else None, ns,
                               _ptr(snap_out), _ptr(snap_E), C.byref(taken), C.byref(final)))
        snapshots = {float(snap_E[i]): snap_out[i].copy() for i in range(taken.value)}
        U_out = Ub if final.value else None
        return U_out, dose, energies[: n_steps.value + 1].copy(), snapshots

    def march_steps(self, steps, U=None):
        """Run at most ``steps`` energy steps (bounded timing sample)."""
        Ub = np.zeros((4, *self.shape)) if U is None else np.array(U, dtype=float, order="C")
        dose = np.empty(self.shape)
        done = C.c_int()
        _check(lib().orc_march_steps(self._h, _ptr(Ub), _ptr(dose), int(steps), C.byref(done)))
        return Ub, dose, done.value
