"""Benchmark of the M1 energy march on B200.

Default workload: pelvis1024, a 1024-spot scanning field on a 256x256x320
synthetic pelvis at 1 mm, in the accelerated form (moving active box,
batched spots, FP32 stencil / FP64 dose, autotuned tile).  A "step" marches
one batch of the field's spots (1/K of them, by decreasing energy) as one
batched march; the K timed steps march the whole field once, and ``value``
is the field's spots/s with inputs resident in HBM, timed with CUDA events
on the march stream.  ``e2e`` is the same through the public
``field_march`` call with host NumPy buffers (upload and copy-back inside
the timed region).  ``gate`` scores a sample of the field's spots against
the plain FP64 full-domain GPU march (gamma 1%/1 mm, max dose).

Single-spot workloads (slab80, water40): a step is one complete march of
the spot.

``--impl reference`` times the reference's own CPU path on the host cores:
one complete moving-box spot march per step, through the unmodified
reference's Numba energy_march where baseline/install_reference.sh installed
it under baseline/_ref, else through the CPU restatement (oracle/).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       [--workload pelvis1024|field256|slab80|water40] [--box heuristic|learned]
       [--precision fp32|fp64]
Under torchrun (N > 1) the field's spots are shared out over the ranks
(longest-processing-time), each rank marches its share, and one all-reduce
sums the FP64 dose; rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "spots/s at gamma1%/1mm>=99.5% vs plain FP64 GPU path; stage-kernel HBM GB/s"
# Algorithmic DRAM bytes per cell-step of the march (three stages), every array
# once per use: U^n read by each stage (96), the stage states U1 and U2 written
# and read (FP64: 128; the FP32 form keeps them as float4: 64), U^{n+1} written
# (32), the marched variable V written, read and written, read (128), the dose
# quadrature part (FP64: 16; FP32: 32, stage B adds its term), the dose read and
# written (16), the int32 material ids per stage (12).
ALG_BYTES_PER_CELL_STEP = {"FP64": 428.0, "FP32_FP64": 380.0}
# Algorithmic floating-point operations per cell-step of the WENO-Z march:
# three stages x (three owned faces x (8 reconstructions, 2 projections, HLL
# with both closures and wave-speed pairs) + divergence and stage update),
# each +, -, *, / and sqrt counted once (oracle/flops.py tallies them; the
# CPU test suite keeps the two equal).
FLOPS_PER_CELL_STEP = 7479
# Non-tensor peaks of the CUDA cores: 148 SMs x lanes per SM x 2 (FMA) x the
# 1965 MHz maximum SM clock; nominal, no measured figure exists for them.
CORE_PEAK_TFLOPS = {"FP32_FP64": 148 * 128 * 2 * 1.965e-3, "FP64": 148 * 64 * 2 * 1.965e-3}
FIELDS = {
    "field256": dict(phantom="ellipsoid", seed=4, n_side=16, pitch=5e-3, energy=(70.0, 220.0),
                     gate_beams=4, precision="fp32",
                     desc="256 spots (16x16 at 5 mm, E~U[70,220] MeV, sigma~U[2,6] mm, sigma_E 1 MeV, "
                          "1e6 protons) on a 128x128x256 @1 mm water phantom with 6-12 seeded ellipsoids "
                          "of water/lung/bone/muscle; Wentzel-VI + nuclear, WENO-Z/HLL/IF-SSPRK3, "
                          "cfl 0.9, max dE 0.5"),
    # the gate scores 8 spots: one spot's maximum dose moves by up to ~1 % with
    # the energy-step sequence (its Bragg peak against the 1 mm voxels), and the
    # plain march's steps are set by cells of rounding-noise fluence
    "pelvis1024": dict(phantom="pelvis", seed=5, n_side=32, pitch=3e-3, energy=(70.0, 230.0),
                       gate_beams=8, precision="fp32",
                       desc="1024 spots (32x32 at 3 mm, E~U[70,230] MeV, sigma~U[2,6] mm, sigma_E 1 MeV, "
                            "1e6 protons) on a 256x256x320 @1 mm synthetic pelvis (water/muscle body, "
                            "ADIPOSE_SYNTH shell = water scaled to 950 kg/m3, bone ring, two bone femoral "
                            "heads, water outside); Wentzel-VI + nuclear, WENO-Z/HLL/IF-SSPRK3, cfl 0.9, "
                            "max dE 0.5"),
}


def workload(name: str):
    from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
    from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
    if name == "slab80":
        geo = Geometry(size=(0.04, 0.04, 0.2), resolution=(80, 80, 400),
                       objects=[Box(-0.02, 0.02, -0.02, 0.02, 0.08, 0.10, Material.BONE_COMPACT)])
        cfg = SolverConfig(
            geometry=geo,
            beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)),
            physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
            numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
        desc = ("80x80x400 @0.5 mm water + 2 cm bone slab at 8 cm depth, 150 MeV, sigma 3 mm, "
                "sigma_E 1 MeV, Wentzel-VI + nuclear, WENO-Z/HLL/IF-SSPRK3, cfl 0.9, max dE 0.5")
        return cfg, desc
    if name == "water40":
        geo = Geometry(size=(0.04, 0.04, 0.2), resolution=(40, 40, 200))
        cfg = SolverConfig(
            geometry=geo,
            beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)),
            numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
        desc = "40x40x200 @1 mm water, 150 MeV, sigma 3 mm, sigma_E 1 MeV, CSDA only"
        return cfg, desc
    raise SystemExit(f"unknown workload {name}")


def field_workload(name: str):
    """(config template, material map, grid, beams, description) of a field workload."""
    from proton_dose_m1_b200 import Numerics, Physics, SolverConfig, phantoms
    from proton_dose_m1_b200.enums import EnergyScheme, Scattering
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    w = FIELDS[name]
    if w["phantom"] == "ellipsoid":
        geo, _ = phantoms.ellipsoid_phantom(w["seed"])
    else:
        geo, _ = phantoms.pelvis_phantom(w["seed"])
    beams = phantoms.spot_grid(w["seed"], w["n_side"], w["pitch"], energy_mev=w["energy"])
    cfg = SolverConfig(geometry=geo, beam=beams[0],
                       physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
    grid = Grid.from_geometry(geo)
    return cfg, MaterialMap.from_geometry(geo, grid), grid, beams, w["desc"]


def gate_sample(beams, n):
    """``n`` spots spread over the field's energy range (quantiles of energy)."""
    order = sorted(range(len(beams)), key=lambda k: beams[k].energy)
    if n >= len(beams):
        return order
    return [order[int(round(q * (len(order) - 1)))] for q in np.linspace(0.1, 0.9, n)]


def problem(cfg):
    from proton_dose_m1_b200.numerics.boundary import BeamInflow
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    grid = Grid.from_geometry(cfg.geometry)
    return MaterialMap.from_geometry(cfg.geometry, grid), grid, BeamInflow.from_beam(cfg.beam, grid)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "0x1") or flag == "1":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def stage_traffic(key, cell_steps, stage_launches):
    """DRAM bytes per stage launch from the committed ncu measurement of this
    workload and method: either bytes per launch, or bytes per cell-step
    (measured over every stage launch of a smaller run of the same kernels)
    scaled by the cell-steps of this run."""
    prof = ROOT / "profiles" / "stage_kernel_traffic.json"
    if not prof.exists():
        return None
    entry = json.loads(prof.read_text()).get(key)
    if entry is None:
        return None
    if "bytes_per_cell_step" in entry:
        return entry["bytes_per_cell_step"] * cell_steps / max(stage_launches, 1)
    return entry.get("bytes_per_launch")


def compute_roofline(cell_steps, stage_ms, precision):
    """The stage kernels are issue-bound on the CUDA cores, not HBM-bound: the
    algorithmic FLOP rate of the stage launches against the nominal core peak
    of the stencil's precision."""
    achieved = cell_steps * FLOPS_PER_CELL_STEP / (stage_ms / 1e3) / 1e12 if stage_ms > 0 else 0.0
    peak = CORE_PEAK_TFLOPS[precision]
    return {"unit": "TFLOP/s", "achieved": achieved, "peak": peak, "frac": achieved / peak,
            "flops_per_cell_step": FLOPS_PER_CELL_STEP,
            "peak_source": f"nominal {'FP32' if precision == 'FP32_FP64' else 'FP64'} CUDA-core peak "
                           "(148 SMs x lanes x 2 x 1965 MHz), not measured"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def static_config(cfg, beam=None):
    """``cfg`` on the full domain (no moving box), optionally with another beam."""
    from dataclasses import replace
    from proton_dose_m1_b200 import SolverConfig
    return SolverConfig(geometry=cfg.geometry, beam=beam or cfg.beam, physics=cfg.physics,
                        numerics=replace(cfg.numerics, moving_active_domain=False))


def reference_sample(workload_name: str, n: int):
    """``n`` spots of a workload for the CPU reference: (config, material map,
    energy) each, on the reference's moving active box (its fastest CPU mode,
    numerics/energy.py:1262-1494, with its own CFL rule).  Fields: the spots at
    the energy quantiles (k + 1/2) / n of the field; single-spot workloads: the
    workload's spot."""
    from dataclasses import replace
    from proton_dose_m1_b200 import SolverConfig
    if workload_name in FIELDS:
        cfg, mm, grid, beams, _ = field_workload(workload_name)
        order = sorted(range(len(beams)), key=lambda k: beams[k].energy)
        picks = [order[min(len(order) - 1, int((k + 0.5) * len(order) / n))] for k in range(n)]
        out = []
        for k in picks:
            c = SolverConfig(geometry=cfg.geometry, beam=beams[k], physics=cfg.physics,
                             numerics=replace(cfg.numerics, moving_active_domain=True))
            out.append((c, mm, beams[k].energy))
        return out
    cfg, _ = workload(workload_name)
    c = SolverConfig(geometry=cfg.geometry, beam=cfg.beam, physics=cfg.physics,
                     numerics=replace(cfg.numerics, moving_active_domain=True))
    return [(c, None, cfg.beam.energy)] * n


def oracle_spots(sample, workers: int, threads_per_worker: int):
    """March every spot of ``sample`` completely with the oracle (moving box),
    ``workers`` spots at a time, each on ``threads_per_worker`` OpenMP
    threads.  Returns (wall seconds, [(energy, steps, seconds)])."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.oracle import OracleProblem, set_threads

    def one(item):
        cfg, mm, energy = item
        set_threads(threads_per_worker)   # per host thread (OpenMP nthreads-var)
        prob = OracleProblem(cfg, mm)
        t0 = time.perf_counter()
        _, _, E, _ = prob.march(None)
        return energy, len(E) - 1, time.perf_counter() - t0

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=workers) as pool:
        rows = list(pool.map(one, sample))
    return time.perf_counter() - t0, rows


def host_split(n_spots: int):
    """(workers, OpenMP threads per worker) over this host's cores.  The
    oracle's per-spot OpenMP loops scale to ~4.6x on 8 threads; several spots
    at once on fewer threads each use the cores better (1.7x on 8 cores)."""
    cores = os.cpu_count() or 1
    workers = max(1, min(n_spots, cores // 2 if cores >= 4 else 1, 8))
    return workers, max(1, cores // workers)


def cpu_baseline(workload_name: str, n: int = 2):
    """Oracle throughput on a bounded sample of the workload: ``n`` complete
    moving-box spots (the reference's fastest CPU mode), marched concurrently
    over the host cores; spots/s = n / wall time."""
    sample = reference_sample(workload_name, n)
    workers, tpw = host_split(len(sample))
    wall, rows = oracle_spots(sample, workers, tpw)
    return {"value": len(sample) / wall, "unit": "spots/s", "cores": workers * tpw, "kind": "port",
            "sample": f"{len(sample)} complete moving-box spot marches (energies "
                      f"{[round(r[0], 1) for r in rows]} MeV, {[r[1] for r in rows]} energy steps) in "
                      f"{wall:.1f} s, {workers} at a time x {tpw} OpenMP threads"}


# The unmodified reference, installed by baseline/install_reference.sh: the
# package under lib/ and its material tables under data/, where the package's
# own path lookups (physics/materials.py:13 and its siblings: three directories
# above the module) find them.
REF_LIB = ROOT / "baseline" / "_ref" / "lib"
# Numba threads per reference worker process: the reference's parallel loops
# scale poorly past ~4 threads (a 89.5 MeV pelvis spot: 18.9 s on 4 threads,
# 16.9 s on 8), so several spots at once on 4 threads each use the cores better.
REF_THREADS_PER_WORKER = 4
# seconds between the reference arm's checks on its workers while it waits
REF_POLL_S = 30.0


def reference_installed() -> bool:
    import importlib.util
    return ((REF_LIB / "proton_solver" / "__init__.py").exists()
            and (REF_LIB.parent / "data" / "materials.csv").exists()
            and importlib.util.find_spec("numba") is not None)


def import_installed_reference():
    """Import the installed reference.  Its package imports plotting and
    gamma-index modules at import time that are not on the energy-march path
    and not in this image (matplotlib, pymedphys): empty stand-ins take their
    names; no reference code is changed."""
    import types
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/pdm1_numba_cache")
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.lines", "matplotlib.patches",
                 "mpl_toolkits", "mpl_toolkits.mplot3d", "mpl_toolkits.mplot3d.art3d", "pymedphys"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["matplotlib.lines"].Line2D = object
    sys.modules["matplotlib.patches"].Patch = object
    sys.modules["mpl_toolkits.mplot3d.art3d"].Poly3DCollection = object
    if str(REF_LIB) not in sys.path:
        sys.path.insert(0, str(REF_LIB))
    import proton_solver
    return proton_solver


def reference_material_map(cfg, mm):
    """The reference's MaterialMap of a workload's phantom, built from its
    voxel ids (``mm``; None: voxelised from ``cfg.geometry``).  Materials are
    keyed by table name, the key of the reference's coefficient tables
    (physics/materials.py:26-60): its Material enum lists only water, compact
    bone and lung, and its data/ tables also hold skeletal muscle and air.
    ADIPOSE_SYNTH (water scaled to 950 kg/m3) takes the tables that
    baseline/synth_tables.py wrote into the installed data, or, where they
    are missing, marches as water."""
    import enum
    from proton_solver.physics.materials import MaterialMap as RefMap
    from proton_dose_m1_b200.numerics.grid import Grid
    from proton_dose_m1_b200.physics.materials import MaterialMap
    if mm is None:
        mm = MaterialMap.from_geometry(cfg.geometry, Grid.from_geometry(cfg.geometry))
    data = REF_LIB.parent / "data"
    names = [m.value if m.value != "ADIPOSE_SYNTH" or (data / "stopping_power" / f"{m.value}.csv").exists()
             else "G4_WATER" for m in mm.materials]
    uniq = list(dict.fromkeys(names))
    G4 = enum.Enum("G4", {n: n for n in uniq})
    remap = np.array([uniq.index(n) for n in names], dtype=np.int32)
    return RefMap(ids=np.ascontiguousarray(remap[np.asarray(mm.ids)]), materials=tuple(G4(n) for n in uniq))


def reference_spot(ps, cfg):
    """The reference's own (config, grid, inflow) for one spot of a workload,
    on its moving active box."""
    from proton_solver.numerics.boundary import BeamInflow as RefInflow
    from proton_solver.numerics.grid import Grid as RefGrid
    b, n = cfg.beam, cfg.numerics
    beam = ps.Beam(n_protons=b.n_protons, energy=b.energy, energy_spread=b.energy_spread,
                   sigma=tuple(b.sigma), center=tuple(b.center), angular_spread=b.angular_spread,
                   cutoff_sigma=b.cutoff_sigma)
    rcfg = ps.SolverConfig(
        geometry=ps.Geometry(size=tuple(cfg.geometry.size), resolution=tuple(cfg.geometry.resolution)),
        beam=beam,
        physics=ps.Physics(scattering=ps.Scattering[cfg.physics.scattering.name],
                           nuclear=cfg.physics.nuclear),
        numerics=ps.Numerics(energy_scheme=ps.EnergyScheme[n.energy_scheme.name], cfl=n.cfl,
                             max_energy_step=n.max_energy_step, moving_active_domain=True),
        backend=ps.Backend.CPU, references=ps.References(reference=ps.Reference.NONE))
    grid = RefGrid.from_geometry(rcfg.geometry, np)
    return rcfg, grid, RefInflow.from_beam(beam, grid, np)


def _reference_warm_inputs(ps):
    """(config, grid, material map, inflow) of a small problem with the
    workloads' physics and scheme (24x24x60 at 1 mm, water with a compact-bone
    block, 45 MeV): marching it compiles every Numba kernel of the reference's
    moving march, untimed."""
    from proton_dose_m1_b200 import Beam, Box, Geometry, Numerics, Physics, SolverConfig
    from proton_dose_m1_b200.enums import EnergyScheme, Material, Scattering
    cfg = SolverConfig(
        geometry=Geometry(size=(0.024, 0.024, 0.06), resolution=(24, 24, 60),
                          objects=[Box(-0.012, 0.012, -0.012, 0.012, 0.01, 0.014, Material.BONE_COMPACT)]),
        beam=Beam(n_protons=1e6, energy=45.0, energy_spread=1.0, sigma=(0.003, 0.003)),
        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
    rcfg, grid, inflow = reference_spot(ps, cfg)
    return rcfg, grid, reference_material_map(cfg, None), inflow


def _reference_worker(workload_name, n_spots, warmup, barrier, todo, done):
    """One reference worker process: build the spots' inputs and compile the
    reference (untimed), wait for the others, then march complete spots from
    ``todo`` with the reference's own energy_march until it is empty."""
    try:
        ps = import_installed_reference()
        from proton_solver.numerics.energy import energy_march as reference_march
        sample = reference_sample(workload_name, n_spots)
        warm = _reference_warm_inputs(ps)
        for _ in range(max(1, warmup)):
            reference_march(None, warm[2], warm[1], warm[3], warm[0], np)
        # fields share one phantom: one material map for all their spots
        ref_map = reference_material_map(sample[0][0], sample[0][1])
        inputs = [(*reference_spot(ps, cfg), ref_map) for cfg, _, _ in sample]
    except BaseException as exc:   # tell the parent instead of leaving it waiting
        barrier.abort()
        done.put(("error", repr(exc)))
        return
    barrier.wait()
    while True:
        k = todo.get()
        if k is None:
            return
        rcfg, grid, inflow, rmm = inputs[k]
        t0 = time.perf_counter()
        _, dose, energies, _ = reference_march(None, rmm, grid, inflow, rcfg, np)
        done.put((k, len(energies) - 1, time.perf_counter() - t0, float(dose.max())))


def run_reference(args, rank, world):
    """The reference's CPU path on the host cores, rank 0 only: every timed
    step marches one complete spot of the workload on the reference's moving
    active box (its fastest CPU mode, numerics/energy.py:1262-1494, with its
    own CFL rule).  The unmodified reference (Numba) when it is installed under
    baseline/_ref, else the oracle."""
    if rank != 0:
        return
    if reference_installed():
        run_reference_numba(args, world)
    else:
        run_reference_port(args, world)


def run_reference_port(args, world):
    """The oracle (CPU restatement of the reference path) on the host cores:
    the K spots run concurrently over the cores (spot-level parallelism on top
    of the oracle's OpenMP loops)."""
    desc = FIELDS[args.workload]["desc"] if args.workload in FIELDS else workload(args.workload)[1]
    sample = reference_sample(args.workload, args.steps)
    workers, tpw = host_split(len(sample))
    # warm-up: the first energy steps of one spot (the oracle has no JIT to warm)
    from oracle.oracle import OracleProblem, set_threads
    set_threads(workers * tpw)
    warm = OracleProblem(sample[0][0], sample[0][1])
    for _ in range(args.warmup):
        warm.march_steps(2)
    del warm
    wall, rows = oracle_spots(sample, workers, tpw)
    value = len(sample) / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "spots/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "strong" if args.workload in FIELDS else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded phantom, no dataset)",
        "config": {"workload": args.workload, "description": desc},
        "cpu_baseline": {"value": value, "unit": "spots/s", "cores": workers * tpw, "kind": "port",
                         "sample": f"{len(sample)} complete moving-box spot marches, one per timed step "
                                   f"(energies {[round(r[0], 1) for r in rows]} MeV; "
                                   f"{[r[1] for r in rows]} energy steps; "
                                   f"{[round(r[2], 1) for r in rows]} s each), {workers} at a time x "
                                   f"{tpw} OpenMP threads, {wall:.1f} s wall"},
        "e2e": {"value": value, "unit": "spots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference_numba(args, world):
    """The unmodified reference's Numba march (its own energy_march, moving
    active box) in ``cores / 4`` spawned worker processes of 4 Numba threads
    each.  The workers build their inputs and compile the reference before the
    clock starts; the K spots go out largest energy first to whichever worker
    is free, and ``value`` = K / the wall time until the last one is done."""
    import multiprocessing as mp
    import queue
    desc = FIELDS[args.workload]["desc"] if args.workload in FIELDS else workload(args.workload)[1]
    k_spots = args.steps
    # the CPUs this process may run on (a container can see more than it gets)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    threads = min(REF_THREADS_PER_WORKER, cores)
    workers = max(1, min(k_spots, cores // threads))
    # Numba reads its thread count when it is first imported: the spawned
    # workers inherit it from this environment
    os.environ["NUMBA_NUM_THREADS"] = str(threads)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/pdm1_numba_cache")
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers + 1)
    todo, done = ctx.Queue(), ctx.Queue()
    energies = [e for _, _, e in reference_sample(args.workload, k_spots)]
    for k in sorted(range(k_spots), key=lambda i: -energies[i]):
        todo.put(k)
    for _ in range(workers):
        todo.put(None)
    procs = [ctx.Process(target=_reference_worker, args=(args.workload, k_spots, args.warmup, barrier, todo, done),
                         daemon=True) for _ in range(workers)]
    for p in procs:
        p.start()
    try:
        barrier.wait(timeout=1800)
    except Exception:
        try:   # a failed worker's message may still be on its way
            err = done.get(timeout=30)[1]
        except queue.Empty:
            err = "a reference worker did not reach the start"
        raise SystemExit(f"reference workers failed before timing: {err}")
    t0 = time.perf_counter()
    rows = {}
    while len(rows) < k_spots:
        try:
            item = done.get(timeout=REF_POLL_S)
        except queue.Empty:
            # a worker with no spot left exits with status 0 while the others
            # still march: only a failed worker, or all of them gone with
            # spots missing, ends the run
            if any(p.exitcode not in (None, 0) for p in procs):
                raise SystemExit("a reference worker failed while marching")
            if all(p.exitcode is not None for p in procs) and done.empty():
                raise SystemExit("the reference workers exited before marching every spot")
            continue
        if item[0] == "error":
            raise SystemExit(f"reference worker failed: {item[1]}")
        rows[item[0]] = item[1:]
    wall = time.perf_counter() - t0
    for p in procs:
        p.join(timeout=60)
    value = k_spots / wall
    order = range(k_spots)
    adipose = (REF_LIB.parent / "data" / "stopping_power" / "ADIPOSE_SYNTH.csv").exists()
    sample = (f"{k_spots} complete moving-box spot marches of the unmodified reference "
              f"(proton_solver energy_march, Numba, NUMBA_NUM_THREADS={threads}), one per timed step: "
              f"energies {[round(energies[k], 1) for k in order]} MeV, "
              f"{[rows[k][0] for k in order]} energy steps, {[round(rows[k][1], 1) for k in order]} s each; "
              f"{workers} worker processes at a time, {wall:.1f} s wall after JIT warm-up"
              + (f"; ADIPOSE_SYNTH shell {'on the tables of baseline/synth_tables.py' if adipose else 'marched as water'}"
                 if args.workload == "pelvis1024" else ""))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "spots/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
        "scaling": "strong" if args.workload in FIELDS else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded phantom, no dataset)",
        "config": {"workload": args.workload, "description": desc},
        "cpu_baseline": {"value": value, "unit": "spots/s", "cores": workers * threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "spots/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Moving box of the accelerated form (--box): fields march the learned proposer
# (24 % fewer cell-steps than the fixed heuristic on pelvis spots, 1.21x the
# spots/s); single spots the heuristic (there the learned box's per-step work
# costs about what the cells it saves do).
BOX = "learned"
# Stencil arithmetic of the accelerated form (--precision): "fp32" (FP32
# stencil / FP64 dose) or "fp64".  Field workloads override the default with
# their own (FIELDS[...]["precision"]).
PRECISION = "fp32"


TILE_OVERRIDE = []   # --tile: a fixed stage tile shape instead of the autotuner's


def accelerated_config(cfg):
    """The accelerated form: moving active box (learned proposer, or the fixed
    heuristic) + FP32 stencil / FP64 dose + autotuned tile shape."""
    from dataclasses import replace
    from proton_dose_m1_b200 import Accel, SolverConfig, learned_box
    from proton_dose_m1_b200.enums import Precision
    model = learned_box.default_model() if BOX == "learned" else None
    precision = Precision.FP32_FP64 if PRECISION == "fp32" else Precision.FP64
    return SolverConfig(geometry=cfg.geometry, beam=cfg.beam, physics=cfg.physics,
                        numerics=replace(cfg.numerics, moving_active_domain=True),
                        accel=Accel(precision=precision, box_model=model,
                                    tile=TILE_OVERRIDE[0] if TILE_OVERRIDE else "auto", phantom_cfl=True))


def accelerated_label():
    arith = "FP32 stencil / FP64 dose" if PRECISION == "fp32" else "FP64"
    return f"moving active box ({BOX}, phantom-wide CFL bound) + {arith} + autotuned tile"


def run_ours(args, cfg, desc, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from proton_dose_m1_b200 import metrics
    from proton_dose_m1_b200.numerics.energy import M1Plan, energy_march

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    mm, grid, inflow = problem(cfg)
    run_cfg = accelerated_config(cfg) if args.method == "accelerated" else cfg
    precision = run_cfg.accel.precision.name
    plan = M1Plan(run_cfg, mm, grid, inflow)
    shape = grid.shape
    stream = torch.cuda.Stream(device=dev)
    U = torch.zeros((4, *shape), dtype=torch.float64, device=dev)
    dose = torch.empty(shape, dtype=torch.float64, device=dev)
    energies = torch.empty(200_001, dtype=torch.float64, device=dev)

    def one_spot(p=plan, d=dose):
        U.zero_()
        return p.march_device(U, d, energies)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one_spot()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stage_ms, stage_launches, launches, n_steps, cell_steps = 0.0, 0, 0, 0, 0.0
        with ClockSampler(local_rank) as clocks:
            start.record(stream)
            for _ in range(args.steps):
                n, _ = one_spot()
                info = plan.last_info
                stage_ms += info.stage_ms
                stage_launches += info.stage_launches
                cell_steps += info.cell_steps
                launches += info.kernel_launches + 1   # + the zero fill
                n_steps = n
            end.record(stream)
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = start.elapsed_time(end)
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        value = world * args.steps / (ms / 1e3)

        # gate: the same spot on the plain FP64 full-domain path (untimed here)
        gate = None
        plain_spots_per_s = None
        if args.method == "accelerated" and rank == 0:
            plain = M1Plan(cfg, mm, grid, inflow)
            dose_plain = torch.empty_like(dose)
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            one_spot(plain, dose_plain)
            s1.record(stream)
            torch.cuda.synchronize()
            plain_spots_per_s = 1e3 / s0.elapsed_time(s1)
            one_spot()
            torch.cuda.synchronize()
            score = metrics.compare(dose, dose_plain, grid)
            gate = {"vs": "plain FP64 GPU path (full domain)",
                    "gamma_1pct_1mm_pass_percent": score["gamma_1pct_1mm_pass_percent"],
                    "max_dose_relative_difference": score["maximum_dose_relative_difference"],
                    "max_abs_difference_over_max": score["max_abs_difference_over_max"],
                    "r80_difference_mm": score["range"]["r80_difference_mm"],
                    "dfw_difference_mm": score["range"]["dfw_difference_mm"],
                    "passed": bool(score["gamma_1pct_1mm_pass_percent"] >= 99.5
                                   and abs(score["maximum_dose_relative_difference"]) <= 0.005)}
            plain.close()

    # end to end through the public API with host buffers
    U_host = np.zeros((4, *shape))
    for _ in range(min(args.warmup, 1)):   # untimed, like the warm-up of `value`
        energy_march(U_host, mm, grid, inflow, run_cfg, np)
    e2e_times = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Uo, doseo, Eo, _ = energy_march(U_host, mm, grid, inflow, run_cfg, np)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = sum(e2e_times) / len(e2e_times)
    h2d = U_host.nbytes + mm.ids.nbytes + inflow.spatial.nbytes
    d2h = (Uo.nbytes if Uo is not None else 0) + doseo.nbytes + Eo.nbytes

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    avg_launch_ms = stage_ms / max(stage_launches, 1)
    # algorithmic bytes of the stage launches: cells marched x bytes per cell-step,
    # a third per stage launch (cell_steps already sums the domain over steps)
    alg_total = cell_steps * ALG_BYTES_PER_CELL_STEP[precision]
    achieved = alg_total / (stage_ms / 1e3) / 1e9 if stage_ms > 0 else 0.0
    traffic = stage_traffic(f"{args.workload}/{args.method}", cell_steps, stage_launches)
    line = {
        "metric": METRIC, "value": value, "unit": "spots/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 stencil / f64 dose" if precision == "FP32_FP64" else "f64",
        "data": "synthetic (analytic phantom, no dataset)",
        "config": {"workload": args.workload, "description": desc,
                   "method": accelerated_label() if args.method == "accelerated" else "plain FP64, full domain",
                   "energy_steps_per_spot": n_steps,
                   "cells_marched_per_spot": cell_steps / max(args.steps, 1),
                   "plain_fp64_spots_per_s": plain_spots_per_s,
                   "l2": "working set (state, two stage states, V, dose: ~350 MB) exceeds the 126 MB L2"},
        "gate": gate,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": f"stage_kernel<{'float' if precision == 'FP32_FP64' else 'double'}> (A/B/C)",
                     "avg_launch_ms": avg_launch_ms,
                     "algorithmic_bytes_per_launch": alg_total / max(stage_launches, 1),
                     "algorithmic_bytes_per_cell_step": ALG_BYTES_PER_CELL_STEP[precision],
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "compute": compute_roofline(cell_steps, stage_ms, precision)},
        "e2e": {"value": 1.0 / e2e_s, "unit": "spots/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, 1)
    print(json.dumps(line), flush=True)


def field_batches(share, beams, k):
    """This rank's spots, highest energy first, in ``k`` contiguous batches of
    near-equal size: the batches of one step take similar numbers of energy
    steps, and the ``k`` timed steps march every spot of the share once."""
    order = sorted(share, key=lambda i: (-beams[i].energy, i))
    n = len(order)
    return [order[(q * n) // k:((q + 1) * n) // k] for q in range(k)]


def run_field(args, rank, world, local_rank):
    """A spot-scanning field.  One step marches one batch of the field's
    spots (1/K of them, by decreasing energy) as one batched field march; the
    K timed steps together march the whole field once, so ``value`` is the
    field's spots over the time of all K steps.  Over N ranks the spots are
    shared out first (sharding.sharded_field_dose, longest-processing-time on
    the moving-box cost model) and one all-reduce sums the FP64 field dose."""
    import torch
    import torch.distributed as dist
    from proton_dose_m1_b200 import metrics
    from proton_dose_m1_b200.numerics.boundary import BeamInflow, transverse_profile
    from proton_dose_m1_b200.numerics.energy import FieldPlan, M1Plan, field_march
    from proton_dose_m1_b200.sharding import assign_spots, sharded_field_dose, spot_cost

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cfg, mm, grid, beams, desc = field_workload(args.workload)
    run_cfg = accelerated_config(cfg)
    costs = [spot_cost(b, run_cfg, grid) for b in beams]
    n_spots = len(beams)
    K = args.steps
    stream = torch.cuda.Stream(device=dev)
    # inflow profiles of every spot: input data, computed once outside the timed region
    profiles = [np.ascontiguousarray(b.n_protons * transverse_profile(b, grid)) for b in beams]

    def reduce_dose(d):
        if world > 1:
            dist.all_reduce(d)

    def march_batches(share, batches, stats=None):
        """Dose of ``share`` marched in ``batches`` steps (device)."""
        dose = torch.zeros(grid.shape, dtype=torch.float64, device=dev)
        part = torch.empty_like(dose)
        for batch in field_batches(share, beams, batches):
            if not batch:
                continue
            plan = FieldPlan(run_cfg, mm, grid, [beams[i] for i in batch],
                             profiles=[profiles[i] for i in batch])
            steps = plan.march_device(part)
            dose.add_(part)
            if stats is not None:
                info = plan.last_info
                stats["stage_ms"] += info.stage_ms
                stats["stage_launches"] += info.stage_launches
                stats["launches"] += info.kernel_launches + 1   # + the dose sum
                stats["cell_steps"] += info.cell_steps
                stats["max_box"] = max(stats["max_box"], info.max_box_cells)
                stats["waves"] += len(plan.waves)
                stats["cap"] = max(stats["cap"], plan.cap)
                stats["retries"] += plan.capacity_retries
                stats["grow"] += info.box_grow_events
                stats["fallbacks"] += info.box_fallbacks
                stats["steps"] += list(steps)
            plan.close()
        return dose

    stats = dict(stage_ms=0.0, stage_launches=0, launches=0, cell_steps=0.0, max_box=0.0, waves=0,
                 cap=0, retries=0, grow=0, fallbacks=0, steps=[])
    with torch.cuda.stream(stream):
        # warm-up: the first W batches of this rank's share (the tile autotuner runs here)
        mine = assign_spots(costs, world)[rank]
        warm = [i for q in field_batches(mine, beams, K)[:args.warmup] for i in q]
        if warm:
            march_batches(warm, min(args.warmup, len(warm)))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as clocks:
            start.record(stream)
            field_dose, share = sharded_field_dose(beams, costs, rank, world,
                                                   lambda idx: march_batches(idx, K, stats), reduce_dose)
            end.record(stream)
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = start.elapsed_time(end)
        if world > 1:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        value = n_spots / (ms / 1e3)
        del field_dose

        gate = None
        plain_spots_per_s = None
        if args.gate_spots != 0:
            # gate: a sample of the field's spots, accelerated (batched, rank 0)
            # vs the plain FP64 full-domain path one spot at a time; over N
            # ranks the plain marches go round-robin by energy, so every rank
            # waits in the sums below for the others' last spot only
            sample = gate_sample(beams, args.gate_spots if args.gate_spots > 0
                                 else FIELDS[args.workload]["gate_beams"])
            sub = [beams[k] for k in sample]
            dose_acc = torch.zeros(grid.shape, dtype=torch.float64, device=dev)
            if rank == 0:
                sp = FieldPlan(run_cfg, mm, grid, sub)
                sp.march_device(dose_acc)
                sp.close()
            dose_plain = torch.zeros_like(dose_acc)
            d1 = torch.empty_like(dose_acc)
            U = torch.empty((4, *grid.shape), dtype=torch.float64, device=dev)
            energies = torch.empty(200_001, dtype=torch.float64, device=dev)
            plain_ms = 0.0
            for b in sub[rank::world]:
                pplan = M1Plan(static_config(cfg, b), mm, grid, BeamInflow.from_beam(b, grid))
                U.zero_()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                pplan.march_device(U, d1, energies)
                s1.record(stream)
                torch.cuda.synchronize()
                plain_ms += s0.elapsed_time(s1)
                dose_plain += d1
                pplan.close()
            del U
            if world > 1:
                t = torch.tensor([plain_ms], dtype=torch.float64, device=dev)
                dist.all_reduce(t)
                plain_ms = float(t.item())
                dist.all_reduce(dose_plain)
            # one GPU's rate: the plain marches' summed device time
            plain_spots_per_s = len(sub) / (plain_ms / 1e3)
        if rank == 0 and args.gate_spots != 0:
            score = metrics.compare(dose_acc, dose_plain, grid)
            gate = {"vs": f"plain FP64 GPU path (full domain, one spot at a time) on {len(sub)} spots "
                          f"of the field (energy quantiles: {[round(b.energy, 1) for b in sub]} MeV)",
                    "gamma_1pct_1mm_pass_percent": score["gamma_1pct_1mm_pass_percent"],
                    "max_dose_relative_difference": score["maximum_dose_relative_difference"],
                    "max_abs_difference_over_max": score["max_abs_difference_over_max"],
                    "passed": bool(score["gamma_1pct_1mm_pass_percent"] >= 99.5
                                   and abs(score["maximum_dose_relative_difference"]) <= 0.005)}
            del dose_acc, dose_plain, d1

    # end to end through the public API with host buffers: field_march per
    # batch (phantom, tables and profiles uploaded, the batch's dose copied
    # back), the sum over batches and ranks on the host side
    def march_batches_host(share):
        dose_h = np.zeros(grid.shape)
        for batch in field_batches(share, beams, K):
            if batch:
                d, _ = field_march(run_cfg, mm, grid, [beams[i] for i in batch])
                dose_h += d
        return torch.from_numpy(dose_h)

    def reduce_host(d):
        if world > 1:
            dd = d.to(dev)
            dist.all_reduce(dd)
            d.copy_(dd.cpu())

    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    _, share_e2e = sharded_field_dose(beams, costs, rank, world, march_batches_host, reduce_host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    nxy = grid.shape[0] * grid.shape[1]
    n_batches = sum(1 for q in field_batches(share_e2e, beams, K) if q)
    h2d = n_batches * mm.ids.nbytes + len(share_e2e) * nxy * 8
    d2h = n_batches * int(np.prod(grid.shape)) * 8

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    precision = "FP32_FP64" if PRECISION == "fp32" else "FP64"
    alg_total = stats["cell_steps"] * ALG_BYTES_PER_CELL_STEP[precision]
    stage_ms = stats["stage_ms"]
    achieved = alg_total / (stage_ms / 1e3) / 1e9 if stage_ms > 0 else 0.0
    traffic = stage_traffic(f"{args.workload}/accelerated", stats["cell_steps"], stats["stage_launches"])
    steps = stats["steps"]
    line = {
        "metric": METRIC, "value": value, "unit": "spots/s", "n_gpus": world,
        "steps": K, "warmup": args.warmup, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 stencil / f64 dose" if PRECISION == "fp32" else "f64",
        "data": "synthetic (seeded phantom and spots, no dataset)",
        "config": {"workload": args.workload, "description": desc,
                   "method": "batched field, " + accelerated_label(),
                   "step": f"one batch of ~{n_spots // max(world, 1) // K} spots (by decreasing energy) "
                           f"per rank; the {K} timed steps march all {n_spots} spots once",
                   "spots": n_spots, "spots_rank0": len(share),
                   "waves": stats["waves"], "box_capacity_cells": stats["cap"],
                   "capacity_retries": stats["retries"],
                   "box_grow_events": stats["grow"], "box_fallbacks": stats["fallbacks"],
                   "parallelism": f"spot sharding over {world} GPU(s), one FP64 dose all-reduce",
                   "max_box_cells": stats["max_box"],
                   "energy_steps_max": max(steps, default=0), "energy_steps_min": min(steps, default=0),
                   "cells_marched_per_field": stats["cell_steps"],
                   "plain_fp64_spots_per_s": plain_spots_per_s,
                   "in_timed_region": "per batch: plan set-up from pooled buffers (phantom ids and inflow "
                                      "profiles uploaded), the batched march, the batch dose summed on device",
                   "l2": "per-spot state buffers (GBs) exceed the 126 MB L2"},
        "gate": gate,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": f"stage_kernel<{'float' if PRECISION == 'fp32' else 'double'}> (A/B/C), "
                               "all spots of a batch per launch",
                     "avg_launch_ms": stage_ms / max(stats["stage_launches"], 1),
                     "algorithmic_bytes_per_launch": alg_total / max(stats["stage_launches"], 1),
                     "algorithmic_bytes_per_cell_step": ALG_BYTES_PER_CELL_STEP[precision],
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "compute": compute_roofline(stats["cell_steps"], stage_ms, precision)},
        "e2e": {"value": n_spots / e2e_s, "unit": "spots/s", "h2d_bytes_per_step": int(h2d / K),
                "d2h_bytes_per_step": int(d2h / K)},
        "gpu_launches": stats["launches"],
        "clocks": clocks.summary(),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload, 2)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="pelvis1024")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--method", choices=("accelerated", "plain"), default="accelerated",
                    help="accelerated: moving box + FP32 stencil/FP64 dose; plain: FP64 full domain")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only run the first K energy steps of one spot (for ncu captures) and exit")
    ap.add_argument("--box", choices=("learned", "heuristic"), default=None,
                    help="moving box of the accelerated form")
    ap.add_argument("--precision", choices=("fp32", "fp64"), default=None,
                    help="stencil arithmetic of the accelerated form (default: fp32; fields: their own)")
    ap.add_argument("--tile", default=None,
                    help="stage tile shape instead of the autotuner's (e.g. 2x8x16, or 'default'; profiling)")
    ap.add_argument("--gate-spots", type=int, default=-1,
                    help="field workloads: spots of the accuracy gate (-1: the workload's own, 0: no gate)")
    ap.add_argument("--profile-spots", type=int, default=0,
                    help="field workloads: march K spots of the field once (for ncu captures) and exit")
    args = ap.parse_args()
    global BOX, PRECISION
    BOX = args.box or ("learned" if args.workload in FIELDS else "heuristic")
    PRECISION = args.precision or (FIELDS[args.workload]["precision"] if args.workload in FIELDS else "fp32")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cfg, desc = (None, None) if args.workload in FIELDS else workload(args.workload)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.tile:
        TILE_OVERRIDE.append(None if args.tile == "default" else tuple(int(v) for v in args.tile.split("x")))
    if args.profile_spots > 0 and args.workload in FIELDS and args.profile_steps > 0:
        # the first K energy steps of the spots (a bounded prefix for profiler captures)
        from proton_dose_m1_b200.numerics.energy import FieldPlan
        import torch
        fcfg, mm, grid, beams, _ = field_workload(args.workload)
        sub = [beams[k] for k in gate_sample(beams, args.profile_spots)]
        plan = FieldPlan(accelerated_config(fcfg), mm, grid, sub)
        plan.march_steps(args.profile_steps)
        torch.cuda.synchronize()
        info = plan.last_info
        print(json.dumps({"profile_spots": len(sub), "profile_steps": args.profile_steps,
                          "stage_launches": info.stage_launches, "stage_ms": info.stage_ms,
                          "cell_steps": info.cell_steps, "box_capacity_cells": plan.cap}))
        return
    if args.profile_spots > 0 and args.workload in FIELDS:
        from proton_dose_m1_b200.numerics.energy import FieldPlan
        import torch
        fcfg, mm, grid, beams, _ = field_workload(args.workload)
        sub = [beams[k] for k in gate_sample(beams, args.profile_spots)]
        plan = FieldPlan(accelerated_config(fcfg), mm, grid, sub)
        dose, steps = plan.march()
        torch.cuda.synchronize()
        info = plan.last_info
        print(json.dumps({"profile_spots": len(sub), "steps": steps, "stage_launches": info.stage_launches,
                          "stage_ms": info.stage_ms, "cell_steps": info.cell_steps,
                          "max_box_cells": info.max_box_cells, "box_capacity_cells": plan.cap}))
        return
    if args.profile_steps > 0:
        from proton_dose_m1_b200.numerics.energy import M1Plan
        import torch
        run_cfg = accelerated_config(cfg) if args.method == "accelerated" else cfg
        plan = M1Plan(run_cfg, *problem(cfg))
        U, dose, E = plan.march_steps(args.profile_steps)
        torch.cuda.synchronize()
        print(json.dumps({"profile_steps": len(E) - 1, "energy": float(E[-1]),
                          "stage_launches": plan.last_info.stage_launches,
                          "stage_ms": plan.last_info.stage_ms, "cell_steps": plan.last_info.cell_steps}))
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        if args.workload in FIELDS:
            run_field(args, rank, world, local_rank)
        else:
            run_ours(args, cfg, desc, rank, world, local_rank)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
