"""Train the learned moving-box proposer and measure what it gains.

    python -m proton_dose_m1_b200.train_box_model [--solves 200] [--test-seeds 1000 1001 1002]
           [--out proton_dose_m1_b200/data/box_model.npz] [--report report.json]

1. ``--solves`` full-domain FP64 marches of the plain method on the lateral
   water/bone interface phantom (80 x 80 x 400 at 0.5 mm, seeds 0..N-1 of
   ``learned_box.training_config``) with the recorder on;
2. samples (features; per face, how far the next step's fluence tail reaches
   beyond the significant box) and the GPU training kernels (Adam,
   asymmetric loss);
3. on held-out seeds, the learned box against the fixed heuristic box, both
   scored against the full-domain march: cell-steps marched, gamma
   (1%/1 mm), maximum-dose difference and max |dD| / max D.
"""

from __future__ import annotations

import argparse
import json
import time
from dataclasses import replace

import numpy as np

from . import learned_box, metrics


def march(config, box_model=None, moving=True, phantom_cfl=False, schedule=None, energies=None):
    """(dose, energy steps, cell-steps, grow events, fallbacks, seconds, grid).
    ``schedule``: march through these energies instead of the CFL steps;
    ``energies``: a list that receives the march's energies."""
    import torch
    from .config import Accel, SolverConfig
    from .numerics.boundary import BeamInflow
    from .numerics.energy import M1Plan
    from .numerics.grid import Grid
    from .physics.materials import MaterialMap
    cfg = SolverConfig(geometry=config.geometry, beam=config.beam, physics=config.physics,
                       numerics=replace(config.numerics, moving_active_domain=moving),
                       accel=Accel(precision=config.accel.precision, box_model=box_model,
                                   phantom_cfl=phantom_cfl))
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    if schedule is not None:
        plan.set_schedule(schedule)
    U = None if moving else torch.zeros((4, *grid.shape), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, dose, E, _ = plan.march(U)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    info = plan.last_info
    plan.close()
    if energies is not None:
        energies.extend(float(e) for e in E)
    return dose, len(E) - 1, info.cell_steps, info.box_grow_events, info.box_fallbacks, dt, grid


_REFERENCE = {}


def _reference(seed, phantom_cfl=False):
    """Full-domain dose and the heuristic-box march of a seed (cached)."""
    if seed not in _REFERENCE:
        cfg = learned_box.training_config(seed)
        full, n_full, cs_full, _, _, t_full, grid = march(cfg, moving=False)
        _REFERENCE[seed] = (cfg, full, grid, {"steps": n_full, "cell_steps": cs_full, "seconds": t_full})
    if (seed, phantom_cfl) not in _REFERENCE:
        cfg = _REFERENCE[seed][0]
        _REFERENCE[seed, phantom_cfl] = march(cfg, box_model=None, phantom_cfl=phantom_cfl)
    return (*_REFERENCE[seed], _REFERENCE[seed, phantom_cfl])


def evaluate(model, seeds, phantom_cfl=False):
    """Learned box vs heuristic box on held-out seeds (FP64 throughout); with
    ``phantom_cfl`` both boxes take the phantom-wide CFL bound."""
    rows = []
    for s in seeds:
        cfg, full, grid, full_info, heuristic = _reference(s, phantom_cfl)
        entry = {"seed": s, "energy_MeV": cfg.beam.energy, "sigma_mm": cfg.beam.sigma[0] * 1e3,
                 "full": full_info, "phantom_cfl": phantom_cfl}
        for name, bm in (("heuristic", None), ("learned", model)):
            d, n, cs, grows, fb, t, _ = (heuristic if bm is None
                                         else march(cfg, box_model=bm, phantom_cfl=phantom_cfl))
            sc = metrics.compare(d, full, grid)
            diff = (d - full)
            entry[name] = {"steps": n, "cell_steps": cs, "grow_events": grows, "fallbacks": fb, "seconds": t,
                           "gamma_1pct_1mm": sc["gamma_1pct_1mm_pass_percent"],
                           "max_dose_rel_diff": sc["maximum_dose_relative_difference"],
                           "max_abs_diff_over_max": float(abs(diff).max() / full.max())}
        rows.append(entry)
        print(json.dumps(entry), flush=True)
    return rows


def interface_case():
    """The reference's extended lateral-interface case of its moving-box study
    (thesis_results/robustness/moving_active_domain/scattering_nuclear/
    transversal_slabs/weno_z/config.json): 100 x 100 x 400 cells on
    24 x 24 x 200 mm, compact bone for x < 0 over the full depth, 150 MeV,
    sigma 2 mm, sigma_E 1 MeV, Wentzel-VI + nuclear, WENO-Z/HLL/IF-SSPRK3,
    cfl 0.9, max dE 0.25, on the reference's moving box (guard 9 cells,
    truncation at 5 sigma).  FP64."""
    from .beam import Beam
    from .config import Numerics, Physics, SolverConfig
    from .enums import EnergyScheme, Material, Scattering
    from .geometry import Box, Geometry
    return SolverConfig(
        geometry=Geometry(size=(0.024, 0.024, 0.2), resolution=(100, 100, 400),
                          objects=[Box(-0.012, 0.0, -0.012, 0.012, 0.0, 0.2, Material.BONE_COMPACT)]),
        beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.002, 0.002)),
        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.25,
                          moving_active_domain=True, active_guard_cells=9, active_truncation_sigma=5.0))


def evaluate_interface(model):
    """Heuristic and learned boxes on the extended lateral-interface case,
    each against the full-domain march: on their own CFL steps, with the
    phantom-wide CFL bound, and through the full-domain march's energies
    (which separates the box's own error from the energy-step sequence)."""
    cfg = interface_case()
    full_E = []
    full, n_full, cs_full, _, _, t_full, grid = march(cfg, moving=False, energies=full_E)
    out = {"full": {"steps": n_full, "cell_steps": cs_full, "seconds": t_full}}
    spacing = (grid.dx * 1e3, grid.dy * 1e3, grid.dz * 1e3)
    m = float(full.max())
    for box, bm in (("heuristic", None), ("learned", model)):
        for mode, kw in (("own", {}), ("phantom_cfl", {"phantom_cfl": True}), ("full_energies", {"schedule": full_E})):
            E = []
            d, n, cs, grows, fb, t, _ = march(cfg, box_model=bm, energies=E, **kw)
            out[f"{box}_{mode}"] = {
                "steps": n, "cell_steps_vs_full": cs / cs_full, "grow_events": grows, "fallbacks": fb,
                "seconds": t, "max_abs_diff_over_max": float((d - full).abs().max()) / m,
                "max_dose_rel_diff": float(d.max()) / m - 1.0,
                "gamma_1pct_1mm": metrics.gamma(d, full, spacing, 1.0, 1.0)[0],
                "energies_equal_full": E == full_E}
            print(json.dumps({f"{box}_{mode}": out[f"{box}_{mode}"]}), flush=True)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--solves", type=int, default=200)
    ap.add_argument("--test-seeds", type=int, nargs="*", default=[1000, 1001, 1002])
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--level", nargs="*", default=["0"],
                    help="tail level per variant (0: 1e-8, 1: 1e-10), or six comma-separated per-face levels")
    ap.add_argument("--safety", type=float, nargs="*", default=[1.0])
    ap.add_argument("--margin-min", type=int, default=3)
    ap.add_argument("--out", default=str(learned_box.MODEL_FILE), help="model of the first variant")
    ap.add_argument("--report", default=None)
    ap.add_argument("--rows", default=None, help="recorded rows: load from this npz if it exists, else save to it")
    ap.add_argument("--evaluate", default=None, help="only evaluate this model file on the test seeds")
    ap.add_argument("--phantom-cfl", action="store_true", help="evaluate with the phantom-wide CFL bound")
    ap.add_argument("--interface-case", action="store_true",
                    help="with --evaluate: the reference's extended lateral-interface case instead of the seeds")
    args = ap.parse_args(argv)
    if args.evaluate and args.interface_case:
        report = {"model": args.evaluate, "interface_case": evaluate_interface(learned_box.BoxModel.load(args.evaluate))}
        if args.report:
            with open(args.report, "w") as f:
                json.dump(report, f, indent=1)
        return report
    if args.evaluate:
        report = {"model": args.evaluate, "phantom_cfl": args.phantom_cfl,
                  "evaluation": evaluate(learned_box.BoxModel.load(args.evaluate), args.test_seeds,
                                         args.phantom_cfl)}
        if args.report:
            with open(args.report, "w") as f:
                json.dump(report, f, indent=1)
        return report
    from pathlib import Path
    t0 = time.perf_counter()
    if args.rows and Path(args.rows).exists():
        with np.load(args.rows) as z:
            all_rows = {k: z[k] for k in z.files}
    else:
        all_rows = {f"seed{s}": learned_box.record(learned_box.training_config(s))[0] for s in range(args.solves)}
        if args.rows:
            np.savez_compressed(args.rows, **all_rows)
    t_rec = time.perf_counter() - t0
    report = {"record_seconds": t_rec, "solves": len(all_rows), "variants": []}
    first = True
    for level_arg in args.level:
        level = tuple(int(v) for v in level_arg.split(",")) if "," in level_arg else int(level_arg)
        parts = [learned_box.samples(r, level=level) for r in all_rows.values()]
        X = np.concatenate([p[0] for p in parts])
        T = np.concatenate([p[1] for p in parts])
        for safety in args.safety:
            t0 = time.perf_counter()
            model, losses = learned_box.train(X, T, epochs=args.epochs, safety=safety, margin_min=args.margin_min)
            t_train = time.perf_counter() - t0
            lv = [level] * 6 if isinstance(level, int) else list(level)
            model.meta.update({"training_solves": len(all_rows),
                               "tail_level_per_face": [learned_box.TAIL_LEVELS[v] if v >= 0 else "significant"
                                                       for v in lv],
                               "record_seconds": t_rec, "train_seconds": t_train,
                               "target_mean": T.mean(0).tolist(), "target_max": T.max(0).tolist()})
            tag = "".join("s" if v < 0 else str(v) for v in lv)
            out = args.out if first else str(Path(args.out).with_suffix("")) + f"_l{tag}_s{safety:g}.npz"
            model.save(out)
            first = False
            print(json.dumps({"level": lv, "safety": safety, "samples": len(X), "train_s": t_train,
                              "loss_first": float(losses[0]), "loss_last": float(losses[-1]), "out": out}),
                  flush=True)
            report["variants"].append({"level": lv, "safety": safety, "model": model.meta, "out": out,
                                       "losses": losses.tolist(), "evaluation": evaluate(model, args.test_seeds)})
            if args.report:
                with open(args.report, "w") as f:
                    json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
