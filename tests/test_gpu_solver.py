"""Solver(config).solve() on the GPU: the reference's public entry point
(proton_solver/solver.py:29-218) returns the march of the oracle and writes
the reference's run directory."""

import json

import numpy as np
import pytest

pytest.importorskip("torch")

from oracle.oracle import OracleProblem
from proton_dose_m1_b200 import OutputConfig, References, Solver, SolverConfig
from proton_dose_m1_b200.enums import Reference
from proton_dose_m1_b200.persistence import config_hash
from tests import cases

pytestmark = pytest.mark.gpu


def test_solver_matches_the_oracle_and_saves(tmp_path):
    spec = cases.march_specs()["hetero_snapshots"]
    base = cases.march_config(spec)
    cfg = SolverConfig(geometry=base.geometry, beam=base.beam, physics=base.physics, numerics=base.numerics,
                       references=References(reference=Reference.NONE),
                       output=OutputConfig(save_results=True, results_directory=str(tmp_path)))
    r = Solver(cfg).solve(snapshot_energies=tuple(spec["snapshots"]))
    _, dose, energies, snaps = OracleProblem(cfg).march(np.zeros((4, *cfg.geometry.resolution)),
                                                        snapshot_energies=tuple(spec["snapshots"]))
    np.testing.assert_array_equal(r.dose, dose)
    np.testing.assert_array_equal(r.energies, energies)
    assert sorted(r.snapshots) == sorted(snaps)
    assert r.primary_label == "Deterministic" and r.reference_dose is None
    meta = json.loads((r.run_directory / "metadata.json").read_text())
    assert meta["config_hash"] == config_hash(cfg)
    with np.load(r.run_directory / "results.npz") as z:
        np.testing.assert_array_equal(z["dose"], dose)
