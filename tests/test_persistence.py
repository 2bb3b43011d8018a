"""Run directories: the canonical configuration and its hash reproduce the
reference's own published run directories (tests/golden/published_configs.json,
copied from thesis_results/**/config.json and metadata.json), and
save_result writes the reference's layout."""

import json

import numpy as np
import pytest

from proton_dose_m1_b200 import Accel, Beam, Geometry, Numerics, OutputConfig, SolverConfig
from proton_dose_m1_b200.enums import Backend, Precision
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.persistence import config_dict, config_from_dict, config_hash, save_result
from proton_dose_m1_b200.result import Result
from tests import cases


def _published():
    return json.loads((cases.GOLDEN / "published_configs.json").read_text())


def _same_schema(a, b):
    if isinstance(a, dict) and isinstance(b, dict):
        return a.keys() == b.keys() and all(_same_schema(a[k], b[k]) for k in a)
    return not isinstance(a, dict) and not isinstance(b, dict)


def test_config_hash_reproduces_published_run_directories():
    runs = _published()
    assert len(runs) >= 40
    checked = 0
    for run in runs:
        cfg = config_from_dict(run["config"])
        ours = config_dict(cfg)
        if not _same_schema(ours, run["config"]):
            continue   # written by an older version of the reference's configuration classes
        assert ours == run["config"], run["source"]
        assert config_hash(cfg) == run["config_hash"], run["source"]
        checked += 1
    assert checked >= 6


def test_gpu_knobs_enter_the_hash_only_when_they_change_the_solution():
    base = SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)), beam=Beam())
    same = SolverConfig(geometry=base.geometry, beam=base.beam, accel=Accel(tile=(8, 8, 4)))
    fp32 = SolverConfig(geometry=base.geometry, beam=base.beam, accel=Accel(precision=Precision.FP32_FP64))
    assert "accel" not in config_dict(base)
    assert config_hash(same) == config_hash(base)
    assert config_hash(fp32) != config_hash(base)


def test_save_result_layout(tmp_path):
    cfg = SolverConfig(geometry=Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10)), beam=Beam(),
                       output=OutputConfig(save_results=True, results_directory=str(tmp_path)))
    grid = Grid.from_geometry(cfg.geometry)
    dose = np.arange(250.0).reshape(5, 5, 10)
    r = Result(phi=dose * 2, J=np.zeros((3, 5, 5, 10)), dose=dose, grid=grid, energies=np.array([3.0, 2.0]),
               runtime=1.5, backend=Backend.GPU)
    run = save_result(r, cfg)
    assert run.parent == tmp_path and run.name.split("__")[1:4] == ["5x5x10", "weno_z", config_hash(cfg)[:8]]
    assert json.loads((run / "config.json").read_text()) == config_dict(cfg)
    meta = json.loads((run / "metadata.json").read_text())
    assert meta["config_hash"] == config_hash(cfg) and meta["runtime_seconds"] == 1.5
    assert meta["backend"] == "GPU" and meta["speedup_vs_bfp_mc_x"] == "-"
    with np.load(run / "results.npz") as z:
        assert set(z.files) == {"x", "y", "z", "phi", "J", "dose", "energies"}
        np.testing.assert_array_equal(z["dose"], dose)


def test_solver_refuses_reference_solutions_it_does_not_hold():
    from proton_dose_m1_b200 import Physics, References, Solver
    from proton_dose_m1_b200.enums import Reference, Scattering
    geo = Geometry(size=(0.01, 0.01, 0.02), resolution=(5, 5, 10))
    cfg = SolverConfig(geometry=geo, beam=Beam(), references=References(reference=Reference.BFP_MC))
    with pytest.raises(NotImplementedError, match="BFP_MC"):
        Solver(cfg).solve()
    cfg = SolverConfig(geometry=geo, beam=Beam(), physics=Physics(scattering=Scattering.WENTZEL),
                       references=References(reference=Reference.ANALYTICAL))
    with pytest.raises(ValueError, match="Analytical reference is not available"):
        Solver(cfg).solve()


def test_interface_case_is_the_published_lateral_interface_run():
    """The box study's extended lateral-interface case (train_box_model
    --interface-case) has the geometry, beam, physics and numerics of the
    reference's own published moving-box run."""
    from proton_dose_m1_b200.train_box_model import interface_case
    src = "thesis_results/robustness/moving_active_domain/scattering_nuclear/transversal_slabs/weno_z"
    run = next(r for r in _published() if r["source"] == src)
    published = cases.published_config(run)
    mine = interface_case()
    for part in ("geometry", "beam", "physics", "numerics"):
        assert getattr(mine, part) == getattr(published, part), part
