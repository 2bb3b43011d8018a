"""The learned moving box on the GPU: training kernels against the CPU
restatement of the network (oracle/mlp.py), the BF16 tensor-core inference,
the recorder's features against the same quantities computed on the host from
the marched state, and the march with a box model."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import mlp as omlp
from oracle.oracle import OracleProblem
from proton_dose_m1_b200 import _native, learned_box, metrics
from proton_dose_m1_b200 import Accel, Beam, Box, Geometry, Numerics, Physics, SolverConfig
from proton_dose_m1_b200.enums import EnergyScheme, Material, Precision, Scattering
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.numerics.energy import M1Plan
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.physics.materials import MaterialMap

pytestmark = pytest.mark.gpu


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device="cuda")


def test_training_gradients_match_the_cpu_network():
    rng = np.random.default_rng(3)
    theta = learned_box.init_params(5) + rng.normal(0, 0.05, omlp.N_PARAMS).astype(np.float32)
    X = rng.normal(size=(300, 16)).astype(np.float32)
    Y = rng.normal(size=(300, 6)).astype(np.float32)
    g = torch.empty(omlp.N_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    t, x, y = _dev(theta), _dev(X), _dev(Y)
    _native.check(_native.lib().pdm1_mlp_gradients(C.c_void_p(t.data_ptr()), C.c_void_p(x.data_ptr()),
                                                   C.c_void_p(y.data_ptr()), len(X), 8.0,
                                                   C.c_void_p(g.data_ptr()), C.c_void_p(loss.data_ptr()),
                                                   _stream()))
    ref_loss, ref_g = omlp.loss_and_grad(theta.astype(np.float64), X.astype(np.float64), Y.astype(np.float64), 8.0)
    got = g.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - ref_loss) <= 1e-5 * ref_loss
    assert np.max(np.abs(got - ref_g)) <= 1e-4 * np.max(np.abs(ref_g))
    # per parameter block as well (the small output layer must not hide in the max)
    o = 0
    for name, shape in omlp.SHAPES:
        n = int(np.prod(shape))
        blk = slice(o, o + n)
        assert np.max(np.abs(got[blk] - ref_g[blk])) <= 1e-4 * np.max(np.abs(ref_g[blk])) + 1e-9, name
        o += n


def test_training_fits_and_forward_matches():
    rng = np.random.default_rng(4)
    X = rng.normal(size=(4000, 16)).astype(np.float32)
    W = rng.normal(size=(16, 6)).astype(np.float32) / 4
    T = np.tanh(X @ W) * 3 + 1
    model, losses = learned_box.train(X, T, epochs=40, batch=256, lr=3e-3, alpha=2.0, seed=1, safety=0.0)
    assert losses[-1] < 0.1 * losses[0]
    xn = (X[:64] - model.x_mean) * model.x_inv_std
    out = torch.empty((64, 6), dtype=torch.float32, device="cuda")
    t = _dev(model.params)
    xd = _dev(xn)
    _native.check(_native.lib().pdm1_mlp_forward(C.c_void_p(t.data_ptr()), C.c_void_p(xd.data_ptr()), 64,
                                                 C.c_void_p(out.data_ptr()), _stream()))
    ref, _ = omlp.forward(model.params.astype(np.float64), xn.astype(np.float64))
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-4, atol=1e-4)
    pred = ref * model.y_scale + model.y_offset
    assert np.sqrt(np.mean((pred - T[:64]) ** 2)) < 0.5


def test_bf16_tensor_core_inference_matches_emulation():
    rng = np.random.default_rng(6)
    theta = learned_box.init_params(7) + rng.normal(0, 0.02, omlp.N_PARAMS).astype(np.float32)
    model = learned_box.BoxModel(params=theta, x_mean=rng.normal(size=16).astype(np.float32),
                                 x_inv_std=rng.uniform(0.5, 2, 16).astype(np.float32),
                                 y_scale=np.ones(6, np.float32), y_offset=np.zeros(6, np.float32))
    X = rng.normal(size=(150, 16)).astype(np.float32) * 2   # 150: a partial last warp tile
    got = model.infer(X)
    xn = (X - model.x_mean) * model.x_inv_std
    ref = omlp.forward_bf16(theta, xn)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= 2e-2 * scale
    exact, _ = omlp.forward(theta.astype(np.float64), xn.astype(np.float64))
    assert np.max(np.abs(got - exact)) <= 5e-2 * scale


def _slab(moving=True, precision=Precision.FP64, box_model=None, guard=9):
    geo = Geometry(size=(0.024, 0.024, 0.06), resolution=(24, 24, 60),
                   objects=[Box(0.0, 0.012, -0.012, 0.012, 0.0, 0.06, Material.BONE_COMPACT)])
    num = Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5,
                   moving_active_domain=moving, active_guard_cells=guard)
    return SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=60.0, energy_spread=1.0,
                                                sigma=(0.003, 0.003)),
                        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True), numerics=num,
                        accel=Accel(precision=precision, box_model=box_model))


def _march(cfg):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    plan = M1Plan(cfg, mm, grid, BeamInflow.from_beam(cfg.beam, grid))
    U = None if cfg.numerics.moving_active_domain else torch.zeros((4, *grid.shape), dtype=torch.float64,
                                                                   device="cuda")
    _, dose, E, _ = plan.march(U)
    info = plan.last_info
    plan.close()
    return dose.cpu().numpy(), E, info, grid


def test_recorder_features_match_the_host_computation():
    cfg = _slab(moving=False)
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    inflow = BeamInflow.from_beam(cfg.beam, grid)
    for steps in (1, 40, 97):
        plan = M1Plan(cfg, mm, grid, inflow)
        rows = torch.zeros((400, 40), dtype=torch.float32, device="cuda")
        _native.check(_native.lib().pdm1_plan_set_recorder(plan._h, C.c_void_p(rows.data_ptr()), 400,
                                                           1e-8, 1e-10))
        U, dose, E = plan.march_steps(steps)
        plan.close()
        r = rows.cpu().numpy()
        assert (r[:steps, 0] > 0).all() and (r[steps:, 0] == 0).all()
        np.testing.assert_array_equal(r[:steps, 0], np.asarray(E[1:], dtype=np.float32))
        Uh = U.cpu().numpy()
        e_last, de_last = float(E[-1]), float(E[-2] - E[-1])
        phi_in = inflow.state(e_last)[0]
        tol = np.exp(-0.5 * cfg.numerics.active_truncation_sigma ** 2)
        sig = omlp.significant_box(Uh[0], phi_in, tol)
        assert tuple(int(v) for v in r[steps - 1, 2:8]) == sig
        assert tuple(int(v) for v in r[steps - 1, 27:33]) == omlp.significant_box(Uh[0], phi_in, 1e-8)
        assert tuple(int(v) for v in r[steps - 1, 33:39]) == omlp.significant_box(Uh[0], phi_in, 1e-10)
        S0 = OracleProblem(cfg, mm).stopping_power(0, e_last)
        f, I = omlp.box_features(Uh, sig, e_last, de_last, cfg.numerics.max_energy_step, S0, grid.spacing)
        np.testing.assert_allclose(r[steps - 1, 8:24], f, rtol=2e-5, atol=2e-5)
        assert r[steps - 1, 25] == pytest.approx(I, rel=1e-5)


def test_constant_guard_model_reproduces_the_heuristic_box():
    """A model whose every margin is the guard and whose flux check never
    fires marches the heuristic boxes exactly."""
    const = learned_box.BoxModel(params=np.zeros(omlp.N_PARAMS, np.float32), x_mean=np.zeros(16, np.float32),
                                 x_inv_std=np.ones(16, np.float32), y_scale=np.zeros(6, np.float32),
                                 y_offset=np.full(6, 9.0, np.float32), margin_min=0, margin_max=64,
                                 leak_tolerance=1e30)
    d_h, E_h, i_h, _ = _march(_slab())
    d_l, E_l, i_l, _ = _march(_slab(box_model=const))
    np.testing.assert_array_equal(E_l, E_h)
    np.testing.assert_array_equal(d_l, d_h)
    assert i_l.cell_steps == i_h.cell_steps and i_l.box_grow_events == 0


def test_flux_check_grows_a_box_that_is_too_small():
    """Margins of zero leak at once: the check grows the faces and the dose
    stays within the gate of the full-domain march."""
    tiny = learned_box.BoxModel(params=np.zeros(omlp.N_PARAMS, np.float32), x_mean=np.zeros(16, np.float32),
                                x_inv_std=np.ones(16, np.float32), y_scale=np.zeros(6, np.float32),
                                y_offset=np.zeros(6, np.float32), margin_min=0, margin_max=64,
                                grow_cells=2, extra_max=40, leak_tolerance=1e-6)
    full, _, _, grid = _march(_slab(moving=False))
    d, _, info, _ = _march(_slab(box_model=tiny))
    assert info.box_grow_events > 0
    score = metrics.compare(d, full, grid)
    assert score["gamma_1pct_1mm_pass_percent"] >= 99.5, score
    assert abs(score["maximum_dose_relative_difference"]) <= 0.005, score


HELD_OUT = (1000, 1001, 1002, 1003, 1004, 1005)


@pytest.fixture(scope="module")
def held_out():
    """Full-domain, heuristic-box and learned-box marches of the six held-out
    interface phantoms (seeds 1000-1005; training used seeds 0-199)."""
    from proton_dose_m1_b200.train_box_model import march
    out = {}
    for seed in HELD_OUT:
        cfg = learned_box.training_config(seed)
        full, _, _, _, _, _, grid = march(cfg, moving=False)
        heur, _, cs_h, _, _, _, _ = march(cfg, box_model=None)
        lrn, _, cs_l, grows, fallbacks, _, _ = march(cfg, box_model=learned_box.default_model())
        out[seed] = dict(full=full, heur=heur, lrn=lrn, grid=grid, cs_h=cs_h, cs_l=cs_l, fallbacks=fallbacks)
    return out


@pytest.mark.parametrize("seed", HELD_OUT)
def test_trained_model_holds_the_gate_on_held_out_seeds(held_out, seed):
    """On every held-out seed both boxes stay within the gate of the
    full-domain march and the learned box never falls back."""
    r = held_out[seed]
    for d in (r["heur"], r["lrn"]):
        sc = metrics.compare(d, r["full"], r["grid"])
        assert sc["gamma_1pct_1mm_pass_percent"] >= 99.5, sc
        assert abs(sc["maximum_dose_relative_difference"]) <= 0.005, sc
    assert r["fallbacks"] == 0
    assert r["cs_l"] <= r["cs_h"], (r["cs_l"], r["cs_h"])


def test_trained_model_gains_over_the_heuristic_box(held_out):
    """Summed over the six held-out seeds the learned box marches at most 0.9x
    the heuristic box's cell-steps (per seed it ranges 0.65-0.95x)."""
    cs_h = sum(r["cs_h"] for r in held_out.values())
    cs_l = sum(r["cs_l"] for r in held_out.values())
    assert cs_l <= 0.9 * cs_h, (cs_l, cs_h)
