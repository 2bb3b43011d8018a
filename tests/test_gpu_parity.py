"""GPU parity: libpdm1.so against the CPU oracle and the reference fixtures.

The FP64 path evaluates every expression in the oracle's order with
separately rounded products and sums and the same double-double exp, so it
is expected to reproduce the oracle bit for bit; the reference fixtures are
matched to the bars in tests/cases.py (reference_rtol).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle.oracle as O
from proton_dose_m1_b200.numerics.energy import M1Plan, energy_march
from proton_dose_m1_b200.numerics.grid import Grid
from proton_dose_m1_b200.numerics.boundary import BeamInflow
from proton_dose_m1_b200.physics.materials import MaterialMap
from proton_dose_m1_b200 import _native
from tests import cases

pytestmark = pytest.mark.gpu


def make_plan(cfg):
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    inflow = BeamInflow.from_beam(cfg.beam, grid)
    return M1Plan(cfg, mm, grid, inflow), (mm, grid, inflow)


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def stream():
    import ctypes
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


@pytest.fixture(scope="module")
def unit():
    return cases.load("unit_vectors.npz")


def test_scalar_kernels_match_oracle(unit):
    L = _native.lib()
    w = dev(unit["weno_in"])
    out = torch.empty(len(w), dtype=torch.float64, device="cuda")
    _native.check(L.pdm1_weno_batch(ptr(w), ptr(out), len(w), stream()))
    np.testing.assert_array_equal(out.cpu().numpy(), unit["weno_out"])

    u = dev(unit["proj_in"]).clone()
    _native.check(L.pdm1_project_batch(ptr(u), len(u), stream()))
    np.testing.assert_array_equal(u.cpu().numpy(), unit["proj_out"])

    e = dev(unit["eig_in"])
    for ax in range(3):
        lohi = torch.empty((len(e), 2), dtype=torch.float64, device="cuda")
        _native.check(L.pdm1_eigen_batch(ptr(e), ax, ptr(lohi), len(e), stream()))
        np.testing.assert_array_equal(lohi.cpu().numpy(), unit["eig_out"][:, ax])

    left, right = dev(unit["hll_left"]), dev(unit["hll_right"])
    for ax in range(3):
        for ws in (0, 1):
            F = torch.empty_like(left)
            _native.check(L.pdm1_hll_batch(ptr(left), ptr(right), ax, ws, ptr(F), len(left), stream()))
            want = np.array([O.hll_flux(l, r, ax, bool(ws)) for l, r in zip(unit["hll_left"], unit["hll_right"])])
            np.testing.assert_array_equal(F.cpu().numpy(), want)


def test_exp_matches_oracle():
    import ctypes
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.uniform(-745, 709, 20000), rng.uniform(-1, 1, 20000), [0.0, -0.0, 700.0, -700.0]])
    y = torch.empty(len(x), dtype=torch.float64, device="cuda")
    xd = dev(x)
    _native.check(_native.lib().pdm1_exp_batch(ptr(xd), ptr(y), len(x), stream()))
    L = O.lib()
    L.orc_exp.argtypes = [ctypes.c_double]
    L.orc_exp.restype = ctypes.c_double
    np.testing.assert_array_equal(y.cpu().numpy(), [L.orc_exp(float(v)) for v in x])


def test_coefficients_match_reference(unit):
    from proton_dose_m1_b200 import Geometry, SolverConfig, Beam, Physics
    from proton_dose_m1_b200.enums import Material, Scattering, CoefficientInterpolation
    E = unit["coef_energy"]
    for interp, tr_key, nuc_key in ((CoefficientInterpolation.LINEAR, "tr_linear", "nuc_linear"),
                                    (CoefficientInterpolation.PCHIP, "tr_pchip", "nuc_pchip")):
        mats = [m for m in Material if m.value.startswith("G4_")]
        ids = np.arange(len(mats), dtype=np.int32).repeat(4 * 4).reshape(len(mats), 4, 4)
        ids = np.ascontiguousarray(np.tile(ids, (1, 1, 1)))
        geo = Geometry.from_ids((0.01, 0.004, 0.004), np.ascontiguousarray(ids.reshape(len(mats), 4, 4)), mats)
        cfg = SolverConfig(geometry=geo, beam=Beam(energy=100.0, sigma=(0.01, 0.01)),
                           physics=Physics(scattering=Scattering.WENTZEL, nuclear=True,
                                           coefficient_interpolation=interp))
        plan, _ = make_plan(cfg)
        got = plan.coefficients(E)
        for m in mats:
            mi = list(unit["coef_materials"]).index(m.value)
            k = mats.index(m)
            np.testing.assert_array_equal(got[:, k, 0], unit["sp"][mi])
            np.testing.assert_array_equal(got[:, k, 1], unit[tr_key][mi])
            np.testing.assert_array_equal(got[:, k, 2], unit[nuc_key][mi])


def test_spatial_operator_and_cfl():
    g = cases.load("operators.npz")
    cfg = cases.operator_config()
    plan, _ = make_plan(cfg)
    orc = O.OracleProblem(cfg)
    E = float(g["E"])
    for bc in (None, g["bc_custom"]):
        got = plan.spatial_operator(g["U"], E, bc).cpu().numpy()
        np.testing.assert_array_equal(got, orc.spatial_operator(g["U"], E, bc))
    assert plan.energy_step(g["U"], E) == float(g["dE_exact"])
    cfg_u = cases.operator_config(wave_speeds=cases.WaveSpeeds.UNIT)
    plan_u, _ = make_plan(cfg_u)
    assert plan_u.energy_step(g["U"], E) == float(g["dE_unit"])
    np.testing.assert_array_equal(plan_u.spatial_operator(g["U"], E).cpu().numpy(),
                                  O.OracleProblem(cfg_u).spatial_operator(g["U"], E))


@pytest.mark.parametrize("name", list(cases.OPERATOR_CASES))
def test_one_step_matches_oracle(name):
    g = cases.load("operators.npz")
    cfg = cases.operator_config(name)
    plan, _ = make_plan(cfg)
    U, edep = plan.advance(g["U"], float(g["E"]), float(g["dE"]))
    U_o, edep_o = O.OracleProblem(cfg).advance(g["U"], float(g["E"]), float(g["dE"]))
    np.testing.assert_array_equal(U.cpu().numpy(), U_o)
    np.testing.assert_array_equal(edep.cpu().numpy(), edep_o)
    ref_U, ref_e = g[f"step_{name}_U"], g[f"step_{name}_edep"]
    assert np.abs(U.cpu().numpy() - ref_U).max() / np.abs(ref_U[0]).max() < 1e-11
    assert np.abs(edep.cpu().numpy() - ref_e).max() / np.abs(ref_e).max() < 1e-11


ALL_MARCHES = list(cases.march_specs())


@pytest.mark.parametrize("name", ALL_MARCHES)
def test_march_matches_oracle_and_reference(name):
    """Static and moving-box marches: bit for bit against the oracle, within the
    rounding-floor bar against the reference's fixtures."""
    spec = cases.march_specs()[name]
    cfg = cases.march_config(spec)
    plan, (mm, grid, inflow) = make_plan(cfg)
    U0 = np.zeros((4, *cfg.geometry.resolution))
    U, dose, energies, snaps = plan.march(U0, snapshot_energies=tuple(spec["snapshots"]))
    U, dose = U.cpu().numpy(), dose.cpu().numpy()
    Uo, dose_o, energies_o, snaps_o = O.OracleProblem(cfg).march(U0, tuple(spec["snapshots"]))
    np.testing.assert_array_equal(energies, energies_o)
    np.testing.assert_array_equal(dose, dose_o)
    np.testing.assert_array_equal(U, Uo)
    assert sorted(snaps) == sorted(snaps_o)
    for e in snaps:
        np.testing.assert_array_equal(snaps[e].cpu().numpy(), snaps_o[e])
    g = cases.load(f"march_{name}.npz")
    np.testing.assert_allclose(energies, g["energies"], rtol=0, atol=1e-12)
    assert np.abs(dose - g["dose"]).max() <= cases.reference_rtol(cfg) * g["dose"].max()


@pytest.mark.parametrize("case", list(cases.published_kats()))
def test_published_kats(case):
    kat = cases.published_kats()[case]
    cfg = cases.published_config(kat)
    plan, _ = make_plan(cfg)
    _, dose, energies, _ = plan.march(None)
    dmax = float(dose.max())
    assert abs(dmax - kat["maximum_dose_Gy"]) <= cases.reference_rtol(cfg) * kat["maximum_dose_Gy"]


def test_energy_march_dropin_numpy_and_torch():
    spec = cases.march_specs()["hetero_snapshots"]
    cfg = cases.march_config(spec)
    grid = Grid.from_geometry(cfg.geometry)
    mm = MaterialMap.from_geometry(cfg.geometry, grid)
    inflow = BeamInflow.from_beam(cfg.beam, grid)
    U0 = np.zeros((4, *grid.shape))
    U, dose, E, snaps = energy_march(U0, mm, grid, inflow, cfg, np, snapshot_energies=(30.0, 55.0))
    assert isinstance(dose, np.ndarray) and isinstance(E, np.ndarray)
    assert list(snaps) == [55.0, 30.0]
    assert np.all(U0 == 0.0)   # the caller's state is not modified
    Ut, doset, Et, snapst = energy_march(torch.zeros((4, *grid.shape), dtype=torch.float64, device="cuda"),
                                         mm, grid, inflow, cfg, torch, snapshot_energies=(30.0, 55.0))
    assert doset.is_cuda
    np.testing.assert_array_equal(doset.cpu().numpy(), dose)
    np.testing.assert_array_equal(Et, E)


def test_march_is_deterministic_at_full_size():
    """40x40x200 at 1 mm: a 30-step prefix matches the oracle bit for bit and
    two full marches give identical dose bits."""
    from proton_dose_m1_b200 import Geometry, SolverConfig, Beam, Numerics
    from proton_dose_m1_b200.enums import EnergyScheme
    cfg = SolverConfig(geometry=Geometry(size=(0.04, 0.04, 0.2), resolution=(40, 40, 200)),
                       beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)),
                       numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))
    plan, _ = make_plan(cfg)
    _, d1, e1, _ = plan.march(None)
    _, d2, e2, _ = plan.march(None)
    assert torch.equal(d1, d2)
    np.testing.assert_array_equal(e1, e2)
    assert 400 < len(e1) - 1 < 520
    assert float(d1.min()) >= 0.0
    U30, dose30, n = O.OracleProblem(cfg).march_steps(30, np.zeros((4, 40, 40, 200)))
    assert n == 30
    Ug, dg, eg = plan.march_steps(30)
    assert len(eg) == 31
    np.testing.assert_array_equal(Ug.cpu().numpy(), U30)
    np.testing.assert_array_equal(dg.cpu().numpy(), dose30)


def test_moving_box_follows_the_beam_at_full_size():
    """40x40x200 water: the moving box reproduces the oracle's step sequence on a
    bounded prefix, and its dose agrees with the static march's within the
    reference heuristic's own truncation error."""
    from proton_dose_m1_b200 import Geometry, SolverConfig, Beam, Numerics
    from proton_dose_m1_b200.enums import EnergyScheme
    base = dict(geometry=Geometry(size=(0.04, 0.04, 0.2), resolution=(40, 40, 200)),
                beam=Beam(n_protons=1e6, energy=150.0, energy_spread=1.0, sigma=(0.003, 0.003)))
    cfg_m = SolverConfig(**base, numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9,
                                                   max_energy_step=0.5, moving_active_domain=True))
    cfg_s = SolverConfig(**base, numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9,
                                                   max_energy_step=0.5))
    pm, _ = make_plan(cfg_m)
    ps, _ = make_plan(cfg_s)
    U40, d40, n = O.OracleProblem(cfg_m).march_steps(40, np.zeros((4, 40, 40, 200)))
    Ug, dg, eg = pm.march_steps(40)
    np.testing.assert_array_equal(dg.cpu().numpy(), d40)
    np.testing.assert_array_equal(Ug.cpu().numpy(), U40)
    _, dm, em, _ = pm.march(None)
    _, ds, es, _ = ps.march(None)
    dm, ds = dm.cpu().numpy(), ds.cpu().numpy()
    assert abs(len(em) - len(es)) <= 2
    assert np.abs(dm - ds).max() <= 1e-3 * ds.max()


@pytest.mark.parametrize("scheme", cases.SCHEMES, ids=lambda s: s.name)
def test_other_reconstructions_match_oracle(scheme):
    """First-order, MUSCL and WENO3 operators and one full step: bit for bit
    against the oracle, which is pinned to the reference's fixtures."""
    g = cases.load("operators.npz")
    E, dE = float(g["E"]), float(g["dE"])
    cfg = cases.operator_config(spatial_scheme=scheme)
    plan, _ = make_plan(cfg)
    orc = O.OracleProblem(cfg)
    for bc in (None, g["bc_custom"]):
        np.testing.assert_array_equal(plan.spatial_operator(g["U"], E, bc).cpu().numpy(),
                                      orc.spatial_operator(g["U"], E, bc))
    cfg = cases.operator_config("if_full", spatial_scheme=scheme)
    plan, _ = make_plan(cfg)
    U, edep = plan.advance(g["U"], E, dE)
    U_o, edep_o = O.OracleProblem(cfg).advance(g["U"], E, dE)
    np.testing.assert_array_equal(U.cpu().numpy(), U_o)
    np.testing.assert_array_equal(edep.cpu().numpy(), edep_o)


@pytest.mark.parametrize("name", list(cases.scheme_march_specs()))
def test_other_reconstruction_marches_match_oracle(name):
    spec = cases.scheme_march_specs()[name]
    cfg = cases.march_config(spec)
    plan, _ = make_plan(cfg)
    U0 = np.zeros((4, *cfg.geometry.resolution))
    U, dose, energies, snaps = plan.march(U0, snapshot_energies=tuple(spec["snapshots"]))
    Uo, dose_o, energies_o, _ = O.OracleProblem(cfg).march(U0, tuple(spec["snapshots"]))
    np.testing.assert_array_equal(energies, energies_o)
    np.testing.assert_array_equal(dose.cpu().numpy(), dose_o)
    g = cases.load(f"march_{name}.npz")
    assert np.abs(dose.cpu().numpy() - g["dose"]).max() <= cases.reference_rtol(cfg) * g["dose"].max()
