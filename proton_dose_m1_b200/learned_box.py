"""The learned moving active box: training data, training and the model.

The reference moves its active box by a fixed rule
(proton_solver/numerics/moving_active_domain.py:107-193): the bounding box of
the cells whose fluence exceeds exp(-s^2/2) of the maximum, widened by
``active_guard_cells`` (9) on every face.  Here a network proposes the widening
per face and per energy step instead, from fluence moments of the beam's
current box; the march checks every step that the particle current through
the box faces stays below ``leak_tolerance`` of the beam current and grows the
faces that leak (``pdm1_plan_set_box_model``).

Pipeline (all on the GPU, through libpdm1.so):

* ``record``: a full-domain march of the plain method with the recorder on
  writes, per energy step, the significant box, the boxes of the fluence tail
  at two lower levels (1e-8 and 1e-10 of the maximum) and the 16 features of
  the state (``pdm1_plan_set_recorder``).
* ``samples``: the target of a step is how far, on each face, the next step's
  fluence tail reaches beyond this step's significant box (in cells): the
  margin that keeps the tail inside the box.  The fixed rule keeps 9 cells on
  every face, which holds a narrow beam's tail at ~1e-11 and a widely
  scattered beam's at ~1e-7; the network keeps one level everywhere.
* ``train``: Adam on the fused forward/backward kernel (``pdm1_mlp_train``);
  the model stores the normalisation and the map from outputs to margins.
* ``BoxModel.attach(plan)``: the march runs the network in BF16 on the tensor
  cores every step.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _native

MODEL_FILE = Path(__file__).resolve().parent / "data" / "box_model.npz"
FACES = ("x-", "x+", "y-", "y+", "z-", "z+")
FEATURES = ("E/100 MeV", "dE/max_dE", "half width x", "half width y", "half depth z",
            "centroid offset x", "centroid offset y", "centroid offset z",
            "rms x", "rms y", "rms z", "mean Jz/phi", "mean |Jx|/phi", "mean |Jy|/phi",
            "front advance (cells/step)", "peak plane share")


@dataclass
class BoxModel:
    """Network parameters and the map of its outputs to margins (cells)."""

    params: np.ndarray                       # float32 (5638,)
    x_mean: np.ndarray                       # float32 (16,)
    x_inv_std: np.ndarray                    # float32 (16,)
    y_scale: np.ndarray                      # float32 (6,)
    y_offset: np.ndarray                     # float32 (6,)
    margin_min: int = 4
    margin_max: int = 24
    grow_cells: int = 4
    extra_max: int = 24
    leak_tolerance: float = 1e-6
    meta: dict = field(default_factory=dict)

    def native(self):
        """The pdm1_box_model struct (keeps the parameter buffer alive on self)."""
        self._buf = np.ascontiguousarray(self.params, dtype=np.float32)
        if self._buf.shape != (_native.BOX_PARAMS,):
            raise ValueError(f"box model needs {_native.BOX_PARAMS} parameters")
        m = _native.BoxModel()
        m.params = self._buf.ctypes.data_as(C.POINTER(C.c_float))
        for name in ("x_mean", "x_inv_std", "y_scale", "y_offset"):
            getattr(m, name)[:] = [float(v) for v in getattr(self, name)]
        m.margin_min, m.margin_max = int(self.margin_min), int(self.margin_max)
        m.grow_cells, m.extra_max = int(self.grow_cells), int(self.extra_max)
        m.leak_tolerance = float(self.leak_tolerance)
        return m

    def attach(self, plan_handle) -> None:
        _native.check(_native.lib().pdm1_plan_set_box_model(plan_handle, C.byref(self.native())))

    def save(self, path=MODEL_FILE) -> None:
        import json
        np.savez_compressed(path, params=self.params.astype(np.float32), x_mean=self.x_mean,
                            x_inv_std=self.x_inv_std, y_scale=self.y_scale, y_offset=self.y_offset,
                            ints=np.array([self.margin_min, self.margin_max, self.grow_cells, self.extra_max]),
                            leak_tolerance=np.array(self.leak_tolerance),
                            meta=np.array(json.dumps(self.meta)))

    @classmethod
    def load(cls, path=MODEL_FILE) -> "BoxModel":
        import json
        with np.load(path) as z:
            ints = [int(v) for v in z["ints"]]
            return cls(params=z["params"].astype(np.float32), x_mean=z["x_mean"].astype(np.float32),
                       x_inv_std=z["x_inv_std"].astype(np.float32), y_scale=z["y_scale"].astype(np.float32),
                       y_offset=z["y_offset"].astype(np.float32), margin_min=ints[0], margin_max=ints[1],
                       grow_cells=ints[2], extra_max=ints[3], leak_tolerance=float(z["leak_tolerance"]),
                       meta=json.loads(str(z["meta"])))

    def infer(self, features):
        """Margins (cells, before clamping and growth) for raw features (n, 16),
        through the march's BF16 tensor-core kernel."""
        import torch
        X = torch.as_tensor(np.ascontiguousarray(features, dtype=np.float32), device="cuda")
        out = torch.empty((len(X), _native.BOX_OUTPUTS), dtype=torch.float32, device="cuda")
        _native.check(_native.lib().pdm1_box_model_infer(
            C.byref(self.native()), C.c_void_p(X.data_ptr()), len(X), C.c_void_p(out.data_ptr()),
            C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return out.cpu().numpy() * self.y_scale + self.y_offset


def default_model() -> BoxModel:
    """The committed model (trained on full-domain solves of the lateral
    water/bone interface phantom)."""
    if not MODEL_FILE.exists():
        raise FileNotFoundError(f"{MODEL_FILE} is missing: train one with learned_box.train")
    return BoxModel.load(MODEL_FILE)


# ---------------------------------------------------------------------------
# Training data
# ---------------------------------------------------------------------------
def training_config(seed: int, shape=(80, 80, 400), spacing=(5e-4, 5e-4, 5e-4)):
    """One training solve: a pencil beam on the lateral water/bone interface
    phantom (bone for x > offset), E ~ U[70, 200] MeV, sigma ~ U[2, 6] mm,
    offset ~ U[-10, 10] mm, full physics (Wentzel-VI + nuclear, IF-SSPRK3)."""
    from . import Beam, Numerics, Physics, SolverConfig
    from .enums import EnergyScheme, Scattering
    from .phantoms import lateral_interface_phantom
    rng = np.random.default_rng(seed)
    E = float(rng.uniform(70.0, 200.0))
    s = float(rng.uniform(2.0, 6.0)) * 1e-3
    off = float(rng.uniform(-10.0, 10.0)) * 1e-3
    geo = lateral_interface_phantom(off, shape, spacing)
    return SolverConfig(geometry=geo, beam=Beam(n_protons=1e6, energy=E, energy_spread=1.0, sigma=(s, s)),
                        physics=Physics(scattering=Scattering.WENTZEL, nuclear=True),
                        numerics=Numerics(energy_scheme=EnergyScheme.IF_SSPRK3, cfl=0.9, max_energy_step=0.5))


TAIL_LEVELS = (1e-8, 1e-10)


def record(config, max_rows: int = 200_000, tails=TAIL_LEVELS):
    """Full-domain march of ``config`` with the recorder: (rows (n, 40) float32,
    dose (device tensor)).  Columns: E, dE, significant box (6), features (16),
    sum phi, beam current, threshold scale, tail boxes at ``tails`` (6 + 6)."""
    import torch
    from .numerics.boundary import BeamInflow
    from .numerics.energy import M1Plan
    from .numerics.grid import Grid
    from .physics.materials import MaterialMap
    grid = Grid.from_geometry(config.geometry)
    mm = MaterialMap.from_geometry(config.geometry, grid)
    plan = M1Plan(config, mm, grid, BeamInflow.from_beam(config.beam, grid))
    rows = torch.zeros((max_rows, _native.RECORD_WIDTH), dtype=torch.float32, device="cuda")
    try:
        _native.check(_native.lib().pdm1_plan_set_recorder(plan._h, C.c_void_p(rows.data_ptr()), max_rows,
                                                           float(tails[0]), float(tails[1])))
        U = torch.zeros((4, *grid.shape), dtype=torch.float64, device="cuda")
        dose = torch.empty(grid.shape, dtype=torch.float64, device="cuda")
        energies = torch.empty(max_rows + 1, dtype=torch.float64, device="cuda")
        n, _ = plan.march_device(U, dose, energies)
    finally:
        plan.close()
    return rows[:min(n, max_rows)].cpu().numpy(), dose


def samples(rows, level=0, horizon: int = 1):
    """(features (n, 16), targets (n, 6)) of a recorded march.  The target of
    step r on each face is how many cells the fluence tail of the next
    ``horizon`` steps reaches beyond the significant box of step r (negative:
    it lies inside).  ``level`` picks the tail (0: 1e-8, 1: 1e-10 of the
    maximum; -1: the significant box itself), one for all faces or one per
    face (x-, x+, y-, y+, z-, z+)."""
    levels = [level] * 6 if isinstance(level, int) else list(level)
    sig = rows[:, 2:8]
    col = lambda lv, f: 2 + f if lv < 0 else 27 + 6 * lv + f
    tail = np.stack([rows[:, col(levels[f], f)] for f in range(6)], axis=1)
    ok = (sig[:, 1] >= 0) & (tail[:, 1] >= 0) & (rows[:, 24] > 0)
    X, T = [], []
    for r in range(len(rows) - horizon):
        if not ok[r] or not ok[r + 1:r + 1 + horizon].all():
            continue
        nxt = tail[r + 1:r + 1 + horizon]
        t = np.array([sig[r, 0] - nxt[:, 0].min(), nxt[:, 1].max() - sig[r, 1],
                      sig[r, 2] - nxt[:, 2].min(), nxt[:, 3].max() - sig[r, 3],
                      sig[r, 4] - nxt[:, 4].min(), nxt[:, 5].max() - sig[r, 5]], dtype=np.float32)
        X.append(rows[r, 8:24])
        T.append(t)
    return np.asarray(X, np.float32).reshape(-1, 16), np.asarray(T, np.float32).reshape(-1, 6)


def train(X, T, epochs: int = 60, batch: int = 512, lr: float = 2e-3, alpha: float = 8.0, seed: int = 0,
          safety: float = 1.0, **limits) -> tuple[BoxModel, np.ndarray]:
    """Fit the proposer on (features, targets) with the GPU training kernels.
    Margins = prediction + ``safety`` cells.  Returns (model, loss per epoch)."""
    import torch
    X = np.asarray(X, np.float32)
    T = np.asarray(T, np.float32)
    x_mean = X.mean(0)
    x_std = X.std(0)
    x_inv = np.where(x_std > 1e-6, 1.0 / np.maximum(x_std, 1e-6), 0.0).astype(np.float32)
    y_mean = T.mean(0)
    y_std = np.maximum(T.std(0), 0.25).astype(np.float32)
    Xn = torch.as_tensor((X - x_mean) * x_inv, device="cuda")
    Yn = torch.as_tensor((T - y_mean) / y_std, device="cuda")
    theta = torch.as_tensor(init_params(seed), device="cuda")
    losses = np.zeros(epochs, np.float32)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _native.check(_native.lib().pdm1_mlp_train(
        C.c_void_p(theta.data_ptr()), C.c_void_p(Xn.data_ptr()), C.c_void_p(Yn.data_ptr()), len(X), epochs,
        batch, lr, alpha, seed, losses.ctypes.data_as(C.POINTER(C.c_float)), stream))
    model = BoxModel(params=theta.cpu().numpy(), x_mean=x_mean.astype(np.float32), x_inv_std=x_inv,
                     y_scale=y_std, y_offset=(y_mean + safety).astype(np.float32), **limits)
    model.meta = {"samples": int(len(X)), "epochs": epochs, "batch": batch, "lr": lr, "alpha": alpha,
                  "seed": seed, "safety_cells": safety, "final_loss": float(losses[-1])}
    return model, losses


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases (the flat layout of the kernels)."""
    rng = np.random.default_rng(seed)
    parts = []
    for n_out, n_in in ((64, 16), (64, 64), (6, 64)):
        parts.append(rng.standard_normal((n_out, n_in)) * np.sqrt(2.0 / n_in))
        parts.append(np.zeros(n_out))
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


__all__ = ["BoxModel", "default_model", "training_config", "record", "samples", "train", "init_params",
           "FACES", "FEATURES"]
