"""CT input (proton_solver/geometry.py:75-134): NPZ keys, orientation and the
validation errors, checked against NumPy's own transpose and flips."""

from __future__ import annotations

import numpy as np
import pytest

from proton_dose_m1_b200 import CTScan


def _npz(tmp_path, name="ct.npz", **arrays):
    p = tmp_path / name
    np.savez(p, **arrays)
    return p


def test_orientation_of_volume_mask_and_spacing(tmp_path):
    hu = np.arange(3 * 4 * 5, dtype=np.float32).reshape(3, 4, 5) - 30.0
    mask = (np.arange(60).reshape(3, 4, 5) % 3) == 0
    p = _npz(tmp_path, HU=hu, body_mask=mask)
    ct = CTScan(p, (1e-3, 2e-3, 3e-3), axis_order=(2, 0, 1), flip_axes=(True, False, True))
    want = np.flip(np.flip(np.transpose(hu, (2, 0, 1)), axis=0), axis=2)
    want_mask = np.flip(np.flip(np.transpose(mask, (2, 0, 1)), axis=0), axis=2)
    assert ct.shape == (5, 3, 4)
    assert np.array_equal(ct.hu, want) and ct.hu.flags.c_contiguous
    assert ct.body_mask.dtype == bool and np.array_equal(ct.body_mask, want_mask)
    assert ct.body_mask.flags.c_contiguous
    assert ct.spacing == (3e-3, 1e-3, 2e-3)


def test_identity_orientation_and_no_mask(tmp_path):
    hu = np.random.default_rng(0).normal(size=(2, 3, 4))
    ct = CTScan(_npz(tmp_path, hu=hu), (1e-3, 1e-3, 1e-3))
    assert np.array_equal(ct.hu, hu) and ct.body_mask is None


def test_key_preference(tmp_path):
    a, b = np.zeros((2, 2, 2)), np.ones((2, 2, 2))
    assert CTScan(_npz(tmp_path, "1.npz", HU=a, hu=b), (1e-3,) * 3).hu.max() == 0.0
    p = tmp_path / "2.npz"
    np.savez(p, b)                               # one unnamed array: arr_0
    assert CTScan(p, (1e-3,) * 3).hu.min() == 1.0
    p = tmp_path / "3.npz"
    np.savez(p, b, a)                            # two unnamed arrays: no volume
    with pytest.raises(ValueError, match="needs a 'HU', 'hu', or single 'arr_0'"):
        CTScan(p, (1e-3,) * 3)


@pytest.mark.parametrize("kwargs, message", [
    (dict(source_spacing_m=(1e-3, 1e-3)), "CT spacing must contain three positive finite metres."),
    (dict(source_spacing_m=(1e-3, 0.0, 1e-3)), "CT spacing must contain three positive finite metres."),
    (dict(source_spacing_m=(1e-3, float("nan"), 1e-3)), "CT spacing must contain three positive finite"),
    (dict(axis_order=(0, 0, 1)), "axis_order must be a permutation of"),
    (dict(flip_axes=(True, 0, False)), "flip_axes must contain three booleans."),
    (dict(flip_axes=(True, False)), "flip_axes must contain three booleans."),
])
def test_orientation_errors_come_before_the_file(tmp_path, kwargs, message):
    args = dict(path=tmp_path / "missing.npz", source_spacing_m=(1e-3, 1e-3, 1e-3))
    args.update(kwargs)
    with pytest.raises(ValueError, match=message.replace("(", r"\(")):
        CTScan(**args)


def test_volume_errors(tmp_path):
    with pytest.raises(ValueError, match="numeric 3D array"):
        CTScan(_npz(tmp_path, "a.npz", HU=np.zeros((2, 2))), (1e-3,) * 3)
    with pytest.raises(ValueError, match="numeric 3D array"):
        CTScan(_npz(tmp_path, "b.npz", HU=np.zeros((2, 2, 2), dtype=bool).astype("U1")), (1e-3,) * 3)
    bad = np.zeros((2, 2, 2))
    bad[1, 1, 1] = np.inf
    with pytest.raises(ValueError, match="non-finite"):
        CTScan(_npz(tmp_path, "c.npz", HU=bad), (1e-3,) * 3)
    with pytest.raises(ValueError, match="body_mask shape must match"):
        CTScan(_npz(tmp_path, "d.npz", HU=np.zeros((2, 2, 2)), body_mask=np.ones((2, 2), bool)), (1e-3,) * 3)
