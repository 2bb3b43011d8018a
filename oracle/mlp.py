"""CPU restatement of the moving-box proposer network (NumPy, float64).

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the GPU training
kernels' gradients and the BF16 inference kernel, never by the product.

The network has no reference counterpart (the reference's moving box is the
fixed heuristic of proton_solver/numerics/moving_active_domain.py:107-193).
Parameters are one flat vector in the order W1 (64x16), b1, W2 (64x64), b2,
W3 (6x64), b3, every matrix row-major [out][in]:

    h1 = relu(W1 x + b1),  h2 = relu(W2 h1 + b2),  y = W3 h2 + b3.

Loss: mean over samples and outputs of w(r) r^2 with r = y - target and
w = alpha where r < 0 (a margin predicted too small costs alpha times more
than one too large), else 1.
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 16, 64, 6
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def forward(theta, X):
    p = unpack(theta)
    a1 = X @ p["W1"].T + p["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = np.maximum(a2, 0.0)
    y = h2 @ p["W3"].T + p["b3"]
    return y, (X, a1, h1, a2, h2)


def loss_and_grad(theta, X, Y, alpha, n_total=None):
    """Loss and gradient; ``n_total`` normalises as if the batch were part of a
    set of that many samples (the GPU kernel's per-minibatch scaling)."""
    p = unpack(theta)
    y, (X, a1, h1, a2, h2) = forward(theta, X)
    n = len(X) if n_total is None else n_total
    r = y - Y
    w = np.where(r < 0.0, alpha, 1.0)
    loss = float(np.sum(w * r * r) / (n * N_OUT))
    dy = 2.0 * w * r / (n * N_OUT)
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ p["W3"]) * (a2 > 0)
    g["W2"] = dh2.T @ h1
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ p["W2"]) * (a1 > 0)
    g["W1"] = dh1.T @ X
    g["b1"] = dh1.sum(0)
    return loss, pack(g)


def bf16(x):
    """Round to bfloat16 (round to nearest even) and back to float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def forward_bf16(theta, X):
    """The inference kernel's arithmetic: BF16 operands (inputs, weights and
    hidden activations), FP32 accumulation and biases."""
    p = unpack(theta)
    f = lambda a: bf16(a).astype(np.float64)
    h1 = np.maximum(f(X) @ f(p["W1"]).T + p["b1"].astype(np.float32), 0.0).astype(np.float32)
    h2 = np.maximum(f(h1) @ f(p["W2"]).T + p["b2"].astype(np.float32), 0.0).astype(np.float32)
    return f(h2) @ f(p["W3"]).T + p["b3"].astype(np.float32)


def significant_box(phi, phi_in, tol):
    """The significant box of the fixed moving-box rule
    (proton_solver/numerics/moving_active_domain.py:107-151): cells whose phi
    exceeds tol * max(max phi, max phi_in), the inflow joining the k = 0
    layer.  Returns (i0, i1, j0, j1, k0, k1) half-open, or None."""
    scale = max(float(phi.max()), float(phi_in.max()))
    if scale == 0.0:
        return None
    thr = tol * scale
    active = phi > thr
    active[:, :, 0] |= phi_in > thr
    ix = np.flatnonzero(active.any(axis=(1, 2)))
    iy = np.flatnonzero(active.any(axis=(0, 2)))
    iz = np.flatnonzero(active.any(axis=(0, 1)))
    if not (ix.size and iy.size and iz.size):
        return None
    return (int(ix[0]), int(ix[-1]) + 1, int(iy[0]), int(iy[-1]) + 1, int(iz[0]), int(iz[-1]) + 1)


def box_features(U, sig, E, dE, max_dE, S0, spacing):
    """The 16 features of a full-domain state U (4, nx, ny, nz) with
    significant box ``sig``, as the recorder and the learned box compute them
    (float64, then float32): energy, last dE, the box half sizes, the fluence
    centroid offset from the box centre and rms widths (cells), mean Jz/phi,
    |Jx|/phi, |Jy|/phi, the cells the front advances per step dE/(S dz) with
    S of material 0, and the largest z-plane current relative to the fluence."""
    dx, dy, dz = spacing
    phi, jx, jy, jz = U
    nx, ny, nz = phi.shape
    M = phi.sum()
    g = [np.arange(n) + 0.5 for n in (nx, ny, nz)]
    mean = [np.einsum("ijk,i->", phi, g[0]) / M, np.einsum("ijk,j->", phi, g[1]) / M,
            np.einsum("ijk,k->", phi, g[2]) / M]
    sq = [np.einsum("ijk,i->", phi, g[0] ** 2) / M, np.einsum("ijk,j->", phi, g[1] ** 2) / M,
          np.einsum("ijk,k->", phi, g[2] ** 2) / M]
    I = jz.sum(axis=(0, 1)).max() * dx * dy
    f = [E / 100.0, dE / max_dE]
    f += [0.5 * (sig[2 * a + 1] - sig[2 * a]) for a in range(3)]
    f += [mean[a] - 0.5 * (sig[2 * a] + sig[2 * a + 1]) for a in range(3)]
    f += [np.sqrt(max(sq[a] - mean[a] ** 2, 0.0)) for a in range(3)]
    f += [jz.sum() / M, np.abs(jx).sum() / M, np.abs(jy).sum() / M]
    f += [dE / (S0 * dz), I / (M * dx * dy * dz) * dz]
    return np.asarray(f, dtype=np.float64).astype(np.float32), float(I)
