"""Floating-point operation count of one cell-step of the fused stage kernels.

TEST INFRASTRUCTURE ONLY (a measurement aid of bench.py's roofline, never the
product).  The scalar building blocks of the march are restated with a
counting number type: every +, -, *, /, sqrt, abs, min/max comparison and
compare-and-select is tallied while one interface flux is evaluated on a
representative forward-peaked state, exactly as the FP64 kernel evaluates it
(reconstruction_methods/weno_z.py:12-87, realizability.py:132-176,
flux.py:10-386).  A cell-step of the IF-SSPRK3 march evaluates three stages;
each stage computes the 3 interface fluxes a cell owns (one per axis) and the
divergence and stage update of the cell (energy.py:878-1130).

Usage:  python -m oracle.flops      (prints the table used in profiles/)
"""

from __future__ import annotations

import math
from collections import Counter

COUNT = Counter()


class F:
    """A float that counts the operations applied to it."""

    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v.v if isinstance(v, F) else float(v)

    @staticmethod
    def _v(x):
        return x.v if isinstance(x, F) else float(x)

    def _op(self, other, name, fn):
        COUNT[name] += 1
        return F(fn(self.v, F._v(other)))

    def __add__(self, o): return self._op(o, "add", lambda a, b: a + b)
    def __radd__(self, o): return self._op(o, "add", lambda a, b: b + a)
    def __sub__(self, o): return self._op(o, "add", lambda a, b: a - b)
    def __rsub__(self, o): return self._op(o, "add", lambda a, b: b - a)
    def __mul__(self, o): return self._op(o, "mul", lambda a, b: a * b)
    def __rmul__(self, o): return self._op(o, "mul", lambda a, b: b * a)
    def __truediv__(self, o): return self._op(o, "div", lambda a, b: a / b)
    def __rtruediv__(self, o): return self._op(o, "div", lambda a, b: b / a)
    def __neg__(self):
        COUNT["add"] += 1
        return F(-self.v)

    def _cmp(self, o, fn):
        COUNT["cmp"] += 1
        return fn(self.v, F._v(o))

    def __lt__(self, o): return self._cmp(o, lambda a, b: a < b)
    def __le__(self, o): return self._cmp(o, lambda a, b: a <= b)
    def __gt__(self, o): return self._cmp(o, lambda a, b: a > b)
    def __ge__(self, o): return self._cmp(o, lambda a, b: a >= b)


def sqrt(x):
    COUNT["sqrt"] += 1
    return F(math.sqrt(F._v(x)))


def fabs(x):
    COUNT["abs"] += 1
    return F(abs(F._v(x)))


def weno_left(v0, v1, v2, v3, v4):
    p0 = v0 / 3 - 7 * v1 / 6 + 11 * v2 / 6
    p1 = -v1 / 6 + 5 * v2 / 6 + v3 / 3
    p2 = v2 / 3 + 5 * v3 / 6 - v4 / 6
    a = v0 - 2 * v1 + v2; b = v0 - 4 * v1 + 3 * v2
    beta0 = (13.0 / 12.0) * (a * a) + 0.25 * (b * b)
    a = v1 - 2 * v2 + v3; b = v1 - v3
    beta1 = (13.0 / 12.0) * (a * a) + 0.25 * (b * b)
    a = v2 - 2 * v3 + v4; b = 3 * v2 - 4 * v3 + v4
    beta2 = (13.0 / 12.0) * (a * a) + 0.25 * (b * b)
    tau5 = fabs(beta2 - beta0)
    r0 = tau5 / (beta0 + 1e-12); r1 = tau5 / (beta1 + 1e-12); r2 = tau5 / (beta2 + 1e-12)
    al0 = 0.1 * (1 + r0 * r0); al1 = 0.6 * (1 + r1 * r1); al2 = 0.3 * (1 + r2 * r2)
    s = al0 + al1 + al2
    return (al0 / s) * p0 + (al1 / s) * p1 + (al2 / s) * p2


def project(u):
    phi, jx, jy, jz = u
    if phi < 0:
        phi = F(0.0)
    jn = sqrt(jx * jx + jy * jy + jz * jz)
    jmax = (1.0 - 1e-10) * phi
    if jn > jmax:
        s = jmax / jn
        jx, jy, jz = jx * s, jy * s, jz * s
    return [phi, jx, jy, jz]


def eigen(u, jn, axis):
    phi = u[0]
    if phi < 1e-10:
        phi = F(1e-10)
    f = jn / phi
    if f > 1.0 - 1e-10:
        f = F(1.0 - 1e-10)
    mu = u[1 + axis] / jn
    chi = (5 - 2 * sqrt(4 - 3 * f * f)) / 3
    den = 5 - 3 * chi
    disc = 4 * f * f * mu * mu - den * (mu * mu * (3 * chi - 1) - 2 * (1 - chi))
    root = sqrt(disc)
    return (2 * f * mu - root) / den, (2 * f * mu + root) / den


def closure(u):
    phi, jx, jy, jz = u
    jn = sqrt(jx * jx + jy * jy + jz * jz)
    f = jn / phi
    if f > 1.0:
        f = F(1.0)
    n = [jx / jn, jy / jn, jz / jn]
    chi = (5 - 2 * sqrt(4 - 3 * f * f)) / 3
    return jn, n, 0.5 * (1 - chi), 0.5 * (3 * chi - 1)


def hll(L, R, axis):
    out = []
    for u in (L, R):
        jn, n, iso, dirc = closure(u)
        Fx = [u[1 + axis]] + [u[0] * ((iso if k == axis else 0.0) + dirc * n[axis] * n[k]) for k in range(3)]
        lo, hi = eigen(u, jn, axis)
        out.append((Fx, lo, hi))
    (FL, lol, hil), (FR, lor, hir) = out
    sl = lor if lor < lol else lol
    sr = hir if hir > hil else hil
    if sl > 0:
        sl = F(0.0)
    if sr < 0:
        sr = F(0.0)
    den = sr - sl
    sp = sl * sr
    return [(sr * FL[c] - sl * FR[c] + sp * (R[c] - L[c])) / den for c in range(4)]


def face():
    """One interface: 8 reconstructions, 2 projections, one HLL flux."""
    import random
    rng = random.Random(1)
    cells = [[F(1.0 + 0.1 * rng.random()), F(0.02 * rng.random()), F(0.02 * rng.random()),
              F(0.9 + 0.05 * rng.random())] for _ in range(6)]
    L = [weno_left(*[cells[q][c] for q in range(5)]) for c in range(4)]
    R = [weno_left(*[cells[5 - q][c] for q in range(5)]) for c in range(4)]
    return hll(project(L), project(R), 2)


def cell_update():
    """Divergence of 4 components and the IF-SSPRK3 update of one stage."""
    Fs = [[F(1.0 + 0.01 * k + 0.001 * c) for c in range(4)] for k in range(6)]
    Lc = [-((Fs[1][c] - Fs[0][c]) / 1e-3 + (Fs[3][c] - Fs[2][c]) / 1e-3 + (Fs[5][c] - Fs[4][c]) / 1e-3)
          for c in range(4)]
    u = [F(1.0), F(0.01), F(0.01), F(0.9)]
    s0, c1, s1 = F(500.0), F(0.99), F(510.0)
    v = [(Lc[c] * 0.3 + s0 * u[c]) * c1 / s1 for c in range(4)]   # stage algebra (representative)
    project(v)


def count(fn):
    COUNT.clear()
    fn()
    return dict(COUNT)


def per_cell_step():
    f, cu = count(face), count(cell_update)
    total = Counter()
    for k, v in f.items():
        total[k] += 3 * 3 * v          # 3 owned faces x 3 stages
    for k, v in cu.items():
        total[k] += 3 * v              # 3 stages
    return f, cu, dict(total)


if __name__ == "__main__":
    f, cu, tot = per_cell_step()
    flops = lambda d: sum(v for k, v in d.items() if k in ("add", "mul", "div", "sqrt"))
    print("per face:", f, "flops", flops(f))
    print("per cell and stage (divergence + update):", cu, "flops", flops(cu))
    print("per cell-step (3 stages):", tot, "flops", flops(tot))
