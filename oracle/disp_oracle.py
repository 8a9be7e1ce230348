"""CPU oracle (test infrastructure only) for Rayleigh dispersion curves.

numpy/scipy restatements of
  propmat.SystemMatrix / LayerPropagator / Compound / HalfSpaceModes / Secular
      internal/propmat/propmat.go:82-315 (the matrix exponential by
      scipy.linalg.expm in place of gonum's mat.Exp)
  disp.Bounds / Modes / Mode / PhaseCurve / GroupVelocity / bisect
      internal/disp/disp.go:62-217
  soil.HalfSpace.RayleighVelocity
      internal/soil/soil.go:136-164
Pinned against the reference's disba goldens (testdata/dispersion/*.json,
committed here under tests/golden/dispersion). Nothing in the product imports
this file.
"""
import math

import numpy as np
from scipy.linalg import expm

PAIRS = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
COMP = [5, 4, 3, 2, 1, 0]
LAPLACE_SIGN = [1, -1, 1, 1, -1, 1]


def _mu(l):
    return l[3] * l[2] * l[2]


def _lam(l):
    return l[3] * l[1] * l[1] - 2 * _mu(l)


def system_matrix(l, k, omega, mu_ref):
    """l = (thickness, vp, vs, density)."""
    mu, lam, rho = _mu(l), _lam(l), l[3]
    l2m = lam + 2 * mu
    rc2 = rho * omega * omega / (k * k)
    a = np.zeros((4, 4))
    a[0, 1] = -1
    a[0, 2] = mu_ref / mu
    a[1, 0] = lam / l2m
    a[1, 3] = mu_ref / l2m
    a[2, 0] = (4 * mu * (lam + mu) / l2m - rc2) / mu_ref
    a[2, 3] = -lam / l2m
    a[3, 1] = -rc2 / mu_ref
    a[3, 2] = 1
    return a


def vertical_wavenumbers(l, k, omega):
    sq = lambda v: math.sqrt(max(0.0, k * k - omega * omega / (v * v)))
    return sq(l[1]), sq(l[2])


def layer_propagator(l, k, omega, mu_ref):
    zeta = k * l[0]
    ra, _ = vertical_wavenumbers(l, k, omega)
    lam_max = ra / k
    shifted = zeta * system_matrix(l, k, omega, mu_ref) - lam_max * zeta * np.eye(4)
    return expm(shifted)


def compound(p):
    c = np.zeros((6, 6))
    for r, (i, j) in enumerate(PAIRS):
        for col, (kk, ll) in enumerate(PAIRS):
            c[r, col] = p[i, kk] * p[j, ll] - p[i, ll] * p[j, kk]
    return c


def half_space_minors(l, k, omega, mu_ref):
    if omega / k >= l[2]:
        return None
    ra, rb = vertical_wavenumbers(l, k, omega)
    mu, rho = _mu(l), l[3]
    rc2 = rho * omega * omega / (k * k)
    a, b = ra / k, rb / k
    p = [1, -a, -2 * (mu / mu_ref) * a, (2 * mu - rc2) / mu_ref]
    sv = [b, -1, (rc2 - 2 * mu) / mu_ref, 2 * (mu / mu_ref) * b]
    return [p[i] * sv[j] - p[j] * sv[i] for (i, j) in PAIRS]


def secular(stack, omega, k):
    """None where the reference returns an error."""
    if k <= 0 or omega <= 0:
        return None
    m = np.array([1.0, 0, 0, 0, 0, 0])
    mu_ref = max(_mu(l) for l in stack)
    for l in stack[:-1]:
        nxt = compound(layer_propagator(l, k, omega, mu_ref)) @ m
        norm = np.abs(nxt).max()
        if norm == 0:
            return None
        m = nxt / norm
    e = half_space_minors(stack[-1], k, omega, mu_ref)
    if e is None:
        return None
    return float(sum(LAPLACE_SIGN[n] * m[n] * e[COMP[n]] for n in range(6)))


def secular_at_velocity(stack, freq, c):
    omega = 2 * math.pi * freq
    return secular(stack, omega, omega / c)


def bounds(stack):
    return 0.85 * min(l[2] for l in stack), stack[-1][2]


def _sign_change(a, b):
    return (a < 0 < b) or (a > 0 > b)


def bisect(f, lo, hi, tol):
    flo = f(lo)
    if flo is None:
        return None
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid == lo or mid == hi or (hi - lo) < tol * mid:
            return mid
        v = f(mid)
        if v is None:
            return None
        if _sign_change(flo, v):
            hi = mid
        else:
            lo, flo = mid, v
    return 0.5 * (lo + hi)


def modes(stack, freq, samples=2000, tol=1e-10):
    """Every mode's phase velocity at freq, slowest first (disp.Modes)."""
    lo, hi = bounds(stack)

    def f(c):
        v = secular_at_velocity(stack, freq, c)
        if v is None or not math.isfinite(v):
            return None
        return v

    step = (hi * (1 - 1e-9) - lo) / samples
    out = []
    prev_c, prev_v = lo, f(lo)
    for i in range(1, samples + 1):
        c = lo + i * step
        v = f(c)
        if v is not None and prev_v is not None and _sign_change(prev_v, v):
            root = bisect(f, prev_c, c, tol)
            if root is not None:
                out.append(root)
        prev_c, prev_v = c, v
    return out


def mode(stack, freq, index, samples=2000, tol=1e-10):
    all_ = modes(stack, freq, samples, tol)
    return all_[index] if 0 <= index < len(all_) else None


def group_velocity(stack, freq, index, samples=2000, tol=1e-10):
    df = freq * 1e-3
    lo, hi, c = (mode(stack, f, index, samples, tol) for f in (freq - df, freq + df, freq))
    if lo is None or hi is None or c is None:
        return None
    dcdf = (hi - lo) / (2 * df)
    den = 1 - freq / c * dcdf
    return None if den == 0 else c / den


def rayleigh_velocity(vp, vs):
    """soil.HalfSpace.RayleighVelocity (soil.go:136-164)."""
    k2 = (vs / vp) ** 2
    f = lambda x: (2 - x) ** 2 - 4 * math.sqrt(1 - x) * math.sqrt(1 - x * k2)
    lo, hi = 1e-9, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid == lo or mid == hi:
            break
        if f(mid) < 0:
            lo = mid
        else:
            hi = mid
    return math.sqrt(0.5 * (lo + hi)) * vs
