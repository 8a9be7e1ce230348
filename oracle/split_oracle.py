"""The tensor-core wavenumber sum's exact-integer splitting, restated in numpy.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the split
(int8-digit) sum's definition and accuracy, never used by the GPU path.

The sum S[f][r] = sum_k rem[f][k] W[k][r] (rem complex, W real: the Hankel
weights w_k J0(k r) dk of internal/fk/fk.go:540-546) is computed the way the
tcgen05 kernel defines it:
- every real row x (the real and the imaginary part of rem[f]) is divided by
  2^e, e = ilogb(max|x| 128/127) + 1, rounded once to N = rint(x 2^(28 - e))
  and cut into balanced base-128 digits
  N = d0 2^21 + d1 2^14 + d2 2^7 + d3 (-64 <= d1, d2, d3 < 64);
- the weights share one exponent e_b from dk (|W| <= dk) and are cut the same
  way;
- the digit products of level l = s + t <= 3 are summed exactly (integers);
- S = 2^(e + e_b) (L0 2^-14 + L1 2^-21 + L2 2^-28 + L3 2^-35), added left to
  right in FP64 as the kernel's epilogue adds them.
"""
import numpy as np


def exponent(mx):
    """ilogb(mx 128/127) + 1 (so that 2^e > mx 128/127), 0 where mx == 0."""
    mx = np.asarray(mx, dtype=np.float64)
    _, e = np.frexp(mx * (128.0 / 127.0))  # y = m 2^e with m in [0.5, 1): ilogb(y) = e - 1
    return np.where(mx > 0, e, 0).astype(np.int64)


def digits(n):
    """Balanced base-128 digits (d0, d1, d2, d3) of integers n (int64 arrays)."""
    n = np.asarray(n, dtype=np.int64)
    out = []
    for _ in range(3):
        d = ((n + 64) & 127) - 64
        n = (n - d) >> 7  # exact: n - d is a multiple of 128
        out.append(d)
    out.append(n)
    return out[::-1]


def cut(x, e):
    """The four digit arrays of x scaled by 2^-e (e broadcast against x)."""
    n = np.rint(np.ldexp(np.asarray(x, dtype=np.float64), 28 - np.asarray(e))).astype(np.int64)
    return digits(n)


LEVEL_WEIGHTS = (2.0 ** -14, 2.0 ** -21, 2.0 ** -28, 2.0 ** -35)


def split_sum_real(a, b, e_b):
    """sum_k a[m][k] b[k][n] for real rows a [M][K] and columns b [K][N] whose
    magnitudes are at most 2^e_b (one shared exponent)."""
    a = np.asarray(a, dtype=np.float64)
    e_a = exponent(np.abs(a).max(axis=1))[:, None]
    da = cut(a, e_a)
    db = cut(b, e_b)
    levels = []
    for lvl in range(4):
        acc = np.zeros((a.shape[0], b.shape[1]), dtype=np.int64)
        for s in range(lvl + 1):
            acc += da[s] @ db[lvl - s]
        levels.append(acc)
    total = levels[0] * LEVEL_WEIGHTS[0]
    for lvl in range(1, 4):
        total = total + levels[lvl] * LEVEL_WEIGHTS[lvl]
    return np.ldexp(total, e_a + e_b), levels


def split_sum(rem, w, dk):
    """The complex integrand rows rem [F][K] times the real weights w [K][N]."""
    e_b = int(exponent(dk))
    re, _ = split_sum_real(np.real(rem), w, e_b)
    im, _ = split_sum_real(np.imag(rem), w, e_b)
    return re + 1j * im


def error_bound(rem_part, dk, k):
    """A bound on |split - exact| for each row of a real part: each operand is
    rounded to 2^-29 of its scale and the dropped levels (s + t >= 4, digits
    below 64) add under 2^-28 more, so one product is off by at most
    2^(e_a + e_b - 27) and a K-term sum by K times that."""
    e_a = exponent(np.abs(rem_part).max(axis=1))
    e_b = int(exponent(dk))
    return k * np.ldexp(1.0, e_a + e_b - 27)
