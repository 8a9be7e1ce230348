"""CPU oracle (test infrastructure only) for bank consumption.

numpy restatements, loop for loop, of
  Bank.prepare            internal/bank/interp.go:66-102
  Bank.bracket            internal/bank/format.go:295-309
  Bank.Response           internal/bank/interp.go:29-54
  CausalImpulseResponseAt internal/dsp/dsp.go:232-261 (IRFFT dsp.go:42-50)
as internal/sensing feeds it (sensing.go:196-204, propagation.go:84-104).
Nothing in the product imports this file.
"""
import math

import numpy as np

NEG_INF = -1e308  # interp.go:56


def go_round(x):
    """Go's math.Round: halves away from zero."""
    return math.copysign(math.floor(abs(x) + 0.5), x)


def prepare(data):
    """data float32 [count][bins][2] -> (logmag, phase) FP64 [count][bins]."""
    count, bins = data.shape[0], data.shape[1]
    logmag = np.zeros((count, bins))
    phase = np.zeros((count, bins))
    for k in range(bins):
        prev = unwrapped = 0.0
        for i in range(count):
            re, im = float(data[i, k, 0]), float(data[i, k, 1])
            mag = math.hypot(re, im)
            if mag == 0:
                logmag[i, k] = NEG_INF
                phase[i, k] = unwrapped
                continue
            logmag[i, k] = math.log(mag)
            w = math.atan2(im, re)
            if i == 0:
                unwrapped = w
            else:
                d = w - prev
                d -= 2 * math.pi * go_round(d / (2 * math.pi))
                unwrapped += d
            prev = w
            phase[i, k] = unwrapped
    return logmag, phase


def bracket(r, min_m, max_m, count):
    if r < min_m or r > max_m:
        raise ValueError(f"bank: range {r:g} m is outside the bank's {min_m:g} to {max_m:g} m")
    if count == 1:
        return 0, 0.0
    x = (r - min_m) / ((max_m - min_m) / (count - 1))
    lo = int(math.floor(x))
    if lo >= count - 1:
        return count - 2, 1.0
    return lo, x - lo


def response(tables, grid, r, k):
    logmag, phase = tables
    count = logmag.shape[0]
    lo, frac = bracket(r, *grid, count)
    hi = lo if count == 1 else lo + 1
    if logmag[lo, k] == NEG_INF or logmag[hi, k] == NEG_INF:
        return 0j
    lm = logmag[lo, k] + frac * (logmag[hi, k] - logmag[lo, k])
    ph = phase[lo, k] + frac * (phase[hi, k] - phase[lo, k])
    return complex(math.exp(lm) * math.cos(ph), math.exp(lm) * math.sin(ph))


def causal_impulse_response_at(n, length, fs, resp):
    nyq = fs / 2
    taper_from = 0.8 * nyq
    coeff = np.zeros(n // 2 + 1, dtype=np.complex128)
    for k in range(n // 2 + 1):
        f = k * fs / n
        h = resp(f)
        if f > taper_from:
            h *= 0.5 * (1 + math.cos(math.pi * (f - taper_from) / (nyq - taper_from)))
        coeff[k] = h
    return np.fft.irfft(coeff, n)[:length]


def impulse_responses(data, grid, fs, samples, ranges, length, sensor=None, velocity=True):
    """[len(ranges)][length], as sensing builds them from a bank."""
    tables = prepare(data)
    bins = data.shape[1]
    out = []
    for r in ranges:
        def resp(f):
            if f <= 0:
                return 0j
            k = int(round(f / (fs / samples)))
            if k >= bins:
                return 0j
            u = response(tables, grid, r, k)
            if velocity:
                u *= 2j * math.pi * f
            if sensor is not None:
                u *= sensor[k]
            return u
        out.append(causal_impulse_response_at(samples, length, fs, resp))
    return np.array(out)
