"""Rayleigh dispersion curves: the reference's internal/disp (with
internal/propmat's secular function) on the GPU.

Same names and behaviour as the Go package: Search, Bounds, Modes, Mode,
PhaseCurve, GroupVelocity (internal/disp/disp.go:30-192); errors are raised
as FkError with the Go message. The root scan and bisection for every
requested frequency run in one libgfk call (gfk_dispersion_modes), one GPU
block per frequency.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .fk import FkError, _c_medium, default_engine


@dataclass
class Search:
    """disp.Search: samples <= 0 uses 2000, tolerance <= 0 uses 1e-10."""
    samples: int = 0
    tolerance: float = 0.0

    def c(self):
        return N.GfkSearch(int(self.samples), 0, float(self.tolerance))


@dataclass
class Curve:
    """disp.Curve: one mode over the frequencies where it exists."""
    mode: int
    frequency: list = field(default_factory=list)
    phase_velocity: list = field(default_factory=list)


def _medium(stack):
    from .fk import Medium
    return Medium(stack)


def bounds(stack):
    """disp.Bounds (disp.go:62-65)."""
    return 0.85 * min(l.vs for l in stack), list(stack)[-1].vs


def modes_many(stack, freqs, opt=None, max_modes=64, engine=None):
    """disp.Modes at every frequency, one GPU call: a list of lists, slowest first."""
    eng = engine or default_engine()
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    vel = np.zeros((len(f), max_modes))
    cnt = np.zeros(len(f), dtype=np.int32)
    with _c_medium(_medium(stack)) as cm:
        st = N.lib().gfk_dispersion_modes(eng.ctx, ctypes.byref(cm), f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          len(f), (opt or Search()).c(), max_modes,
                                          vel.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                          cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    eng.check(st)
    return [list(vel[i, :cnt[i]]) for i in range(len(f))]


def modes(stack, freq, opt=None, engine=None):
    """disp.Modes (disp.go:68-103)."""
    return modes_many(stack, [freq], opt, engine=engine)[0]


def mode(stack, freq, index, opt=None, engine=None):
    """disp.Mode (disp.go:111-123)."""
    if index < 0:
        raise FkError(N.EARG, f"disp: mode index must not be negative, got {index}")
    all_ = modes(stack, freq, opt, engine)
    if index >= len(all_):
        raise FkError(N.EARG, f"disp: mode {index} does not exist at {freq:g} Hz (found {len(all_)})")
    return all_[index]


def phase_curve(stack, freqs, index, opt=None, engine=None):
    """disp.PhaseCurve (disp.go:135-152): frequencies without the mode are skipped."""
    c = Curve(index)
    for f, ms in zip(freqs, modes_many(stack, freqs, opt, engine=engine)):
        if index < len(ms):
            c.frequency.append(float(f))
            c.phase_velocity.append(ms[index])
    if not c.frequency:
        raise FkError(N.EARG, f"disp: mode {index} exists at none of the {len(freqs)} frequencies given")
    return c


def group_velocity(stack, freq, index, opt=None, engine=None):
    """disp.GroupVelocity (disp.go:164-186): U = c / (1 - (f/c) dc/df) by
    central difference at +-1e-3 f."""
    df = freq * 1e-3
    lo, hi, c = (mode(stack, f, index, opt, engine) for f in (freq - df, freq + df, freq))
    den = 1 - freq / c * ((hi - lo) / (2 * df))
    if den == 0:
        raise FkError(N.EARG, f"disp: group velocity is singular at {freq:g} Hz")
    return c / den


def secular_at_velocity(stack, freqs, velocities, engine=None):
    """propmat.SecularAtVelocity at (frequency, velocity) pairs: (values, ok)."""
    eng = engine or default_engine()
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    c = np.ascontiguousarray(velocities, dtype=np.float64)
    out = np.zeros(len(f))
    ok = np.zeros(len(f), dtype=np.int32)
    with _c_medium(_medium(stack)) as cm:
        eng.check(N.lib().gfk_secular(eng.ctx, ctypes.byref(cm), f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(f),
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      ok.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
    return out, ok.astype(bool)
