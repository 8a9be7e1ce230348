"""The reference's finite-difference validator (internal/fdtd) on the GPU.

Same names and behaviour as the Go package: Model (model.go:30-100), Ricker
and RickerSpectrum (run.go:14-44), Shot / Trace / Result / Run
(run.go:46-127), SpacingFor (model.go:102-120). Run executes every time
step on the device (gfk_fdtd_run: one velocity and one stress kernel per
step over the whole grid) and returns the surface traces.
"""
import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .fk import SLS, FkError, Medium, Stack, _c_medium, default_engine


@dataclass
class Model:
    """fdtd.Model: zero fields take the reference's defaults."""
    stack: Stack
    relax: SLS = None
    ref_freq: float = 0.0
    max_range: float = 0.0
    depth: float = 0.0
    spacing: float = 0.0
    pml_cells: int = 0
    pml_reflection: float = 0.0
    dominant_freq: float = 0.0
    courant: float = 0.0

    def c(self, cmedium):
        return N.GfkFdtdModel(cmedium, float(self.max_range), float(self.depth), float(self.spacing),
                              int(self.pml_cells), 0, float(self.pml_reflection), float(self.dominant_freq),
                              float(self.courant))

    def _medium(self):
        return Medium(self.stack, ref_freq=self.ref_freq, relax=self.relax)

    def grid(self):
        """(dt, nr, nz) of the simulation New builds (fdtd.go:45-64)."""
        with _c_medium(self._medium()) as cm:
            dt, nr, nz = ctypes.c_double(), ctypes.c_int32(), ctypes.c_int32()
            st = N.lib().gfk_fdtd_grid(ctypes.byref(self.c(cm)), ctypes.byref(dt), ctypes.byref(nr),
                                       ctypes.byref(nz))
        if st:
            raise FkError(st, f"fdtd: invalid model ({N.status_string(st)})")
        return dt.value, nr.value, nz.value

    def spacing_for(self, max_freq, cells_per_wavelength):
        """Model.SpacingFor (model.go:102-120)."""
        if max_freq <= 0 or cells_per_wavelength <= 0:
            raise FkError(N.EARG, "fdtd: bandwidth and cells per wavelength must be positive")
        self.stack.validate()
        v = min(l.vs for l in self.stack)
        if self.relax and self.relax.tau_eps > self.relax.tau_sigma:
            f_ref = self.ref_freq if self.ref_freq > 0 else 30.0
            w = 2j * math.pi * f_ref
            mod = (1 + w * self.relax.tau_eps) / (1 + w * self.relax.tau_sigma)
            v = v * (1 / np.sqrt(mod)).real
        return v / (max_freq * cells_per_wavelength)


def ricker(peak, f0, dt, n):
    """fdtd.Ricker (run.go:14-27)."""
    if f0 <= 0 or dt <= 0 or n <= 0:
        raise FkError(N.EARG, "fdtd: Ricker needs a positive frequency, step and length")
    t0 = 1.5 / f0
    a = math.pi * math.pi * f0 * f0
    tau = np.arange(n) * dt - t0
    return peak * (1 - 2 * a * tau * tau) * np.exp(-a * tau * tau)


def ricker_spectrum(peak, f0, f):
    """fdtd.RickerSpectrum (run.go:33-44)."""
    fr = f / f0
    mag = 2 / math.sqrt(math.pi) * fr * fr * np.exp(-fr * fr) / f0
    phase = -2 * math.pi * f * 1.5 / f0
    return peak * mag * np.exp(1j * phase)


@dataclass
class Trace:
    range: float
    vertical: np.ndarray


@dataclass
class Result:
    dt: float
    t0: float
    traces: list
    cells: tuple
    peak: float


@dataclass
class Shot:
    model: Model
    force: np.ndarray
    ranges: list
    steps: int


def run(shot, engine=None):
    """fdtd.Run (run.go:78-127) on the GPU."""
    eng = engine or default_engine()
    force = np.ascontiguousarray(shot.force, dtype=np.float64)
    r = np.ascontiguousarray(shot.ranges, dtype=np.float64)
    traces = np.zeros((len(r), max(int(shot.steps), 1)))
    snapped = np.zeros(len(r))
    meta = np.zeros(5)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    with _c_medium(shot.model._medium()) as cm:
        st = N.lib().gfk_fdtd_run(eng.ctx, ctypes.byref(shot.model.c(cm)), dp(force), len(force), dp(r), len(r),
                                  int(shot.steps), dp(traces), dp(snapped), dp(meta))
    eng.check(st)
    return Result(meta[0], meta[1], [Trace(float(snapped[i]), traces[i]) for i in range(len(r))],
                  (int(meta[3]), int(meta[4])), meta[2])
