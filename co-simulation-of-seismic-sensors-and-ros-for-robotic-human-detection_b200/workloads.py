"""The seeded synthetic workloads the engine is tested and measured on.

There is no public dataset for this path; each workload is a medium, a range
grid, a frequency grid and a wavenumber integration, exactly as stated here.

  single_soil    2 viscoelastic layers over a half-space (0.5 m and 2 m), 512
                 bins on fs = 1 kHz (Samples = 1024, bins 1..512), 4096
                 wavenumbers to k_max = 2.5 w_max/Vs_min, 64 ranges 1..64 m,
                 w_I = pi/T with T = 1.024 s, Qp as given.
  graded_soil    10 finite layers of 0.8 m (Vs 120 -> 600 m/s linear in layer
                 index, Vp = 2 Vs, rho 1600 -> 2100, Qs 10 -> 60, Qp = 2 Qs) over
                 a half-space with the last layer's properties; 2048 bins on
                 fs = 1 kHz (Samples = 4096), 16384 wavenumbers to
                 k_max = max(2.5 w_max/Vs_min, 40/r_min) = 80 rad/m, 1024 ranges
                 0.5..512 m, w_I = pi/T with T = Samples/fs.
  batched_soils  seeded soils with layer counts 2..12 (stack entries including
                 the half-space), Vs log-uniform 80..600, Vp/Vs uniform 1.7..3.0,
                 rho uniform 1500..2200, Qs uniform 10..60 with Qp = 2 Qs,
                 thickness log-uniform 0.2..5 m; frequency counts uniform in
                 256..2048 over 0..500 Hz (Samples = 2 Nf); 8192 wavenumbers on
                 one shared grid to k_max = 2.5 w_max/80; 128 ranges 1..128 m.

The fixed grid of a workload is expressed through the reference's own
Integration: Samples = Nk and KMaxFactor = 2.5 f_max/f make GridFor return
k_max = max(2.5 w_max/Vs_min, 40/r_min) at every frequency
(internal/fk/fk.go:479), so one wavenumber grid serves every frequency.
"""
import math
from dataclasses import dataclass

import numpy as np

from .fk import Integration, Layer, Medium, Stack
from . import _native as N


@dataclass
class Workload:
    name: str
    stack: Stack
    ranges: np.ndarray
    freqs: np.ndarray
    samples: int          # wavenumber samples
    kmax: float           # wavenumber cut
    omega_imag: float
    fs: float
    transform_samples: int

    def integration(self):
        """The workload's one wavenumber grid at every frequency."""
        return Integration(self.samples, 0.0, self.kmax)

    def kmax_factor_at(self, f):
        """The reference's per-frequency expression of the same cut."""
        slowest, _ = self.stack.velocity_bounds()
        return self.kmax / (2 * math.pi * f / slowest)

    def medium(self, formulation=N.DUNKIN, **kw):
        return Medium(self.stack, formulation=formulation,
                      omega_imag=self.omega_imag if formulation == N.DUNKIN else 0.0, **kw)

    def cells(self):
        return len(self.freqs) * len(self.ranges)


def single_soil():
    stack = Stack([Layer(0.5, 300.0, 150.0, 1700.0, 15.0, 30.0),
                   Layer(2.0, 500.0, 250.0, 1800.0, 25.0, 50.0),
                   Layer(0.0, 800.0, 400.0, 2000.0, 40.0, 80.0)])
    fs, n = 1000.0, 1024
    freqs = np.arange(1, n // 2 + 1) * fs / n
    ranges = np.arange(1, 65, dtype=np.float64)
    kmax = max(2.5 * 2 * math.pi * freqs.max() / 150.0, 40 / ranges.min())
    return Workload("single_soil", stack, ranges, freqs, 4096, kmax, math.pi / (n / fs), fs, n)


def graded_soil():
    layers = []
    for i in range(10):
        x = i / 9
        vs = 120.0 + (600.0 - 120.0) * x
        qs = 10.0 + 50.0 * x
        layers.append(Layer(0.8, 2 * vs, vs, 1600.0 + 500.0 * x, qs, 2 * qs))
    last = layers[-1]
    layers.append(Layer(0.0, last.vp, last.vs, last.density, last.qs, last.qp))
    fs, n = 1000.0, 4096
    freqs = np.arange(1, n // 2 + 1) * fs / n
    ranges = np.arange(1, 1025, dtype=np.float64) * 0.5
    kmax = max(2.5 * 2 * math.pi * freqs.max() / 120.0, 40 / ranges.min())
    return Workload("graded_soil", Stack(layers), ranges, freqs, 16384, kmax, math.pi / (n / fs), fs, n)


def batched_soils(count=4096, seed=20240611):
    """The seeded uneven soils; returns a list of (Stack, freqs) and the shared
    ranges and wavenumber grid."""
    rng = np.random.default_rng(seed)
    soils = []
    for _ in range(count):
        nl = int(rng.integers(2, 13))
        vs = np.exp(rng.uniform(math.log(80), math.log(600), nl))
        ratio = rng.uniform(1.7, 3.0, nl)
        rho = rng.uniform(1500, 2200, nl)
        qs = rng.uniform(10, 60, nl)
        h = np.exp(rng.uniform(math.log(0.2), math.log(5.0), nl))
        stack = Stack(Layer(float(h[i]) if i < nl - 1 else 0.0, float(vs[i] * ratio[i]), float(vs[i]),
                            float(rho[i]), float(qs[i]), float(2 * qs[i])) for i in range(nl))
        nf = int(rng.integers(256, 2049))
        fs = 1000.0
        freqs = np.arange(1, nf + 1) * fs / (2 * nf)
        soils.append((stack, freqs))
    ranges = np.arange(1, 129, dtype=np.float64)
    kmax = 2.5 * 2 * math.pi * 500.0 / 80.0
    return soils, ranges, 8192, kmax


def shard(units, rank, world):
    """The units (e.g. (stack, freqs) soils) one rank of `world` builds:
    greedy longest-processing-time assignment on the cost rows x layers, so
    ranks finish together; deterministic, every rank computes the same split."""
    if world <= 1:
        return list(units)
    cost = [len(fr) * len(st) for st, fr in units]
    order = sorted(range(len(units)), key=lambda i: (-cost[i], i))
    load = [0] * world
    owner = [0] * len(units)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += cost[i]
    return [u for i, u in enumerate(units) if owner[i] == rank]
