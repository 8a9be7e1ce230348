"""The learned part: a network answering G(soil, range, frequency).

The reference has no learned component; this module serves the Sobol and
sweep workloads (py/analysis/sobol.py, internal/sweep) with a network trained
on banks the batched solver produces, the plain GPU f-k solve being both its
fallback and the measure of its error.

Soil family (the 11 scalars): three finite layers over a half-space drawn
from the batched-soil ranges (Vs log-uniform 80-600 m/s, Vp/Vs uniform 1.7-3,
Qs uniform 10-60 with Qp = 2 Qs, thickness log-uniform 0.2-5 m):

    vs1, vpvs1, qs1, h1, vs2, vpvs2, qs2, h2, vs3, h3, vs_hs

Densities are fixed per layer (1700, 1850, 2000 kg/m3, half-space 2000);
layer 3 and the half-space have Vp/Vs 2 and Qs 40. The Sobol workload's soils
(two layers with a 2 m second layer over a half-space, ``sobol.soil_of``) are
members: h2 = 2 and a third layer identical to the half-space (vs3 = vs_hs,
any h3), which leaves the response unchanged.

Labels are FP64 banks from the Dunkin solver on the Sobol traces' grid
(bins k fs/n, k = 1..512 at fs 1 kHz, n 1024; complex frequency offset pi/T)
at ranges 1..64 m: t0 = log|G| and t1 = -phi/(w r), phi the phase unwrapped
along range like internal/bank/interp.go:66-102 (see gfk_mlp.cu k_labels).
"""
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .fk import Batch, FkError, Integration, Layer, Stack, default_engine

PARAMS = [
    ("vs1", 80.0, 600.0, True), ("vpvs1", 1.7, 3.0, False), ("qs1", 10.0, 60.0, False), ("h1", 0.2, 5.0, True),
    ("vs2", 80.0, 600.0, True), ("vpvs2", 1.7, 3.0, False), ("qs2", 10.0, 60.0, False), ("h2", 0.2, 5.0, True),
    ("vs3", 80.0, 600.0, True), ("h3", 0.2, 5.0, True), ("vs_hs", 80.0, 600.0, True),
]
NPARAM = len(PARAMS)
DENSITY = (1700.0, 1850.0, 2000.0, 2000.0)
DEEP_VPVS, DEEP_QS = 2.0, 40.0


def soil_of(p):
    """The stack for one row of the 11 scalars."""
    vs1, r1, q1, h1, vs2, r2, q2, h2, vs3, h3, vsh = (float(x) for x in p)
    return Stack([Layer(h1, r1 * vs1, vs1, DENSITY[0], q1, 2 * q1),
                  Layer(h2, r2 * vs2, vs2, DENSITY[1], q2, 2 * q2),
                  Layer(h3, DEEP_VPVS * vs3, vs3, DENSITY[2], DEEP_QS, 2 * DEEP_QS),
                  Layer(0.0, DEEP_VPVS * vsh, vsh, DENSITY[3], DEEP_QS, 2 * DEEP_QS)])


def layer_table(params):
    """soil_of for many rows at once: ([4 n, 6] layer entries, [n] counts)."""
    p = np.asarray(params, dtype=np.float64)
    vs1, r1, q1, h1, vs2, r2, q2, h2, vs3, h3, vsh = p.T
    n = len(p)
    c = lambda x: np.full(n, x)
    out = np.empty((n, 4, 6))
    out[:, 0] = np.stack([h1, r1 * vs1, vs1, c(DENSITY[0]), q1, 2 * q1], axis=1)
    out[:, 1] = np.stack([h2, r2 * vs2, vs2, c(DENSITY[1]), q2, 2 * q2], axis=1)
    out[:, 2] = np.stack([h3, DEEP_VPVS * vs3, vs3, c(DENSITY[2]), c(DEEP_QS), c(2 * DEEP_QS)], axis=1)
    out[:, 3] = np.stack([c(0.0), DEEP_VPVS * vsh, vsh, c(DENSITY[3]), c(DEEP_QS), c(2 * DEEP_QS)], axis=1)
    return out.reshape(4 * n, 6), np.full(n, 4, dtype=np.int32)


def draw(n, seed):
    """n soils uniform on the family's box (log-uniform where marked)."""
    u = np.random.default_rng(seed).random((n, NPARAM))
    return from_unit(u)


def from_unit(u):
    out = np.empty_like(u, dtype=np.float64)
    for j, (_, lo, hi, log) in enumerate(PARAMS):
        out[:, j] = np.exp(np.log(lo) + u[:, j] * (np.log(hi) - np.log(lo))) if log else lo + u[:, j] * (hi - lo)
    return out


def to_scalars(params):
    """Network inputs: each parameter mapped onto [-1, 1] (its log where log-uniform)."""
    params = np.asarray(params, dtype=np.float64)
    out = np.empty_like(params)
    for j, (_, lo, hi, log) in enumerate(PARAMS):
        x = params[:, j]
        out[:, j] = (2 * (np.log(x / lo) / np.log(hi / lo)) - 1) if log else (2 * (x - lo) / (hi - lo) - 1)
    return out


def travel_times(params):
    """Vertical S and P travel times of the three finite layers (s): the
    network's resonance features, [h1/vs1, h2/vs2, h3/vs3, h1/vp1, h2/vp2, h3/vp3]."""
    p = np.asarray(params, dtype=np.float64)
    vs1, r1, _, h1, vs2, r2, _, h2, vs3, h3, _ = p.T
    return np.ascontiguousarray(np.stack([h1 / vs1, h2 / vs2, h3 / vs3, h1 / (r1 * vs1), h2 / (r2 * vs2),
                                          h3 / (DEEP_VPVS * vs3)], axis=1))


def from_sobol(p8, h3=0.2):
    """Sobol rows (vs1, vpvs1, qs1, vs2, vpvs2, qs2, h1, vs_hs) as family rows."""
    p8 = np.asarray(p8, dtype=np.float64)
    vs1, r1, q1, vs2, r2, q2, h1, vsh = p8.T
    n = len(p8)
    return np.stack([vs1, r1, q1, h1, vs2, r2, q2, np.full(n, 2.0), vsh, np.full(n, h3), vsh], axis=1)


@dataclass
class LabelGrid:
    """The grid banks are solved and labelled on."""
    ranges: np.ndarray = field(default_factory=lambda: np.arange(1.0, 65.0))
    fs: float = 1000.0
    n: int = 1024
    nk: int = 8192
    kmax: float = 2.5 * 2 * math.pi * 500.0 / 80.0

    @property
    def freqs(self):
        return np.arange(1, self.n // 2 + 1) * self.fs / self.n

    @property
    def omega_imag(self):
        return math.pi / (self.n / self.fs)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def solve_media(params, grid, engine, ranges=None, batch_soils=8192, each=None):
    """Solves the family's soils on the grid with the Dunkin formulation and
    plain FP64 quadrature, batch by batch; `each(plan, first, count)` sees
    every executed plan (its result stays on the device). Returns the GPU
    milliseconds spent in the solver."""
    ranges = grid.ranges if ranges is None else np.asarray(ranges, dtype=np.float64)
    freqs = grid.freqs
    opt = Integration(grid.nk, 0.0, grid.kmax)
    ms = 0.0
    for b0 in range(0, len(params), batch_soils):
        chunk = params[b0:b0 + batch_soils]
        lay, cnt = layer_table(chunk)
        plan = Batch.from_layers(lay, cnt, freqs, ranges, opt, (N.DUNKIN, N.PLAIN_FP64, grid.omega_imag),
                                 engine=engine)
        try:
            plan.execute()
            st = plan.statuses()
            if (st != 0).any():
                bad = int(np.nonzero(st)[0][0])
                raise FkError(int(st[bad]), f"soil {b0 + bad // len(freqs)}: {N.STATUS_NAMES[int(st[bad])]}")
            a, b, c = plan.kernel_times()
            ms += a + b + c
            if each:
                each(plan, b0, len(chunk))
        finally:
            plan.close()
    return ms


class Dataset:
    """Labels of a set of family soils, in device memory (gfk_dataset)."""

    def __init__(self, params, grid=None, floor_rel=1e-6, engine=None):
        self.engine = engine or default_engine()
        self.grid = grid or LabelGrid()
        self.params = np.ascontiguousarray(params, dtype=np.float64)
        self.scalars = np.ascontiguousarray(to_scalars(self.params))
        self.times = travel_times(self.params)
        self.floor_rel = floor_rel
        h = ctypes.c_void_p()
        r = np.ascontiguousarray(self.grid.ranges, dtype=np.float64)
        f = np.ascontiguousarray(self.grid.freqs, dtype=np.float64)
        self.engine.check(N.lib().gfk_dataset_create(self.engine.ctx, NPARAM, len(self.params), _dp(self.scalars),
                                                     _dp(self.times), _dp(r), len(r), _dp(f), len(f), floor_rel,
                                                     ctypes.byref(h)))
        self.p = h
        self.engine._plans.add(self)
        self.solve_ms = 0.0

    def fill(self, batch_soils=8192):
        """Solves every soil and turns its bank into labels on the device."""
        def each(plan, first, count):
            self.engine.check(N.lib().gfk_dataset_fill(self.p, ctypes.c_void_p(plan.result_device_ptr()),
                                                       first, count))
        self.solve_ms += solve_media(self.params, self.grid, self.engine, batch_soils=batch_soils, each=each)
        return self

    def stats(self):
        """(mean t0, std t0, mean t1, std t1, phase-cell fraction)."""
        s = np.zeros(6)
        self.engine.check(N.lib().gfk_dataset_stats(self.p, _dp(s)))
        n0, s0, q0, n1, s1, q1 = s
        m0, m1 = s0 / n0, s1 / max(n1, 1)
        return (m0, math.sqrt(max(q0 / n0 - m0 * m0, 1e-30)), m1, math.sqrt(max(q1 / max(n1, 1) - m1 * m1, 1e-30)),
                n1 / n0)

    def labels(self, soil):
        out = np.zeros((len(self.grid.ranges), len(self.grid.freqs), 2), dtype=np.float32)
        self.engine.check(N.lib().gfk_dataset_labels(self.p, int(soil), _fp(out)))
        return out

    def close(self):
        if self.p:
            if self.engine.ctx:
                N.lib().gfk_dataset_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class NetConfig:
    batch: int = 8192
    warmup_steps: int = 500
    total_steps: int = 40000
    lr_max: float = 3e-4
    lr_min: float = 1e-5
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    weight_decay: float = 0.0
    phase_weight: float = 1.0
    fourier_sigma: float = 8.0
    loss_mode: int = N.LOSS_AMPLITUDE
    weight_floor: float = 0.1
    phase_cap: float = 1e4
    seed: int = 1

    def c(self):
        return N.GfkNetConfig(NPARAM, self.batch, self.warmup_steps, self.total_steps, self.lr_max, self.lr_min,
                              self.beta1, self.beta2, self.eps, self.weight_decay, self.phase_weight,
                              self.fourier_sigma, self.loss_mode, self.weight_floor, self.phase_cap, 0, self.seed)


class Net:
    """One surrogate network (gfk_net): BF16 MLP trained by libgfk's kernels."""

    def __init__(self, config=None, engine=None):
        self.engine = engine or default_engine()
        self.config = config or NetConfig()
        h = ctypes.c_void_p()
        self.engine.check(N.lib().gfk_net_create(self.engine.ctx, ctypes.byref(self.config.c()), ctypes.byref(h)))
        self.p = h
        self.engine._plans.add(self)
        self.scales = None
        self.steps_done = 0

    # -- parameters ---------------------------------------------------------
    @property
    def nparam(self):
        return int(N.lib().gfk_net_param_count(self.p))

    def params(self):
        out = np.zeros(self.nparam, dtype=np.float32)
        self.engine.check(N.lib().gfk_net_params(self.p, _fp(out), len(out), 0))
        return out

    def set_params(self, v):
        v = np.ascontiguousarray(v, dtype=np.float32)
        self.engine.check(N.lib().gfk_net_params(self.p, _fp(v), len(v), 1))

    def fourier(self):
        out = np.zeros(2 * N.NET_FOURIER, dtype=np.float32)
        self.engine.check(N.lib().gfk_net_fourier(self.p, _fp(out), 0))
        return out.reshape(N.NET_FOURIER, 2)

    def set_fourier(self, b):
        b = np.ascontiguousarray(b, dtype=np.float32).ravel()
        self.engine.check(N.lib().gfk_net_fourier(self.p, _fp(b), 1))

    def set_scales(self, r_lo, r_hi, f_lo, f_hi, mean_std):
        ms = np.ascontiguousarray(mean_std, dtype=np.float32)
        self.engine.check(N.lib().gfk_net_set_scales(self.p, r_lo, r_hi, f_lo, f_hi, _fp(ms)))
        self.scales = (float(r_lo), float(r_hi), float(f_lo), float(f_hi), [float(x) for x in ms])

    def scales_from(self, ds):
        m0, s0, m1, s1, _ = ds.stats()
        g = ds.grid
        self.set_scales(float(g.ranges.min()), float(g.ranges.max()), float(g.freqs.min()), float(g.freqs.max()),
                        [m0, s0, m1, s1])

    # -- training -----------------------------------------------------------
    def train(self, ds, soils, steps, ranges=None):
        """`steps` AdamW steps on cells of the given data set soils (and, if
        given, only the data set's range indices [ranges[0], ranges[1]));
        returns the per-step (amplitude, phase) mean squared errors."""
        soils = np.ascontiguousarray(soils, dtype=np.int32)
        loss = np.zeros((steps, 2), dtype=np.float32)
        r0, r1 = ranges if ranges is not None else (0, len(ds.grid.ranges))
        self.engine.check(N.lib().gfk_net_train_ranges(self.p, ds.p, _ip(soils), len(soils), int(r0), int(r1 - r0),
                                                       int(steps), _fp(loss)))
        self.steps_done += steps
        return loss

    def probe(self, X, Y, C=None):
        """One forward/backward pass on a given batch with loss coefficients
        C [batch][2] (None: 1 and phase_weight): (gradient, loss[2])."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        Cp = None if C is None else _fp(np.ascontiguousarray(C, dtype=np.float32))
        grad = np.zeros(self.nparam, dtype=np.float32)
        loss = np.zeros(2, dtype=np.float32)
        self.engine.check(N.lib().gfk_net_probe(self.p, _fp(X), _fp(Y), Cp, _fp(grad), _fp(loss)))
        return grad, loss

    # -- inference ----------------------------------------------------------
    def predict(self, params, ranges, freqs, out_device_ptr=None):
        """G [soil, freq, range] for family rows `params`; written to device
        memory instead when out_device_ptr is given."""
        sc = np.ascontiguousarray(to_scalars(params))
        tt = travel_times(params)
        r = np.ascontiguousarray(ranges, dtype=np.float64)
        f = np.ascontiguousarray(freqs, dtype=np.float64)
        if out_device_ptr is not None:
            self.engine.check(N.lib().gfk_net_predict(self.p, _dp(sc), _dp(tt), len(sc), _dp(r), len(r), _dp(f),
                                                      len(f), ctypes.c_void_p(out_device_ptr), 1))
            return None
        out = np.zeros((len(sc), len(f), len(r), 2))
        self.engine.check(N.lib().gfk_net_predict(self.p, _dp(sc), _dp(tt), len(sc), _dp(r), len(r), _dp(f), len(f),
                                                  out.ctypes.data_as(ctypes.c_void_p), 0))
        return out[..., 0] + 1j * out[..., 1]

    def evaluate(self, ds, soils):
        """Held-out error over the data set grid: rel-L2 of complex G, RMS of
        the log-amplitude error, RMS phase error (rad), over the listed soils."""
        soils = np.ascontiguousarray(soils, dtype=np.int32)
        o = np.zeros(7)
        self.engine.check(N.lib().gfk_net_evaluate(self.p, ds.p, _ip(soils), len(soils), _dp(o)))
        cells, e0, n1, e1, eph, dg, g2 = o
        return {"cells": int(cells), "rel_l2": math.sqrt(dg / g2), "rms_log_amp": math.sqrt(e0 / cells),
                "rms_t1": math.sqrt(e1 / max(n1, 1)), "rms_phase_rad": math.sqrt(eph / max(n1, 1)),
                "phase_cells": int(n1)}

    # -- persistence --------------------------------------------------------
    def save(self, path):
        np.savez(path, params=self.params(), fourier=self.fourier(), scales=np.array(self.scales[:4]),
                 mean_std=np.array(self.scales[4]), seed=self.config.seed, steps=self.steps_done)

    @classmethod
    def load(cls, path, config=None, engine=None):
        z = np.load(path)
        cfg = config or NetConfig(seed=int(z["seed"]))
        net = cls(cfg, engine)
        net.set_params(z["params"])
        net.set_fourier(z["fourier"])
        net.set_scales(*[float(x) for x in z["scales"]], z["mean_std"])
        net.steps_done = int(z["steps"])
        return net

    def close(self):
        if self.p:
            if self.engine.ctx:
                N.lib().gfk_net_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def split_soils(n, holdout=0.05, seed=0):
    """(train, held-out) soil indices; every 1/holdout-th soil of a seeded permutation is held out."""
    perm = np.random.default_rng(seed).permutation(n)
    k = max(1, int(round(n * holdout)))
    return np.sort(perm[k:]).astype(np.int32), np.sort(perm[:k]).astype(np.int32)


def train_ensemble(ds, train, members=4, steps=40000, config=None, engine=None, log=None, ranges=None):
    """`members` networks differing in initial weights, Fourier frequencies and
    batches; `ranges` restricts training to range indices [r0, r1)."""
    nets = []
    for m in range(members):
        cfg = NetConfig(**{**(config.__dict__ if config else {}), "seed": (config.seed if config else 1) + 7919 * m,
                           "total_steps": steps})
        net = Net(cfg, engine)
        net.scales_from(ds)
        t = time.perf_counter()
        loss = net.train(ds, train, steps, ranges)
        if log:
            log(f"member {m}: {steps} steps in {time.perf_counter() - t:.1f} s, final loss "
                f"{loss[-100:, 0].mean():.3e} / {loss[-100:, 1].mean():.3e}")
        nets.append(net)
    return nets


__all__ = ["PARAMS", "NPARAM", "soil_of", "draw", "from_unit", "to_scalars", "travel_times", "from_sobol", "LabelGrid", "Dataset",
           "NetConfig", "Net", "solve_media", "split_soils", "train_ensemble"]
