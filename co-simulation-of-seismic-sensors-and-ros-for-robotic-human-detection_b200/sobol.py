"""Sobol sensitivity of footstep metrics to the soil, with every soil's
Green's function at the sensor solved on the GPU.

The Sobol workload: a Saltelli design over 8 soil parameters (two finite
layers' Vs, Vp/Vs and Qs, the top layer's thickness and the half-space Vs),
N(d+2) soils; for each, the vertical velocity at 10 m from one footstep
(double-hump ground reaction force: 75 kg, 1.2 body-weight peaks, 30 ms
heel-strike rise) through an SM-24-like geophone (10 Hz, damping 0.7) is
reduced to its peak and its 2-400 Hz spectral centroid, and first-order and
total indices are estimated.

Restated on the host (cheap, O(soils x samples)):
  saltelli / indices / bootstrap   py/analysis/sobol.py:44-99
  Stance (GRF profile)             internal/grf/grf.go:34-330
  Geophone response                internal/geophone/geophone.go:36-203
  measure (peak, centroid)         internal/sweep/sweep.go:128-169
  causal taper above 0.8 Nyquist   internal/dsp/dsp.go:232-261
The banks (the f-k solve, all of the cost) run in libgfk as batches.

Choices the workload statement leaves open, fixed here: layer 2 is 2 m
thick; densities are 1700, 1850 and 2000 kg/m^3 (top, layer 2, half-space);
the half-space has Vp/Vs = 2, Qs = 40; every layer has Qp = 2 Qs; the trace is
1024 samples at 1 kHz (bins 1..512 solved), heel strike 50 ms in; the solve
uses the complex frequency offset w_I = pi/T (T = 1.024 s), undone after the
inverse transform; wavenumbers: 8192 to k_max = 2.5 w_max/80 m/s.
"""
import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from .fk import Batch, Integration, Layer, Medium, Stack
from . import _native as N

# ------------------------------------------------------------------ design --

# (name, low, high, log-scaled)
PARAMS = [
    ("vs1", 80.0, 600.0, True),
    ("vpvs1", 1.7, 3.0, False),
    ("qs1", 10.0, 60.0, False),
    ("vs2", 80.0, 600.0, True),
    ("vpvs2", 1.7, 3.0, False),
    ("qs2", 10.0, 60.0, False),
    ("h1", 0.2, 5.0, True),
    ("vs_hs", 80.0, 600.0, True),
]


def saltelli(n, k, seed=0):
    """(N(k+2), k) unit-cube design, blocks A, B, AB_0..AB_{k-1}
    (py/analysis/sobol.py:44-57): A and B from one scrambled Sobol sequence of
    dimension 2k."""
    from scipy.stats import qmc
    sample = qmc.Sobol(d=2 * k, scramble=True, seed=seed).random(n)
    a, b = sample[:, :k], sample[:, k:]
    blocks = [a, b]
    for i in range(k):
        ab = a.copy()
        ab[:, i] = b[:, i]
        blocks.append(ab)
    return np.vstack(blocks)


def indices(y, n, k):
    """First-order (Saltelli 2010) and total (Jansen 1999) indices
    (py/analysis/sobol.py:60-79)."""
    ya, yb = y[:n], y[n:2 * n]
    var = np.var(np.concatenate([ya, yb]), ddof=1)
    if var == 0:
        return np.zeros(k), np.zeros(k)
    s1, st = np.empty(k), np.empty(k)
    for i in range(k):
        yab = y[(i + 2) * n:(i + 3) * n]
        s1[i] = np.mean(yb * (yab - ya)) / var
        st[i] = np.mean((ya - yab) ** 2) / (2 * var)
    return s1, st


def bootstrap(y, n, k, draws=400, seed=0):
    """5-95% intervals, resampling matched rows across every block
    (py/analysis/sobol.py:82-99)."""
    rng = np.random.default_rng(seed)
    s1s, sts = np.empty((draws, k)), np.empty((draws, k))
    for d in range(draws):
        idx = rng.integers(0, n, n)
        resampled = np.concatenate([y[b * n:(b + 1) * n][idx] for b in range(k + 2)])
        s1s[d], sts[d] = indices(resampled, n, k)
    return np.percentile(s1s, [5, 95], axis=0), np.percentile(sts, [5, 95], axis=0)


def unit_to_params(u):
    """Maps the unit cube to parameter values (log-uniform where marked)."""
    out = np.empty_like(u)
    for j, (_, lo, hi, log) in enumerate(PARAMS):
        out[:, j] = np.exp(np.log(lo) + u[:, j] * (np.log(hi) - np.log(lo))) if log else lo + u[:, j] * (hi - lo)
    return out


def soil_of(p):
    """The stack for one parameter row."""
    vs1, r1, q1, vs2, r2, q2, h1, vsh = (float(x) for x in p)
    return Stack([Layer(h1, r1 * vs1, vs1, 1700.0, q1, 2 * q1),
                  Layer(2.0, r2 * vs2, vs2, 1850.0, q2, 2 * q2),
                  Layer(0.0, 2.0 * vsh, vsh, 2000.0, 40.0, 80.0)])


def layer_table(params):
    """soil_of for many rows at once: ([3 n, 6] layer entries, [n] counts),
    the arrays Batch.from_layers takes."""
    p = np.asarray(params, dtype=np.float64)
    vs1, r1, q1, vs2, r2, q2, h1, vsh = p.T
    n = len(p)
    out = np.empty((n, 3, 6))
    out[:, 0] = np.stack([h1, r1 * vs1, vs1, np.full(n, 1700.0), q1, 2 * q1], axis=1)
    out[:, 1] = np.stack([np.full(n, 2.0), r2 * vs2, vs2, np.full(n, 1850.0), q2, 2 * q2], axis=1)
    out[:, 2] = np.stack([np.zeros(n), 2.0 * vsh, vsh, np.full(n, 2000.0), np.full(n, 40.0), np.full(n, 80.0)],
                         axis=1)
    return out.reshape(3 * n, 6), np.full(n, 3, dtype=np.int32)


# ------------------------------------------------------------------ source --

@dataclass
class Stance:
    """grf.Stance (internal/grf/grf.go:34-105): vertical GRF of one stance."""
    mass: float = 75.0
    duration: float = 0.62
    first_peak: float = 1.2
    second_peak: float = 1.2
    valley: float = 0.75
    hump_width: float = 0.11          # defaultHumpWidth
    transient_peak: float = 0.35      # defaultTransientPeak
    transient_rise: float = 0.030
    taper: float = 0.098              # defaultTaperFraction

    def body_weight(self):
        return self.mass * 9.80665

    def profile(self, tau):
        """ProfileAt (grf.go:280-300) in body weights, vectorised."""
        tau = np.asarray(tau, dtype=np.float64)
        inside = (tau > 0) & (tau < 1)
        w = self.hump_width
        g1 = np.exp(-((tau - 0.25) / w) ** 2)
        g2 = np.exp(-((tau - 0.75) / w) ** 2)
        body = self.valley + (self.first_peak - self.valley) * g1 + (self.second_peak - self.valley) * g2
        r = self.taper
        tuk = np.where(tau < r, 0.5 * (1 - np.cos(np.pi * tau / r)),
                       np.where(tau > 1 - r, 0.5 * (1 - np.cos(np.pi * (1 - tau) / r)), 1.0))
        # transientAt (grf.go:230-240): a damped sine from heel contact
        crest, crest_phase = 0.63790, 0.20090
        period = self.transient_rise / crest_phase / self.duration
        decay = period / 2
        tr = np.where(tau > 0, self.transient_peak / crest * np.exp(-np.maximum(tau, 0) / decay)
                      * np.sin(2 * np.pi * tau / period), 0.0)
        return np.where(inside, tuk * body + tr, 0.0)

    def force(self, fs, n, lead):
        """ForceAt on n samples at fs, heel strike at `lead` seconds (newtons)."""
        t = np.arange(n) / fs - lead
        return self.profile(t / self.duration) * self.body_weight()


@dataclass
class Geophone:
    """geophone.Geophone (internal/geophone/geophone.go:36-62), SM-24 values
    (:64-77) with the natural frequency and damping the workload sets."""
    natural_freq: float = 10.0
    sensitivity: float = 28.8
    coil: float = 375.0
    shunt: float = 0.0
    open_circuit_damping: float = 0.7
    moving_mass: float = 0.011
    coupling_freq: float = 200.0      # WellPlantedSpike
    coupling_damping: float = 0.5

    def damping(self):
        if self.shunt <= 0:
            return self.open_circuit_damping
        w0 = 2 * np.pi * self.natural_freq
        return self.open_circuit_damping + self.sensitivity ** 2 / (2 * w0 * self.moving_mass * (self.coil + self.shunt))

    def response(self, s):
        """Response = CouplingResponse * TransducerResponse (geophone.go:175-203)
        at the Laplace variable s (i w on the real axis, i w_c off it), V/(m/s)."""
        w0 = 2 * np.pi * self.natural_freq
        div = 1.0 if self.shunt <= 0 else self.shunt / (self.coil + self.shunt)
        trans = (self.sensitivity * div) * s * s / (s * s + 2 * self.damping() * w0 * s + w0 * w0)
        if self.coupling_freq <= 0:
            return trans
        wc = 2 * np.pi * self.coupling_freq
        return wc * wc / (s * s + 2 * self.coupling_damping * wc * s + wc * wc) * trans


# ---------------------------------------------------------------- synthesis --

@dataclass
class TraceSetup:
    fs: float = 1000.0
    n: int = 1024
    lead: float = 0.05
    r: float = 10.0
    stance: Stance = field(default_factory=Stance)
    geophone: Geophone = field(default_factory=Geophone)

    @property
    def omega_imag(self):
        return math.pi / (self.n / self.fs)

    def freqs(self):
        return np.arange(1, self.n // 2 + 1) * self.fs / self.n


def traces(G, setup):
    """Geophone output traces (volts) from displacement spectra G[soil, bin]
    (bins 1..n/2) evaluated at w_c = 2 pi f - i w_I. The response is tapered to
    zero over the top fifth of the band (dsp.go:232-261) and the damping
    e^(-w_I t) is undone after the inverse transform."""
    n, fs, wi = setup.n, setup.fs, setup.omega_imag
    f = np.arange(n // 2 + 1) * fs / n
    wc = 2 * np.pi * f - 1j * wi
    s = 1j * wc
    t = np.arange(n) / fs
    force = setup.stance.force(fs, n, setup.lead) * np.exp(-wi * t)
    F = np.fft.rfft(force)
    H = np.zeros((G.shape[0], n // 2 + 1), dtype=np.complex128)
    H[:, 1:] = G * (1j * wc[1:])            # velocity per newton
    H *= setup.geophone.response(s)[None, :]
    nyq = fs / 2
    taper_from = 0.8 * nyq
    w = np.where(f > taper_from, 0.5 * (1 + np.cos(np.pi * (f - taper_from) / (nyq - taper_from))), 1.0)
    Y = H * (w * F)[None, :]
    y = np.fft.irfft(Y, n=n, axis=1)
    return y * np.exp(wi * t)[None, :]


def measure(y, fs):
    """Peak |y| and the 2-400 Hz magnitude-weighted spectral centroid
    (sweep.go:137-169), per trace."""
    peak = np.max(np.abs(y), axis=1)
    npad = 1 << int(math.ceil(math.log2(y.shape[1])))
    Y = np.fft.rfft(y, n=npad, axis=1)
    f = np.arange(npad // 2 + 1) * fs / npad
    band = (f >= 2) & (f <= 400)
    a = np.abs(Y[:, band])
    den = a.sum(axis=1)
    cen = np.where(den > 0, (a * f[band][None, :]).sum(axis=1) / np.where(den > 0, den, 1), 0.0)
    return peak, cen


# -------------------------------------------------------------------- solve --

NK = 8192
KMAX = 2.5 * 2 * math.pi * 500.0 / 80.0


def solve_banks(params, setup, engine, batch_soils=20000, nk=NK, kmax=KMAX, formulation=N.DUNKIN):
    """G[soil, bin] at setup.r for every parameter row, batched on the GPU.
    Returns (G, seconds of GPU execute, rows)."""
    freqs = setup.freqs()
    opt = Integration(nk, 0.0, kmax)
    out = np.zeros((len(params), len(freqs)), dtype=np.complex128)
    gpu_s = 0.0
    for b0 in range(0, len(params), batch_soils):
        chunk = params[b0:b0 + batch_soils]
        media = [Medium(soil_of(p), formulation=formulation, omega_imag=setup.omega_imag, engine=engine)
                 for p in chunk]
        plan = Batch(media, [freqs] * len(media), [setup.r], opt, engine=engine)
        plan.execute()
        g, status = plan.download()
        prop, quad, other = plan.kernel_times()
        gpu_s += (prop + quad + other) * 1e-3
        plan.close()
        if (status != 0).any():
            bad = int(np.nonzero(status)[0][0])
            raise RuntimeError(f"soil {b0 + bad // len(freqs)}: status {N.STATUS_NAMES[int(status[bad])]}")
        out[b0:b0 + len(chunk)] = g.reshape(len(chunk), len(freqs))
    return out, gpu_s, len(params) * len(freqs)


@dataclass
class SobolResult:
    n: int
    s1: dict
    st: dict
    metrics: dict
    seconds: dict


def shaping(setup):
    """S_k, k = 0..n/2: what traces() multiplies G[k-1] by (velocity per
    newton, sensor, taper above 0.8 Nyquist, footstep spectrum) at w_c."""
    n, fs, wi = setup.n, setup.fs, setup.omega_imag
    f = np.arange(n // 2 + 1) * fs / n
    wc = 2 * np.pi * f - 1j * wi
    t = np.arange(n) / fs
    F = np.fft.rfft(setup.stance.force(fs, n, setup.lead) * np.exp(-wi * t))
    nyq = fs / 2
    taper_from = 0.8 * nyq
    w = np.where(f > taper_from, 0.5 * (1 + np.cos(np.pi * (f - taper_from) / (nyq - taper_from))), 1.0)
    S = (1j * wc) * setup.geophone.response(1j * wc) * (w * F)
    S[0] = 0.0
    return S


def band(setup, lo=2.0, hi=400.0):
    """First and last rfft bin of measure()'s centroid band."""
    npad = 1 << int(math.ceil(math.log2(setup.n)))
    f = np.arange(npad // 2 + 1) * setup.fs / npad
    idx = np.nonzero((f >= lo) & (f <= hi))[0]
    return int(idx[0]), int(idx[-1])


def metrics_device(engine, d_G, stride, ns, setup):
    """(peak, centroid) of ns soils whose spectra G[s][k-1] (bins 1..n/2) are
    device (re, im) pairs at d_G + 16 s stride: gfk_trace_metrics."""
    Sc = shaping(setup)
    S = np.ascontiguousarray(np.stack([Sc.real, Sc.imag], axis=1).ravel())
    k_lo, k_hi = band(setup)
    peak = np.zeros(ns)
    cen = np.zeros(ns)

    def dp(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    engine.check(N.lib().gfk_trace_metrics(engine.ctx, ctypes.c_void_p(d_G), int(stride), int(ns), setup.n // 2,
                                           dp(S), setup.n, setup.fs, setup.omega_imag, k_lo, k_hi, dp(peak),
                                           dp(cen)))
    return peak, cen


def solve_metrics(params, setup, engine, batch_soils=20000, nk=NK, kmax=KMAX, formulation=N.DUNKIN):
    """(peak, centroid) of every parameter row through the GPU f-k solve and
    the GPU trace metrics; the banks never leave the device. Returns
    (peak, centroid, GPU solver seconds). The host tables of the next group's
    plan are built while the previous group executes on the device."""
    freqs = setup.freqs()
    opt = Integration(nk, 0.0, kmax)
    peak = np.zeros(len(params))
    cen = np.zeros(len(params))
    gpu_s = 0.0

    def build(b0):
        lay, cnt = layer_table(params[b0:b0 + batch_soils])
        return b0, Batch.from_layers(lay, cnt, freqs, [setup.r], opt, (formulation, N.PLAIN_FP64, setup.omega_imag),
                                     engine=engine)

    def finish(b0, plan):
        nonlocal gpu_s
        ns = len(params[b0:b0 + batch_soils])
        status = plan.statuses()
        if (status != 0).any():
            bad = int(np.nonzero(status)[0][0])
            raise RuntimeError(f"soil {b0 + bad // len(freqs)}: status {N.STATUS_NAMES[int(status[bad])]}")
        a, b, c = plan.kernel_times()
        gpu_s += (a + b + c) * 1e-3
        peak[b0:b0 + ns], cen[b0:b0 + ns] = metrics_device(engine, plan.result_device_ptr(), len(freqs), ns, setup)

    pending = []
    try:
        for b0 in range(0, len(params), batch_soils):
            pending.append(build(b0))
            if len(pending) == 2:
                finish(*pending[0])
                pending.pop(0)[1].close()
            pending[-1][1].execute()
        while pending:
            finish(*pending[0])
            pending.pop(0)[1].close()
    finally:
        for _, plan in pending:
            plan.close()
    return peak, cen, gpu_s


def _result(n, k, peak, cen, seconds):
    s1p, stp = indices(peak, n, k)
    s1c, stc = indices(cen, n, k)
    names = [p[0] for p in PARAMS]
    return SobolResult(n, {"peak": dict(zip(names, s1p)), "centroid": dict(zip(names, s1c))},
                       {"peak": dict(zip(names, stp)), "centroid": dict(zip(names, stc))},
                       {"peak": peak, "centroid": cen}, seconds)


def run_plain(engine, n=16384, seed=0, setup=None, batch_soils=20000, host_metrics=False):
    """The all-plain Sobol run: every soil through the GPU f-k solve. The
    metrics run on the GPU (gfk_trace_metrics) unless host_metrics, which
    downloads the banks and uses traces()/measure()."""
    setup = setup or TraceSetup()
    k = len(PARAMS)
    t0 = time.perf_counter()
    u = saltelli(n, k, seed)
    params = unit_to_params(u)
    if host_metrics:
        G, gpu_s, rows = solve_banks(params, setup, engine, batch_soils)
        t1 = time.perf_counter()
        peak, cen = measure(traces(G, setup), setup.fs)
    else:
        peak, cen, gpu_s = solve_metrics(params, setup, engine, batch_soils)
        t1 = time.perf_counter()
    res = _result(n, k, peak, cen, {})
    t2 = time.perf_counter()
    res.seconds = {"solve_wall": t1 - t0, "solve_gpu": gpu_s, "post": t2 - t1, "total": t2 - t0,
                   "rows": len(params) * len(setup.freqs()), "soils": len(params)}
    return res


def ensemble_metrics(nets, params8, setup, engine, chunk_soils=32768):
    """Every network's (peak, centroid) for the Sobol rows: each network
    predicts G at the sensor range on the device and the trace metrics run
    on that device buffer. Returns arrays [members][soils]."""
    import torch  # device buffers only

    from .surrogate import from_sobol
    p11 = from_sobol(params8)
    freqs = setup.freqs()
    nb = len(freqs)
    peaks = np.zeros((len(nets), len(p11)))
    cens = np.zeros((len(nets), len(p11)))
    buf = torch.empty(min(chunk_soils, len(p11)) * nb * 2, dtype=torch.float64, device=f"cuda:{engine.device}")
    for e, net in enumerate(nets):
        for b0 in range(0, len(p11), chunk_soils):
            chunk = p11[b0:b0 + chunk_soils]
            net.predict(chunk, [setup.r], freqs, out_device_ptr=buf.data_ptr())
            pk, ce = metrics_device(engine, buf.data_ptr(), nb, len(chunk), setup)
            peaks[e, b0:b0 + len(chunk)] = pk
            cens[e, b0:b0 + len(chunk)] = ce
    del buf
    return peaks, cens


def spread(values):
    """Relative spread (max - min) / |mean| over the ensemble axis 0."""
    v = np.asarray(values)
    return (v.max(axis=0) - v.min(axis=0)) / np.maximum(np.abs(v.mean(axis=0)), 1e-300)


def _solve_rows(params, bins_per_soil, setup, engine, batch_soils, nk=NK, kmax=KMAX, formulation=N.DUNKIN):
    """Yields (plan, soil indices) for the listed rows of each soil: one batch
    plan per group of soils, each soil with its own bins. The next group's
    plan is built while the previous one executes."""
    freqs = setup.freqs()
    opt = Integration(nk, 0.0, kmax)
    soils = [i for i, b in enumerate(bins_per_soil) if len(b)]

    def build(group):
        lay, cnt = layer_table(params[group])
        return Batch.from_layers(lay, cnt, None, [setup.r], opt, (formulation, N.PLAIN_FP64, setup.omega_imag),
                                 engine=engine, freqs_per_medium=[freqs[bins_per_soil[i]] for i in group])

    def checked(plan):
        status = plan.statuses()
        if (status != 0).any():
            bad = int(np.nonzero(status)[0][0])
            raise RuntimeError(f"fallback row {bad}: status {N.STATUS_NAMES[int(status[bad])]}")

    pending = []
    try:
        for b0 in range(0, len(soils), batch_soils):
            group = soils[b0:b0 + batch_soils]
            pending.append((build(group), group))
            if len(pending) == 2:
                checked(pending[0][0])
                yield pending[0]
                pending.pop(0)[0].close()
            pending[-1][0].execute()
        while pending:
            checked(pending[0][0])
            yield pending[0]
            pending.pop(0)[0].close()
    finally:
        for plan, _ in pending:
            plan.close()


def run_surrogate(engine, nets, n=16384, seed=0, setup=None, threshold=0.01, batch_soils=20000, gate="rows",
                  chunk_soils=32768, amp_threshold=0.001):
    """The Sobol run with the surrogate answering and the plain GPU f-k solve
    as fallback and as the measure of its error.

    gate="rows": every network predicts each soil's spectrum at the sensor;
    the ensemble mean answers, except on the rows (soil, bin) where the
    members disagree by more than `threshold` of the soil's trace-spectrum
    peak (gfk_ensemble_gate), which the f-k solve recomputes in place
    (gfk_scatter_rows); metrics then run on the merged device spectra.
    With amp_threshold > 0 the rows whose predicted |G S_k| exceeds
    amp_threshold of that peak are re-solved too: members trained on the same
    data can agree on an energetic row and all be wrong, and those rows carry
    the trace.
    gate="soil": each network's metrics are computed; where the ensemble's
    relative spread of either metric exceeds `threshold` the whole soil is
    re-solved and its plain metrics replace the ensemble mean."""
    import torch  # device buffers only

    from .surrogate import from_sobol
    setup = setup or TraceSetup()
    k = len(PARAMS)
    t0 = time.perf_counter()
    u = saltelli(n, k, seed)
    params = unit_to_params(u)
    nb = len(setup.freqs())
    if gate == "soil":
        peaks, cens = ensemble_metrics(nets, params, setup, engine)
        t1 = time.perf_counter()
        peak, cen = peaks.mean(axis=0), cens.mean(axis=0)
        sp = np.maximum(spread(peaks), spread(cens))
        fb = np.nonzero(sp > threshold)[0]
        gpu_s = 0.0
        if len(fb):
            pk, ce, gpu_s = solve_metrics(params[fb], setup, engine, batch_soils)
            peak[fb], cen[fb] = pk, ce
        t2 = time.perf_counter()
        res = _result(n, k, peak, cen, {})
        res.seconds = {"surrogate": t1 - t0, "fallback_wall": t2 - t1, "fallback_gpu": gpu_s,
                       "total": time.perf_counter() - t0, "soils": len(params), "fallback_soils": int(len(fb)),
                       "fallback_fraction": len(fb) / len(params), "members": len(nets), "threshold": threshold,
                       "gate": gate}
        res.metrics["spread"] = sp
        return res

    p11 = from_sobol(params)
    Sc = shaping(setup)
    S = np.ascontiguousarray(np.stack([Sc.real, Sc.imag], axis=1).ravel())
    dev = f"cuda:{engine.device}"
    cs = min(chunk_soils, len(p11))
    bufs = [torch.empty(cs * nb * 2, dtype=torch.float64, device=dev) for _ in nets]
    mean = torch.empty(cs * nb * 2, dtype=torch.float64, device=dev)
    ptrs = (ctypes.c_void_p * len(nets))(*[b.data_ptr() for b in bufs])
    peak = np.zeros(len(p11))
    cen = np.zeros(len(p11))
    spread_s = np.zeros(len(p11))
    t_pred = t_fb = gpu_s = 0.0
    rows_fb = 0
    soils_fb = 0
    for c0 in range(0, len(p11), cs):
        chunk = p11[c0:c0 + cs]
        m = len(chunk)
        ta = time.perf_counter()
        for net, b in zip(nets, bufs):
            net.predict(chunk, [setup.r], setup.freqs(), out_device_ptr=b.data_ptr())
        flags = np.zeros((m, nb), dtype=np.uint8)
        sp = np.zeros(m)
        engine.check(N.lib().gfk_ensemble_gate(
            engine.ctx, ptrs, len(nets), nb, m, nb, S.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), threshold,
            amp_threshold, ctypes.c_void_p(mean.data_ptr()), flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            sp.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        tb = time.perf_counter()
        t_pred += tb - ta
        bins = [np.nonzero(flags[i])[0] for i in range(m)]
        rows_fb += int(flags.sum())
        soils_fb += int((flags.sum(axis=1) > 0).sum())
        for plan, group in _solve_rows(params[c0:c0 + m], bins, setup, engine, batch_soils):
            idx = np.ascontiguousarray(np.concatenate([g * nb + bins[g] for g in group]).astype(np.int64))
            engine.check(N.lib().gfk_scatter_rows(engine.ctx, ctypes.c_void_p(plan.result_device_ptr()), 1,
                                                  idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(idx),
                                                  ctypes.c_void_p(mean.data_ptr())))
            a, b_, c_ = plan.kernel_times()
            gpu_s += (a + b_ + c_) * 1e-3
        pk, ce = metrics_device(engine, mean.data_ptr(), nb, m, setup)
        peak[c0:c0 + m], cen[c0:c0 + m], spread_s[c0:c0 + m] = pk, ce, sp
        t_fb += time.perf_counter() - tb
    del bufs, mean
    res = _result(n, k, peak, cen, {})
    total = time.perf_counter() - t0
    res.seconds = {"surrogate": t_pred, "fallback_wall": t_fb, "fallback_gpu": gpu_s, "total": total,
                   "soils": len(params), "fallback_soils": soils_fb, "fallback_rows": rows_fb,
                   "fallback_fraction": rows_fb / (len(params) * nb), "members": len(nets), "threshold": threshold,
                   "gate": gate}
    res.metrics["spread"] = spread_s
    return res
