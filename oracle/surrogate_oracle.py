"""CPU oracle (test infrastructure only) for the surrogate network's kernels.

numpy FP64 restatements of what libgfk's surrogate kernels compute, used by
the tests to check the GPU path; nothing in the product imports this file.

* labels(): the label construction of k_labels — log-amplitude with an
  amplitude floor and the phase unwrapped along range, each range step's
  cycle count predicted from the same step one frequency bin lower (the
  range-unwrap rule of internal/bank/interp.go:66-102 with the fold taken
  about that prediction).
* features(): the 128 input features of one (soil, range, frequency) point.
* forward()/backward(): the MLP (five SiLU layers of width 512, FP32 output
  layer) and the gradient of the loss (1/B) sum_b [e0^2 + w m_b e1^2], with
  an option that rounds to BF16 wherever the GPU stores BF16, so the GPU's
  gradients can be checked to FP32-accumulation accuracy.
"""
import math

import numpy as np

WIDTH, INPUTS, LAYERS, SCALARS, TIMES = 512, 128, 5, 16, 6
TIME_FEAT = SCALARS                      # sin, cos(2 pi f T_q)
LOG_TIME_FEAT = TIME_FEAT + 2 * TIMES    # (ln(f T_q) + 2) / 3 clamped to [-2, 2]
FOURIER_FEAT = LOG_TIME_FEAT + TIMES     # Fourier pairs of (range, frequency)
FOURIER = (INPUTS - FOURIER_FEAT) // 2


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


# ------------------------------------------------------------------ labels --

def labels(G, ranges, freqs, floor_rel):
    """G [nf][nr] complex -> labels [nr][nf][2] (t0, t1; t1 NaN where not learnt)."""
    G = np.asarray(G)
    nf, nr = G.shape
    amp = np.hypot(G.real, G.imag)
    floor = amp.max() * floor_rel
    w = np.arctan2(G.imag, G.real)
    two_pi = 2 * math.pi
    n_cyc = np.zeros((nr, nf), dtype=np.int64)
    ok = np.zeros((nr, nf), dtype=bool)
    # first range: along frequency
    n, good, dprev = 0, True, 0.0
    for j in range(nf):
        if j > 0:
            dw = w[j, 0] - w[j - 1, 0]
            m = np.rint((dprev - dw) / two_pi)
            dprev = dw + two_pi * m
            n += int(m)
        good = good and amp[j, 0] > floor
        n_cyc[0, j], ok[0, j] = n, good
    for i in range(1, nr):
        good, dprev = True, 0.0
        for j in range(nf):
            dw = w[j, i] - w[j, i - 1]
            pred = dprev * (freqs[j] / freqs[j - 1]) if j > 0 else 0.0
            m = np.rint((pred - dw) / two_pi)
            dprev = dw + two_pi * m
            good = good and amp[j, i] > floor and amp[j, i - 1] > floor
            n_cyc[i, j], ok[i, j] = int(m), good
    out = np.zeros((nr, nf, 2))
    for j in range(nf):
        n, valid = n_cyc[0, j], ok[0, j]
        for i in range(nr):
            if i > 0:
                valid = valid and ok[i, j]
                if valid:
                    n += n_cyc[i, j]
            out[i, j, 0] = math.log(max(amp[j, i], floor))
            out[i, j, 1] = -(w[j, i] + two_pi * n) / (two_pi * freqs[j] * ranges[i]) if valid else np.nan
    return out


# ---------------------------------------------------------------- features --

def features(scalars, times, r, f, dom, fourier):
    """Input rows for points (soil scalars [n][<=11], travel times [n][6],
    r [n], f [n]); dom = (r_lo, r_hi, f_lo, f_hi); fourier [47][2]."""
    scalars = np.atleast_2d(scalars)
    times = np.atleast_2d(times)
    r = np.asarray(r, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    n = len(r)
    r_lo, r_hi, f_lo, f_hi = dom
    ur = (r - r_lo) / (r_hi - r_lo)
    uf = (f - f_lo) / (f_hi - f_lo)
    X = np.zeros((n, INPUTS))
    X[:, :scalars.shape[1]] = scalars
    X[:, 11] = 2 * ur - 1
    X[:, 12] = 2 * uf - 1
    X[:, 13] = 2 * np.log(r / r_lo) / math.log(r_hi / r_lo) - 1
    X[:, 14] = 2 * np.log(f / f_lo) / math.log(f_hi / f_lo) - 1
    ft = f[:, None] * times
    X[:, TIME_FEAT:LOG_TIME_FEAT:2] = np.sin(2 * math.pi * ft)
    X[:, TIME_FEAT + 1:LOG_TIME_FEAT:2] = np.cos(2 * math.pi * ft)
    with np.errstate(divide="ignore"):
        lt = np.where(ft > 0, (np.log(np.where(ft > 0, ft, 1.0)) + 2) / 3, -2.0)
    X[:, LOG_TIME_FEAT:FOURIER_FEAT] = np.clip(lt, -2, 2)
    B = np.asarray(fourier, dtype=np.float64).reshape(FOURIER, 2)
    arg = 2 * math.pi * (ur[:, None] * B[None, :, 0] + uf[:, None] * B[None, :, 1])
    X[:, FOURIER_FEAT::2] = np.sin(arg)
    X[:, FOURIER_FEAT + 1::2] = np.cos(arg)
    return X


# --------------------------------------------------------------------- MLP --

def layout():
    """(offset of W_l, offset of b_l, fan-in) per layer, then W6, b6 offsets and the total."""
    off, layers = 0, []
    for l in range(LAYERS):
        fan_in = INPUTS if l == 0 else WIDTH
        w = off
        off += WIDTH * fan_in
        b = off
        off += WIDTH
        layers.append((w, b, fan_in))
    w6 = off
    off += 2 * WIDTH
    b6 = off
    off += 2
    return layers, w6, b6, off


def unpack(p):
    layers, w6, b6, n = layout()
    p = np.asarray(p, dtype=np.float64)
    assert len(p) == n
    Ws = [p[w:w + WIDTH * fi].reshape(WIDTH, fi) for (w, _, fi) in layers]
    bs = [p[b:b + WIDTH] for (_, b, _) in layers]
    return Ws, bs, p[w6:w6 + 2 * WIDTH].reshape(2, WIDTH), p[b6:b6 + 2]


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, X, emulate=True):
    """Returns (output [B][2], cache). With emulate, operands and stored
    activations are BF16-rounded where the GPU stores BF16."""
    Ws, bs, W6, b6 = unpack(p)
    rnd = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    h = rnd(X)
    cache = {"in": [], "z": [], "Wb": []}
    for l in range(LAYERS):
        Wb = rnd(Ws[l])
        z = h @ Wb.T + (f32(bs[l]) if emulate else bs[l])
        cache["in"].append(h)
        cache["Wb"].append(Wb)
        cache["z"].append(rnd(z))
        h = rnd(z * _sig(z))
    cache["h"] = h
    y = h @ W6.T + b6
    return y, cache


def coefficients(Y, phase_weight=1.0):
    """The plain loss's coefficients: (1, phase_weight), 0 where no phase."""
    Y = np.asarray(Y, dtype=np.float64)
    return np.stack([np.ones(len(Y)), np.where(np.isnan(Y[:, 1]), 0.0, phase_weight)], axis=1)


def backward(p, X, Y, C=None, emulate=True):
    """(gradient in the flat parameter layout, (weighted mse0, weighted mse1))
    of (1/B) sum_b c0 e0^2 + c1 e1^2 for targets Y [B][2] (NaN phase: no
    phase term) and coefficients C [B][2] (None: plain, weight 1)."""
    layers, w6o, b6o, n = layout()
    Ws, bs, W6, b6 = unpack(p)
    rnd = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    y, c = forward(p, X, emulate)
    B = len(X)
    Y = np.asarray(Y, dtype=np.float64)
    C = coefficients(Y) if C is None else np.asarray(C, dtype=np.float64)
    m = ~np.isnan(Y[:, 1]) & (C[:, 1] > 0)
    e0 = y[:, 0] - Y[:, 0]
    e1 = np.where(m, y[:, 1] - np.where(m, Y[:, 1], 0.0), 0.0)
    c1 = np.where(m, C[:, 1], 0.0)
    d = np.stack([2 * C[:, 0] * e0 / B, 2 * c1 * e1 / B], axis=1)
    g = np.zeros(n)
    h5 = c["h"]
    g[w6o:w6o + 2 * WIDTH] = (d.T @ h5).ravel()
    g[b6o:b6o + 2] = d.sum(axis=0)
    dh = d @ W6
    for l in range(LAYERS - 1, -1, -1):
        z = c["z"][l]
        s = _sig(z)
        dz = rnd(dh * (s * (1 + z * (1 - s))))
        w, b, fi = layers[l]
        g[w:w + WIDTH * fi] = (dz.T @ c["in"][l]).ravel()
        g[b:b + WIDTH] = dz.sum(axis=0)
        dh = dz @ c["Wb"][l]
    mse0 = float(np.sum(C[:, 0] * e0 ** 2) / max(C[:, 0].sum(), 1e-300))
    mse1 = float(np.sum(c1 * e1 ** 2) / max(c1.sum(), 1e-300))
    return g, (mse0, mse1)


def loss(p, X, Y, C=None):
    """The training loss (1/B) sum c0 e0^2 + c1 e1^2 in FP64 without rounding."""
    y, _ = forward(p, X, emulate=False)
    Y = np.asarray(Y, dtype=np.float64)
    C = coefficients(Y) if C is None else np.asarray(C, dtype=np.float64)
    m = ~np.isnan(Y[:, 1]) & (C[:, 1] > 0)
    e0 = y[:, 0] - Y[:, 0]
    e1 = np.where(m, y[:, 1] - np.where(m, Y[:, 1], 0.0), 0.0)
    return float(np.mean(C[:, 0] * e0 ** 2 + np.where(m, C[:, 1], 0.0) * e1 ** 2))


def loss_coefficients(labels_t0, labels_t1, lmax, f, r, mean_std, phase_weight=1.0, weight_floor=1e-4,
                      phase_cap=1e4):
    """The complex loss's coefficients (k_batch, loss mode 1) for cells with
    labels (t0, t1), log max_f |G| at their range, frequency and range."""
    s0, s1 = mean_std[1], mean_std[3]
    w = np.maximum(np.exp(2 * (np.asarray(labels_t0) - lmax)), weight_floor)
    wr = 2 * math.pi * np.asarray(f) * np.asarray(r) * (s1 / s0)
    c1 = np.where(np.isnan(labels_t1), 0.0, phase_weight * w * np.minimum(wr * wr, phase_cap))
    return np.stack([w, c1], axis=1)


def adam_step(p, m, v, g, t, lr, beta1=0.9, beta2=0.999, eps=1e-8, wd=0.0):
    """AdamW (Loshchilov & Hutter 2019), as k_adam applies it."""
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** t)
    vh = v / (1 - beta2 ** t)
    return p - lr * (mh / (np.sqrt(vh) + eps) + wd * p), m, v
