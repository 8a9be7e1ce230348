"""Host side of the Sobol workload: the estimators against Ishigami's exact
indices (the reference's self test, py/analysis/sobol.py:127-158), the GRF and
geophone restatements against their analytic properties, and the trace
synthesis and metrics on closed-form cases. No GPU."""
import math

import numpy as np
import pytest


@pytest.fixture(scope="module")
def S(gfk):
    return gfk.sobol


def ishigami(x, a=7.0, b=0.1):
    return np.sin(x[:, 0]) + a * np.sin(x[:, 1]) ** 2 + b * x[:, 2] ** 4 * np.sin(x[:, 0])


def ishigami_exact(a=7.0, b=0.1):
    v1 = 0.5 * (1 + b * np.pi ** 4 / 5) ** 2
    v2 = a ** 2 / 8
    v13 = 8 * b ** 2 * np.pi ** 8 / 225
    var = v1 + v2 + v13
    return np.array([v1, v2, 0.0]) / var, np.array([v1 + v13, v2, v13]) / var


def test_estimators_recover_ishigami(S):
    n, k = 1 << 14, 3
    x = S.saltelli(n, k, seed=1) * (2 * np.pi) - np.pi
    y = ishigami(x)
    s1, st = S.indices(y, n, k)
    xs1, xst = ishigami_exact()
    assert abs(s1[2]) <= 0.02 and abs(st[2] - xst[2]) <= 0.02
    assert max(np.max(np.abs(s1 - xs1)), np.max(np.abs(st - xst))) <= 0.02
    (lo1, hi1), (lo_t, hi_t) = S.bootstrap(y, n, k, draws=100, seed=1)
    assert (lo1 <= s1 + 1e-12).all() and (s1 <= hi1 + 1e-12).all()


def test_design_blocks(S):
    n, k = 64, 8
    u = S.saltelli(n, k, seed=0)
    assert u.shape == (n * (k + 2), k)
    a, b = u[:n], u[n:2 * n]
    for i in range(k):
        ab = u[(i + 2) * n:(i + 3) * n]
        assert np.array_equal(np.delete(ab, i, axis=1), np.delete(a, i, axis=1))
        assert np.array_equal(ab[:, i], b[:, i])
    p = S.unit_to_params(u)
    for j, (_, lo, hi, _) in enumerate(S.PARAMS):
        assert (p[:, j] >= lo - 1e-9).all() and (p[:, j] <= hi + 1e-9).all()
    st = S.soil_of(p[0])
    st.validate()


def test_stance_profile(S):
    s = S.Stance()
    tau = np.linspace(0, 1, 20001)
    prof = s.profile(tau)
    assert prof[0] == 0 and prof[-1] == 0
    assert s.profile(np.array([-0.1, 1.5])).tolist() == [0.0, 0.0]
    # the heel-strike transient crests at its rise time with its stated height
    tr_only = S.Stance(first_peak=1e-9, second_peak=1e-9, valley=1e-9 / 2)
    t = np.linspace(0, 0.1, 100001)
    tr = tr_only.profile(t / s.duration)
    i = int(np.argmax(tr))
    assert abs(t[i] - s.transient_rise) < 2e-4
    assert abs(tr[i] - s.transient_peak) < 2e-3
    # the smooth curve reaches its peaks and valley (grf.go:280-300)
    smooth = S.Stance(transient_peak=1e-12)
    assert abs(smooth.profile(np.array([0.25]))[0] - 1.2) < 0.01
    assert abs(smooth.profile(np.array([0.5]))[0] - 0.75) < 0.01


def test_geophone_limits(S):
    """geophone_test.go:27-60: flat above resonance, sens/(2 zeta) at it,
    rising as f^2 below it (coupling off)."""
    g = S.Geophone(coupling_freq=0.0)
    w0 = 2 * np.pi * g.natural_freq
    h500 = g.response(1j * 2 * np.pi * 500)
    assert abs(abs(h500) - g.sensitivity) / g.sensitivity < 1e-3
    w = 2 * np.pi * 500
    assert abs(np.angle(h500) - math.atan2(2 * g.damping() * w0 * w, w * w - w0 * w0)) < 1e-12
    h0 = g.response(1j * w0)
    assert abs(abs(h0) - g.sensitivity / (2 * g.damping())) / abs(h0) < 1e-12
    lo = g.response(1j * 2 * np.pi * 0.1)
    assert abs(abs(lo) - g.sensitivity * (0.1 / g.natural_freq) ** 2) / abs(lo) < 1e-3


def test_traces_are_linear_and_real(S):
    setup = S.TraceSetup()
    f = setup.freqs()
    wc = 2 * np.pi * f - 1j * setup.omega_imag
    G = (np.exp(-1j * wc * 0.05) / (1j * wc))[None, :] * np.array([[1.0], [2.0]])
    y = S.traces(G, setup)
    assert y.shape == (2, setup.n)
    assert np.allclose(y[1], 2 * y[0], rtol=1e-12, atol=1e-18)


def test_centroid_of_a_tone(S):
    fs, n = 1000.0, 1024
    t = np.arange(n) / fs
    f0 = 125.0  # on the 1024-point grid
    y = np.sin(2 * np.pi * f0 * t)[None, :]
    peak, cen = S.measure(y, fs)
    assert abs(peak[0] - 1) < 1e-3
    assert abs(cen[0] - f0) < 1.0
