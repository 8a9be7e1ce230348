"""The finite-difference validator on the GPU (gfk_fdtd_run): parity with the
CPU restatement (oracle/fdtd_oracle.py), the reference's V5 comparison
against the wavenumber solve (internal/fdtd/v5_test.go: Richardson-
extrapolated peak ratio and residual within 2% homogeneous, 3% layered),
and its stability, elastic-limit and argument checks."""
import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import fdtd_oracle as FO  # noqa: E402

pytestmark = pytest.mark.gpu

LAYERED = [(2.0, 350.0, 140.0, 1600.0), (0.0, 800.0, 320.0, 2000.0)]
LOAM = [(0.0, 500.0, 200.0, 1700.0)]


@pytest.fixture(scope="module")
def pkg():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    return g.load_package()


@pytest.fixture(scope="module")
def eng(pkg):
    e = pkg.Engine(0)
    yield e
    e.close()


def stack(pkg, layers):
    return pkg.Stack([pkg.Layer(h, vp, vs, rho, 0, 0) for (h, vp, vs, rho) in layers])


@pytest.mark.parametrize("lossy", [False, True])
def test_matches_oracle(pkg, eng, lossy):
    sls = pkg.SLS.fit(25, 30) if lossy else None
    md = pkg.fdtd.Model(stack(pkg, LAYERED), relax=sls, ref_freq=30, max_range=8, depth=6, spacing=0.2,
                        dominant_freq=25)
    dt, nr, nz = md.grid()
    steps = 400
    force = pkg.fdtd.ricker(1000, 25, dt, steps)
    res = pkg.fdtd.run(pkg.fdtd.Shot(md, force, [0.0, 3.0, 6.0], steps), engine=eng)
    sim = FO.Sim(LAYERED, FO.SLS.fit(25, 30) if lossy else None, 30, 8, 6, 0.2, dominant_freq=25)
    assert (sim.nr, sim.nz) == res.cells and sim.dt == dt
    want = FO.run(sim, FO.ricker(1000, 25, dt, steps), [0.0, 3.0, 6.0], steps)
    got = np.array([t.vertical for t in res.traces])
    assert [t.range for t in res.traces] == [0.0, 3.0, 6.0]
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-9 * scale, np.abs(got - want).max() / scale


def synthesise(pkg, eng, layers, sls, ranges, peak, dt, t0, n):
    """v5_test.go synthesise: the f-k response through the Ricker wavelet, as velocity."""
    nfft = 1 << int(math.ceil(math.log2(n)))
    fs = 1 / dt
    df = fs / nfft
    nb = int(90.0 / df)
    freqs = np.arange(1, nb + 1) * df
    med = pkg.Medium(stack(pkg, layers), ref_freq=30, relax=sls, formulation=pkg.DUNKIN, engine=eng)
    u, st = med.bank_spectra(ranges, freqs)
    assert (st == 0).all()
    w = pkg.fdtd.ricker_spectrum(peak, 25.0, freqs)
    jw = 2j * np.pi * freqs
    shift = np.exp(-2j * np.pi * freqs * t0)
    coeff = np.zeros((len(ranges), nfft // 2 + 1), dtype=np.complex128)
    coeff[:, 1:nb + 1] = (u * (w * jw * shift * fs)[:, None]).T
    return np.fft.irfft(coeff, nfft, axis=1)[:, :n]


def compare(got, want, dt):
    pa, pb = np.abs(got).max(), np.abs(want).max()
    n = len(want)
    max_lag = n // 8
    full = np.correlate(got, want, "full")  # full[k + n - 1] = sum_i got[i] want[i - k]
    lags = np.arange(-max_lag, max_lag + 1)
    c = full[lags + n - 1]
    b = int(np.argmax(c))
    best_at = lags[b]
    l, r, best = full[best_at - 1 + n - 1], full[best_at + 1 + n - 1], c[b]
    lag = (best_at - 0.5 * (r - l) / (l - 2 * best + r)) * dt if l - 2 * best + r != 0 else best_at * dt
    shifted = np.zeros(n)
    idx = np.arange(n) - best_at
    ok = (idx >= 0) & (idx < n)
    shifted[ok] = want[idx[ok]]
    residual = math.sqrt(((got - shifted) ** 2).sum() / (shifted ** 2).sum())
    return pa / pb, lag, residual


def shoot(pkg, eng, layers, spacing, rmax, depth, ranges, seconds):
    sls = pkg.SLS.fit(25.0, 30.0)
    md = pkg.fdtd.Model(stack(pkg, layers), relax=sls, ref_freq=30, max_range=rmax, depth=depth, spacing=spacing,
                        dominant_freq=25)
    dt, _, _ = md.grid()
    steps = int(seconds / dt)
    res = pkg.fdtd.run(pkg.fdtd.Shot(md, pkg.fdtd.ricker(1000, 25.0, dt, steps), ranges, steps), engine=eng)
    snapped = [t.range for t in res.traces]
    ref = synthesise(pkg, eng, layers, sls, snapped, 1000, dt, res.t0, steps)
    return [compare(t.vertical, ref[i], dt) for i, t in enumerate(res.traces)]


@pytest.mark.parametrize("case", ["homogeneous", "layered"])
def test_v5_against_wavenumber_solve(pkg, eng, case):
    if case == "homogeneous":
        args, tol = (LOAM, 26, 18, [4.0, 8.0, 16.0]), 0.02
        coarse = shoot(pkg, eng, args[0], 0.111, *args[1:], 0.3)
        fine = shoot(pkg, eng, args[0], 0.0555, *args[1:], 0.3)
    else:
        args, tol = (LAYERED, 16, 10, [3.0, 6.0, 10.0]), 0.03
        coarse = shoot(pkg, eng, args[0], 0.1, *args[1:], 0.3)
        fine = shoot(pkg, eng, args[0], 0.05, *args[1:], 0.3)
    for c, f in zip(coarse, fine):
        peak = 2 * f[0] - c[0]
        residual = 2 * f[2] - c[2]
        assert abs(peak - 1) <= tol, (case, c, f)
        assert abs(residual) <= tol, (case, c, f)


def test_stability_limit(pkg, eng):
    md = pkg.fdtd.Model(stack(pkg, LOAM), max_range=6, depth=5, spacing=0.2)
    dt, _, _ = md.grid()
    force = pkg.fdtd.ricker(1000, 25, dt, 600)
    res = pkg.fdtd.run(pkg.fdtd.Shot(md, force, [2.0], 600), engine=eng)
    assert math.isfinite(res.peak) and res.peak > 0
    md.courant = 1.4
    dt2, _, _ = md.grid()
    with pytest.raises(pkg.FkError) as e:
        pkg.fdtd.run(pkg.fdtd.Shot(md, pkg.fdtd.ricker(1000, 25, dt2, 3000), [2.0], 3000), engine=eng)
    assert e.value.status == pkg._native.ENONFINITE and "diverged" in str(e.value)


def test_zero_relaxation_is_elastic(pkg, eng):
    base = dict(max_range=6, depth=5, spacing=0.2, dominant_freq=25)
    el = pkg.fdtd.Model(stack(pkg, LAYERED), **base)
    zr = pkg.fdtd.Model(stack(pkg, LAYERED), relax=pkg.SLS(0.001, 0.001), **base)
    dt, _, _ = el.grid()
    f = pkg.fdtd.ricker(1000, 25, dt, 300)
    a = pkg.fdtd.run(pkg.fdtd.Shot(el, f, [1.0, 3.0], 300), engine=eng)
    b = pkg.fdtd.run(pkg.fdtd.Shot(zr, f, [1.0, 3.0], 300), engine=eng)
    for x, y in zip(a.traces, b.traces):
        assert np.array_equal(x.vertical, y.vertical)


def test_rejects_bad_shots(pkg, eng):
    md = pkg.fdtd.Model(stack(pkg, LOAM), max_range=6, depth=5, spacing=0.2)
    f = np.zeros(10)
    with pytest.raises(pkg.FkError):
        pkg.fdtd.run(pkg.fdtd.Shot(md, f, [7.0], 10), engine=eng)
    with pytest.raises(pkg.FkError):
        pkg.fdtd.run(pkg.fdtd.Shot(md, f, [1.0], 0), engine=eng)
    bad = pkg.fdtd.Model(stack(pkg, LOAM), max_range=6, depth=5, spacing=-1)
    with pytest.raises(pkg.FkError):
        pkg.fdtd.run(pkg.fdtd.Shot(bad, f, [1.0], 10), engine=eng)
