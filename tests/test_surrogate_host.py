"""Host-side checks of the surrogate: the oracle's own gradient against finite
differences, BF16 rounding, the label unwrapping on phases too fast for a
plain range unwrap, the soil family's embedding of the Sobol soils, and the
feature layout. No GPU."""
import math
import sys
import pathlib

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import surrogate_oracle as SO  # noqa: E402


@pytest.fixture(scope="module")
def pkg():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    return g.load_package()


def small_params(seed=0, scale=1.0):
    layers, w6, b6, n = SO.layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n)
    for (w, b, fi) in layers:
        a = scale / math.sqrt(fi)
        p[w:w + SO.WIDTH * fi] = rng.uniform(-a, a, SO.WIDTH * fi)
        p[b:b + SO.WIDTH] = rng.uniform(-a, a, SO.WIDTH)
    a = 1 / math.sqrt(SO.WIDTH)
    p[w6:b6 + 2] = rng.uniform(-a, a, 2 * SO.WIDTH + 2)
    return p


def test_oracle_gradient_matches_finite_differences():
    p = small_params(1)
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (6, SO.INPUTS))
    Y = rng.normal(size=(6, 2))
    Y[2, 1] = np.nan  # a row without a phase term
    C = rng.uniform(0.1, 3.0, (6, 2))  # per-sample loss coefficients
    g, _ = SO.backward(p, X, Y, C, emulate=False)
    layers, w6, b6, n = SO.layout()
    picks = [layers[0][0] + 5, layers[0][1] + 3, layers[2][0] + 1000, layers[4][0] + 77, layers[4][1] + 9,
             w6 + 3, w6 + SO.WIDTH + 11, b6, b6 + 1]
    for i in picks:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (SO.loss(pp, X, Y, C) - SO.loss(pm, X, Y, C)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_bf16_rounding():
    vals = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -2.5, 3.140625, 1e-3])
    got = SO.bf16(vals)
    # ties go to even: 1 + 2^-8 -> 1, 1 + 3 2^-8 -> 1 + 2^-6
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1 + 2 ** -6
    assert got[3] == -2.5 and got[4] == 3.140625
    assert abs(got[5] - 1e-3) / 1e-3 < 2 ** -8


def test_labels_unwrap_fast_phase_and_floor():
    """A dispersive wave whose phase advances up to ~40 rad per 1 m range
    step (far past a half cycle): the prediction-guided unwrap recovers the
    exact phase slowness; cells past the amplitude floor carry no phase."""
    ranges = np.arange(1.0, 65.0)
    freqs = np.arange(1, 513) * 1000 / 1024
    c = 80.0 + 0.2 * freqs                     # phase velocity per frequency
    k = 2 * np.pi * freqs / c
    amp = np.exp(-0.0004 * freqs[:, None] * ranges[None, :]) / ranges[None, :]
    G = amp * np.exp(-1j * k[:, None] * ranges[None, :])
    L = SO.labels(G, ranges, freqs, floor_rel=1e-6)
    floor = amp.max() * 1e-6
    ok = ~np.isnan(L[..., 1])
    want = np.broadcast_to(1.0 / c[None, :], ok.shape)
    assert ok.sum() > 0.8 * ok.size
    assert np.allclose(L[..., 1][ok], want[ok], rtol=1e-12, atol=0)
    # the cells without a phase label are exactly those behind a sub-floor cell
    below = (amp.T <= floor)
    reach = np.zeros_like(below)
    for j in range(len(freqs)):
        reach[:, j] = np.maximum.accumulate(below[:, j] | (below[:, j - 1] if j else False))
    assert (~ok == np.maximum.accumulate(reach, axis=1)).mean() > 0.99
    assert np.allclose(L[..., 0], np.log(np.maximum(amp.T, floor)), rtol=0, atol=1e-12)


def test_labels_plain_unwrap_would_alias():
    """The same wave through interp.go's plain fold (about zero) loses cycles."""
    ranges = np.arange(1.0, 9.0)
    f = 400.0
    k = 2 * np.pi * f / 90.0
    w = np.angle(np.exp(-1j * k * ranges))
    d = np.diff(w)
    d -= 2 * np.pi * np.round(d / (2 * np.pi))
    plain = w[0] + np.concatenate([[0], np.cumsum(d)])
    assert np.abs(plain - (-k * ranges)).max() > 1.0


def test_sobol_soils_are_family_members(pkg):
    sob, sur = pkg.sobol, pkg.surrogate
    p8 = sob.unit_to_params(np.random.default_rng(3).random((5, 8)))
    p11 = sur.from_sobol(p8)
    for a, b in zip(p8, p11):
        s2, s3 = sob.soil_of(a), sur.soil_of(b)
        assert len(s3) == len(s2) + 1
        for la, lb in zip(list(s2)[:2], list(s3)[:2]):
            assert (la.thickness, la.vp, la.vs, la.density, la.qs, la.qp) == \
                   (lb.thickness, lb.vp, lb.vs, lb.density, lb.qs, lb.qp)
        hs2, l3, hs3 = list(s2)[2], list(s3)[2], list(s3)[3]
        for lb in (l3, hs3):
            assert (lb.vp, lb.vs, lb.density, lb.qs, lb.qp) == (hs2.vp, hs2.vs, hs2.density, hs2.qs, hs2.qp)


def test_sobol_embedding_gives_same_response(pkg):
    """A third layer identical to the half-space changes nothing (CPU oracle)."""
    import oracle as O
    sob, sur = pkg.sobol, pkg.surrogate
    p8 = sob.unit_to_params(np.random.default_rng(4).random((2, 8)))
    p11 = sur.from_sobol(p8)
    for a, b in zip(p8, p11):
        m2 = O.OracleMedium([(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in sob.soil_of(a)])
        m3 = O.OracleMedium([(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in sur.soil_of(b)])
        f = np.array([5.0, 60.0, 250.0])
        g2 = O.bank_spectra(m2, [10.0], f, samples=2048, kmax=98.17, formulation=O.DUNKIN, omega_imag=3.07)
        g3 = O.bank_spectra(m3, [10.0], f, samples=2048, kmax=98.17, formulation=O.DUNKIN, omega_imag=3.07)
        g2 = g2[0] if isinstance(g2, tuple) else g2
        g3 = g3[0] if isinstance(g3, tuple) else g3
        assert np.allclose(g2, g3, rtol=1e-9, atol=0)


def test_scalars_and_features(pkg):
    sur = pkg.surrogate
    lo = np.array([[p[1] for p in sur.PARAMS]])
    hi = np.array([[p[2] for p in sur.PARAMS]])
    assert np.allclose(sur.to_scalars(lo), -1) and np.allclose(sur.to_scalars(hi), 1)
    B = np.random.default_rng(5).normal(0, 8, (SO.FOURIER, 2))
    T = sur.travel_times(lo)
    X = SO.features(sur.to_scalars(lo), T, np.array([1.0]), np.array([500.0]), (1.0, 64.0, 500 / 512, 500.0), B)
    assert X.shape == (1, 128) and SO.FOURIER == 47
    assert X[0, 11] == -1 and X[0, 12] == 1 and X[0, 13] == -1 and X[0, 14] == 1 and X[0, 15] == 0
    ft = 500.0 * T[0]
    assert np.allclose(X[0, 16:28:2], np.sin(2 * np.pi * ft)) and np.allclose(X[0, 17:28:2], np.cos(2 * np.pi * ft))
    assert np.allclose(X[0, 28:34], np.clip((np.log(ft) + 2) / 3, -2, 2))
    assert np.allclose(X[0, 34::2], np.sin(2 * np.pi * B[:, 1]))
    assert np.allclose(X[0, 35::2], np.cos(2 * np.pi * B[:, 1]))
    # the first soil's S travel time through layer 1 is h1 / vs1
    assert np.isclose(T[0, 0], lo[0, 3] / lo[0, 0]) and np.isclose(T[0, 5], lo[0, 9] / (2 * lo[0, 8]))


def test_draw_and_split(pkg):
    sur = pkg.surrogate
    p = sur.draw(1000, 7)
    assert p.shape == (1000, 11)
    for j, (_, lo, hi, _) in enumerate(sur.PARAMS):
        assert lo <= p[:, j].min() and p[:, j].max() <= hi
    tr, ho = sur.split_soils(1000, 0.05, 0)
    assert len(ho) == 50 and len(np.intersect1d(tr, ho)) == 0 and len(tr) + len(ho) == 1000


def test_adam_oracle_first_step():
    """The first AdamW step moves every parameter by lr in the sign of its gradient."""
    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -1e-3, 2.0])
    q, m, v = SO.adam_step(p, np.zeros(3), np.zeros(3), g, 1, 1e-2)
    assert np.allclose(q, p - 1e-2 * np.sign(g), atol=1e-9)


def test_layer_tables_equal_stacks(pkg):
    """The vectorised layer tables the batch solves use equal the per-soil stacks."""
    sob, sur = pkg.sobol, pkg.surrogate
    p8 = sob.unit_to_params(np.random.default_rng(11).random((7, 8)))
    lay, cnt = sob.layer_table(p8)
    want = np.array([[l.thickness, l.vp, l.vs, l.density, l.qs, l.qp] for p in p8 for l in sob.soil_of(p)])
    assert np.array_equal(lay, want) and (cnt == 3).all()
    p11 = sur.draw(7, 12)
    lay, cnt = sur.layer_table(p11)
    want = np.array([[l.thickness, l.vp, l.vs, l.density, l.qs, l.qp] for p in p11 for l in sur.soil_of(p)])
    assert np.array_equal(lay, want) and (cnt == 4).all()
