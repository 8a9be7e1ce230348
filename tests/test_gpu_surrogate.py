"""GPU checks of the surrogate kernels and the trace metrics against the CPU
oracle (oracle/surrogate_oracle.py) and the host restatement of the Sobol
post-processing."""
import ctypes
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import surrogate_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu


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


def seg_rel(a, b, lo, hi):
    return np.linalg.norm(a[lo:hi] - b[lo:hi]) / max(np.linalg.norm(b[lo:hi]), 1e-300)


def test_gradients_match_oracle(pkg, eng):
    """One forward/backward pass of libgfk's BF16 kernels against the FP64
    oracle with BF16 rounding at the same places (tolerance: FP32
    accumulation order), and against the unrounded FP64 gradient."""
    sur = pkg.surrogate
    net = sur.Net(sur.NetConfig(batch=256, seed=3), eng)
    net.set_scales(1.0, 64.0, 1.0, 500.0, [0.0, 1.0, 0.0, 1.0])
    p = net.params().astype(np.float64)
    rng = np.random.default_rng(4)
    X = rng.uniform(-1, 1, (256, 128)).astype(np.float32)
    Y = rng.normal(size=(256, 2)).astype(np.float32)
    Y[::7, 1] = np.nan
    C = rng.uniform(0.05, 2.0, (256, 2)).astype(np.float32)  # complex-loss-like per-sample weights
    C[::7, 1] = 0.0
    g_gpu, loss = net.probe(X, Y, C)
    g_emu, (m0, m1) = SO.backward(p, X, Y, C, emulate=True)
    g_ref, _ = SO.backward(p, X, Y, C, emulate=False)
    assert abs(loss[0] - m0) <= 2e-3 * m0 and abs(loss[1] - m1) <= 2e-3 * m1
    layers, w6, b6, n = SO.layout()
    segs = [(w, w + SO.WIDTH * fi) for (w, _, fi) in layers] + [(b, b + SO.WIDTH) for (_, b, _) in layers]
    segs += [(w6, w6 + 2 * SO.WIDTH), (b6, b6 + 2)]
    for lo, hi in segs:
        assert seg_rel(g_gpu, g_emu, lo, hi) < 1e-2, (lo, seg_rel(g_gpu, g_emu, lo, hi))
        assert seg_rel(g_gpu, g_ref, lo, hi) < 5e-2, (lo, seg_rel(g_gpu, g_ref, lo, hi))
    net.close()


def test_predict_matches_oracle_forward(pkg, eng):
    """Features, inference GEMMs and the output mapping against the oracle."""
    sur = pkg.surrogate
    net = sur.Net(sur.NetConfig(batch=256, seed=5), eng)
    ms = [-20.0, 2.0, 0.006, 0.002]
    net.set_scales(1.0, 64.0, 500 / 512, 500.0, ms)
    params = sur.draw(3, 11)
    ranges = np.array([1.0, 2.0, 3.5])
    freqs = np.array([500 / 512, 10.0, 30.0, 45.0])
    G = net.predict(params, ranges, freqs)
    assert G.shape == (3, 4, 3)
    p = net.params().astype(np.float64)
    B = net.fourier()
    sc = sur.to_scalars(params)
    tt = sur.travel_times(params)
    for s in range(3):
        rr, ff = np.meshgrid(ranges, freqs)
        X = SO.features(np.repeat(sc[s:s + 1], rr.size, axis=0), np.repeat(tt[s:s + 1], rr.size, axis=0),
                        rr.ravel(), ff.ravel(), (1.0, 64.0, 500 / 512, 500.0), B)
        y, _ = SO.forward(p, X, emulate=True)
        t0 = y[:, 0] * ms[1] + ms[0]
        t1 = y[:, 1] * ms[3] + ms[2]
        want = np.exp(t0) * np.exp(-1j * t1 * 2 * np.pi * ff.ravel() * rr.ravel())
        got = G[s].ravel()
        assert np.allclose(np.log(np.abs(got)), t0, atol=2e-2)
        assert np.abs(got - want).max() / np.abs(want).max() < 5e-2
    net.close()


def test_labels_match_oracle(pkg, eng):
    """Bank -> labels on the device against the oracle's restatement."""
    sur = pkg.surrogate
    grid = sur.LabelGrid(ranges=np.arange(1.0, 33.0), nk=4096)
    params = sur.draw(3, 21)
    ds = sur.Dataset(params, grid, floor_rel=1e-6, engine=eng)
    banks = []

    def each(plan, first, count):
        eng.check(pkg._native.lib().gfk_dataset_fill(ds.p, ctypes.c_void_p(plan.result_device_ptr()), first,
                                                     count))
        g, _ = plan.download()
        banks.append(g.reshape(count, len(grid.freqs), len(grid.ranges)))

    sur.solve_media(params, grid, eng, batch_soils=2, each=each)
    G = np.concatenate(banks)
    for s in range(3):
        want = SO.labels(G[s], grid.ranges, grid.freqs, 1e-6)
        got = ds.labels(s)
        assert np.array_equal(np.isnan(got[..., 1]), np.isnan(want[..., 1]))
        ok = ~np.isnan(want[..., 1])
        assert ok.mean() > 0.3
        assert np.allclose(got[..., 0], want[..., 0], rtol=1e-6, atol=1e-6)
        assert np.allclose(got[..., 1][ok], want[..., 1][ok], rtol=1e-6, atol=0)
    m0, s0, m1, s1, frac = ds.stats()
    assert s0 > 0 and s1 > 0 and 0 < frac <= 1
    ds.close()


def test_trace_metrics_match_host(pkg, eng):
    """gfk_trace_metrics against traces()/measure() on the same spectra."""
    import torch
    sob = pkg.sobol
    setup = sob.TraceSetup()
    rng = np.random.default_rng(6)
    f = setup.freqs()
    G = (rng.normal(size=(40, 512)) + 1j * rng.normal(size=(40, 512))) * 1e-9 * np.exp(-f / 80.0)[None, :]
    peak, cen = sob.measure(sob.traces(G, setup), setup.fs)
    d = torch.from_numpy(np.stack([G.real, G.imag], axis=-1).ravel()).to("cuda:0")
    pk, ce = sob.metrics_device(eng, d.data_ptr(), 512, 40, setup)
    assert np.allclose(pk, peak, rtol=1e-10, atol=0)
    assert np.allclose(ce, cen, rtol=1e-10, atol=0)


def test_sobol_plain_gpu_metrics_equal_host(pkg, eng):
    """The plain Sobol run with device metrics equals the host path."""
    sob = pkg.sobol
    a = sob.run_plain(eng, n=8, seed=2, host_metrics=True)
    b = sob.run_plain(eng, n=8, seed=2)
    assert np.allclose(a.metrics["peak"], b.metrics["peak"], rtol=1e-9)
    assert np.allclose(a.metrics["centroid"], b.metrics["centroid"], rtol=1e-9)


def test_training_reduces_loss_and_beats_mean(pkg, eng):
    """A short training run on a small data set: the loss falls, the fit on
    the training soils is close, and on held-out soils (36 training soils in
    11 dimensions generalise only roughly) it beats the best constant."""
    sur = pkg.surrogate
    grid = sur.LabelGrid(ranges=np.arange(1.0, 17.0), nk=2048)
    params = sur.draw(40, 31)
    ds = sur.Dataset(params, grid, engine=eng).fill(batch_soils=40)
    train, held = sur.split_soils(40, 0.1, 1)
    net = sur.Net(sur.NetConfig(batch=1024, warmup_steps=50, total_steps=600, lr_max=2e-3, seed=9,
                                loss_mode=pkg._native.LOSS_PLAIN), eng)
    net.scales_from(ds)
    loss = net.train(ds, train, 600)
    assert np.isfinite(loss).all()
    assert loss[-50:, 0].mean() < 0.2 * loss[:50, 0].mean()
    # the complex (energy-weighted) loss trains as well
    cnet = sur.Net(sur.NetConfig(batch=1024, warmup_steps=50, total_steps=600, lr_max=2e-3, seed=9), eng)
    cnet.scales_from(ds)
    closs = cnet.train(ds, train, 600)
    assert np.isfinite(closs).all() and closs[-50:].sum(axis=1).mean() < 0.2 * closs[:50].sum(axis=1).mean()
    cnet.close()
    # the constant predictor (t = mean) has RMS s0 on log-amplitude
    m0, s0, _, _, _ = ds.stats()
    assert net.evaluate(ds, train)["rms_log_amp"] / s0 < 0.3
    assert net.evaluate(ds, held)["rms_log_amp"] / s0 < 0.9
    ds.close()
    net.close()


def test_surrogate_sobol_plumbing(pkg, eng):
    """End to end with an untrained two-member ensemble. Soil gate: every
    soil the ensemble disagrees on is re-solved and those soils' metrics
    equal the plain run's. Row gate: with a negative threshold every row is
    re-solved in place and all metrics equal the plain run's; with an
    unreachable one (and the amplitude rule off) nothing is, and no solver
    row runs."""
    sob, sur = pkg.sobol, pkg.surrogate
    nets = [sur.Net(sur.NetConfig(batch=256, seed=s), eng) for s in (1, 2)]
    for n_ in nets:
        n_.set_scales(1.0, 64.0, 500 / 512, 500.0, [-22.0, 2.0, 0.006, 0.002])
    plain = sob.run_plain(eng, n=8, seed=2)
    res = sob.run_surrogate(eng, nets, n=8, seed=2, threshold=0.01, gate="soil")
    fb = np.nonzero(res.metrics["spread"] > 0.01)[0]
    assert res.seconds["fallback_soils"] == len(fb) and len(fb) > 0
    assert np.allclose(res.metrics["peak"][fb], plain.metrics["peak"][fb], rtol=1e-12)
    rows = sob.run_surrogate(eng, nets, n=8, seed=2, threshold=-1.0, gate="rows")
    assert rows.seconds["fallback_fraction"] == 1.0
    assert np.allclose(rows.metrics["peak"], plain.metrics["peak"], rtol=1e-12)
    assert np.allclose(rows.metrics["centroid"], plain.metrics["centroid"], rtol=1e-12)
    none = sob.run_surrogate(eng, nets, n=8, seed=2, threshold=1e30, gate="rows", amp_threshold=0.0)
    assert none.seconds["fallback_rows"] == 0 and np.isfinite(none.metrics["peak"]).all()
    for n_ in nets:
        n_.close()


def test_ensemble_gate_and_scatter_match_numpy(pkg, eng):
    """gfk_ensemble_gate (mean, trace-weighted spread flags, per-soil worst
    ratio) and gfk_scatter_rows against numpy on random member spectra."""
    import torch
    sob = pkg.sobol
    setup = sob.TraceSetup()
    S = sob.shaping(setup)
    rng = np.random.default_rng(9)
    E, ns, nb = 3, 7, 512
    G = (rng.normal(size=(E, ns, nb)) + 1j * rng.normal(size=(E, ns, nb))) * 1e-9
    G[1:] = G[0] + 0.05 * (G[1:] - G[0])  # members close to each other
    dev = [torch.from_numpy(np.stack([g.real, g.imag], axis=-1).ravel()).to("cuda:0") for g in G]
    mean = torch.zeros(ns * nb * 2, dtype=torch.float64, device="cuda:0")
    ptrs = (ctypes.c_void_p * E)(*[d.data_ptr() for d in dev])
    Sh = np.ascontiguousarray(np.stack([S.real, S.imag], axis=1).ravel())
    flags = np.zeros((ns, nb), dtype=np.uint8)
    spread = np.zeros(ns)
    thr = 0.02
    m = G.mean(axis=0)
    d = np.abs(G - m[None]).max(axis=0) * np.abs(S[1:])[None]
    peak = np.abs(m * S[1:][None]).max(axis=1, keepdims=True)
    ratio = d / peak
    for amp in (0.0, 0.05):
        eng.check(pkg._native.lib().gfk_ensemble_gate(
            eng.ctx, ptrs, E, nb, ns, nb, Sh.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), thr, amp,
            ctypes.c_void_p(mean.data_ptr()), flags.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            spread.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        got = mean.cpu().numpy().reshape(ns, nb, 2)
        assert np.allclose(got[..., 0] + 1j * got[..., 1], m, rtol=1e-14, atol=1e-30)
        want = ratio > thr
        if amp > 0:
            loud = np.abs(m * S[1:][None]) > amp * peak
            assert (loud & ~want).any()  # the amplitude rule adds rows
            want |= loud
        assert np.array_equal(flags.astype(bool), want)
        assert np.allclose(spread, ratio.max(axis=1), rtol=1e-12)
    # scatter three rows back from a packed source
    src = torch.from_numpy(np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])).to("cuda:0")
    idx = np.array([5, 700, 3583], dtype=np.int64)
    eng.check(pkg._native.lib().gfk_scatter_rows(eng.ctx, ctypes.c_void_p(src.data_ptr()), 1,
                                                 idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), 3,
                                                 ctypes.c_void_p(mean.data_ptr())))
    out = mean.cpu().numpy().reshape(-1, 2)
    assert np.array_equal(out[idx], [[1, 2], [3, 4], [5, 6]])


def test_trained_surrogate_gain_over_plain_solve(pkg, eng):
    """What the trained network gains over the method without it. Three
    members, trained for 20,000 steps on FP64 f-k labels of 16,384 soils from
    the Sobol soils' box (sensor range only), answer a Saltelli N = 256 sweep
    (2560 soils x 512 bins at 10 m); the row gate sends to the plain f-k solve
    the rows where the members disagree by more than 1% of the soil's
    trace-spectrum peak or whose predicted |G S| exceeds 0.1% of it. Against
    the all-plain run, which solves every row: about a quarter of the rows are
    never solved, the Sobol indices stay within 0.02 and the peak metric within
    1% at the 90th percentile. Untrained members under the same gate leave far
    fewer rows to the network — the training is what earns the saving."""
    sob, sur = pkg.sobol, pkg.surrogate
    rng = np.random.default_rng(20240611)
    p11 = sur.from_sobol(sob.unit_to_params(rng.random((16384, 8))))
    ds = sur.Dataset(p11, sur.LabelGrid(), floor_rel=1e-6, engine=eng).fill(batch_soils=8192)
    train, _ = sur.split_soils(len(p11), 0.05, 0)
    cfg = sur.NetConfig(total_steps=20000, lr_max=1e-3, warmup_steps=200)
    nets = sur.train_ensemble(ds, train, members=3, steps=20000, config=cfg, engine=eng, ranges=(9, 10))
    untrained = [sur.Net(sur.NetConfig(seed=s), eng) for s in (1, 7920, 15839)]
    for n_ in untrained:
        n_.scales_from(ds)
    plain = sob.run_plain(eng, n=256, seed=0)
    got = sob.run_surrogate(eng, nets, n=256, seed=0, threshold=0.01, gate="rows", amp_threshold=0.001)
    base = sob.run_surrogate(eng, untrained, n=256, seed=0, threshold=0.01, gate="rows", amp_threshold=0.001)
    frac = got.seconds["fallback_fraction"]
    assert frac <= 0.80, frac
    assert base.seconds["fallback_fraction"] >= frac + 0.1, (base.seconds["fallback_fraction"], frac)
    worst = max(abs(getattr(got, kind)[out][q] - getattr(plain, kind)[out][q])
                for kind in ("s1", "st") for out in ("peak", "centroid") for q in getattr(got, kind)[out])
    assert worst <= 0.02, worst
    assert np.percentile(np.abs(got.metrics["peak"] / plain.metrics["peak"] - 1), 90) <= 0.01
    for n_ in nets + untrained:
        n_.close()
    ds.close()
