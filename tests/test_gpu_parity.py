"""GPU parity: libgfk through its C ABI against the CPU oracle and the
high-precision golden values. Tolerances: rel-L2 <= 1e-9 for the FP64 Dunkin
path (same algorithm, different rounding), <= 1e-6 for the reference-direct
path (the direct eigenbasis loses digits at large k/k_body in both
implementations, differently)."""
import ctypes
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN, as_tuples, rel_l2

import closed_forms as CF

pytestmark = pytest.mark.gpu
MP = json.loads((GOLDEN / "surface_response_mp.json").read_text())


def medium_of(gfk, tuples, **kw):
    return gfk.Medium(gfk.Stack(gfk.Layer(*t) for t in tuples), **kw)


@pytest.mark.parametrize("form", [0, 1], ids=["reference_direct", "dunkin"])
def test_surface_response_against_high_precision(gfk, engine, form):
    worst = 0.0
    groups = {}
    for c in MP["cases"]:
        st = MP["media"][c["medium"]]
        if form == 0 and (c["qp_mode"] != "reference" or c["kh"] > 16):
            continue
        if form == 1 and c["qp_mode"] == "reference":
            st = [tuple(l[:5]) + (0.0,) for l in st]
        groups.setdefault((c["medium"], c["qp_mode"], c["omega_imag"]), (st, []))[1].append(c)
    n = 0
    for (name, qpm, wi), (st, cases) in groups.items():
        m = medium_of(gfk, st, formulation=form, omega_imag=wi, engine=engine)
        k = np.array([c["k"] for c in cases])
        f = np.array([c["f"] for c in cases])
        got = m.surface_response(k, f)
        want = np.array([complex(*c["u"]) for c in cases])
        worst = max(worst, float(np.max(np.abs(got - want) / np.abs(want))))
        n += len(cases)
    assert n > 40
    assert worst < (1e-6 if form == 0 else 1e-12), worst


def test_surface_response_matches_oracle_pointwise(gfk, engine, oracle):
    wl = gfk.workloads.graded_soil()
    st = as_tuples(wl.stack)
    rng = np.random.default_rng(7)
    k = rng.uniform(0.005, 80.0, 400)
    f = rng.uniform(0.2, 500.0, 400)
    m = medium_of(gfk, st, formulation=1, omega_imag=wl.omega_imag, engine=engine)
    got = m.surface_response(k, f)
    want = np.array([oracle.surface_response(st, ki, fi, 1, wl.omega_imag) for ki, fi in zip(k, f)])
    assert np.max(np.abs(got - want) / np.abs(want)) < 1e-11


def test_thick_layer_start_matches_full_propagation(gfk, engine, oracle):
    """The solve starts at the shallowest layer thick enough to isolate the
    layers beneath it; the oracle propagates every layer. Uneven seeded soils
    (2-12 layers, 0.2-5 m) put the start at every depth across the k range."""
    soils, _, _, kmax = gfk.workloads.batched_soils(count=8, seed=3)
    rng = np.random.default_rng(11)
    worst = 0.0
    for st, _ in soils:
        tup = as_tuples(st)
        k = rng.uniform(0.01, kmax, 150)
        f = rng.uniform(1.0, 500.0, 150)
        m = medium_of(gfk, tup, formulation=1, omega_imag=1.5, engine=engine)
        got = m.surface_response(k, f)
        want = np.array([oracle.surface_response(tup, ki, fi, 1, 1.5) for ki, fi in zip(k, f)])
        worst = max(worst, float(np.max(np.abs(got - want) / np.abs(want))))
    assert worst < 1e-11, worst


def test_reference_mode_per_frequency_grid(gfk, engine, oracle):
    """VerticalDisplacementMulti with the reference's own GridFor grids (the
    ragged path), soft_over_stiff and loam, against the oracle."""
    for st in ([(3.0, 400.0, 160.0, 1600.0, 0.0, 0.0), (0.0, 900.0, 400.0, 2000.0, 0.0, 0.0)],
               CF.uniform(CF.LOAM)):
        m = medium_of(gfk, st, engine=engine)
        ranges = np.array([2.0, 5.0, 10.0, 20.0])
        freqs = np.array([5.0, 20.0, 60.0, 110.0])
        got, status = m.bank_spectra(ranges, freqs)
        assert (status == 0).all()
        want, ost = oracle.bank_spectra(st, ranges, freqs)
        assert (ost == 0).all()
        assert rel_l2(got, want) < 1e-6
        single = m.vertical_displacement_multi(ranges, 20.0)
        assert np.allclose(single, got[1], rtol=1e-12, atol=0)


def test_single_range_vertical_displacement(gfk, engine, oracle):
    h = CF.LOAM
    m = gfk.Medium(gfk.uniform(*h), engine=engine)
    lam = CF.rayleigh_velocity(h) / 30.0
    for mult in (1.5, 3.0):
        got = m.vertical_displacement(mult * lam, 30.0)
        want = oracle.vertical_displacement(CF.uniform(h), mult * lam, 30.0)
        assert abs(got - want) / abs(want) < 1e-8


def test_single_soil_full_bank_against_oracle(gfk, engine, oracle):
    """The whole 512 x 64 bank of the single-soil workload, Dunkin, shared grid."""
    wl = gfk.workloads.single_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine)
    got, status = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    assert (status == 0).all()
    want, ost = oracle.bank_spectra(as_tuples(wl.stack), wl.ranges, wl.freqs, samples=wl.samples, kmax=wl.kmax,
                                    formulation=oracle.DUNKIN, omega_imag=wl.omega_imag)
    assert (ost == 0).all()
    assert rel_l2(got, want) < 1e-9


def test_single_soil_reference_parity_band(gfk, engine, oracle):
    """The reference's semantics (real frequency, Qp = 2.25 Qs, guard) on the
    single-soil grid: bins the reference answers match the oracle's
    restatement, the rest are refused with EGUARD as fk.go:251-266 refuses."""
    wl = gfk.workloads.single_soil()
    st = [(l.thickness, l.vp, l.vs, l.density, l.qs, 0.0) for l in wl.stack]
    m = medium_of(gfk, st, engine=engine)
    got, status = m.bank_spectra(wl.ranges, wl.freqs, wl.integration(), raise_on_error=False)
    answered = status == 0
    band = wl.freqs[answered]
    assert band.max() < 170 and band.max() > 160   # 16*0.87*150/(2 pi 2) = 166 Hz
    assert (status[~answered] == gfk._native.EGUARD).all()
    sample = np.nonzero(answered)[0][::6]
    want, ost = oracle.bank_spectra(st, wl.ranges, wl.freqs[sample], samples=wl.samples, kmax=wl.kmax)
    assert (ost == 0).all()
    assert rel_l2(got[sample], want) < 1e-6
    # and the Dunkin solve agrees with the reference-direct one in that band
    md = medium_of(gfk, st, formulation=gfk.DUNKIN, engine=engine)
    gd, sd = md.bank_spectra(wl.ranges, band, wl.integration())
    assert (sd == 0).all()
    assert rel_l2(gd, got[answered]) < 1e-6


def test_graded_soil_full_size_sampled_rows(gfk, engine, oracle):
    """The 2048 x 1024 graded-soil bank on the GPU; rows at 8 frequencies
    across the band recomputed by the oracle at the same full grid."""
    wl = gfk.workloads.graded_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine)
    got, status = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    assert (status == 0).all() and np.isfinite(got).all()
    rows = np.linspace(0, len(wl.freqs) - 1, 8).astype(int)
    want, ost = oracle.bank_spectra(as_tuples(wl.stack), wl.ranges, wl.freqs[rows], samples=wl.samples,
                                    kmax=wl.kmax, formulation=oracle.DUNKIN, omega_imag=wl.omega_imag)
    assert (ost == 0).all()
    assert rel_l2(got[rows], want) < 1e-9


def test_split_layer_invariance_above_the_guard(gfk, engine):
    """stability_test.go:30-92 carried past 400 Hz: a half-space cut into
    identical 2 m layers is the half-space, to 1e-9, on the GPU."""
    h = CF.LOAM
    half = gfk.Medium(gfk.uniform(*h), formulation=gfk.DUNKIN, default_q=30, engine=engine)
    l = gfk.Layer(2.0, h[0], h[1], h[2], h[3])
    split = gfk.Medium(gfk.Stack([l, l, gfk.Layer(0, h[0], h[1], h[2], h[3])]), formulation=gfk.DUNKIN,
                       default_q=30, engine=engine)
    freqs = np.array([10.0, 100.0, 400.0, 800.0, 1400.0])
    ranges = np.array([10.0])
    a, _ = half.bank_spectra(ranges, freqs)
    b, _ = split.bank_spectra(ranges, freqs)
    assert np.max(np.abs(a - b) / np.abs(a)) < 1e-9
    ref = gfk.Medium(split.stack, engine=engine)
    _, st = ref.bank_spectra(ranges, freqs, raise_on_error=False)
    assert list(st) == [0, 0, gfk._native.EGUARD, gfk._native.EGUARD, gfk._native.EGUARD]


def test_static_limit_and_boussinesq(gfk, engine):
    h = CF.LOAM
    m = gfk.Medium(gfk.Stack([gfk.Layer(0, h[0], h[1], h[2], 1e9)]), default_q=1e9, formulation=gfk.DUNKIN,
                   engine=engine)
    want = CF.boussinesq_coefficient(h)
    u = m.surface_response(np.array([1.0, 10.0, 200.0, 4000.0]), 0.05)
    assert np.max(np.abs(np.abs(u * np.array([1.0, 10.0, 200.0, 4000.0])) - want) / want) < 1e-5
    mu, nu = CF.shear_modulus(h), CF.poisson_ratio(h)
    for r in (2.0, 10.0):
        got = m.vertical_displacement(r, 0.02, gfk.Integration(8000))
        assert abs(abs(got) - (1 - nu) / (2 * math.pi * mu * r)) / ((1 - nu) / (2 * math.pi * mu * r)) < 0.02


def test_linearity_in_force_scale(gfk, engine):
    """Doubling every density doubles mu_ref and halves the response."""
    wl = gfk.workloads.single_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine)
    heavy = gfk.Stack(gfk.Layer(l.thickness, l.vp, l.vs, 2 * l.density, l.qs, l.qp) for l in wl.stack)
    m2 = gfk.Medium(heavy, formulation=gfk.DUNKIN, omega_imag=wl.omega_imag, engine=engine)
    a, _ = m.bank_spectra(wl.ranges[::16], wl.freqs[::32], wl.integration())
    b, _ = m2.bank_spectra(wl.ranges[::16], wl.freqs[::32], wl.integration())
    assert rel_l2(2 * b, a) < 1e-12


def test_error_statuses(gfk, engine):
    E = gfk._native
    m = gfk.Medium(gfk.uniform(*CF.LOAM), engine=engine)
    with pytest.raises(gfk.FkError) as e:
        m.surface_response(0.0, 10.0)
    assert e.value.status == E.EARG
    with pytest.raises(gfk.FkError) as e:
        m.vertical_displacement(-1.0, 10.0)
    assert e.value.status == E.EARG
    bad = gfk.Medium(gfk.Stack([gfk.Layer(0, 100, 200, 1700)]), engine=engine)
    with pytest.raises(gfk.FkError) as e:
        bad.surface_response(1.0, 10.0)
    assert e.value.status == E.ESTACK
    _, st = bad.bank_spectra([1.0, 2.0], [10.0, 20.0], raise_on_error=False)
    assert (st == E.ESTACK).all()
    nanm = gfk.Medium(gfk.Stack([gfk.Layer(1, 500, float("nan"), 1700), gfk.Layer(0, 500, 200, 1700)]),
                      formulation=gfk.DUNKIN, engine=engine)
    with pytest.raises(gfk.FkError) as e:
        nanm.bank_spectra([1.0], [10.0])
    assert e.value.status == E.ESTACK
    with pytest.raises(gfk.FkError) as e:
        gfk.Medium(gfk.uniform(*CF.LOAM), omega_imag=1.0, engine=engine).bank_spectra([1.0], [10.0])
    assert e.value.status == E.EARG  # the reference formulation is real-frequency only
    with pytest.raises(gfk.FkError) as e:
        m.bank_spectra([], [10.0])
    assert e.value.status == E.EARG
    got, st = m.bank_spectra([1.0], [-5.0, 10.0], raise_on_error=False)
    assert st[0] == E.EARG and st[1] == 0 and got[0, 0] == 0
    # a failed call leaves the context usable
    assert np.isfinite(m.vertical_displacement_multi([1.0, 2.0], 10.0)).all()


def test_plan_is_deterministic_and_timed(gfk, engine):
    wl = gfk.workloads.single_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine)
    p = gfk.Plan(m, wl.ranges, wl.freqs, wl.integration(), engine=engine)
    p.execute()
    a, _ = p.download()
    before = engine.kernel_launches()
    p.execute()
    b, _ = p.download()
    assert engine.kernel_launches() - before == p.launches_per_execute()
    assert np.array_equal(a, b)
    prop, quad, other = p.kernel_times()
    assert prop > 0 and quad > 0
    ref, _ = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    assert np.array_equal(a, ref)
    p.close()


@pytest.mark.parametrize("quadrature", ["fp64", "split"])
def test_plans_share_hankel_weights(gfk, engine, quadrature):
    """Plans on the same grid and ranges share one device copy of the Hankel
    weights: the second plan's first execute builds none, and every plan keeps
    giving its bank after the plan that built them is closed and after the
    context's cached copy has moved on to other ranges."""
    wl = gfk.workloads.single_soil()
    q = gfk.SPLIT_INT8 if quadrature == "split" else gfk.PLAIN_FP64
    m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=q)
    ranges = wl.ranges * 1.37  # not any other test's ranges
    opt = wl.integration()
    a = gfk.Plan(m, ranges, wl.freqs, opt, engine=engine)
    before = engine.kernel_launches()
    a.execute()
    assert engine.kernel_launches() - before >= a.launches_per_execute() + 1  # the weights were built
    a.download()
    # as many rows as a (the tuned launch shapes are the ones a chose), other frequencies
    freqs_b = wl.freqs * 1.01
    b = gfk.Plan(m, ranges, freqs_b, opt, engine=engine)
    before = engine.kernel_launches()
    b.execute()
    assert engine.kernel_launches() - before == b.launches_per_execute()  # and reused
    got_b, _ = b.download()
    fp64_b, _ = wl.medium(gfk.DUNKIN, engine=engine).bank_spectra(ranges, freqs_b, opt)
    assert rel_l2(got_b, fp64_b) < (1e-6 if quadrature == "split" else 1e-12)
    a.close()
    other = ranges[:17] * 0.5
    c = gfk.Plan(m, other, wl.freqs, opt, engine=engine)
    c.execute()
    got_c, _ = c.download()
    ref_c, _ = wl.medium(gfk.DUNKIN, engine=engine).bank_spectra(other, wl.freqs, opt)
    assert rel_l2(got_c, ref_c) < (1e-6 if quadrature == "split" else 1e-12)
    b.execute()
    again, _ = b.download()
    assert np.array_equal(again, got_b)
    b.close()
    c.close()


def test_every_propagator_shape_gives_the_same_bank(gfk, engine, monkeypatch):
    """Every tuned launch shape of the propagator (one item per block or
    persistent over the device queue; 1-8 runs per item; with and without the
    fused slicing) computes each (row, k) with the same code, so the banks are
    bit-identical. 1000 wavenumbers fill no run evenly."""
    wl = gfk.workloads.single_soil()
    opt = gfk.Integration(1000, 0.0, wl.kmax)
    freqs = wl.freqs[1::3]
    shapes = []
    v = 0
    while True:
        try:
            shapes.append(gfk.prop_shape(v))
        except gfk.FkError:
            break
        v += 1
    assert any(s["persistent"] for s in shapes)
    for q in (gfk.PLAIN_FP64, gfk.SPLIT_INT8):
        m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=q)
        banks = []
        for s in shapes:
            monkeypatch.setenv("GFK_PROP_VARIANT", str(s["index"]))
            p = gfk.Plan(m, wl.ranges, freqs, opt, engine=engine)
            p.execute()
            assert p.tuning()[0] == s["index"]
            b, st = p.download()
            assert (st == 0).all()
            p.execute()  # a second launch on the same queue and counters
            again, _ = p.download()
            assert np.array_equal(again, b)
            banks.append(b)
            p.close()
        for s, b in zip(shapes, banks):
            assert np.array_equal(b, banks[0]), s
    # one row of the smallest grid (64 wavenumbers, less than one item of any shape)
    tiny = []
    for q in (gfk.PLAIN_FP64, gfk.SPLIT_INT8):
        m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=q)
        for s in shapes:
            monkeypatch.setenv("GFK_PROP_VARIANT", str(s["index"]))
            b, st = m.bank_spectra(wl.ranges[:40], wl.freqs[100:101], gfk.Integration(64, 0.0, wl.kmax))
            assert (st == 0).all() and np.isfinite(b).all()
            tiny.append((q, b))
    for q, b in tiny:
        ref = next(x for qq, x in tiny if qq == q)
        assert np.array_equal(b, ref)
    # per-frequency grids (GridFor): rows of different lengths in one launch
    m = gfk.Medium(wl.stack, formulation=gfk.DUNKIN, omega_imag=wl.omega_imag, engine=engine)
    f2 = wl.freqs[5:300:7]
    banks = []
    for s in shapes:
        monkeypatch.setenv("GFK_PROP_VARIANT", str(s["index"]))
        b, st = m.bank_spectra(wl.ranges[:9], f2)
        assert (st == 0).all()
        banks.append(b)
    for s, b in zip(shapes, banks):
        assert np.array_equal(b, banks[0]), s
    monkeypatch.delenv("GFK_PROP_VARIANT")


def test_build_and_write_bank(gfk, engine, tmp_path):
    """geobank build on the GPU (cmd/geobank/main.go:51-178) round-tripped
    through the file format."""
    st = gfk.Stack([gfk.Layer(3.0, 400, 160, 1600), gfk.Layer(0, 900, 400, 2000)])
    h = gfk.Header(gfk.Provenance("gfk-b200 fk (layered wavenumber integration)"), st, 2000.0, 512,
                   gfk.RangeGrid(1.0, 10.0, 40), "vertical surface displacement per unit vertical surface point force",
                   "m/N")
    m = gfk.Medium(st, default_q=30, engine=engine)
    b, spectra = gfk.build_bank(m, h, 100.0, spectra=True)
    path = tmp_path / "g.bank"
    b.write(path)
    r = gfk.open_bank(path)
    top = int(100.0 / (2000.0 / 512))
    assert np.array_equal(r.data, b.data)
    assert (r.data[:, 0] == 0).all() and (r.data[:, top + 1:] == 0).all()
    assert np.array_equal(r.data[:, 1:top + 1, 0], spectra.T.real.astype(np.float32))


@pytest.mark.parametrize("name", ["single_soil", "graded_soil"])
def test_split_quadrature_against_fp64(gfk, engine, name):
    """The tensor-core (exact int8 slice) wavenumber sum against the FP64 one on
    the same integrand: rel-L2 <= 1e-6 over the whole bank, the bar the
    split-precision path is held to."""
    wl = getattr(gfk.workloads, name)()
    plain = wl.medium(gfk.DUNKIN, engine=engine)
    split = wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8)
    a, sa = plain.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    b, sb = split.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    assert (sa == 0).all() and (sb == 0).all()
    rel = rel_l2(b, a)
    assert rel < 1e-6, rel
    # every bin, not just the aggregate
    per_bin = np.linalg.norm(b - a, axis=1) / np.linalg.norm(a, axis=1)
    assert per_bin.max() < 1e-5, per_bin.max()


def test_split_quadrature_ragged_shapes(gfk, engine, oracle):
    """Sizes that are not multiples of the 128 x 128 x 64 tiles."""
    wl = gfk.workloads.single_soil()
    ranges = wl.ranges[:45] * 1.5
    freqs = wl.freqs[3:70:2]
    opt = gfk.Integration(1000, 0.0, wl.kmax)
    split = wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8)
    got, st = split.bank_spectra(ranges, freqs, opt)
    assert (st == 0).all()
    want, ost = oracle.bank_spectra(as_tuples(wl.stack), ranges, freqs, samples=1000, kmax=wl.kmax,
                                    formulation=oracle.DUNKIN, omega_imag=wl.omega_imag)
    assert rel_l2(got, want) < 1e-6


def test_split_quadrature_refuses_per_frequency_grids(gfk, engine):
    m = gfk.Medium(gfk.uniform(500, 200, 1700, 25), formulation=gfk.DUNKIN, quadrature=gfk.SPLIT_INT8,
                   engine=engine)
    with pytest.raises(gfk.FkError) as e:
        m.bank_spectra([1.0, 2.0], [10.0, 20.0])
    assert e.value.status == gfk._native.EARG


def test_batch_of_uneven_soils_matches_single_plans(gfk, engine, oracle):
    """Media with different layer counts and frequency lists in one batch give
    the rows each medium gives on its own; a medium that fails validation
    marks only its own rows."""
    soils, ranges, nk, kmax = gfk.workloads.batched_soils(count=6, seed=11)
    ranges = ranges[::4]
    opt = gfk.Integration(2048, 0.0, kmax)
    media, freqs = [], []
    for st, fr in soils:
        media.append(gfk.Medium(st, formulation=gfk.DUNKIN, omega_imag=1.5, engine=engine))
        freqs.append(fr[::97])
    bad = gfk.Medium(gfk.Stack([gfk.Layer(0, 100, 200, 1700)]), formulation=gfk.DUNKIN, omega_imag=1.5,
                     engine=engine)
    media.insert(2, bad)
    freqs.insert(2, np.array([10.0, 20.0]))
    for quad in (gfk.PLAIN_FP64, gfk.SPLIT_INT8):
        for m in media:
            m.quadrature = quad
        b = gfk.Batch(media, freqs, ranges, opt, engine=engine)
        b.execute()
        got, status = b.download(raise_on_error=False)
        parts, stats = b.split(got), b.split(status)
        assert (stats[2] == gfk._native.ESTACK).all()
        for i, (m, fr) in enumerate(zip(media, freqs)):
            if i == 2:
                continue
            assert (stats[i] == 0).all()
            want, _ = m.bank_spectra(ranges, fr, opt)
            assert rel_l2(parts[i], want) < 1e-12
        st0 = soils[0][0]
        w0, _ = oracle.bank_spectra(as_tuples(st0), ranges, freqs[0], samples=2048, kmax=kmax,
                                    formulation=oracle.DUNKIN, omega_imag=1.5)
        assert rel_l2(parts[0], w0) < 1e-6
        b.close()


@pytest.mark.parametrize("quad", ["plain", "split"])
def test_split_k_sum_matches_one_pass(gfk, engine, quad):
    """A bank too small to fill the SMs (512 x 64 cells) divides the
    wavenumber sum among blocks and adds the partial sums in a fixed order;
    the same soil inside a large batch takes the one-pass sum. Both must agree
    to rounding, and the split result must be bit-reproducible."""
    wl = gfk.workloads.single_soil()
    q = gfk.PLAIN_FP64 if quad == "plain" else gfk.SPLIT_INT8
    m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=q)
    a, sa = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    a2, _ = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    assert (sa == 0).all()
    assert np.array_equal(a, a2)
    copies = 24
    b = gfk.Batch([m] * copies, [wl.freqs] * copies, wl.ranges, wl.integration(), engine=engine)
    b.execute()
    got, st = b.download()
    assert (st == 0).all()
    parts = b.split(got)
    b.close()
    per_bin = np.linalg.norm(parts[copies - 1] - a, axis=1) / np.linalg.norm(a, axis=1)
    assert per_bin.max() < 1e-11, per_bin.max()
    assert np.array_equal(parts[0], parts[copies - 1])


def test_graph_execute_matches_stream_execute(gfk, engine):
    wl = gfk.workloads.single_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8)
    p = gfk.Plan(m, wl.ranges, wl.freqs, wl.integration(), engine=engine)
    p.execute()
    a, _ = p.download()
    p.use_graph(True)
    p.execute()  # captures
    p.execute()  # relaunches
    b, _ = p.download()
    assert np.array_equal(a, b)
    p.close()


def test_fused_sum_for_few_ranges(gfk, engine, oracle):
    """Up to 8 ranges on a shared grid: the sum is fused into the propagator
    (the integrand never reaches HBM) and must give what the GEMM path and the
    oracle give."""
    wl = gfk.workloads.single_soil()
    m = wl.medium(gfk.DUNKIN, engine=engine)
    few = wl.ranges[[0, 4, 9, 31, 63]]
    many = np.concatenate([few, wl.ranges[[1, 2, 3, 5, 6]]])  # 10 ranges: GEMM path
    a, sa = m.bank_spectra(few, wl.freqs, wl.integration())
    b, sb = m.bank_spectra(many, wl.freqs, wl.integration())
    assert (sa == 0).all() and (sb == 0).all()
    assert rel_l2(a, b[:, :5]) < 1e-12
    rows = np.arange(0, len(wl.freqs), 37)
    want, _ = oracle.bank_spectra(as_tuples(wl.stack), few, wl.freqs[rows], samples=wl.samples, kmax=wl.kmax,
                                  formulation=oracle.DUNKIN, omega_imag=wl.omega_imag)
    assert rel_l2(a[rows], want) < 1e-9
    a2, _ = m.bank_spectra(few, wl.freqs, wl.integration())
    assert np.array_equal(a, a2)  # fixed reduction order: bit-reproducible


def test_sobol_banks_and_metrics_against_oracle(gfk, engine, oracle):
    """The Sobol workload's per-soil responses at 10 m (fused single-range
    path) against the oracle, and the metrics computed from them."""
    S = gfk.sobol
    setup = S.TraceSetup()
    u = S.saltelli(4, len(S.PARAMS), seed=2)
    params = S.unit_to_params(u)
    G, gpu_s, rows = S.solve_banks(params, setup, engine, batch_soils=16, nk=2048)
    assert G.shape == (len(params), setup.n // 2) and np.isfinite(G).all()
    for i in (0, 17):
        st = S.soil_of(params[i])
        want, _ = oracle.bank_spectra(as_tuples(st), [setup.r], setup.freqs(), samples=2048, kmax=S.KMAX,
                                      formulation=oracle.DUNKIN, omega_imag=setup.omega_imag)
        assert rel_l2(G[i], want[:, 0]) < 1e-9
        y = S.traces(np.vstack([G[i], want[:, 0]]), setup)
        pk, cen = S.measure(y, setup.fs)
        assert abs(pk[0] - pk[1]) / pk[1] < 1e-8 and abs(cen[0] - cen[1]) < 1e-6


def test_plan_execute_download_overlaps_chunks(gfk, engine):
    """gfk_plan_execute_download on a plan of two row chunks (71,680 rows: over
    the 65,535-row grid limit): into page-locked memory each chunk is copied
    out while the next computes; the bank, statuses and zeroed failed rows
    equal execute + download, with the plan's CUDA graph on before and after."""
    import torch
    wl = gfk.workloads.single_soil()
    opt = gfk.Integration(256, 0.0, wl.kmax)
    ranges = np.array([1.0, 3.0, 7.5, 20.0, 41.0])
    freqs = wl.freqs.copy()
    bad = freqs.copy()
    bad[17] = -5.0
    media = [wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8) for _ in range(140)]
    fl = [bad if i == 70 else freqs for i in range(140)]
    p = gfk.Batch(media, fl, ranges, opt, engine=engine)
    p.use_graph(True)
    p.execute()
    want, sw = p.download(raise_on_error=False)
    rows = len(p.freqs)
    assert rows == 140 * len(freqs) and (sw != 0).sum() == 1
    pinned = torch.full((rows, 2 * len(ranges)), 7.0, dtype=torch.float64, pin_memory=True).numpy()
    pinned = pinned.view(np.complex128)
    got, sg = p.execute_download(raise_on_error=False, out=pinned)
    assert np.array_equal(sg, sw) and np.array_equal(got, want)
    assert (got[70 * len(freqs) + 17] == 0).all()
    p.execute()  # the captured graph again
    again, _ = p.download(raise_on_error=False)
    assert np.array_equal(again, want)
    plain, _ = p.execute_download(raise_on_error=False)  # pageable memory: execute, then download
    assert np.array_equal(plain, want)
    p.close()


def test_pinned_bank_download_overlaps_and_matches(gfk, engine):
    """Into page-locked memory gfk_bank_spectra computes a larger bank in row
    chunks and downloads each while the next computes; the bank equals the
    one-piece call to rounding (the split sums differ only in their split
    count), and failing rows come back zeroed with their statuses."""
    import torch
    wl = gfk.workloads.single_soil()
    wl.ranges = np.linspace(1.0, 64.0, 2048)  # 512 x 2048 cells = 16 MB: the chunked path
    for q in (gfk.PLAIN_FP64, gfk.SPLIT_INT8):
        m = wl.medium(gfk.DUNKIN, engine=engine, quadrature=q)
        want, sw = m.bank_spectra(wl.ranges, wl.freqs, wl.integration())
        pinned = torch.zeros((len(wl.freqs), 2 * len(wl.ranges)), dtype=torch.float64, pin_memory=True).numpy()
        got, sg = m.bank_spectra(wl.ranges, wl.freqs, wl.integration(), out=pinned)
        assert (sw == 0).all() and (sg == 0).all()
        per_bin = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
        assert per_bin.max() < 1e-11, per_bin.max()
        got2, _ = m.bank_spectra(wl.ranges, wl.freqs, wl.integration(), out=pinned)
        assert np.array_equal(got, got2)
    # per-frequency grids (GridFor): the sequential per-row sum, so chunking changes nothing
    m = gfk.Medium(wl.stack, formulation=gfk.DUNKIN, omega_imag=wl.omega_imag, engine=engine)
    f2 = wl.freqs[:256]
    want, _ = m.bank_spectra(wl.ranges, f2)
    pinned2 = torch.zeros((len(f2), 2 * len(wl.ranges)), dtype=torch.float64, pin_memory=True).numpy()
    got, st = m.bank_spectra(wl.ranges, f2, out=pinned2)
    assert (st == 0).all() and np.array_equal(got, want)
    freqs = wl.freqs.copy()
    freqs[300] = -5.0
    m = wl.medium(gfk.DUNKIN, engine=engine)
    pinned = torch.full((len(freqs), 2 * len(wl.ranges)), 7.0, dtype=torch.float64, pin_memory=True).numpy()
    got, st = m.bank_spectra(wl.ranges, freqs, wl.integration(), raise_on_error=False, out=pinned)
    want, stw = m.bank_spectra(wl.ranges, freqs, wl.integration(), raise_on_error=False)
    assert st[300] == gfk._native.EARG and (st == stw).all()
    assert (got[300] == 0).all() and np.abs(got[:300] - want[:300]).max() <= 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("form", [0, 1], ids=["reference_direct", "dunkin"])
def test_layered_causality_known_answers(gfk, engine, form):
    """TestLayeredResponseHasNoPrecursor (internal/fk/causality_test.go:45-141)
    through libgfk: 1228 bins to 120 Hz of the 2 m layer over a half-space,
    each on GridFor's own wavenumber grid, shaped and transformed as the
    reference's test does. The peak times, the precursor and the negative-time
    residue equal what the reference's run logged, to its printed digits
    (docs/validation-report.md:278-280), in both formulations (Dunkin with the
    reference's Qp = 2.25 Qs at real frequencies)."""
    import causality_case as CC
    KA = json.loads((GOLDEN / "known_answers.json").read_text())
    st = CC.STACK if form == 0 else [tuple(l[:5]) + (2.25 * l[4],) for l in CC.STACK]
    m = medium_of(gfk, st, default_q=CC.DEFAULT_Q, formulation=form, engine=engine)
    _, freqs = CC.bins()
    spectra, status = m.bank_spectra(CC.RANGES, freqs)
    assert (status == 0).all()
    CC.check_against_logged(CC.metrics(spectra), KA["causality_precursor"])


@pytest.mark.parametrize("form", [0, 1], ids=["reference_direct", "dunkin"])
def test_sls_medium_matches_oracle(gfk, engine, oracle, form):
    """Medium.Relax: one standard linear solid replaces constant Q for P and S
    alike (internal/fk/fk.go:44-52, 84-88, 96-102; internal/visco/visco.go:55-108),
    on a two-layer stack. GPU against the oracle's restatement: pointwise
    surface responses and a bank, Dunkin at a complex frequency offset."""
    st = [(1.5, 400.0, 170.0, 1650.0, 0.0, 0.0), (3.0, 650.0, 260.0, 1850.0, 0.0, 0.0),
          (0.0, 900.0, 420.0, 2000.0, 0.0, 0.0)]
    sls = gfk.SLS.fit(25.0, 30.0)
    wi = 0.0 if form == 0 else 1.5
    m = medium_of(gfk, st, relax=sls, ref_freq=30.0, formulation=form, omega_imag=wi, engine=engine)
    om = oracle.OracleMedium(st, ref_freq=30.0, sls=(sls.tau_sigma, sls.tau_eps))
    rng = np.random.default_rng(3)
    f = rng.uniform(1.0, 80.0, 200)
    k = rng.uniform(0.01, 4.0, 200) * 2 * np.pi * f / 170.0
    got = m.surface_response(k, f)
    want = np.array([oracle.surface_response(om, ki, fi, form, wi) for ki, fi in zip(k, f)])
    assert np.max(np.abs(got - want) / np.abs(want)) < (1e-6 if form == 0 else 1e-11)
    ranges = np.arange(1.0, 33.0)
    freqs = np.linspace(2.0, 80.0, 40)
    kmax = 2.5 * 2 * np.pi * 80.0 / 170.0
    opt = gfk.Integration(4096, 0.0, kmax)
    g, gs = m.bank_spectra(ranges, freqs, opt)
    w, ws = oracle.bank_spectra(om, ranges, freqs, samples=4096, kmax=kmax, formulation=form, omega_imag=wi)
    assert (gs == 0).all() and (ws == 0).all()
    assert rel_l2(g, w) < (1e-6 if form == 0 else 1e-9)
    # the relaxation is not constant Q: the same stack at Q = 25 differs
    mq = medium_of(gfk, [l[:4] + (25.0, 0.0) for l in st], ref_freq=30.0, formulation=form, omega_imag=wi,
                   engine=engine)
    gq, _ = mq.bank_spectra(ranges, freqs, opt)
    assert rel_l2(gq, g) > 1e-3


def _hardest_batched_soils(soils, count):
    """The seeded uneven soils whose split sums cancel most: the lowest
    min(Vs Qs) (slow, lossy layers) and the highest min(Qs) (sharp poles)."""
    by_vsq = sorted(range(len(soils)), key=lambda i: min(l.vs * l.qs for l in soils[i][0]))
    by_q = sorted(range(len(soils)), key=lambda i: -min(l.qs for l in soils[i][0]))
    return list(dict.fromkeys(by_vsq[:count // 2] + by_q[:count // 2]))


def test_split_sum_on_hardest_batched_soils(gfk, engine):
    """The exact int8-slice wavenumber sum against the FP64 sum on the same
    integrand, on the 64 hardest of the 4096 seeded uneven soils at their full
    size (256-2048 bins each, 8192 wavenumbers, 128 ranges): rel-L2 <= 1e-6 per
    soil, and <= 1e-5 in every bin."""
    soils, ranges, nk, kmax = gfk.workloads.batched_soils()
    pick = _hardest_batched_soils(soils, 64)
    assert len(pick) >= 60
    opt = gfk.Integration(nk, 0.0, kmax)
    out = {}
    for quad in (gfk.PLAIN_FP64, gfk.SPLIT_INT8):
        media = [gfk.Medium(soils[i][0], formulation=gfk.DUNKIN, quadrature=quad, engine=engine) for i in pick]
        b = gfk.Batch(media, [soils[i][1] for i in pick], ranges, opt, engine=engine)
        b.execute()
        got, status = b.download()
        assert (status == 0).all() and np.isfinite(got).all()
        out[quad] = b.split(got)
        b.close()
    worst_soil = worst_bin = 0.0
    for a, s in zip(out[gfk.PLAIN_FP64], out[gfk.SPLIT_INT8]):
        worst_soil = max(worst_soil, rel_l2(s, a))
        worst_bin = max(worst_bin, float(np.max(np.linalg.norm(s - a, axis=1) / np.linalg.norm(a, axis=1))))
    assert worst_soil < 1e-6, worst_soil
    assert worst_bin < 1e-5, worst_bin


def test_tensor_core_wait_timeout_is_reported_and_context_survives(gfk, engine):
    """Failure detection without a GPU fault: the tensor-core sum's producer is
    told to issue no loads, so the MMA issuer's bounded mbarrier wait runs out
    (after 2^22 SM clocks, ~2 ms). The kernel must drain, free its tensor
    memory, exit and mark the tile's 64 rows GFK_ETIMEOUT, and the same context
    must then compute a split-sum bank as before."""
    N = gfk._native
    rows = ctypes.c_int32()
    st = N.lib().gfk_selftest_wait_timeout(engine.ctx, 1 << 22, ctypes.byref(rows))
    assert st == N.ETIMEOUT and rows.value == 64, (N.status_string(st), rows.value)
    wl = gfk.workloads.single_soil()
    split = wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8)
    plain = wl.medium(gfk.DUNKIN, engine=engine)
    a, sa = split.bank_spectra(wl.ranges, wl.freqs[::8], wl.integration())
    b, sb = plain.bank_spectra(wl.ranges, wl.freqs[::8], wl.integration())
    assert (sa == 0).all() and (sb == 0).all()
    assert rel_l2(a, b) < 1e-6


@pytest.mark.parametrize("shape", [0, 1, 2, 3], ids=["n128_s3", "n128_s2", "n64_s4", "n64_s3"])
def test_split_sum_every_tile_shape(gfk, engine, shape, monkeypatch):
    """Every tile shape the plan's tuner can choose for the tensor-core sum
    (128 or 64 ranges per CTA, 2-4 pipeline stages), forced in turn, on ragged
    sizes (200 ranges, 3000 wavenumbers, 171 frequencies): the same bank as
    the FP64 sum within the split sum's 1e-6."""
    monkeypatch.setenv("GFK_QUAD_TC_VARIANT", str(shape))
    wl = gfk.workloads.single_soil()
    ranges = np.arange(1.0, 201.0) * 0.5
    freqs = wl.freqs[::3]
    opt = gfk.Integration(3000, 0.0, wl.kmax)
    split = wl.medium(gfk.DUNKIN, engine=engine, quadrature=gfk.SPLIT_INT8)
    plan = gfk.Plan(split, ranges, freqs, opt, engine=engine)
    plan.execute()
    got, st = plan.download()
    tn, ns, _ = plan.quad_shape()
    plan.close()
    assert (tn, ns) == [(128, 3), (128, 2), (64, 4), (64, 3)][shape]
    want, sw = wl.medium(gfk.DUNKIN, engine=engine).bank_spectra(ranges, freqs, opt)
    assert (st == 0).all() and (sw == 0).all()
    assert rel_l2(got, want) < 1e-6


def test_bank_payload_packed_on_device(gfk, engine):
    """gfk_bank_payload: the bank file's float32 range-major payload packed on
    the device equals the host packing (gfk_bank_pack) of the FP64 spectra,
    bins outside the computed ones stay zero, and frequencies the reference
    formulation's guard refuses come back with their status and zero columns,
    the call returning the first failure as geobank aborts on it."""
    N = gfk._native
    st = gfk.Stack([gfk.Layer(2.0, 400, 160, 1600, 20), gfk.Layer(0, 900, 400, 2000, 40)])
    ranges = np.linspace(1.0, 30.0, 37)
    bins, first = 300, 5
    freqs = (np.arange(first, first + 250) * 1.0)  # 5..254 Hz, the guard refuses the top ones
    for form in (N.DUNKIN, N.REFERENCE_DIRECT):
        m = gfk.Medium(st, formulation=form, engine=engine)
        pay, status = m.bank_payload(ranges, freqs, first, bins, raise_on_error=False)
        spec, sst = m.bank_spectra(ranges, freqs, raise_on_error=False)
        assert np.array_equal(status, sst)
        host = np.zeros(2 * len(ranges) * bins, dtype=np.float32)
        sp = np.ascontiguousarray(np.stack([spec.real, spec.imag], axis=-1))
        assert N.lib().gfk_bank_pack(sp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(freqs), len(ranges),
                                     first, bins, host.ctypes.data_as(ctypes.POINTER(ctypes.c_float))) == 0
        assert np.array_equal(pay.ravel(), host)
        assert (pay[:, :first] == 0).all() and (pay[:, first + len(freqs):] == 0).all()
        if form == N.REFERENCE_DIRECT:
            refused = status == N.EGUARD
            assert refused.any() and not refused.all()
            assert (pay[:, first + np.nonzero(refused)[0]] == 0).all()
            with pytest.raises(gfk.FkError) as e:
                m.bank_payload(ranges, freqs, first, bins)
            assert e.value.status == N.EGUARD
        else:
            assert (status == 0).all()
    with pytest.raises(gfk.FkError):
        gfk.Medium(st, engine=engine).bank_payload(ranges, freqs, 100, bins)  # bins beyond the payload
