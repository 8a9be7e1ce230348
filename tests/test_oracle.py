"""The CPU oracle pinned before it is trusted: against 40-3000-digit
evaluations of the reference algorithm, and against every number the
reference's own test run logged for this path (docs/validation-report.md)."""
import cmath
import json
import math

import numpy as np
import pytest

from conftest import GOLDEN

import closed_forms as CF

MP = json.loads((GOLDEN / "surface_response_mp.json").read_text())
KA = json.loads((GOLDEN / "known_answers.json").read_text())


def _mp_cases():
    return [c for c in MP["cases"]]


@pytest.mark.parametrize("form", [0, 1], ids=["reference_direct", "dunkin"])
def test_surface_response_against_high_precision(oracle, form):
    """Both formulations against the reference algorithm at 40+ digits. The
    direct form loses digits with k*h and k/k_body (fk.go:224-242,
    fk_test.go:48-57), so it is held only where the reference's guard lets it
    answer; Dunkin is held everywhere."""
    worst = 0.0
    for c in _mp_cases():
        st = MP["media"][c["medium"]]
        if form == 0:
            if c["qp_mode"] != "reference" or c["kh"] > 16:
                continue
        elif c["qp_mode"] == "reference":
            st = [tuple(l[:5]) + (0.0,) for l in st]
        want = complex(*c["u"])
        got = oracle.surface_response(st, c["k"], c["f"], form, c["omega_imag"])
        rel = abs(got - want) / abs(want)
        worst = max(worst, rel)
    assert worst < (1e-6 if form == 0 else 1e-12), worst


def test_integrand_at_zero_wavenumber_known_answer(oracle):
    """fk_test.go:317-347, logged at docs/validation-report.md:67-70."""
    m = CF.uniform(CF.LOAM)
    kb = 2 * math.pi * 40 / 200
    c = oracle.static_coefficient(m, 40.0, 200 * kb)
    for row in KA["integrand_at_zero_k"]:
        assert abs(abs(c) - row["minus_C_abs"]) / row["minus_C_abs"] < 5e-7
        u = oracle.surface_response(m, row["k"], 40.0)
        g = row["k"] * u - c
        assert abs(abs(g) - row["integrand_abs"]) / row["integrand_abs"] < 5e-7
        assert abs(abs(g + c) / abs(c) - row["apart"]) / row["apart"] < 5e-3


def test_quadrature_order_known_answer(oracle):
    """fk_test.go:270-312: GridFor's 6000 samples and the logged errors
    (docs/validation-report.md:60-62)."""
    m = CF.uniform(CF.LOAM)
    kmax, n = oracle.grid_for(m, [16.0], 60.0)
    assert n == 6000
    fine = oracle.vertical_displacement(m, 16.0, 60.0, samples=16 * n)
    finer = oracle.vertical_displacement(m, 16.0, 60.0, samples=32 * n)
    ref = (4 * finer - fine) / 3
    for row in KA["quadrature_order"]:
        got = oracle.vertical_displacement(m, 16.0, 60.0, samples=row["n"])
        rel = abs(got - ref) / abs(ref)
        assert abs(rel - row["rel"]) / row["rel"] < 2e-3, (row, rel)


def test_far_field_phase_known_answer(oracle):
    """fk_test.go:184-223 against the closed-form far field (green.go:218-266),
    logged at docs/validation-report.md:53-55."""
    h = CF.LOAM
    lam = CF.rayleigh_velocity(h) / 30.0
    for row in KA["far_field_phase"]:
        r = row["wavelengths"] * lam
        u = oracle.vertical_displacement(CF.uniform(h), r, 30.0)
        ratio = 1j * 2 * math.pi * 30.0 * u / CF.far_field_velocity_response(h, r, 30.0)
        assert abs(abs(ratio) - row["abs_ratio"]) < 6e-5
        assert abs(math.degrees(cmath.phase(ratio)) - row["phase_deg"]) < 0.06
        assert abs(abs(ratio - 1) - row["gap"]) < 6e-5


def test_guard_band_known_answer(oracle):
    """stability_test.go:97-121, logged at docs/validation-report.md:155-157."""
    for row in KA["guard_band"]:
        st = [(row["thickness_m"], 500, 200, 1700, 25, 0), (0, 500, 200, 1700, 25, 0)]
        lo, hi = 1.0, 4000.0
        for _ in range(40):
            mid = 0.5 * (lo + hi)
            if oracle.check_layer_phase(st, mid) == 0:
                lo = mid
            else:
                hi = mid
        assert round(lo) == row["usable_hz"]


def test_fastest_velocity_known_answer():
    """complexVelocity(800, 2.25*20, 120 Hz) real part, causality_test.go:86-93
    (docs/validation-report.md:278)."""
    import mp_direct
    v = complex(mp_direct.complex_velocity(800.0, 2.25 * 20, 120.0))
    assert round(v.real, 1) == KA["fastest_velocity"][0]["mps"]


def test_split_layer_invariance(oracle):
    """stability_test.go:30-92: identical layers over their own half-space.
    The direct form stays within 1e-5 below the guard and is refused above;
    the Dunkin form agrees everywhere, 400-1400 Hz included."""
    half = oracle.OracleMedium(CF.uniform(CF.LOAM), default_q=30)
    l = (2.0, 500.0, 200.0, 1700.0, 25.0, 0.0)
    split = oracle.OracleMedium([l, l, (0.0, 500.0, 200.0, 1700.0, 25.0, 0.0)], default_q=30)
    logged = {row["freq_hz"]: row["rel"] for row in KA["split_layer"]}
    for f in (10, 30, 100, 200):
        a = oracle.vertical_displacement(half, 10.0, f)
        b = oracle.vertical_displacement(split, 10.0, f)
        rel = abs(a - b) / abs(a)
        assert rel < 1e-5
        assert rel < 100 * logged[f]  # same rounding-level size as the reference logged
        d = oracle.vertical_displacement(split, 10.0, f, formulation=oracle.DUNKIN)
        assert abs(a - d) / abs(a) < 1e-10
    with pytest.raises(oracle.OracleError) as e:
        oracle.vertical_displacement(split, 10.0, 400.0)
    assert e.value.status == 3
    for f in (400, 600, 1000, 1400):
        a = oracle.vertical_displacement(half, 10.0, f)
        d = oracle.vertical_displacement(split, 10.0, f, formulation=oracle.DUNKIN)
        assert abs(a - d) / abs(a) < 1e-9


@pytest.mark.parametrize("name,h", [("loam", CF.LOAM), ("dry sand", CF.DRY_SAND), ("rock", CF.WEATHERED_ROCK)])
def test_boussinesq_large_wavenumber(oracle, name, h):
    """fk_test.go:33-64: k|u| -> (1-nu)/(2 pi mu) within 1e-3; the Dunkin
    form holds 1e-6, since it has no eigenvector ill-conditioning at large k."""
    m = oracle.OracleMedium(CF.uniform(h, 1e9), default_q=1e9)
    want = CF.boussinesq_coefficient(h)
    for k in (1.0, 10.0, 200.0):
        for form, tol in ((0, 1e-3), (1, 1e-5)):
            got = k * abs(oracle.surface_response(m, k, 0.05, form))
            assert abs(got - want) / want < tol


def test_static_limit(oracle):
    """fk_test.go:71-87: at 0.02 Hz the displacement at range is Boussinesq's."""
    h = CF.LOAM
    m = oracle.OracleMedium(CF.uniform(h, 1e9), default_q=1e9)
    mu, nu = CF.shear_modulus(h), CF.poisson_ratio(h)
    for r in (2.0, 5.0, 10.0, 20.0):
        want = (1 - nu) / (2 * math.pi * mu * r)
        for form in (0, 1):
            got = oracle.vertical_displacement(m, r, 0.02, samples=8000, formulation=form)
            assert abs(abs(got) - want) / want < 0.02


def test_static_coefficient_follows_surface_layer(oracle):
    """fk_test.go:230-253."""
    top = (3.0, 400.0, 160.0, 1600.0, 1e9, 0.0)
    stacked = oracle.OracleMedium([top, (0.0, 2200.0, 1100.0, 2400.0, 1e9, 0.0)], default_q=1e9)
    alone = oracle.OracleMedium([(0.0,) + top[1:]], default_q=1e9)
    for form in (0, 1):
        a = oracle.static_coefficient(stacked, 1.0, 40.0, form)
        b = oracle.static_coefficient(alone, 1.0, 40.0, form)
        assert abs(a - b) / abs(b) < 1e-6


def test_multi_matches_single_range(oracle):
    """multi_test.go:14-37: the shared grid changes nothing beyond 5%."""
    m = CF.uniform(CF.LOAM)
    ranges = [2.0, 5.0, 10.0, 20.0]
    kmax, n = oracle.grid_for(m, ranges, 20.0)
    multi = oracle.vertical_displacement_multi(m, ranges, 20.0)
    for i, r in enumerate(ranges):
        single = oracle.vertical_displacement(m, r, 20.0, samples=n, kmax_factor=kmax / (2 * math.pi * 20 / 200))
        assert abs(multi[i] - single) / abs(single) < 0.05


def test_grid_rules_and_errors(oracle):
    """multi_test.go:42-61 and fk_test.go:349-367."""
    m = CF.uniform(CF.LOAM)
    kmax, n = oracle.grid_for(m, [1.0, 50.0], 20.0)
    assert kmax >= 40 and kmax / n <= 2 * math.pi / (8 * 50)
    with pytest.raises(oracle.OracleError):
        oracle.grid_for(m, [], 20.0)
    with pytest.raises(oracle.OracleError):
        oracle.grid_for(m, [0.0], 20.0)
    with pytest.raises(oracle.OracleError):
        oracle.surface_response(m, 0.0, 10.0)
    with pytest.raises(oracle.OracleError):
        oracle.surface_response(m, 1.0, 0.0)
    with pytest.raises(oracle.OracleError):
        oracle.vertical_displacement(m, 0.0, 10.0)
    with pytest.raises(oracle.OracleError):
        oracle.surface_response([(0, 100, 200, 1700, 0, 0)], 1.0, 10.0)


def test_near_field_departure_grows(oracle):
    """fk_test.go:102-167: inside a wavelength the full solution exceeds the far
    field, increasingly so as range shrinks (the plan's table,
    docs/wp1-forward-model-plan.md:476-485, to its two digits where stable)."""
    h = CF.LOAM
    lam = CF.rayleigh_velocity(h) / 10.0
    prev = 0.0
    for mult in (0.6, 0.4, 0.25, 0.15, 0.08):
        r = mult * lam
        u = oracle.vertical_displacement(CF.uniform(h), r, 10.0, samples=6000)
        ratio = abs(1j * 2 * math.pi * 10 * u) / abs(CF.far_field_velocity_response(h, r, 10.0))
        assert ratio > prev
        prev = ratio
    r = 0.05 * lam
    u = oracle.vertical_displacement(CF.uniform(h), r, 10.0, samples=6000)
    assert abs(1j * 2 * math.pi * 10 * u) / abs(CF.far_field_velocity_response(h, r, 10.0)) > 2


def test_dunkin_matches_direct_in_guarded_band(oracle, gfk):
    """Where the reference answers, both formulations give one bank to the
    1e-6 parity bar. They differ at ~1e-7, concentrated in the lowest bins,
    where k/k_body reaches ~1e3 and the direct eigenbasis loses digits
    (fk_test.go:48-57); the Dunkin values are the ones that match the
    high-precision evaluation there."""
    wl = gfk.workloads.single_soil()
    st = [tuple(l[:5]) + (0.0,) for l in [(x.thickness, x.vp, x.vs, x.density, x.qs) for x in wl.stack]]
    freqs = wl.freqs[wl.freqs <= 160][::40]
    a, sa = oracle.bank_spectra(st, wl.ranges[::8], freqs, samples=1024, kmax=wl.kmax, formulation=0)
    b, sb = oracle.bank_spectra(st, wl.ranges[::8], freqs, samples=1024, kmax=wl.kmax, formulation=1)
    assert (sa == 0).all() and (sb == 0).all()
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-6


def test_layered_causality_known_answers(oracle):
    """TestLayeredResponseHasNoPrecursor (internal/fk/causality_test.go:45-141):
    the oracle's reference-direct spectra of the 2 m layer over a half-space,
    shaped and transformed as the reference's test does, reproduce the logged
    peak times, precursor and negative-time values to their printed digits
    (docs/validation-report.md:278-280) — a pin on layered output."""
    import causality_case as CC
    m = oracle.OracleMedium(CC.STACK, default_q=CC.DEFAULT_Q)
    _, freqs = CC.bins()
    spectra, status = oracle.bank_spectra(m, CC.RANGES, freqs)
    assert (status == 0).all()
    CC.check_against_logged(CC.metrics(spectra), KA["causality_precursor"])


def test_split_sum_restatement_on_the_oracle_integrand(oracle, gfk):
    """The tensor-core sum's definition (oracle/split_oracle.py: one rounding to
    28 bits per operand, balanced base-128 digits, exact level sums up to
    s + t = 3) on the graded soil's own integrand from the oracle: the digits
    rebuild their integers exactly, every sum stays inside the rigorous bound
    K 2^(e_a + e_b - 27), and the whole result is within the 1e-6 bar of the
    FP64 sum (fk.go:534-546 with the oracle's J0)."""
    import split_oracle as S
    from conftest import as_tuples, rel_l2
    rng = np.random.default_rng(5)
    lim = 127 * 2 ** 21  # |x 2^(28 - e)| <= 127/128 2^28
    n = np.concatenate([np.array([0, 1, -1, 63, 64, -64, -65, lim, -lim, lim - 1, 1 - lim]),
                        rng.integers(-lim, lim + 1, 20000)])
    d = S.digits(n)
    assert np.array_equal(d[0] * 2 ** 21 + d[1] * 2 ** 14 + d[2] * 2 ** 7 + d[3], n)
    assert all(((x >= -64) & (x < 64)).all() for x in d[1:]) and (np.abs(d[0]) <= 127).all()
    mx = np.array([1.0, 127 / 128, 0.5, 3.0, 1e-300, 7e12])
    e = S.exponent(mx)
    y = mx * (128 / 127)
    assert (np.ldexp(1.0, e) > y).all() and (np.ldexp(1.0, e - 1) <= y).all()  # e = ilogb(y) + 1
    assert S.exponent(0.0) == 0

    wl = gfk.workloads.graded_soil()
    st = as_tuples(wl.stack)
    nk = 2048
    dk = wl.kmax / nk
    k = np.arange(1, nk + 1) * dk
    freqs = wl.freqs[[64, 400, 800, 1200, 1600, 2040]]
    ranges = wl.ranges[::32]
    vs_min = min(l[2] for l in st)
    rem = np.empty((len(freqs), nk), dtype=complex)
    for i, f in enumerate(freqs):
        kfar = max(200 * 2 * math.pi * f / vs_min, 400 / ranges.min())
        c = oracle.static_coefficient(st, f, kfar, oracle.DUNKIN, wl.omega_imag)
        u = np.array([oracle.surface_response(st, kk, f, oracle.DUNKIN, wl.omega_imag) for kk in k])
        rem[i] = k * u - c
    w = np.array([[oracle.j0(kk * r) for r in ranges] for kk in k]) * dk
    w[-1] *= 0.5
    exact = rem @ w
    got = S.split_sum(rem, w, dk)
    for part in (np.real, np.imag):
        bound = S.error_bound(part(rem), dk, nk)[:, None]
        assert (np.abs(part(got) - part(exact)) <= bound).all()
    # heavy cancellation: |sum| far below sum |terms| (the reason 28 bits are needed)
    assert (np.abs(rem) @ np.abs(w) / np.abs(exact)).max() > 100
    assert rel_l2(got, exact) < 1e-6
