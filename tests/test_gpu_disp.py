"""Dispersion curves on the GPU (gfk_dispersion_modes, gfk_secular) against
the reference's disba goldens at the reference's own tolerance (1e-4,
internal/disp/disp_test.go:41-79), against the CPU oracle's roots, and the
reference's property tests (disp_test.go:107-261)."""
import json
import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import disp_oracle as D  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = sorted((ROOT / "tests" / "golden" / "dispersion").glob("*.json"))


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


def stack_of(pkg, g):
    return pkg.Stack([pkg.Layer(l["thickness_m"], l["vp_mps"], l["vs_mps"], l["density_kgm3"], 0, 0)
                      for l in g["layers"]])


SOFT = [(3.0, 400.0, 160.0, 1600.0), (0.0, 900.0, 400.0, 2000.0)]


def soft(pkg):
    return pkg.Stack([pkg.Layer(h, vp, vs, rho, 20, 40) for (h, vp, vs, rho) in SOFT])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_matches_disba(pkg, eng, path):
    g = json.loads(path.read_text())
    st = stack_of(pkg, g)
    for ms, want in g["modes"].items():
        fr, pv = want["frequency_hz"], want["phase_velocity_mps"]
        got = pkg.disp.modes_many(st, fr, engine=eng)
        for f, w, all_ in zip(fr, pv, got):
            assert int(ms) < len(all_), f"mode {ms} at {f:.3f} Hz: disba {w:.2f} m/s, none found"
            assert abs(all_[int(ms)] / w - 1) < 1e-4, (ms, f, all_[int(ms)], w)
        lo, hi = pkg.disp.bounds(st)
        for all_ in got:
            assert all(lo < c < hi for c in all_) and all(b > a for a, b in zip(all_, all_[1:]))


def test_roots_match_oracle(pkg, eng):
    g = json.loads(GOLDEN[-1].read_text())
    layers = [(l["thickness_m"], l["vp_mps"], l["vs_mps"], l["density_kgm3"]) for l in g["layers"]]
    st = stack_of(pkg, g)
    freqs = [3.0, 25.0, 90.0]
    for f, got in zip(freqs, pkg.disp.modes_many(st, freqs, engine=eng)):
        want = D.modes(layers, f)
        assert len(got) == len(want)
        assert np.allclose(got, want, rtol=1e-9, atol=0)


def test_secular_matches_oracle(pkg, eng):
    g = json.loads(GOLDEN[-1].read_text())
    layers = [(l["thickness_m"], l["vp_mps"], l["vs_mps"], l["density_kgm3"]) for l in g["layers"]]
    st = stack_of(pkg, g)
    rng = np.random.default_rng(1)
    f = rng.uniform(1, 120, 40)
    c = rng.uniform(130, 1099, 40)
    v, ok = pkg.disp.secular_at_velocity(st, f, c, engine=eng)
    for i in range(40):
        w = D.secular_at_velocity(layers, f[i], c[i])
        assert ok[i] == (w is not None)
        if w is not None:
            assert abs(v[i] - w) <= 1e-9 * max(1.0, abs(w)), (f[i], c[i], v[i], w)
    _, ok2 = pkg.disp.secular_at_velocity(st, [10.0], [1100.0], engine=eng)  # at Vs of the half-space
    assert not ok2[0]


def test_homogeneous_does_not_disperse(pkg, eng):
    st = pkg.uniform(500.0, 200.0, 1700.0, 25.0)
    want = D.rayleigh_velocity(500.0, 200.0)
    for c in pkg.disp.modes_many(st, [2.0, 20.0, 120.0], engine=eng):
        assert abs(c[0] / want - 1) < 1e-6
    u = pkg.disp.group_velocity(st, 20.0, 0, engine=eng)
    assert abs(u / want - 1) < 1e-4


def test_soft_over_stiff_dispersion_cutoffs_group(pkg, eng):
    st = soft(pkg)
    freqs = [2, 5, 10, 20, 40, 80, 120]
    c0 = [m[0] for m in pkg.disp.modes_many(st, freqs, engine=eng)]
    assert all(b < a for a, b in zip(c0, c0[1:]))
    slow = D.rayleigh_velocity(400.0, 160.0)
    assert abs(c0[-1] - slow) / slow < 0.05
    with pytest.raises(pkg.FkError):
        pkg.disp.mode(st, 2.0, 1, engine=eng)
    pkg.disp.mode(st, 100.0, 1, engine=eng)
    curve = pkg.disp.phase_curve(st, freqs, 1, engine=eng)
    assert len(curve.frequency) == len(curve.phase_velocity) and 0 < len(curve.frequency) < len(freqs)
    for f in (10.0, 20.0, 40.0):
        c = pkg.disp.mode(st, f, 0, engine=eng)
        u = pkg.disp.group_velocity(st, f, 0, engine=eng)
        assert 0 < u < c


def test_rejects_bad_arguments(pkg, eng):
    st = pkg.uniform(500.0, 200.0, 1700.0, 25.0)
    with pytest.raises(pkg.FkError):
        pkg.disp.modes(st, 0.0, engine=eng)
    with pytest.raises(pkg.FkError):
        pkg.disp.mode(st, 20.0, -1, engine=eng)
    with pytest.raises(pkg.FkError):
        pkg.disp.mode(st, 20.0, 9, engine=eng)
    bad = pkg.Stack([pkg.Layer(3, 100, 200, 1600, 0, 0), pkg.Layer(0, 900, 400, 2000, 0, 0)])
    with pytest.raises(pkg.FkError) as e:
        pkg.disp.modes(bad, 20.0, engine=eng)
    assert e.value.status == pkg._native.ESTACK


def _sequential_roots(secular, lo, hi, samples, tol):
    """disp.Modes' one-thread search (internal/disp/disp.go:68-196, restated in
    oracle/disp_oracle.py): the scan's sign changes, then one bisection per
    bracket with the reference's stopping rules, over the given secular
    function (a callable on a list of velocities returning values and
    defined-flags)."""
    step = (hi * (1 - 1e-9) - lo) / samples
    cs = [lo] + [lo + i * step for i in range(1, samples + 1)]
    vals, ok = secular(cs)
    roots = []
    for i in range(1, samples + 1):
        if not (ok[i] and ok[i - 1] and D._sign_change(vals[i - 1], vals[i])):
            continue
        blo, bhi, flo = cs[i - 1], cs[i], vals[i - 1]
        root = None
        for it in range(201):
            mid = 0.5 * (blo + bhi)
            if it == 200 or mid == blo or mid == bhi or (bhi - blo) < tol * mid:
                root = mid
                break
            v, vok = secular([mid])
            if not vok[0]:
                break  # undefined inside the bracket: no root
            if D._sign_change(flo, v[0]):
                bhi = mid
            else:
                blo, flo = mid, v[0]
        if root is not None:
            roots.append(root)
    return roots


@pytest.mark.parametrize("tol", [0.0, 1e-300], ids=["default_tol", "to_the_last_bit"])
def test_roots_equal_sequential_search_exactly(pkg, eng, tol):
    """k_modes evaluates three bisection steps' midpoints at once and walks the
    path the one-thread search takes; its roots must be the sequential
    search's doubles exactly, when both use the GPU's own secular function
    (gfk_secular). With tolerance 1e-300 every bracket runs until its midpoint
    equals an end (~40 halvings)."""
    for path in GOLDEN:
        g = json.loads(path.read_text())
        st = stack_of(pkg, g)
        lo, hi = pkg.disp.bounds(st)
        for f in (4.0, 37.0, 110.0):
            def secular(cs, f=f):
                v, ok = pkg.disp.secular_at_velocity(st, [f] * len(cs), cs, engine=eng)
                return list(v), [bool(o) and math.isfinite(x) for o, x in zip(ok, v)]
            want = _sequential_roots(secular, lo, hi, 2000, tol if tol > 0 else 1e-10)
            got = pkg.disp.modes_many(st, [f], opt=pkg.disp.Search(0, tol), engine=eng)[0]
            assert got == want, (path.stem, f, got, want)
