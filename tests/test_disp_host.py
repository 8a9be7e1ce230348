"""The dispersion oracle (oracle/disp_oracle.py, a restatement of
internal/propmat + internal/disp) against the reference's disba goldens and
the closed-form Rayleigh velocity. No GPU."""
import json
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import disp_oracle as D  # noqa: E402

GOLDEN = sorted((ROOT / "tests" / "golden" / "dispersion").glob("*.json"))


def load(p):
    g = json.loads(p.read_text())
    st = [(l["thickness_m"], l["vp_mps"], l["vs_mps"], l["density_kgm3"]) for l in g["layers"]]
    return g, st


def test_four_goldens_present():
    assert len(GOLDEN) == 4


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_disba(path):
    g, st = load(path)
    for ms, want in g["modes"].items():
        fr, pv = want["frequency_hz"], want["phase_velocity_mps"]
        for i in (0, len(fr) // 2, len(fr) - 1):
            got = D.mode(st, fr[i], int(ms))
            assert got is not None and abs(got / pv[i] - 1) < 2e-6, (ms, fr[i], got, pv[i])


def test_homogeneous_is_rayleigh_velocity():
    st = [(0.0, 500.0, 200.0, 1700.0)]  # soil.Loam
    want = D.rayleigh_velocity(500.0, 200.0)
    for f in (2.0, 20.0, 120.0):
        assert abs(D.mode(st, f, 0) / want - 1) < 1e-6


def _speculative_bisect(f, lo, hi, flo, tol, depth=3, cap=200):
    """The root phase of csrc/gfk_disp.cu's k_modes, restated: per round the
    2^depth - 1 midpoints the next `depth` halvings could visit are evaluated
    (each bracket built by the same halvings), then the path the one-thread
    search takes is walked through them."""
    it = 0
    while True:
        vals = {}
        for h in range(1, 2 ** depth):
            d = h.bit_length() - 1
            nlo, nhi = lo, hi
            for sh in range(d - 1, -1, -1):
                mid = 0.5 * (nlo + nhi)
                if (h >> sh) & 1:
                    nlo = mid
                else:
                    nhi = mid
            vals[h] = f(0.5 * (nlo + nhi))
        h = 1
        for _ in range(depth):
            if it >= cap:
                return 0.5 * (lo + hi)
            mid = 0.5 * (lo + hi)
            if mid == lo or mid == hi or (hi - lo) < tol * mid:
                return mid
            it += 1
            v = vals[h]
            if v is None:
                return None
            if D._sign_change(flo, v):
                hi, h = mid, 2 * h
            else:
                lo, flo, h = mid, v, 2 * h + 1


def test_speculative_bisection_equals_sequential():
    """The GPU's several-steps-per-round bisection visits the same midpoints
    and takes the same decisions as disp.bisect (disp.go:194-217), so it
    returns the same double, with the stopping rules, the 200-step cap and
    undefined values inside the bracket included."""
    import math
    import random
    rng = random.Random(7)
    cases = 0
    for _ in range(400):
        root = rng.uniform(100.0, 500.0)
        scale = rng.choice([1e-3, 1.0, 1e6])
        hole = rng.random() < 0.2
        hole_at = root + rng.uniform(-2.0, 2.0)

        def f(c, root=root, scale=scale, hole=hole, hole_at=hole_at):
            if hole and abs(c - hole_at) < 0.05:
                return None  # undefined, as the secular function can be
            return scale * math.tanh(c - root) + 1e-18 * math.sin(c)

        lo = root - rng.uniform(0.01, 3.0)
        hi = root + rng.uniform(0.01, 3.0)
        flo = f(lo)
        if flo is None or f(hi) is None:
            continue
        for tol in (1e-10, 1e-14, 0.0):  # 0: runs into the 200-step cap or mid == lo / hi
            want = D.bisect(f, lo, hi, tol)
            got = _speculative_bisect(f, lo, hi, flo, tol)
            assert got == want, (root, lo, hi, tol, got, want)
            cases += 1
    assert cases > 900
