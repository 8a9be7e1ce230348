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
