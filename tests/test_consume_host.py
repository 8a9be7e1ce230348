"""Host checks of the bank-consumption oracle (oracle/bank_oracle.py) on the
reference's conformance banks: the tables reproduce every stored value, the
unwrapped phase steps stay within half a cycle, and the impulse response
equals a direct inverse transform of the interpolated spectrum. No GPU."""
import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import bank_oracle as BO  # noqa: E402


@pytest.fixture(scope="module")
def pkg():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    return g.load_package()


@pytest.mark.parametrize("name", ["python_written.bank", "go_written.bank"])
def test_tables_reproduce_grid_values(pkg, name):
    b = pkg.open_bank(ROOT / "tests" / "golden" / name)
    lm, ph = BO.prepare(b.data)
    v = b.data[..., 0].astype(np.float64) + 1j * b.data[..., 1].astype(np.float64)
    nz = np.abs(v) > 0
    rec = np.exp(lm) * np.exp(1j * ph)
    assert np.allclose(rec[nz], v[nz], rtol=1e-12, atol=0)
    assert (lm[~nz] == BO.NEG_INF).all()
    assert (np.abs(np.diff(ph, axis=0)) <= math.pi + 1e-12).all()
    grid = (b.header.ranges.min_m, b.header.ranges.max_m)
    for i in range(b.header.ranges.count):
        for k in range(b.header.bins()):
            assert abs(BO.response((lm, ph), grid, b.header.ranges.at(i), k) - v[i, k]) <= 1e-12 * abs(v[i, k])


def test_bracket_edges():
    assert BO.bracket(1.0, 1.0, 4.0, 7) == (0, 0.0)
    assert BO.bracket(4.0, 1.0, 4.0, 7) == (5, 1.0)
    lo, frac = BO.bracket(2.25, 1.0, 4.0, 7)
    assert lo == 2 and abs(frac - 0.5) < 1e-12
    with pytest.raises(ValueError):
        BO.bracket(4.5, 1.0, 4.0, 7)


def test_impulse_response_is_inverse_of_tapered_spectrum(pkg):
    b = pkg.open_bank(ROOT / "tests" / "golden" / "python_written.bank")
    h = b.header
    n, fs, r = h.samples, h.sample_rate_hz, 2.25
    got = BO.impulse_responses(b.data, (h.ranges.min_m, h.ranges.max_m), fs, n, [r], 20)[0]
    lm, ph = BO.prepare(b.data)
    f = np.arange(n // 2 + 1) * fs / n
    c = np.array([BO.response((lm, ph), (h.ranges.min_m, h.ranges.max_m), r, k) for k in range(n // 2 + 1)])
    c = c * 2j * np.pi * f
    c[0] = 0
    w = np.where(f > 0.8 * fs / 2, 0.5 * (1 + np.cos(np.pi * (f - 0.8 * fs / 2) / (0.2 * fs / 2))), 1.0)
    want = np.fft.irfft(c * w, n)[:20]
    assert np.allclose(got, want, rtol=1e-12, atol=1e-18)
