"""Host-side checks of the FDTD validator's set-up (no GPU): gfk_fdtd_grid
against the numpy restatement (time step and cell counts of fdtd.New for
elastic and lossy models), its argument errors, and the Ricker wavelet
against its closed-form spectrum (internal/fdtd/run.go:14-44)."""
import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
import fdtd_oracle as FO  # noqa: E402

LAYERED = [(2.0, 350.0, 140.0, 1600.0), (0.0, 800.0, 320.0, 2000.0)]


@pytest.fixture(scope="module")
def pkg():
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as g
    return g.load_package()


def stack(pkg, layers):
    return pkg.Stack([pkg.Layer(h, vp, vs, rho, 0, 0) for (h, vp, vs, rho) in layers])


@pytest.mark.parametrize("lossy,courant,spacing", [(False, 0.0, 0.2), (True, 0.0, 0.1), (True, 0.4, 0.0555)])
def test_grid_matches_oracle(pkg, lossy, courant, spacing):
    sls = pkg.SLS.fit(25, 30) if lossy else None
    md = pkg.fdtd.Model(stack(pkg, LAYERED), relax=sls, ref_freq=30, max_range=16, depth=10, spacing=spacing,
                        courant=courant)
    dt, nr, nz = md.grid()
    sim = FO.Sim(LAYERED, FO.SLS.fit(25, 30) if lossy else None, 30, 16, 10, spacing,
                 courant=courant if courant > 0 else 0.5)
    assert (nr, nz) == (sim.nr, sim.nz)
    assert dt == pytest.approx(sim.dt, rel=1e-15)


def test_grid_rejects_bad_models(pkg):
    st = stack(pkg, LAYERED)
    for kw in (dict(spacing=0.0, max_range=5, depth=5), dict(spacing=0.1, max_range=0, depth=5),
               dict(spacing=0.1, max_range=5, depth=-1)):
        with pytest.raises(pkg.FkError) as e:
            pkg.fdtd.Model(st, **kw).grid()
        assert e.value.status == pkg._native.EARG
    with pytest.raises(pkg.FkError) as e:
        pkg.fdtd.Model(st, relax=pkg.SLS(0.002, 0.001), spacing=0.1, max_range=5, depth=5).grid()
    assert e.value.status == pkg._native.EARG
    bad = pkg.Stack([pkg.Layer(3, 100, 200, 1600, 0, 0), pkg.Layer(0, 900, 400, 2000, 0, 0)])
    with pytest.raises(pkg.FkError) as e:
        pkg.fdtd.Model(bad, spacing=0.1, max_range=5, depth=5).grid()
    assert e.value.status == pkg._native.ESTACK


def test_ricker_spectrum_is_the_wavelets_transform(pkg):
    dt, n, f0 = 1e-4, 1 << 15, 25.0
    w = pkg.fdtd.ricker(1.0, f0, dt, n)
    assert w.max() == pytest.approx(1.0, rel=1e-3)
    spec = np.fft.rfft(w) * dt
    f = np.fft.rfftfreq(n, dt)
    band = (f > 2) & (f < 90)
    want = pkg.fdtd.ricker_spectrum(1.0, f0, f[band])
    assert np.abs(spec[band] - want).max() < 1e-6 * np.abs(want).max()


def test_spacing_for(pkg):
    md = pkg.fdtd.Model(stack(pkg, LAYERED))
    assert md.spacing_for(100.0, 10.0) == pytest.approx(140.0 / 1000.0)
    md.relax = pkg.SLS.fit(25, 30)
    h = md.spacing_for(100.0, 10.0)
    assert 0.13 < h < 0.14
    with pytest.raises(pkg.FkError):
        md.spacing_for(0.0, 10.0)
