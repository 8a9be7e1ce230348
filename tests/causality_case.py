"""The reference's layered causality check (internal/fk/causality_test.go:45-141),
restated so that any solver's spectra can be put through it.

A 2 m soft layer (Vp 350, Vs 140, rho 1600, Qs 20) over a half-space (800, 320,
2000, 20), Medium.DefaultQ 20, receivers at 10 and 20 m. Bins k df up to
120 Hz of a 4096-point record at fs = 400 Hz, each VerticalDisplacementMulti
with the default Integration (GridFor's own grid per frequency). The spectra
are shaped by a 20 Hz Ricker delayed by 1.5/f0, turned into velocity (i 2 pi f)
and scaled by fs (causality_test.go:64-84); the trace is dsp.IRFFT (an inverse
real transform scaled 1/n, internal/dsp/dsp.go:42-50). The reference's run
logged the peak times, the largest sample before the first possible arrival
and the largest at negative time (docs/validation-report.md:278-280).
"""
import math

import numpy as np

FS, N, BAND, F0 = 400.0, 4096, 120.0, 20.0
STACK = [(2.0, 350.0, 140.0, 1600.0, 20.0, 0.0), (0.0, 800.0, 320.0, 2000.0, 20.0, 0.0)]
DEFAULT_Q = 20.0
RANGES = np.array([10.0, 20.0])
# real(complexVelocity(800, 2.25 * 20, 120 Hz)) (causality_test.go:86-93)
FASTEST_MPS = 807.8


def bins():
    """Bin indices k = 1.. with k df <= BAND, and their frequencies."""
    df = FS / N
    ks = np.arange(1, N // 2 + 1)
    ks = ks[ks * df <= BAND]
    return ks, ks * df


def metrics(spectra):
    """spectra: [nbins][2] complex displacement per newton at RANGES. Returns
    one dict per range: peak time (s), first possible arrival (s), the largest
    |sample| / peak before it and the largest at negative time."""
    ks, freqs = bins()
    fr = freqs / F0
    mag = 2 / math.sqrt(math.pi) * fr * fr * np.exp(-fr * fr) / F0
    wavelet = mag * np.exp(1j * (-2 * math.pi * freqs * 1.5 / F0))
    out = []
    for i, r in enumerate(RANGES):
        coeff = np.zeros(N // 2 + 1, dtype=np.complex128)
        coeff[ks] = 1j * 2 * math.pi * freqs * spectra[:, i] * wavelet * FS
        trace = np.fft.irfft(coeff, N)
        a = np.abs(trace)
        peak = a.max()
        arrival = int(math.floor(r / FASTEST_MPS * FS))
        early = float((a[:max(arrival - 1, 0)] / peak).max())
        back = float(max(a[N - b] / peak for b in range(1, N // 4)))
        out.append({"range_m": float(r), "peak_s": int(a.argmax()) / FS, "arrival_s": arrival / FS,
                    "early": early, "negative_time": back})
    return out


def check_against_logged(got, logged):
    """The logged values are printed to three significant digits; the peak
    and arrival times are sample-exact."""
    assert len(got) == len(logged)
    for g, want in zip(got, logged):
        assert g["range_m"] == want["range_m"]
        assert g["peak_s"] == {10.0: 0.1850, 20.0: 0.3150}[g["range_m"]]
        assert g["arrival_s"] == {10.0: 0.0100, 20.0: 0.0225}[g["range_m"]]
        for key in ("early", "negative_time"):
            assert float(f"{g[key]:.2e}") == want[key], (g["range_m"], key, g[key], want[key])
        # the reference's own bounds (causality_test.go:129-139)
        assert g["early"] < 1e-4 and g["negative_time"] < 1e-4
