"""Closed-form comparators the reference's fk tests use, restated in Python.

TEST INFRASTRUCTURE ONLY (the checker, never the product):
  - soil.HalfSpace presets, PoissonRatio, RayleighVelocity
    (internal/soil/soil.go:46-66, 103-106, 136-164)
  - green.HalfSpaceGF far-field Rayleigh velocity response
    (internal/green/green.go:58-125, 130-145, 169-266)
  - the Boussinesq static coefficient (1-nu)/(2 pi mu) that
    internal/fk/fk_test.go:33-87 pins the wavenumber solve against.
"""
import cmath
import math

# (vp, vs, density, qs) — internal/soil/soil.go:46-60
DRY_SAND = (350.0, 150.0, 1600.0, 20.0)
LOAM = (500.0, 200.0, 1700.0, 25.0)
FIRM_SOIL = (750.0, 300.0, 1900.0, 40.0)
WEATHERED_ROCK = (1800.0, 800.0, 2300.0, 80.0)


def uniform(h, qs=None):
    """layer.Uniform (internal/layer/layer.go:45-47) as an oracle layer list."""
    vp, vs, rho, q = h
    return [(0.0, vp, vs, rho, q if qs is None else qs, 0.0)]


def poisson_ratio(h):
    vp, vs = h[0], h[1]
    return (vp * vp - 2 * vs * vs) / (2 * (vp * vp - vs * vs))


def shear_modulus(h):
    return h[2] * h[1] * h[1]


def boussinesq_coefficient(h):
    """(1 - nu) / (2 pi mu): the large-k limit of k*u (fk_test.go:41)."""
    return (1 - poisson_ratio(h)) / (2 * math.pi * shear_modulus(h))


def rayleigh_velocity(h):
    """Bisection on the irrational Rayleigh equation (soil.go:136-164)."""
    vp, vs = h[0], h[1]
    k2 = (vs / vp) ** 2

    def f(x):
        return (2 - x) ** 2 - 4 * math.sqrt(1 - x) * math.sqrt(1 - x * k2)

    lo, hi = 1e-9, 1.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mid == lo or mid == hi:
            break
        if f(mid) < 0:
            lo = mid
        else:
            hi = mid
    return math.sqrt(0.5 * (lo + hi)) * vs


def far_field_velocity_response(h, r, f, ref_freq=30.0):
    """green.HalfSpaceGF.VelocityResponse (green.go:218-266), (m/s)/N."""
    vp, vs, rho, qs = h
    cr = rayleigh_velocity(h)
    gam = math.atan(1 / qs) / math.pi
    c = cr * (f / ref_freq) ** gam
    c0 = cr * math.cos(math.pi * gam / 2)
    omega = 2 * math.pi * f
    mag = omega / c0 * (f / ref_freq) ** (-gam)
    kc = mag * cmath.exp(complex(0, -math.pi * gam / 2))
    # eigenfunctions (green.go:58-80) at the elastic Rayleigh velocity
    k = omega / cr
    q = k * math.sqrt(1 - cr * cr / (vp * vp))
    s = k * math.sqrt(1 - cr * cr / (vs * vs))
    k2, s2 = k * k, s * s
    xq, xs = k, -2 * k * q * s / (k2 + s2)
    zq, zs = -q, 2 * k2 * q / (k2 + s2)

    def sq(a, b):
        return a * a / (2 * q) + 2 * a * b / (q + s) + b * b / (2 * s)

    i1 = 0.5 * rho * (sq(xq, xs) + sq(zq, zs))
    uz = zq + zs
    amp = uz * uz / (8 * c * c * i1) * math.sqrt(2 / (math.pi * kc.real * r))
    prop = cmath.exp(complex(0, -math.pi / 4) - 1j * kc * r)
    return complex(0, omega) * amp * prop
