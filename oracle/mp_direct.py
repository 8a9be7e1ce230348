"""High-precision (mpmath) restatement of the reference's SurfaceResponse.

TEST INFRASTRUCTURE ONLY. The reference's direct algorithm
(internal/fk/fk.go:119-327: eigenvectors of fk.go:138-168, propagators
E diag(e^(lambda k h)) E^-1, the 4x4 surface solve of fk.go:299-326) evaluated
with enough digits that its loss of precision at large k*h and large k/k_body
cannot reach the result. It is the ground truth both formulations are checked
against. Layers are (thickness, vp, vs, rho, qs, qp); qp_mode "reference"
uses Qp = 2.25 Qs (fk.go:122), "layer" uses the layer's qp when > 0.
"""
import math

import mpmath as mp


def complex_velocity(v, q, f, ref_freq=30.0, omega_imag=0.0):
    """fk.go:96-110 at the complex frequency 2 pi f - i omega_imag."""
    if q <= 0 or f <= 0:
        return mp.mpc(v)
    gam = mp.atan(1 / mp.mpf(q)) / mp.pi
    c0 = v * mp.cos(mp.pi * gam / 2)
    wc = mp.mpc(2 * mp.pi * f, -omega_imag)
    return c0 * mp.exp(gam * mp.log(mp.mpc(0, 1) * wc / (2 * mp.pi * ref_freq)))


def surface_response(stack, k, f, omega_imag=0.0, qp_mode="reference", ref_freq=30.0, default_q=30.0, dps=None):
    """u_z(k, f) per newton (fk.go:276-327) as a Python complex."""
    tot = sum(k * l[0] for l in stack[:-1])
    with mp.workdps(dps or int(40 + 2 * tot / 2.3)):
        muref = max(mp.mpf(l[3]) * mp.mpf(l[2]) ** 2 for l in stack)
        wc = mp.mpc(2 * mp.pi * f, -omega_imag)
        kk = mp.mpf(k)

        def eig(l):
            q = l[4] if l[4] > 0 else default_q
            qp = l[5] if (qp_mode == "layer" and l[5] > 0) else 2.25 * q
            a = complex_velocity(l[1], qp, f, ref_freq, omega_imag)
            b = complex_velocity(l[2], q, f, ref_freq, omega_imag)
            rho = mp.mpf(l[3])
            mu = rho * b * b
            w2 = wc * wc
            ra = mp.sqrt(1 - w2 / (kk * kk * a * a))
            rb = mp.sqrt(1 - w2 / (kk * kk * b * b))
            if mp.re(ra) < 0:
                ra = -ra
            if mp.re(rb) < 0:
                rb = -rb
            rc2 = rho * w2 / (kk * kk)
            pd = [1, -ra, -2 * mu / muref * ra, (2 * mu - rc2) / muref]
            pu = [1, ra, 2 * mu / muref * ra, (2 * mu - rc2) / muref]
            sd = [rb, -1, (rc2 - 2 * mu) / muref, 2 * mu / muref * rb]
            su = [-rb, -1, (rc2 - 2 * mu) / muref, -2 * mu / muref * rb]
            E = mp.matrix(4, 4)
            for i in range(4):
                E[i, 0], E[i, 1], E[i, 2], E[i, 3] = pd[i], sd[i], pu[i], su[i]
            return [-ra, -rb, ra, rb], E

        total = mp.eye(4)
        for l in stack[:-1]:
            lam, E = eig(l)
            D = mp.matrix(4, 4)
            for i in range(4):
                D[i, i] = mp.exp(lam[i] * kk * l[0])
            total = (E * D * E ** -1) * total
        _, E = eig(stack[-1])
        b4 = mp.mpc(0, -1) / (2 * mp.pi * muref * kk)
        A = mp.matrix(4, 4)
        rhs = mp.matrix(4, 1)
        for i in range(4):
            A[i, 0], A[i, 1] = total[i, 0], total[i, 1]
            A[i, 2], A[i, 3] = -E[i, 0], -E[i, 1]
            rhs[i] = -b4 * total[i, 3]
        x = mp.lu_solve(A, rhs)
        return complex(mp.mpc(0, -1) * x[1])
