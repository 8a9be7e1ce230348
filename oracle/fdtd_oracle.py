"""CPU oracle (test infrastructure only) for the finite-difference validator.

A numpy restatement of internal/fdtd (fdtd.go:45-345, model.go:30-246,
pml.go:30-70, run.go:78-127): the same grid, materials, C-PML profiles and
per-cell updates, each phase vectorised over the grid (every phase reads only
the previous phase's fields, so the order of cells does not matter).
Nothing in the product imports this file.
"""
import cmath
import math

import numpy as np


class SLS:
    def __init__(self, tau_sigma=0.0, tau_eps=0.0):
        self.ts, self.te = tau_sigma, tau_eps

    @staticmethod
    def fit(q, f0):
        w0 = 2 * math.pi * f0
        root = math.sqrt(1 + 1 / (q * q))
        return SLS((root - 1 / q) / w0, (root + 1 / q) / w0)

    def lossy(self):
        return self.te > self.ts

    def delta(self):
        return self.te / self.ts - 1

    def modulus(self, f):
        w = 2j * math.pi * f
        return (1 + w * self.te) / (1 + w * self.ts)

    def relaxed_velocity(self, v, fref):
        return v * (1 / cmath.sqrt(self.modulus(fref))).real


def ricker(peak, f0, dt, n):
    """fdtd.Ricker (run.go:14-27)."""
    t0 = 1.5 / f0
    a = math.pi * math.pi * f0 * f0
    tau = np.arange(n) * dt - t0
    return peak * (1 - 2 * a * tau * tau) * np.exp(-a * tau * tau)


def _profile(n, h, offset, inner, thickness, vmax, refl, dominant, dt):
    a, b, first = np.zeros(n), np.ones(n), n
    if thickness <= 0:
        return a, b, first
    d0 = -3 * vmax * math.log(refl) / (2 * thickness)
    amax = math.pi * dominant
    for i in range(n):
        s = (i + offset) * h - inner
        if s <= 0:
            continue
        x = min(s / thickness, 1.0)
        d = d0 * x ** 2
        alpha = amax * (1 - x)
        if d + alpha <= 0:
            continue
        bb = math.exp(-(d + alpha) * dt)
        a[i] = d * (bb - 1) / (d + alpha)
        b[i] = bb
        first = min(first, i)
    return a, b, first


class Sim:
    """stack: [(thickness, vp, vs, density)], last = half-space."""

    def __init__(self, stack, sls=None, ref_freq=30.0, max_range=10.0, depth=8.0, spacing=0.25, pml_cells=20,
                 pml_reflection=1e-4, dominant_freq=0.0, courant=0.5):
        self.stack, self.sls, self.fref = stack, sls or SLS(), ref_freq
        h = spacing
        self.h, self.max_range, self.depth = h, max_range, depth
        self.nr = int(round(max_range / h)) + 1 + pml_cells
        self.nz = int(round(depth / h)) + 1 + pml_cells
        lossy = self.sls.lossy()
        vmax = 0.0
        for l in stack:
            v = l[1]
            if lossy:
                v = self.sls.relaxed_velocity(v, ref_freq) * math.sqrt(1 + self.sls.delta())
            vmax = max(vmax, v)
        self.dt = courant * (h / (vmax * math.sqrt(2)))
        if dominant_freq > 0:
            dom = dominant_freq
        else:
            v = min(l[2] for l in stack)
            if lossy:
                v = self.sls.relaxed_velocity(v, ref_freq)
            dom = v / (20 * h)
        nz, nr = self.nz, self.nr
        rho, lam, mu = np.zeros(nz), np.zeros(nz), np.zeros(nz)
        for j in range(nz):
            z, top, l = j * h, 0.0, stack[-1]
            for ll in stack[:-1]:
                top += ll[0]
                if z < top:
                    l = ll
                    break
            r, vp, vs = l[3], l[1], l[2]
            if lossy:
                cp, cs = self.sls.relaxed_velocity(vp, ref_freq), self.sls.relaxed_velocity(vs, ref_freq)
                mp, ms = r * cp * cp * (1 + self.sls.delta()), r * cs * cs * (1 + self.sls.delta())
            else:
                mp, ms = r * vp * vp, r * vs * vs
            rho[j], mu[j], lam[j] = r, ms, mp - 2 * ms
        k = np.minimum(np.arange(nz) + 1, nz - 1)
        self.rho, self.lam, self.mu = rho, lam, mu
        self.rhoZ = 0.5 * (rho + rho[k])
        self.muZ = np.where((mu <= 0) | (mu[k] <= 0), 0.0, 2 * mu * mu[k] / np.where(mu + mu[k] == 0, 1, mu + mu[k]))
        th = pml_cells * h
        self.pRi = _profile(nr, h, 0, max_range, th, vmax, pml_reflection, dom, self.dt)
        self.pRh = _profile(nr, h, 0.5, max_range, th, vmax, pml_reflection, dom, self.dt)
        self.pZi = _profile(nz, h, 0, depth, th, vmax, pml_reflection, dom, self.dt)
        self.pZh = _profile(nz, h, 0.5, depth, th, vmax, pml_reflection, dom, self.dt)
        self.lossy = lossy
        if lossy:
            tau, kappa = self.sls.ts, self.sls.delta() / (1 + self.sls.delta())
            den = 1 + self.dt / (2 * tau)
            self.decay, self.drive = (1 - self.dt / (2 * tau)) / den, (self.dt * kappa / tau) / den
        z = lambda: np.zeros((nz, nr))
        self.vr, self.vz, self.trr, self.tqq, self.tzz, self.trz = z(), z(), z(), z(), z(), z()
        self.rrr, self.rqq, self.rzz, self.rrz = z(), z(), z(), z()
        self.psi = {name: z() for name in ("TrrR", "TrzZ", "TrzR", "TzzZ", "VrR", "VzZ", "VzR", "VrZ")}
        self.src_area = math.pi * h * h / 4
        self.step = 0
        self.force = np.zeros(0)

    def _cpml(self, name, prof, axis, deriv, sl):
        """psi = b psi + a deriv on the cells of slice sl whose index along axis is >= first."""
        a, b, first = prof
        idx = np.arange(deriv.shape[axis])
        full_idx = idx + (sl[axis].start or 0)
        mask = full_idx >= first
        shape = [1, 1]
        shape[axis] = -1
        av, bv, m = a[full_idx].reshape(shape), b[full_idx].reshape(shape), mask.reshape(shape)
        psi = self.psi[name][sl]
        new = bv * psi + av * deriv
        new = np.where(m, new, psi)
        self.psi[name][sl] = new
        return deriv + np.where(m, new, 0.0)

    def _relax(self, r, e):
        nxt = self.decay * r - self.drive * e
        avg = 0.5 * (r + nxt)
        return nxt, avg

    def force_at(self, n):
        return self.force[n] if 0 <= n < len(self.force) else 0.0

    def do_step(self):
        nr, nz, h, dt = self.nr, self.nz, self.h, self.dt
        self.tzz[0, 0] = -self.force_at(self.step) / self.src_area
        trr, tqq, tzz, trz = self.trr, self.tqq, self.tzz, self.trz
        # radial velocity, cells [0, nz-1) x [0, nr-1)
        S = (slice(0, nz - 1), slice(0, nr - 1))
        i = np.arange(nr - 1)[None, :]
        dtrr = (trr[:nz - 1, 1:] - trr[:nz - 1, :nr - 1]) / h
        dtrr = self._cpml("TrrR", self.pRh, 1, dtrr, S)
        dtrz = np.empty((nz - 1, nr - 1))
        dtrz[0] = 2 * trz[0, :nr - 1] / h
        dtrz[1:] = (trz[1:nz - 1, :nr - 1] - trz[0:nz - 2, :nr - 1]) / h
        dtrz = self._cpml("TrzZ", self.pZi, 0, dtrz, S)
        hoop = 0.5 * ((trr[:nz - 1, :nr - 1] - tqq[:nz - 1, :nr - 1]) + (trr[:nz - 1, 1:] - tqq[:nz - 1, 1:])) / \
            ((i + 0.5) * h)
        self.vr[S] += dt / self.rho[:nz - 1, None] * (dtrr + dtrz + hoop)
        # vertical velocity
        dtzz = (tzz[1:nz, :nr - 1] - tzz[:nz - 1, :nr - 1]) / h
        dtzz = self._cpml("TzzZ", self.pZh, 0, dtzz, S)
        radial = np.empty((nz - 1, nr - 1))
        radial[:, 0] = 4 * trz[:nz - 1, 0] / h
        d = (trz[:nz - 1, 1:nr - 1] - trz[:nz - 1, 0:nr - 2]) / h
        d = self._cpml("TrzR", self.pRi, 1, d, (slice(0, nz - 1), slice(1, nr - 1)))
        ii = np.arange(1, nr - 1)[None, :]
        radial[:, 1:] = d + 0.5 * (trz[:nz - 1, 1:nr - 1] + trz[:nz - 1, 0:nr - 2]) / (ii * h)
        self.vz[S] += dt / self.rhoZ[:nz - 1, None] * (dtzz + radial)
        # normal stresses, all cells
        vr, vz = self.vr, self.vz
        dTdt = (self.force_at(self.step + 1) - self.force_at(self.step)) / dt
        dvr = np.empty((nz, nr))
        vrr = np.empty((nz, nr))
        dvr[:, 0] = 2 * vr[:, 0] / h
        vrr[:, 0] = dvr[:, 0]
        dvr[:, 1:] = (vr[:, 1:] - vr[:, :nr - 1]) / h
        vrr[:, 1:] = 0.5 * (vr[:, 1:] + vr[:, :nr - 1]) / (np.arange(1, nr)[None, :] * h)
        dvr = self._cpml("VrR", self.pRi, 1, dvr, (slice(0, nz), slice(0, nr)))
        lam, mu = self.lam[:, None], self.mu[:, None]
        l2m = lam + 2 * mu
        dvz = np.empty((nz, nr))
        applied = np.zeros(nr)
        applied[0] = dTdt
        dvz[0] = (applied - self.lam[0] * (dvr[0] + vrr[0])) / (self.lam[0] + 2 * self.mu[0])
        dz_ = (vz[1:] - vz[:nz - 1]) / h
        dvz[1:] = self._cpml("VzZ", self.pZi, 0, dz_, (slice(1, nz), slice(0, nr)))
        err = l2m * dvr + lam * (vrr + dvz)
        eqq = lam * (dvr + dvz) + l2m * vrr
        ezz = lam * (dvr + vrr) + l2m * dvz
        if self.lossy:
            self.rrr, a1 = self._relax(self.rrr, err)
            self.rqq, a2 = self._relax(self.rqq, eqq)
            trr += dt * (err + a1)
            tqq += dt * (eqq + a2)
            rzz_new, a3 = self._relax(self.rzz[1:], ezz[1:])
            self.rzz[1:] = rzz_new
            tzz[1:] += dt * (ezz[1:] + a3)
        else:
            trr += dt * err
            tqq += dt * eqq
            tzz[1:] += dt * ezz[1:]
        # shear stress
        dvzdr = (vz[:nz - 1, 1:] - vz[:nz - 1, :nr - 1]) / h
        dvzdr = self._cpml("VzR", self.pRh, 1, dvzdr, S)
        dvrdz = (vr[1:, :nr - 1] - vr[:nz - 1, :nr - 1]) / h
        dvrdz = self._cpml("VrZ", self.pZh, 0, dvrdz, S)
        e = self.muZ[:nz - 1, None] * (dvzdr + dvrdz)
        if self.lossy:
            rrz_new, a4 = self._relax(self.rrz[S], e)
            self.rrz[S] = rrz_new
            trz[S] += dt * (e + a4)
        else:
            trz[S] += dt * e
        self.step += 1

    def surface_velocity(self, i):
        h = self.h
        if i == 0:
            dvr = 2 * self.vr[0, 0] / h
            vrr = dvr
        else:
            dvr = (self.vr[0, i] - self.vr[0, i - 1]) / h
            vrr = 0.5 * (self.vr[0, i] + self.vr[0, i - 1]) / (i * h)
        lam, mu = self.lam[0], self.mu[0]
        dvz = -lam / (lam + 2 * mu) * (dvr + vrr)
        return self.vz[0, i] - 0.5 * h * dvz

    def column(self, r):
        i = int(math.floor(r / self.h + 0.5))
        return max(0, min(i, self.nr - 2))


def run(sim, force, ranges, steps):
    """fdtd.Run: traces [len(ranges)][steps]."""
    sim.force = np.asarray(force, dtype=np.float64)
    cols = [sim.column(r) for r in ranges]
    out = np.zeros((len(ranges), steps))
    for n in range(steps):
        sim.do_step()
        for q, c in enumerate(cols):
            out[q, n] = sim.surface_velocity(c)
    return out
