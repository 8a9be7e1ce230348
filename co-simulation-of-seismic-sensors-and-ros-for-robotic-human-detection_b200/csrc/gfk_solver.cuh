// gfk_solver.cuh — the per-(f, k) layered boundary-value solve, as device code.
//
// Two formulations of the reference's Medium.SurfaceResponse
// (internal/fk/fk.go:276-327):
//   direct_u  — the reference algorithm restated: 4x4 complex eigenvector
//               propagators and a pivoted 4x4 surface solve (fk.go:138-327,
//               internal/fk/cmat.go:57-96).
//   dunkin_u  — the complex second-compound (minor) propagation of the
//               half-space's decaying 2-plane up to the surface, in closed form
//               with no k*h limit (design source internal/propmat/propmat.go:168-315),
//               started at the shallowest layer thick enough to isolate the
//               layers beneath it.
#pragma once
#include "gfk_math.cuh"

namespace gfk {

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kPi = 3.141592653589793238462643383280;
constexpr int kMaxLayers = 64;

// Per-(frequency, layer) constants, written once per build by the layer kernel.
// Dunkin:  c[0] = 1/alpha^2, c[1] = 1/beta^2, c[2] = beta^2/alpha^2, c[3] = rho beta^2/mu_ref
// direct:  c[0] = alpha,     c[1] = beta,     c[2] = mu = rho beta^2, c[3] = (rho, 0)
struct LayerC {
    cd c[4];
    double h;
    double pad;
};

// Layer description on the device (mirrors gfk_layer).
struct LayerP {
    double h, vp, vs, rho, qs, qp;
};

// One medium of a plan: fk.Medium's defaults plus what the kernels derive.
struct MediumP {
    double ref_freq, default_q, tau_sigma, tau_eps;
    double mu_ref;  // max rho Vs^2 (fk.go:216-222)
    int count;      // stack entries, the last one the half-space
    int sls;        // nonzero: SLS relaxation replaces constant Q
    int lp_off;     // first layer in the plan's LayerP table
    int pad;
};

// One frequency of a plan (a bank row).
struct FreqDesc {
    double freq;     // Hz
    double dk;       // wavenumber step; k_i = i dk, i = 1..nk
    double kfar;     // k of the static coefficient (fk.go:515-521); 0 skips the row
    int64_t off;     // integrand row offset within its chunk
    int64_t lc_off;  // first of the row's layer constants
    int nk;          // wavenumber samples
    int soil;        // index into the medium table
};

GFK_HD double q_of(const MediumP& m, const LayerP& l) {  // fk.go:67-75
    if (l.qs > 0) return l.qs;
    if (m.default_q > 0) return m.default_q;
    return 30.0;
}

GFK_HD double ref_freq(const MediumP& m) { return m.ref_freq > 0 ? m.ref_freq : 30.0; }

GFK_HD cd sls_modulus(const MediumP& m, cd w) {  // visco.go:78-81 at complex w
    cd iw = cmul_i(w);
    return (1.0 + iw * m.tau_eps) / (1.0 + iw * m.tau_sigma);
}

// Medium.complexVelocity (fk.go:96-110) at the complex frequency 2 pi f - i wi.
// Kjartansson c0 (i w_c / w_ref)^gamma on the principal branch; with wi = 0 the
// reference's own factorisation c0 (f/f_ref)^gamma e^(i pi gamma/2) is used.
GFK_HD cd complex_velocity(const MediumP& m, double v, double q, double f, double wi) {
    if (m.sls) {
        cd rel = 1.0 / csqrt_(sls_modulus(m, mk(kTwoPi * ref_freq(m))));
        double relaxed = v * rel.re;  // visco.go:100-102
        if (f <= 0) return mk(relaxed);
        return relaxed * csqrt_(sls_modulus(m, mk(kTwoPi * f, -wi)));  // visco.go:106-108
    }
    if (q <= 0 || f <= 0) return mk(v);
    double gam = atan(1.0 / q) / kPi;
    double c0 = v * cos(kPi * gam / 2);
    if (wi == 0.0) return (c0 * pow(f / ref_freq(m), gam)) * cexp_(mk(0.0, kPi * gam / 2));
    cd z = cmul_i(mk(kTwoPi * f, -wi)) / (kTwoPi * ref_freq(m));
    return c0 * cexp_(gam * clog_(z));
}

// ---------------------------------------------------------------- Dunkin --
//
// Minor order n <-> row pair: 0:(0,1) 1:(0,2) 2:(0,3) 3:(1,2) 4:(1,3) 5:(2,3)
// (propmat.go:168-174). Each layer's basis is F = [pd, g, pu, h]:
//   pd, pu = P eigenvectors (fk.go:158-159);  t = mu'(1 + rb^2)
//   g = (sd - rb pd)/eb = (0, -u1, -mu' x2,  mu' rb)
//   h = (su + rb pu)/eb = (0, -u1, -mu' x2, -mu' rb)
// with eb = c^2/beta^2 = 1 - rb^2, u1 = (1 - ra rb)/eb, x2 = (1 + rb^2 - 2 ra rb)/eb,
// r2 = ((1 + rb^2)^2 - 4 ra rb)/eb. In F the system matrix is block upper
// triangular, T = [[-ra, tau, 0, 0], [0, -rb, 0, 0], [0, 0, ra, tau], [0, 0, 0, rb]],
// tau = rb (ra - rb)/eb, so the layer's compound C(F) C(exp(-T k h)) C(F)^-1 is
// closed form with no 0/0 as c -> 0 and a single growth exp((ra + rb) k h),
// divided out. C(F)^-1 = Q C(F)^T Q / det F (Q the Laplace pairing); det F
// and every other common scale cancel in the surface ratio M_12/M_23.

struct Terms {
    cd ra, rb, ea, eb, ieb, mup, u1, x2, r2;
};

GFK_HD Terms layer_terms(const LayerC& L, cd c2) {
    Terms t;
    t.ea = c2 * L.c[0];
    t.eb = c2 * L.c[1];
    const cd kap = L.c[2];
    t.mup = L.c[3];
    t.ra = csqrt_fast(1.0 - t.ea);  // principal root: Re >= 0, the decaying branch
    t.rb = csqrt_fast(1.0 - t.eb);
    const cd ra = t.ra, rb = t.rb, ea = t.ea, eb = t.eb;
    const cd rarb = ra * rb;
    const cd rb2p1 = 1.0 + rb * rb;
    if (cnorm1(eb) < 0.35) {
        // small c: the O(eb) numerators written without cancellation; the four
        // denominators share one reciprocal
        const cd d1 = 1.0 + rarb;
        const cd s = ra + rb;
        const cd d2 = s * s;
        const cd d3 = rb2p1 * rb2p1 + 4.0 * rarb;
        const cd d12 = d1 * d2, d34 = d3 * eb;
        const cd ip = crcp_(d12 * d34);
        const cd i12 = d34 * ip, i34 = d12 * ip;  // 1/(d1 d2), 1/(d3 eb)
        const cd omk = 1.0 - kap;
        t.u1 = (kap + 1.0 - ea) * (d2 * i12);
        t.x2 = (eb * omk * omk) * (d1 * i12) + kap;
        const cd num = 16.0 * (kap - 1.0) + eb * (24.0 - 16.0 * kap + eb * (eb - 8.0));
        t.r2 = num * (eb * i34);
        t.ieb = d3 * i34;
    } else {
        const cd ieb = crcp_(eb);
        t.ieb = ieb;
        t.u1 = (1.0 - rarb) * ieb;
        t.x2 = (rb2p1 - 2.0 * rarb) * ieb;
        t.r2 = (rb2p1 * rb2p1 - 4.0 * rarb) * ieb;
    }
    return t;
}

// pd ^ g: minors of a layer's two downward-decaying solutions.
GFK_HD void decaying_minors(const Terms& t, cd m[6]) {
    const cd mu = t.mup;
    m[0] = -t.u1;
    m[1] = -(mu * t.x2);
    m[2] = mu * t.rb;
    m[3] = -(mu * t.ra);
    m[4] = mu * t.x2;
    m[5] = (mu * mu) * t.r2;
}

// m <- C(exp(-A zeta)) m up to a scalar: one layer, bottom to top. With
// renorm the result is rescaled by a power of two (exact) so its largest part
// is in [1, 2); a layer changes the magnitude by a bounded factor, so callers
// rescale every few layers (kRenormEvery) and at the surface.
GFK_HD void dunkin_layer_up(const Terms& t, double zeta, cd m[6], bool renorm = true) {
    const cd ra = t.ra, rb = t.rb, mu = t.mup, u1 = t.u1, x2 = t.x2, r2 = t.r2;
    const cd rarb = ra * rb;
    const cd tt = mu * (1.0 + rb * rb);
    const cd p13 = x2 + 2.0 * rarb;
    const cd p23 = r2 + 4.0 * rarb;
    const cd mx2 = mu * x2, mrb = mu * rb, mra = mu * ra, mu2 = mu * mu;
    // a = Q m
    const cd a0 = m[5], a1 = -m[4], a2 = m[3], a3 = m[2], a4 = -m[1], a5 = m[0];
    // D = C(F)^T a, column by column (zeros of C(F) skipped)
    const cd S = -(u1 * a0) - mx2 * a1;
    const cd P = mrb * a2;
    const cd R = mra * a3;
    const cd T0 = mx2 * a4 + (mu2 * r2) * a5;
    const cd T2 = (mu * p13) * a4 + (mu2 * p23) * a5;
    const cd D0 = S + P - R + T0;
    const cd D1 = 2.0 * ra * (a0 + 2.0 * mu * a1 - tt * a4 - 2.0 * mu * tt * a5);
    const cd D2 = S - P - R + T2;
    const cd D3 = -(S + P + R + T2);
    const cd D4 = 2.0 * mrb * (u1 * a4 + mx2 * a5);
    const cd D5 = S - P + R + T0;
    // y = Q D
    const cd y0 = D5, y1 = -D4, y2 = D3, y3 = D2, y4 = -D1, y5 = D0;
    // exp(-T zeta) compound over exp((ra + rb) zeta): 1, a 4x4 Kronecker block, (EaEb)^2
    const cd Eb = cexp_(-(rb * zeta));
    const cd delta = (t.eb - t.ea) * crcp_(ra + rb);  // ra - rb, cancellation-free
    const cd dz = delta * zeta;
    cd Ea, W;  // W = tau (Eb - Ea)/(ra - rb) = rb (Eb - Ea)/eb
    if (cnorm1(dz) < 0.5) {
        const cd em1 = cexpm1_(-dz);  // Ea = Eb exp(-dz), Eb - Ea = -Eb expm1(-dz)
        const cd e = Eb * em1;
        Ea = Eb + e;
        W = (rb * (-e)) * t.ieb;
    } else {
        Ea = cexp_(-(ra * zeta));
        W = (rb * (Eb - Ea)) * t.ieb;
    }
    const cd EaEb = Ea * Eb;
    const cd z0 = y0;
    const cd z1 = EaEb * y1 - (Eb * W) * y2 - (W * Ea) * y3 + (W * W) * y4;
    const cd z2 = (Eb * Eb) * y2 - (W * Eb) * y4;
    const cd z3 = (Ea * Ea) * y3 - (W * Ea) * y4;
    const cd z4 = EaEb * y4;
    const cd z5 = (EaEb * EaEb) * y5;
    // m = C(F) z
    const cd s05 = z0 + z5, d23 = z2 - z3;
    const cd e0 = z0 + z2 - z3 + z5;
    m[0] = 2.0 * ra * z1 - u1 * e0;
    m[1] = 4.0 * mra * z1 - mx2 * e0;
    m[2] = mrb * (z0 - z2 - z3 - z5);
    m[3] = -(mra * (z0 + z2 + z3 - z5));
    m[4] = mx2 * s05 + (mu * p13) * d23 - (2.0 * ra * tt) * z1 + (2.0 * mrb * u1) * z4;
    m[5] = (mu2 * r2) * s05 + (mu2 * p23) * d23 - (4.0 * mra * tt) * z1 + (2.0 * mu2 * rb * x2) * z4;
    // renormalise by a power of two (exact; the common scale cancels)
    if (!renorm) return;
    double mx = 0.0;
#pragma unroll
    for (int i = 0; i < 6; i++) mx = fmax(mx, cnorm1(m[i]));
    if (mx > 0.0 && mx < INFINITY) {
        const double sc = pow2i(-ilogb(mx));
#pragma unroll
        for (int i = 0; i < 6; i++) m[i] = m[i] * sc;
    }
}

// Thick-layer start. Through a finite layer whose P and S factors
// exp(-Re(ra) k h) and exp(-Re(rb) k h) are both below e^-kThick, the
// minors leave as z0 C(F) e0 plus terms carrying products of two such
// factors (z1..z5 in dunkin_layer_up). C(F) e0 is the layer's own decaying
// minors, so above that layer the minors are those of a half-space of its
// material up to scale, to ~e^(-2 kThick) relative, and the layers beneath it
// cannot reach the surface in FP64. Propagation therefore starts at the
// shallowest such layer. Re(sqrt(1 - e)) >= sqrt(Re(1 - e)) gives a cheap
// sufficient test without the square roots. Against the full propagation on
// the graded, single and 40 seeded uneven soils the difference stays at
// rounding level down to kThick = 20; below that it grows as C e^(-2 kThick)
// with C = 260-550 at kThick = 8-12 (rising slowly with kThick), so at 26 the
// neglected part is ~1e-19 relative, three orders below FP64 rounding.
constexpr double kThick = 26.0;

// Layers between power-of-two rescalings of the minor vector (the scale is
// exact and cancels, so the result does not depend on it while nothing
// overflows; one layer changes the magnitude by far less than 2^64).
constexpr int kRenormEvery = 4;

GFK_HD bool thick_layer(const LayerC& L, cd c2, double zeta) {
    const double pa = 1.0 - (c2.re * L.c[0].re - c2.im * L.c[0].im);  // Re(1 - ea)
    const double pb = 1.0 - (c2.re * L.c[1].re - c2.im * L.c[1].im);  // Re(1 - eb)
    return fmin(pa, pb) * (zeta * zeta) > kThick * kThick;
}

// The layer the upward propagation starts from: the shallowest thick finite
// layer, else the half-space.
GFK_HD int start_layer(const LayerC* L, int n, cd c2, double k) {
    for (int i = 0; i < n - 1; i++)
        if (thick_layer(L[i], c2, k * L[i].h)) return i;
    return n - 1;
}

// Surface vertical displacement per newton (fk.go:276-327) by minor
// propagation: u_z = i b4 M_12/M_23 with b4 = -i/(2 pi mu_ref k).
GFK_HD cd dunkin_u(const LayerC* L, int n, cd wc2, double k, double mu_ref) {
    const cd c2 = wc2 * rcp_(k * k);  // rcp_ is the correctly rounded 1/x
    const int top = start_layer(L, n, c2, k);
    cd m[6];
    {
        Terms t = layer_terms(L[top], c2);
        decaying_minors(t, m);
    }
    for (int i = top - 1; i >= 0; i--) {
        Terms t = layer_terms(L[i], c2);
        dunkin_layer_up(t, k * L[i].h, m, i % kRenormEvery == 0);
    }
    // the minors end rescaled into [1, 2), so |denominator|^2 stays in range
    // for one real reciprocal
    return cdiv_fast(m[3], (kTwoPi * mu_ref * k) * m[5]);
}

// Two wavenumbers of one frequency in lockstep through the layers: two
// independent dependency chains per thread, for latency hiding at low occupancy.
GFK_HD void dunkin_u2(const LayerC* L, int n, cd wc2, double k0, double k1, double mu_ref, cd& u0, cd& u1) {
    const cd c20 = wc2 * rcp_(k0 * k0);
    const cd c21 = wc2 * rcp_(k1 * k1);
    const int top0 = start_layer(L, n, c20, k0), top1 = start_layer(L, n, c21, k1);
    cd m0[6], m1[6];
    {
        Terms t0 = layer_terms(L[top0], c20);
        Terms t1 = layer_terms(L[top1], c21);
        decaying_minors(t0, m0);
        decaying_minors(t1, m1);
    }
    for (int i = (top0 > top1 ? top0 : top1) - 1; i >= 0; i--) {
        if (i < top0) {
            Terms t0 = layer_terms(L[i], c20);
            dunkin_layer_up(t0, k0 * L[i].h, m0, i % kRenormEvery == 0);
        }
        if (i < top1) {
            Terms t1 = layer_terms(L[i], c21);
            dunkin_layer_up(t1, k1 * L[i].h, m1, i % kRenormEvery == 0);
        }
    }
    u0 = cdiv_fast(m0[3], (kTwoPi * mu_ref * k0) * m0[5]);
    u1 = cdiv_fast(m1[3], (kTwoPi * mu_ref * k1) * m1[5]);
}

// ------------------------------------------------------ reference direct --

struct M4 {
    cd a[4][4];
};

// cmat.solve (cmat.go:57-96): Gaussian elimination with partial pivoting.
__device__ __forceinline__ bool m4_solve(M4 m, cd x[4], cd out[4]) {
#pragma unroll
    for (int col = 0; col < 4; col++) {
        double best = 0.0;
        int brow = col;
#pragma unroll
        for (int r = col; r < 4; r++) {
            double v = cabs_(m.a[r][col]);
            if (v > best) { best = v; brow = r; }
        }
        if (best == 0.0) return false;
#pragma unroll
        for (int r = col + 1; r < 4; r++) {
            if (r == brow) {
#pragma unroll
                for (int c = 0; c < 4; c++) { cd t = m.a[col][c]; m.a[col][c] = m.a[r][c]; m.a[r][c] = t; }
                cd t = x[col]; x[col] = x[r]; x[r] = t;
            }
        }
        const cd p = m.a[col][col];
#pragma unroll
        for (int r = col + 1; r < 4; r++) {
            const cd f = m.a[r][col] / p;
            if (f.re == 0.0 && f.im == 0.0) continue;
#pragma unroll
            for (int c = col; c < 4; c++) m.a[r][c] -= f * m.a[col][c];
            x[r] -= f * x[col];
        }
    }
#pragma unroll
    for (int i = 3; i >= 0; i--) {
        cd s = x[i];
#pragma unroll
        for (int j = i + 1; j < 4; j++) s -= m.a[i][j] * out[j];
        out[i] = s / m.a[i][i];
    }
    return true;
}

// props.eigen (fk.go:138-168): columns (P down, SV down, P up, SV up).
__device__ __forceinline__ void eigen4(const LayerC& L, double k, double omega, double mu_ref, cd lam[4], M4& e) {
    const cd alpha = L.c[0], beta = L.c[1], mu = L.c[2];
    const double rho = L.c[3].re;
    const double w2 = omega * omega;
    const double k2 = k * k;
    cd ra = csqrt_(1.0 - mk(w2) / ((k2 * alpha) * alpha));
    cd rb = csqrt_(1.0 - mk(w2) / ((k2 * beta) * beta));
    if (ra.re < 0) ra = -ra;
    if (rb.re < 0) rb = -rb;
    const double rc2 = rho * w2 / k2;
    const cd mr = mk(mu_ref);
    lam[0] = -ra; lam[1] = -rb; lam[2] = ra; lam[3] = rb;
    const cd two_mu_mr = (2.0 * mu) / mr;
    const cd p3 = (2.0 * mu - rc2) / mr;
    const cd s2 = (rc2 - 2.0 * mu) / mr;
    e.a[0][0] = mk(1.0);            e.a[0][1] = rb;               e.a[0][2] = mk(1.0);          e.a[0][3] = -rb;
    e.a[1][0] = -ra;                e.a[1][1] = mk(-1.0);         e.a[1][2] = ra;               e.a[1][3] = mk(-1.0);
    e.a[2][0] = -(two_mu_mr * ra);  e.a[2][1] = s2;               e.a[2][2] = two_mu_mr * ra;   e.a[2][3] = s2;
    e.a[3][0] = p3;                 e.a[3][1] = two_mu_mr * rb;   e.a[3][2] = p3;               e.a[3][3] = -(two_mu_mr * rb);
}

// Medium.SurfaceResponse restated (fk.go:276-327). ok = false where the
// reference reports a singular propagator or surface system.
__device__ __forceinline__ cd direct_u(const LayerC* L, int n, double omega, double k, double mu_ref, bool& ok) {
    M4 total;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) total.a[i][j] = mk(i == j ? 1.0 : 0.0);
    ok = true;
    for (int l = 0; l < n - 1; l++) {
        cd lam[4];
        M4 e;
        eigen4(L[l], k, omega, mu_ref, lam, e);
        const double zeta = k * L[l].h;
        double max_re = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) max_re = fmax(max_re, lam[i].re);
        cd d[4];
#pragma unroll
        for (int i = 0; i < 4; i++) d[i] = cexp_((lam[i] - max_re) * zeta);
        M4 inv;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            cd ej[4] = {mk(0), mk(0), mk(0), mk(0)};
            ej[j] = mk(1.0);
            cd col[4];
            if (!m4_solve(e, ej, col)) { ok = false; return mk(0.0); }
#pragma unroll
            for (int i = 0; i < 4; i++) inv.a[i][j] = col[i];
        }
        // p = (e d) inv; total = p total
        M4 p;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                cd s = mk(0.0);
#pragma unroll
                for (int q = 0; q < 4; q++) s += (e.a[i][q] * d[q]) * inv.a[q][j];
                p.a[i][j] = s;
            }
        M4 nt;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                cd s = mk(0.0);
#pragma unroll
                for (int q = 0; q < 4; q++) s += p.a[i][q] * total.a[q][j];
                nt.a[i][j] = s;
            }
        total = nt;
    }
    cd lam[4];
    M4 e;
    eigen4(L[n - 1], k, omega, mu_ref, lam, e);
    const cd b4 = mk(0.0, -1.0 / (kTwoPi * mu_ref * k));
    M4 a;
    cd rhs[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        a.a[i][0] = total.a[i][0];
        a.a[i][1] = total.a[i][1];
        a.a[i][2] = -e.a[i][0];
        a.a[i][3] = -e.a[i][1];
        rhs[i] = -(b4 * total.a[i][3]);
    }
    cd x[4];
    if (!m4_solve(a, rhs, x)) { ok = false; return mk(0.0); }
    return mk(x[1].im, -x[1].re);  // -i * x1
}

}  // namespace gfk
