/*
 * gfk_oracle.c — CPU FP64 restatement of the reference's Green's-function path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for libgfk: the tests, the
 * smoke check and the benchmark's CPU-baseline leg call it through ctypes. No
 * product code links it or routes through it.
 *
 * Two formulations:
 *   - reference-direct: a behavioural restatement of internal/fk/fk.go and
 *     internal/fk/cmat.go (direct 4x4 propagators, pivoted solves, Qp = 2.25 Qs,
 *     MaxLayerPhase guard, GridFor, static subtraction, closed k = 0 panel,
 *     trapezoid with w = 1/2 at the last sample, J0 from glibc's j0, which is
 *     fdlibm-derived like Go's math.J0). Go's math/cmplx is replaced by C99
 *     complex functions; values agree to rounding, not bit for bit.
 *   - Dunkin: the complex second-compound (minor) propagation libgfk runs on
 *     the GPU, written independently here in plain C99 complex arithmetic.
 *
 * Citations are path:line within the reference project.
 */
#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "../include/gfk.h"

typedef double complex cx;

#define TWO_PI (2.0 * M_PI)
#define MAX_LAYER_PHASE 16.0 /* internal/fk/fk.go:242 */
#define MAX_LAYERS 64

/* ---------------------------------------------------------------- medium -- */

static double ref_freq(const gfk_medium *m) { /* fk.go:60-65 */
    return m->ref_freq_hz > 0 ? m->ref_freq_hz : 30.0;
}

static double q_of(const gfk_medium *m, const gfk_layer *l) { /* fk.go:67-75 */
    if (l->qs > 0) return l->qs;
    if (m->default_q > 0) return m->default_q;
    return 30.0;
}

static int has_sls(const gfk_medium *m) {
    return m->sls_tau_sigma > 0 && m->sls_tau_eps > 0;
}

/* visco.SLS.Modulus at complex angular frequency w (visco.go:78-81). */
static cx sls_modulus(const gfk_medium *m, cx w) {
    cx iw = I * w;
    return (1.0 + iw * m->sls_tau_eps) / (1.0 + iw * m->sls_tau_sigma);
}

/* visco.SLS.Q (visco.go:84-90). */
static double sls_q(const gfk_medium *m, double f) {
    cx mm = sls_modulus(m, TWO_PI * f);
    if (cimag(mm) == 0) return INFINITY;
    return creal(mm) / cimag(mm);
}

/* visco.SLS.RelaxedVelocity (visco.go:100-102). */
static double sls_relaxed(const gfk_medium *m, double v) {
    return v * creal(1.0 / csqrt(sls_modulus(m, TWO_PI * ref_freq(m))));
}

/* Medium.poleQ (fk.go:83-88). */
static double pole_q(const gfk_medium *m, double f) {
    if (has_sls(m)) return sls_q(m, f);
    return q_of(m, &m->layers[m->count - 1]);
}

/* Medium.complexVelocity (fk.go:96-110) generalised to a complex frequency
 * w - i*wi: Kjartansson c0*(i*w_c/w_ref)^gamma on the principal branch. With
 * wi = 0 it is evaluated exactly as the reference writes it. */
static cx complex_velocity(const gfk_medium *m, double v, double q, double f, double wi) {
    if (has_sls(m)) {
        if (f <= 0) return sls_relaxed(m, v);
        cx w = TWO_PI * f - I * wi;
        return sls_relaxed(m, v) * csqrt(sls_modulus(m, w));
    }
    if (q <= 0 || f <= 0) return v;
    double gam = atan(1.0 / q) / M_PI;
    double c0 = v * cos(M_PI * gam / 2);
    if (wi == 0) return c0 * pow(f / ref_freq(m), gam) * cexp(I * (M_PI * gam / 2));
    cx z = I * (TWO_PI * f - I * wi) / (TWO_PI * ref_freq(m));
    return c0 * cexp(gam * clog(z));
}

/* layer.Stack.Validate (layer.go:53-73), plus a finiteness check the
 * reference does not make (a NaN passes its comparisons). */
int or_validate(const gfk_medium *m) {
    if (!m || !m->layers || m->count <= 0 || m->count > MAX_LAYERS) return GFK_ESTACK;
    for (int i = 0; i < m->count; i++) {
        const gfk_layer *l = &m->layers[i];
        if (!isfinite(l->vs_mps) || !isfinite(l->vp_mps) || !isfinite(l->density_kgm3) ||
            !isfinite(l->qs) || !isfinite(l->qp) || (i < m->count - 1 && !isfinite(l->thickness_m)))
            return GFK_ESTACK;
        if (l->vs_mps <= 0 || l->vp_mps <= 0 || l->density_kgm3 <= 0) return GFK_ESTACK;
        if (l->vp_mps <= M_SQRT2 * l->vs_mps) return GFK_ESTACK;
        if (i < m->count - 1 && l->thickness_m <= 0) return GFK_ESTACK;
    }
    return GFK_OK;
}

static double slowest_vs(const gfk_medium *m) { /* layer.go:93-100 */
    double s = m->layers[0].vs_mps;
    for (int i = 0; i < m->count; i++) s = fmin(s, m->layers[i].vs_mps);
    return s;
}

static double reference_modulus(const gfk_medium *m) { /* fk.go:216-222 */
    double r = m->layers[0].density_kgm3 * m->layers[0].vs_mps * m->layers[0].vs_mps;
    for (int i = 0; i < m->count; i++)
        r = fmax(r, m->layers[i].density_kgm3 * m->layers[i].vs_mps * m->layers[i].vs_mps);
    return r;
}

/* Medium.checkLayerPhase (fk.go:251-266). */
int or_check_layer_phase(const gfk_medium *m, double f) {
    if (!m || m->count <= 0) return GFK_ESTACK;
    double k = TWO_PI * f / (0.87 * slowest_vs(m));
    for (int i = 0; i < m->count - 1; i++)
        if (k * m->layers[i].thickness_m > MAX_LAYER_PHASE) return GFK_EGUARD;
    return GFK_OK;
}

/* ----------------------------------------------- reference-direct (4x4) -- */

typedef struct { cx a[4][4]; } cmat;

/* cmat.solve (cmat.go:57-96): Gaussian elimination, partial pivoting on |.|. */
static int cmat_solve(const cmat *a, const cx b[4], cx out[4]) {
    cmat m = *a;
    cx x[4];
    memcpy(x, b, sizeof x);
    for (int col = 0; col < 4; col++) {
        double best = 0;
        int brow = col;
        for (int r = col; r < 4; r++) {
            double v = cabs(m.a[r][col]);
            if (v > best) { best = v; brow = r; }
        }
        if (best == 0) return 0;
        for (int c = 0; c < 4; c++) { cx t = m.a[col][c]; m.a[col][c] = m.a[brow][c]; m.a[brow][c] = t; }
        { cx t = x[col]; x[col] = x[brow]; x[brow] = t; }
        cx p = m.a[col][col];
        for (int r = col + 1; r < 4; r++) {
            cx f = m.a[r][col] / p;
            if (f == 0) continue;
            for (int c = col; c < 4; c++) m.a[r][c] -= f * m.a[col][c];
            x[r] -= f * x[col];
        }
    }
    for (int i = 3; i >= 0; i--) {
        cx s = x[i];
        for (int j = i + 1; j < 4; j++) s -= m.a[i][j] * out[j];
        out[i] = s / m.a[i][i];
    }
    return 1;
}

static void cmat_mul(const cmat *a, const cmat *b, cmat *out) { /* cmat.go:16-28 */
    cmat o;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            cx s = 0;
            for (int k = 0; k < 4; k++) s += a->a[i][k] * b->a[k][j];
            o.a[i][j] = s;
        }
    *out = o;
}

typedef struct { cx mu, alpha, beta; double rho; } props;

/* Medium.propsOf (fk.go:119-128): Qp = 2.25*Qs hard-coded. */
static props props_of(const gfk_medium *m, const gfk_layer *l, double f) {
    double q = q_of(m, l);
    props p;
    p.alpha = complex_velocity(m, l->vp_mps, 2.25 * q, f, 0);
    p.beta = complex_velocity(m, l->vs_mps, q, f, 0);
    p.rho = l->density_kgm3;
    p.mu = p.rho * p.beta * p.beta;
    return p;
}

/* props.eigen (fk.go:138-168). */
static void eigen(const props *p, double k, double omega, double mu_ref, cx lam[4], cmat *vec) {
    cx kc = k, w2 = omega * omega;
    cx ra = csqrt(1 - w2 / (kc * kc * p->alpha * p->alpha));
    cx rb = csqrt(1 - w2 / (kc * kc * p->beta * p->beta));
    if (creal(ra) < 0) ra = -ra;
    if (creal(rb) < 0) rb = -rb;
    cx rc2 = p->rho * w2 / (kc * kc);
    cx mr = mu_ref, mu = p->mu;
    lam[0] = -ra; lam[1] = -rb; lam[2] = ra; lam[3] = rb;
    cx pd[4] = {1, -ra, -2 * mu / mr * ra, (2 * mu - rc2) / mr};
    cx pu[4] = {1, ra, 2 * mu / mr * ra, (2 * mu - rc2) / mr};
    cx sd[4] = {rb, -1, (rc2 - 2 * mu) / mr, 2 * mu / mr * rb};
    cx su[4] = {-rb, -1, (rc2 - 2 * mu) / mr, -2 * mu / mr * rb};
    for (int i = 0; i < 4; i++) {
        vec->a[i][0] = pd[i]; vec->a[i][1] = sd[i]; vec->a[i][2] = pu[i]; vec->a[i][3] = su[i];
    }
}

/* props.propagator (fk.go:177-196) with invert (fk.go:199-213). */
static int propagator(const props *p, double k, double omega, double mu_ref, double h, cmat *out) {
    cx lam[4];
    cmat e;
    eigen(p, k, omega, mu_ref, lam, &e);
    cx zeta = k * h;
    double max_re = 0;
    for (int i = 0; i < 4; i++) max_re = fmax(max_re, creal(lam[i]));
    cmat d;
    memset(&d, 0, sizeof d);
    for (int i = 0; i < 4; i++) d.a[i][i] = cexp((lam[i] - max_re) * zeta);
    cmat inv;
    for (int j = 0; j < 4; j++) {
        cx ej[4] = {0, 0, 0, 0}, col[4];
        ej[j] = 1;
        if (!cmat_solve(&e, ej, col)) return 0;
        for (int i = 0; i < 4; i++) inv.a[i][j] = col[i];
    }
    cmat ed;
    cmat_mul(&e, &d, &ed);
    cmat_mul(&ed, &inv, out);
    return 1;
}

/* Medium.SurfaceResponse (fk.go:276-327). */
static int surface_response_direct(const gfk_medium *m, double k, double f, cx *u) {
    if (k <= 0 || f <= 0) return GFK_EARG;
    int st = or_validate(m);
    if (st) return st;
    double omega = TWO_PI * f, mu_ref = reference_modulus(m);
    cmat total;
    memset(&total, 0, sizeof total);
    for (int i = 0; i < 4; i++) total.a[i][i] = 1;
    for (int i = 0; i < m->count - 1; i++) {
        props p = props_of(m, &m->layers[i], f);
        cmat pm;
        if (!propagator(&p, k, omega, mu_ref, m->layers[i].thickness_m, &pm)) return GFK_ESINGULAR;
        cmat_mul(&pm, &total, &total);
    }
    props hp = props_of(m, &m->layers[m->count - 1], f);
    cx lam[4];
    cmat e;
    eigen(&hp, k, omega, mu_ref, lam, &e);
    cx b4 = -I / (TWO_PI * mu_ref * k);
    cmat a;
    cx rhs[4], x[4];
    for (int i = 0; i < 4; i++) {
        a.a[i][0] = total.a[i][0];
        a.a[i][1] = total.a[i][1];
        a.a[i][2] = -e.a[i][0];
        a.a[i][3] = -e.a[i][1];
        rhs[i] = -b4 * total.a[i][3];
    }
    if (!cmat_solve(&a, rhs, x)) return GFK_ESINGULAR;
    *u = -I * x[1];
    return GFK_OK;
}

/* ------------------------------------------------ Dunkin (6x6 compounds) -- */
/*
 * Minor index n <-> row pair: 0:(0,1) 1:(0,2) 2:(0,3) 3:(1,2) 4:(1,3) 5:(2,3),
 * the ordering of internal/propmat/propmat.go:168-174. The Laplace pairing
 * (u^v).Q.(x^y) = det[u,v,x,y] uses Q[n][5-n] = sign[n], sign = (+,-,+,+,-,+).
 *
 * Each layer's motion-stress basis is F = [pd, g, pu, h] with pd, pu the P
 * eigenvectors of fk.go:158-159 and g = (sd - rb*pd)/eb, h = (su + rb*pu)/eb
 * (eb = 1 - rb^2 = c^2/beta^2). In F, A is block upper-triangular
 *   T = [[-ra, tau, 0, 0], [0, -rb, 0, 0], [0, 0, ra, tau], [0, 0, 0, rb]],
 * tau = rb (ra - rb)/eb, so exp(-A k h) = F exp(-T k h) F^-1 has closed-form
 * entries with no 0/0 as c -> 0 (where pd and sd coalesce) and no growing
 * exponential other than exp((ra+rb) k h), which is divided out.
 * The compound satisfies C(F)^-1 = Q C(F)^T Q / det F; det F is a per-layer
 * scalar and is dropped, as is every common scale: only the ratio
 * M_12/M_23 of the surface minors is used.
 */

typedef struct { cx inv_a2, inv_b2, kap, mup; double h; } lconst;

typedef struct { cx ra, rb, ea, eb, kap, mup, u1, x2, r2; } lterms;

static cx csqrt_re_pos(cx z) {
    cx r = csqrt(z);
    return creal(r) < 0 ? -r : r;
}

static void layer_terms(const lconst *L, cx c2, lterms *t) {
    t->ea = c2 * L->inv_a2;
    t->eb = c2 * L->inv_b2;
    t->kap = L->kap;
    t->mup = L->mup;
    t->ra = csqrt_re_pos(1 - t->ea);
    t->rb = csqrt_re_pos(1 - t->eb);
    cx ra = t->ra, rb = t->rb, ea = t->ea, eb = t->eb, kap = t->kap;
    if (fmax(fabs(creal(eb)), fabs(cimag(eb))) < 0.35) {
        /* the small-c forms: every O(eb) numerator written without cancellation */
        t->u1 = (kap + 1 - ea) / (1 + ra * rb);
        cx s = ra + rb;
        t->x2 = eb * (1 - kap) * (1 - kap) / (s * s) + kap;
        cx num = 16 * (kap - 1) + eb * (24 - 16 * kap + eb * (-8 + eb));
        cx den = (1 + rb * rb) * (1 + rb * rb) + 4 * ra * rb;
        t->r2 = num / den;
    } else {
        t->u1 = (1 - ra * rb) / eb;
        t->x2 = (1 + rb * rb - 2 * ra * rb) / eb;
        t->r2 = ((1 + rb * rb) * (1 + rb * rb) - 4 * ra * rb) / eb;
    }
}

/* pd ^ g of one layer: the minors of its two downward-decaying solutions. */
static void decaying_minors(const lterms *t, cx m[6]) {
    cx mu = t->mup;
    m[0] = -t->u1;
    m[1] = -mu * t->x2;
    m[2] = mu * t->rb;
    m[3] = -mu * t->ra;
    m[4] = mu * t->x2;
    m[5] = mu * mu * t->r2;
}

static double max_abs6(const cx m[6]) {
    double s = 0;
    for (int i = 0; i < 6; i++) s = fmax(s, fmax(fabs(creal(m[i])), fabs(cimag(m[i]))));
    return s;
}

/* One layer, bottom to top: m <- C(exp(-A k h)) m, up to a scalar. */
static void dunkin_layer_up(const lterms *t, double zeta, cx m[6]) {
    cx ra = t->ra, rb = t->rb, mu = t->mup, u1 = t->u1, x2 = t->x2, r2 = t->r2;
    cx tt = mu * (1 + rb * rb);
    cx p13 = x2 + 2 * ra * rb;
    cx p23 = r2 + 4 * ra * rb;
    /* C(F) columns, pairs of F's columns in minor order:
       0:(pd,g) 1:(pd,pu) 2:(pd,h) 3:(g,pu) 4:(g,h) 5:(pu,h) */
    cx cf[6][6] = {
        {-u1, -mu * x2, mu * rb, -mu * ra, mu * x2, mu * mu * r2},
        {2 * ra, 4 * mu * ra, 0, 0, -2 * ra * tt, -4 * mu * ra * tt},
        {-u1, -mu * x2, -mu * rb, -mu * ra, mu * p13, mu * mu * p23},
        {u1, mu * x2, -mu * rb, -mu * ra, -mu * p13, -mu * mu * p23},
        {0, 0, 0, 0, 2 * mu * rb * u1, 2 * mu * mu * rb * x2},
        {-u1, -mu * x2, -mu * rb, mu * ra, mu * x2, mu * mu * r2},
    }; /* cf[column][row] */
    /* Q m */
    cx qm[6] = {m[5], -m[4], m[3], m[2], -m[1], m[0]};
    cx d[6];
    for (int q = 0; q < 6; q++) {
        cx s = 0;
        for (int n = 0; n < 6; n++) s += cf[q][n] * qm[n];
        d[q] = s;
    }
    cx y[6] = {d[5], -d[4], d[3], d[2], -d[1], d[0]};
    /* exp(-T zeta) compound, normalised by exp(-(ra+rb) zeta) */
    cx Ea = cexp(-ra * zeta), Eb = cexp(-rb * zeta);
    cx delta = (t->eb - t->ea) / (ra + rb); /* ra - rb without cancellation */
    cx W, dz = delta * zeta;
    if (fmax(fabs(creal(dz)), fabs(cimag(dz))) < 0.5) {
        /* Eb - Ea = Eb (1 - exp(-dz)) = -Eb expm1(-dz), expm1 of a complex
           argument as expm1(x) cos y - 2 sin^2(y/2) + i e^x sin y */
        double x = -creal(dz), y = -cimag(dz);
        cx em1 = (expm1(x) * cos(y) - 2 * sin(y / 2) * sin(y / 2)) + I * (exp(x) * sin(y));
        W = rb * (-Eb * em1) / t->eb;
    } else {
        W = rb * (Eb - Ea) / t->eb;
    }
    cx z[6];
    z[0] = y[0];
    z[1] = Ea * Eb * y[1] - Eb * W * y[2] - W * Ea * y[3] + W * W * y[4];
    z[2] = Eb * Eb * y[2] - W * Eb * y[4];
    z[3] = Ea * Ea * y[3] - W * Ea * y[4];
    z[4] = Ea * Eb * y[4];
    z[5] = (Ea * Eb) * (Ea * Eb) * y[5];
    for (int n = 0; n < 6; n++) {
        cx s = 0;
        for (int p = 0; p < 6; p++) s += cf[p][n] * z[p];
        m[n] = s;
    }
    /* renormalise by a power of two: exact, and the scale cancels */
    double mx = max_abs6(m);
    if (mx > 0 && isfinite(mx)) {
        int e;
        frexp(mx, &e);
        for (int n = 0; n < 6; n++) m[n] = ldexp(creal(m[n]), -e) + I * ldexp(cimag(m[n]), -e);
    }
}

static void layer_constants(const gfk_medium *m, const gfk_solve *s, double f, double mu_ref,
                            lconst *out) {
    for (int i = 0; i < m->count; i++) {
        const gfk_layer *l = &m->layers[i];
        double q = q_of(m, l);
        double qp = l->qp > 0 ? l->qp : 2.25 * q;
        cx a = complex_velocity(m, l->vp_mps, qp, f, s->omega_imag);
        cx b = complex_velocity(m, l->vs_mps, q, f, s->omega_imag);
        cx a2 = a * a, b2 = b * b;
        out[i].inv_a2 = 1.0 / a2;
        out[i].inv_b2 = 1.0 / b2;
        out[i].kap = b2 / a2;
        out[i].mup = l->density_kgm3 * b2 / mu_ref;
        out[i].h = l->thickness_m;
    }
}

static cx dunkin_u(const lconst *L, int n, cx wc2, double k, double mu_ref) {
    cx c2 = wc2 / (k * k);
    lterms t;
    layer_terms(&L[n - 1], c2, &t);
    cx m[6];
    decaying_minors(&t, m);
    for (int i = n - 2; i >= 0; i--) {
        layer_terms(&L[i], c2, &t);
        dunkin_layer_up(&t, k * L[i].h, m);
    }
    return m[3] / (TWO_PI * mu_ref * k * m[5]);
}

/* ------------------------------------------------------ solve dispatch -- */

typedef struct {
    const gfk_medium *m;
    const gfk_solve *s;
    double f, mu_ref;
    cx wc2;
    lconst L[MAX_LAYERS];
} fctx;

static int fctx_init(fctx *c, const gfk_medium *m, const gfk_solve *s, double f) {
    int st = or_validate(m);
    if (st) return st;
    if (s->formulation == GFK_REFERENCE_DIRECT && s->omega_imag != 0) return GFK_EARG;
    if (s->omega_imag < 0 || !isfinite(s->omega_imag)) return GFK_EARG;
    c->m = m; c->s = s; c->f = f;
    c->mu_ref = reference_modulus(m);
    cx wc = TWO_PI * f - I * s->omega_imag;
    c->wc2 = wc * wc;
    if (s->formulation == GFK_DUNKIN) layer_constants(m, s, f, c->mu_ref, c->L);
    return GFK_OK;
}

static int fctx_u(const fctx *c, double k, cx *u) {
    if (k <= 0 || c->f <= 0) return GFK_EARG;
    if (c->s->formulation == GFK_REFERENCE_DIRECT) return surface_response_direct(c->m, k, c->f, u);
    *u = dunkin_u(c->L, c->m->count, c->wc2, k, c->mu_ref);
    if (!isfinite(creal(*u)) || !isfinite(cimag(*u))) return GFK_ENONFINITE;
    return GFK_OK;
}

/* ------------------------------------------------------------ public -- */

int or_surface_response(const gfk_medium *m, const gfk_solve *s, double k, double f, double *out) {
    if (k <= 0 || f <= 0) return GFK_EARG;
    fctx c;
    int st = fctx_init(&c, m, s, f);
    if (st) return st;
    cx u;
    st = fctx_u(&c, k, &u);
    if (st) return st;
    out[0] = creal(u); out[1] = cimag(u);
    return GFK_OK;
}

int or_static_coefficient(const gfk_medium *m, const gfk_solve *s, double f, double k_far, double *out) {
    double u[2];
    int st = or_surface_response(m, s, k_far, f, u);
    if (st) return st;
    out[0] = k_far * u[0]; out[1] = k_far * u[1];
    return GFK_OK;
}

/* Medium.GridFor (fk.go:464-495). */
int or_grid_for(const gfk_medium *m, const double *ranges, int nr, double f, gfk_integration opt,
                gfk_grid *out) {
    if (nr <= 0 || !ranges) return GFK_EARG;
    if (!m || m->count <= 0) return GFK_ESTACK;
    double rmin = INFINITY, rmax = 0;
    for (int i = 0; i < nr; i++) {
        if (!(ranges[i] > 0)) return GFK_EARG;
        rmin = fmin(rmin, ranges[i]);
        rmax = fmax(rmax, ranges[i]);
    }
    double kbody = TWO_PI * f / slowest_vs(m);
    double kmf = opt.kmax_factor > 0 ? opt.kmax_factor : 30;
    double kmax = fmax(opt.kmax > 0 ? opt.kmax : kmf * kbody, 40 / rmin);
    double dk = TWO_PI / (8 * rmax);
    double q = pole_q(m, f);
    if (kbody > 0 && q > 0) dk = fmin(dk, kbody / (2 * q) / 4);
    double nn = ceil(kmax / dk);
    int n = nn > 2e9 ? 2000000000 : (int)nn;
    if (opt.samples > 0) n = opt.samples;
    if (n < 64) n = 64;
    out->kmax = kmax;
    out->samples = n;
    out->_pad = 0;
    return GFK_OK;
}

/* Medium.VerticalDisplacementMulti (fk.go:506-550). out: nr (re, im). */
int or_vertical_displacement_multi(const gfk_medium *m, const gfk_solve *s, const double *ranges, int nr,
                                   double f, gfk_integration opt, double *out) {
    int guard = s->guard || s->formulation == GFK_REFERENCE_DIRECT;
    if (!m || m->count <= 0) return GFK_ESTACK;
    if (guard) {
        int st = or_check_layer_phase(m, f);
        if (st) return st;
    }
    gfk_grid g;
    int st = or_grid_for(m, ranges, nr, f, opt, &g);
    if (st) return st;
    double kbody = TWO_PI * f / slowest_vs(m);
    double rmin = INFINITY;
    for (int i = 0; i < nr; i++) rmin = fmin(rmin, ranges[i]);
    if (f <= 0) return GFK_EARG;
    fctx c;
    st = fctx_init(&c, m, s, f);
    if (st) return st;
    double kfar = fmax(200 * kbody, 400 / rmin);
    cx uf;
    st = fctx_u(&c, kfar, &uf);
    if (st) return st;
    cx C = kfar * uf;
    double dk = g.kmax / g.samples;
    cx *acc = malloc(sizeof(cx) * nr);
    if (!acc) return GFK_ENOMEM;
    for (int j = 0; j < nr; j++) acc[j] = C / ranges[j] - (0.5 * dk) * C;
    for (int i = 1; i <= g.samples; i++) {
        double k = i * dk;
        cx u;
        st = fctx_u(&c, k, &u);
        if (st) { free(acc); return st; }
        double w = i == g.samples ? 0.5 : 1.0;
        cx rem = k * u - C;
        for (int j = 0; j < nr; j++) acc[j] += (w * j0(k * ranges[j]) * dk) * rem;
    }
    for (int j = 0; j < nr; j++) { out[2 * j] = creal(acc[j]); out[2 * j + 1] = cimag(acc[j]); }
    free(acc);
    return GFK_OK;
}

/* Medium.VerticalDisplacement (fk.go:396-443). */
int or_vertical_displacement(const gfk_medium *m, const gfk_solve *s, double r, double f,
                             gfk_integration opt, double *out) {
    if (r <= 0 || f <= 0) return GFK_EARG;
    if (!m || m->count <= 0) return GFK_ESTACK;
    if (s->guard || s->formulation == GFK_REFERENCE_DIRECT) {
        int st = or_check_layer_phase(m, f);
        if (st) return st;
    }
    double kbody = TWO_PI * f / slowest_vs(m);
    double kmf = opt.kmax_factor > 0 ? opt.kmax_factor : 30;
    double kmax = fmax(opt.kmax > 0 ? opt.kmax : kmf * kbody, 40 / r);
    fctx c;
    int st = fctx_init(&c, m, s, f);
    if (st) return st;
    double kfar = fmax(200 * kbody, 400 / r);
    cx uf;
    st = fctx_u(&c, kfar, &uf);
    if (st) return st;
    cx C = kfar * uf;
    int n = opt.samples > 0 ? opt.samples : 20000;
    double dk = kmax / n;
    cx sum = (0.5 * dk) * (-C);
    for (int i = 1; i <= n; i++) {
        double k = i * dk;
        cx u;
        st = fctx_u(&c, k, &u);
        if (st) return st;
        double w = i == n ? 0.5 : 1.0;
        cx rem = k * u - C;
        sum += (w * j0(k * r) * dk) * rem;
    }
    cx v = C / r + sum;
    out[0] = creal(v); out[1] = cimag(v);
    return GFK_OK;
}

/* ------------------------------------- threaded bank spectra (geobank) -- */

typedef struct {
    const gfk_medium *m;
    const gfk_solve *s;
    const double *ranges, *freqs;
    int nr, nf;
    gfk_integration opt;
    double *out;
    int32_t *status;
    atomic_int next;
} bank_job;

static void *bank_worker(void *arg) {
    bank_job *j = arg;
    for (;;) {
        int i = atomic_fetch_add(&j->next, 1);
        if (i >= j->nf) break;
        int st = or_vertical_displacement_multi(j->m, j->s, j->ranges, j->nr, j->freqs[i], j->opt,
                                                j->out + (size_t)2 * j->nr * i);
        if (st) memset(j->out + (size_t)2 * j->nr * i, 0, sizeof(double) * 2 * j->nr);
        if (j->status) j->status[i] = st;
    }
    return NULL;
}

/* VerticalDisplacementMulti at nf frequencies on nthreads host threads, one
 * frequency per task, as cmd/geobank/main.go:133-167 does with goroutines.
 * Returns the first failing status in frequency order. */
int or_bank_spectra(const gfk_medium *m, const gfk_solve *s, const double *ranges, int nr,
                    const double *freqs, int nf, gfk_integration opt, double *out, int32_t *status,
                    int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 1024) nthreads = 1024;
    int32_t *st = status ? status : calloc(nf > 0 ? nf : 1, sizeof(int32_t));
    if (!st) return GFK_ENOMEM;
    bank_job job = {m, s, ranges, freqs, nr, nf, opt, out, st, 0};
    pthread_t th[1024];
    int started = 0;
    for (int t = 0; t < nthreads; t++)
        if (pthread_create(&th[t], NULL, bank_worker, &job) == 0) started++;
    if (started == 0) bank_worker(&job);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    int first = GFK_OK;
    for (int i = 0; i < nf; i++)
        if (st[i]) { first = st[i]; break; }
    if (!status) free(st);
    return first;
}

/* Bessel J0 as the oracle evaluates it (glibc, fdlibm-derived). */
double or_j0(double x) { return j0(x); }
