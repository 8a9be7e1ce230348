// gfk_math.cuh — complex FP64 arithmetic for the f-k kernels.
//
// A plain struct rather than cuComplex/thrust so every operation is visible and
// the compiler keeps everything in registers. The elementary functions call
// CUDA's real sqrt/exp/expm1/sincos/hypot/atan/pow/log; the complex forms
// are the textbook identities named at each function.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#define GFK_HD __host__ __device__ __forceinline__

struct cd {
    double re, im;
};

GFK_HD cd mk(double r, double i = 0.0) { return cd{r, i}; }
GFK_HD cd operator+(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
GFK_HD cd operator-(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
GFK_HD cd operator-(cd a) { return cd{-a.re, -a.im}; }
GFK_HD cd operator*(cd a, cd b) { return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
GFK_HD cd operator*(double s, cd a) { return cd{s * a.re, s * a.im}; }
GFK_HD cd operator*(cd a, double s) { return cd{s * a.re, s * a.im}; }
GFK_HD cd operator+(cd a, double s) { return cd{a.re + s, a.im}; }
GFK_HD cd operator+(double s, cd a) { return cd{a.re + s, a.im}; }
GFK_HD cd operator-(double s, cd a) { return cd{s - a.re, -a.im}; }
GFK_HD cd operator-(cd a, double s) { return cd{a.re - s, a.im}; }
GFK_HD cd& operator+=(cd& a, cd b) { a.re += b.re; a.im += b.im; return a; }
GFK_HD cd& operator-=(cd& a, cd b) { a.re -= b.re; a.im -= b.im; return a; }
GFK_HD cd cmul_i(cd a) { return cd{-a.im, a.re}; }  // i*a

// Smith's algorithm (R. L. Smith, CACM 5(8):435, 1962), the robust complex
// division Go's runtime also uses.
GFK_HD cd operator/(cd n, cd m) {
    if (fabs(m.re) >= fabs(m.im)) {
        double ratio = m.im / m.re;
        double denom = m.re + ratio * m.im;
        return cd{(n.re + n.im * ratio) / denom, (n.im - n.re * ratio) / denom};
    }
    double ratio = m.re / m.im;
    double denom = m.im + ratio * m.re;
    return cd{(n.re * ratio + n.im) / denom, (n.im * ratio - n.re) / denom};
}
GFK_HD cd operator/(cd n, double s) { return cd{n.re / s, n.im / s}; }
GFK_HD cd operator/(double s, cd m) { return cd{s, 0.0} / m; }

GFK_HD double cabs_(cd a) { return hypot(a.re, a.im); }
GFK_HD double cnorm1(cd a) { return fmax(fabs(a.re), fabs(a.im)); }

// Principal square root: with t = sqrt((|x| + |z|)/2), sqrt(z) is (t, y/2t)
// for x >= 0 and (|y|/2t, copysign(t, y)) otherwise. Re >= 0 always.
GFK_HD cd csqrt_(cd z) {
    if (z.re == 0.0 && z.im == 0.0) return cd{0.0, z.im};
    double t = sqrt(0.5 * (fabs(z.re) + hypot(z.re, z.im)));
    if (z.re >= 0.0) return cd{t, z.im / (2.0 * t)};
    return cd{fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

// exp(x + iy) = e^x (cos y + i sin y).
GFK_HD cd cexp_(cd z) {
    double s, c;
    sincos(z.im, &s, &c);
    double e = exp(z.re);
    return cd{e * c, e * s};
}

// exp(z) - 1 without cancellation for small |z|:
//   Re = expm1(x) cos y - 2 sin^2(y/2),  Im = e^x sin y.
GFK_HD cd cexpm1_(cd z) {
    double sh, ch;
    sincos(0.5 * z.im, &sh, &ch);
    double s = 2.0 * sh * ch;
    double c = 1.0 - 2.0 * sh * sh;
    double em = expm1(z.re);
    return cd{em * c - 2.0 * sh * sh, (em + 1.0) * s};
}

// Reciprocal and reciprocal square root on the device: the hardware's FP64
// approximations (rcp.approx / rsqrt.approx, ~2^-20 relative) refined by one
// third-order Newton-type step (Markstein, "IA-64 and Elementary Functions",
// 2000): for 1/x, y (1 + e + e^2) with e = 1 - x y; for 1/sqrt(x),
// y (1 + e/2 + 3e^2/8) with e = 1 - x y^2. Measured over 4M log-uniform
// arguments in [2^-200, 2^200] on a B200: at most 0.50 ulp (1/x) and 0.62 ulp
// (1/sqrt(x)) from the exact values. Inputs are the solver's moderate
// magnitudes (subnormals flush to zero). The host versions exist so the
// solver can be compiled and checked on the CPU.
GFK_HD double rcp_(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
#else
    return 1.0 / x;
#endif
}
GFK_HD double rsqrt_(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x * y, y, 1.0);
    return fma(y, e * fma(e, 0.375, 0.5), y);
#else
    return 1.0 / sqrt(x);
#endif
}

// 1/b = conj(b)/|b|^2 with one real reciprocal. For the moderate magnitudes of
// the solver's quantities (|b| within 1e-150..1e150) this is accurate to a few
// ulp and much cheaper than Smith's division.
GFK_HD cd crcp_(cd b) {
    const double t = rcp_(fma(b.re, b.re, b.im * b.im));
    return cd{b.re * t, -b.im * t};
}
GFK_HD cd cdiv_fast(cd a, cd b) { return a * crcp_(b); }

// Principal square root from two reciprocal square roots: with r = |z|
// (= |z|^2 / sqrt(|z|^2)),
// s = (|x| + r)/2 and t = sqrt(s): (t, y/2t) for x >= 0, (|y|/2t, copysign(t, y))
// otherwise.
GFK_HD cd csqrt_fast(cd z) {
    const double n2 = fma(z.re, z.re, z.im * z.im);
    const double r = n2 > 0.0 ? n2 * rsqrt_(n2) : 0.0;
    const double s = 0.5 * (fabs(z.re) + r);
    if (s == 0.0) return cd{0.0, z.im};
    const double ti = rsqrt_(s);
    const double t = s * ti;
    const double h = 0.5 * ti;
    if (z.re >= 0.0) return cd{t, z.im * h};
    return cd{fabs(z.im) * h, copysign(t, z.im)};
}

// 2^e as a double, built from its bits (|e| < 1000).
GFK_HD double pow2i(int e) {
#ifdef __CUDA_ARCH__
    return __hiloint2double((e + 1023) << 20, 0);
#else
    return ldexp(1.0, e);
#endif
}

// log(z) = log|z| + i arg z.
GFK_HD cd clog_(cd z) { return cd{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }

// Scale by 2^e exactly.
GFK_HD cd cldexp(cd a, int e) { return cd{ldexp(a.re, e), ldexp(a.im, e)}; }
