// gfk_slice.cuh — exact int8 digits for the tensor-core wavenumber sum.
//
// An operand row x with |x| <= mx is scaled by 2^-e (2^e >= mx 128/127) into
// (-1, 1) and rounded once to the integer N = rint(x 2^(28 - e)), |N| < 2^28,
// which is written as four balanced base-128 digits,
//     N = d0 2^21 + d1 2^14 + d2 2^7 + d3,  -64 <= d1, d2, d3 < 64, |d0| <= 127,
// so x 2^-e 128 = d0 + d1/128 + d2/128^2 + d3/128^3 + O(128^-3). The digits
// are taken with integer operations: one FP64 multiply and one conversion per
// value, the rest off the FP64 pipe the propagator saturates.
#pragma once
#include <stdint.h>

#include "gfk_math.cuh"

namespace gfk {

// The digits of N, d0 in the lowest byte.
__device__ __forceinline__ uint32_t digits4(int n) {
    const int d3 = ((n + 64) & 127) - 64;
    n = (n - d3) >> 7;  // exact: n - d3 is a multiple of 128
    const int d2 = ((n + 64) & 127) - 64;
    n = (n - d2) >> 7;
    const int d1 = ((n + 64) & 127) - 64;
    n = (n - d1) >> 7;
    return (uint32_t)(n & 255) | (uint32_t)(d1 & 255) << 8 | (uint32_t)(d2 & 255) << 16 | (uint32_t)(d3 & 255) << 24;
}

// x 2^(28 - e) rounded to the nearest integer; sc = 2^(28 - e).
__device__ __forceinline__ int scaled_int(double x, double sc) { return __double2int_rn(x * sc); }

// The power of two a row with maximum magnitude mx is divided by.
__device__ __forceinline__ int slice_exp(double mx) { return mx > 0 ? ilogb(mx * (128.0 / 127.0)) + 1 : 0; }

// Where the propagator leaves the sliced integrand: rowmax[2f + p] the bits of
// max_k |part p of row f| (p = 0 real, 1 imaginary), done[f] the row's count
// of finished blocks, row_exp[2f + p] the row's exponents, and the four digit
// planes A[4][Mp][Kp] (rows 2f, 2f + 1 of each).
struct SliceOut {
    unsigned long long* rowmax;
    unsigned long long* done;
    int* row_exp;
    int8_t* A;
    int Mp, Kp;
};

// Slices integrand row f (src[0..nk), zero beyond, up to Kp) with the block's
// THREADS threads. The row is read from L2 (other blocks wrote it) in passes
// of THREADS x 8 values through `tile`: coalesced 16-byte loads, the next
// pass's issued before this pass is cut, into shared memory (16-byte units
// XOR-swizzled within each run of 8, so neither the row-order stores nor each
// thread's 8-unit reads conflict); each thread then cuts 8 consecutive values
// and writes 8 bytes per digit plane and part.
template <int THREADS>
__device__ void slice_row(const cd* src, int nk, bool live, const int e[2], const SliceOut& so, int f, cd* tile) {
    constexpr int P = THREADS * 8;
    const int t = threadIdx.x;
    const double sc0 = ldexp(1.0, 28 - e[0]), sc1 = ldexp(1.0, 28 - e[1]);
    double2 next[8];
    auto fetch = [&](int kb) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int k = kb + t + THREADS * i;
            next[i] = (live && k < nk) ? __ldcg(reinterpret_cast<const double2*>(src + k)) : make_double2(0.0, 0.0);
        }
    };
    fetch(0);
    for (int kb = 0; kb < so.Kp; kb += P) {
        __syncthreads();  // the previous pass's reads of the tile are done
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int el = t + THREADS * i;
            const int r = el >> 3, c = el & 7;
            tile[(r << 3) | (c ^ (r & 7))] = cd{next[i].x, next[i].y};
        }
        __syncthreads();
        if (kb + P < so.Kp) fetch(kb + P);
        const int k0 = kb + 8 * t;
        if (k0 >= so.Kp) continue;  // Kp is a multiple of 64: a thread's 8 values are all in or all out
        uint32_t w[2][8];  // digit words: part, value
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const cd v = tile[(t << 3) | (i ^ (t & 7))];
            w[0][i] = digits4(scaled_int(v.re, sc0));
            w[1][i] = digits4(scaled_int(v.im, sc1));
        }
        // byte q of each word is plane q's digit: gather the 8 values' plane-q
        // bytes with byte permutes (pairs, then the pairs of pairs)
#pragma unroll
        for (int p = 0; p < 2; p++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t pick = (uint32_t)q | (uint32_t)(q + 4) << 4;  // byte q of x, then of y
                const uint32_t v01 = __byte_perm(w[p][0], w[p][1], pick), v23 = __byte_perm(w[p][2], w[p][3], pick);
                const uint32_t v45 = __byte_perm(w[p][4], w[p][5], pick), v67 = __byte_perm(w[p][6], w[p][7], pick);
                const uint2 o = make_uint2(__byte_perm(v01, v23, 0x5410), __byte_perm(v45, v67, 0x5410));
                *reinterpret_cast<uint2*>(so.A + ((size_t)q * so.Mp + 2 * f + p) * so.Kp + k0) = o;
            }
    }
}

}  // namespace gfk
