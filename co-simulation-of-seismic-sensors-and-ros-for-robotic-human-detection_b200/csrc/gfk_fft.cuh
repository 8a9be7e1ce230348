// gfk_fft.cuh — FP64 complex radix-2 FFT of one power-of-two record in shared
// memory, by the block that calls it.
//
// The autosort (Stockham) formulation of Govindaraju et al., SC 2008: at the
// stage with sub-transform length ns, butterfly j (< n/2) reads x[j] and
// x[j + n/2] and writes y[2 ns (j / ns) + j % ns] and that + ns, with twiddle
// e^{-2 pi i (j % ns) / (2 ns)} = tw[(j % ns) (n / (2 ns))], tw[m] =
// e^{-2 pi i m / n}. Results come out in natural order.
#pragma once
#include "gfk_math.cuh"

namespace gfk {

// Forward transform (e^{-i}) of x[0, n); y is scratch of the same size. The
// result ends in x when log2(n) is even, in y otherwise; the return value
// points at it. Every thread of the block must call it.
__device__ inline cd* fft_pow2(cd* x, cd* y, int n, const cd* __restrict__ tw) {
    cd* src = x;
    cd* dst = y;
    for (int ns = 1; ns < n; ns <<= 1) {
        for (int j = threadIdx.x; j < n / 2; j += blockDim.x) {
            const int k = j & (ns - 1);
            const cd w = tw[k * (n / (2 * ns))];
            const cd a0 = src[j];
            const cd a1 = src[j + n / 2] * w;
            const int d = ((j - k) << 1) + k;
            dst[d] = a0 + a1;
            dst[d + ns] = a0 - a1;
        }
        __syncthreads();
        cd* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// In-place iterative radix-2 decimation in time (Cooley-Tukey): x holds the
// input in bit-reversed order (element k at index bitrev(k)); the forward
// transform (e^{-i}) ends in x in natural order. Half the shared memory of
// fft_pow2; every thread of the block must call it.
__device__ inline void fft_pow2_dit_inplace(cd* x, int n, const cd* __restrict__ tw, int tw_n = 0) {
    // tw holds e^{-2 pi i m / tw_n}, m < tw_n / 2 (tw_n = n by default; a
    // multiple of n reuses a larger transform's table)
    const int tn = tw_n > 0 ? tw_n : n;
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = tn / len;
        for (int j = threadIdx.x; j < n / 2; j += blockDim.x) {
            const int pos = j & (half - 1);
            const int i0 = ((j - pos) << 1) + pos;
            const cd w = tw[pos * step];
            const cd a = x[i0];
            const cd b = x[i0 + half] * w;
            x[i0] = a + b;
            x[i0 + half] = a - b;
        }
        __syncthreads();
    }
}

// Index of element k in the bit-reversed order of a 2^logn record.
__device__ __forceinline__ int bitrev(int k, int logn) { return (int)(__brev((unsigned)k) >> (32 - logn)); }

}  // namespace gfk
