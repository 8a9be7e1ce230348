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

}  // namespace gfk
