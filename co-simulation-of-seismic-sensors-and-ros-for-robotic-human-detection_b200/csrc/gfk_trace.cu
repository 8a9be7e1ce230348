// gfk_trace.cu — geophone traces and their sweep metrics, one soil per CTA.
//
// For a displacement spectrum G[k-1] on bins k = 1..n/2 at the complex
// frequency w_c = 2 pi f - i w_I, the recorded trace is
//     Y_k = G[k-1] S_k,   S_k = (i w_c) geophone(i w_c) taper_k F_k
// (velocity per newton through the sensor, times the footstep spectrum, the
// host precomputes S once per setup), y = irfft(Y, n) e^{w_I t}
// (internal/dsp/dsp.go:232-261 taper and inverse transform; the damping
// undone after it). The metrics follow sweep.Measure
// (internal/sweep/sweep.go:128-169): the peak |y| and the magnitude-weighted
// centroid of |rfft(y)| over the band bins [k_lo, k_hi].
//
// Both transforms are n = 1024 complex radix-2 FFTs in FP64 in shared memory
// (gfk_fft.cuh). The inverse transform of the Hermitian spectrum is
// Re(FFT(conj(Y~))) / n.
#include "gfk_fft.cuh"
#include "gfk_kernels.cuh"
#include "gfk_mlp.cuh"

namespace gfk {
namespace trace {

constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_metrics(const cd* __restrict__ G, long long stride, int nbins,
                                                      const cd* __restrict__ S, const cd* __restrict__ tw, double fs,
                                                      double wi, int k_lo, int k_hi, double* peak,
                                                      double* centroid) {
    __shared__ cd buf[2][kN];
    __shared__ double red[2][kThreads];
    const int s = blockIdx.x, tid = threadIdx.x;
    const cd* g = G + (size_t)s * stride;
    // conj of the Hermitian extension of Y: k = 0 and n/2 real parts only
    for (int k = tid; k <= kN / 2; k += blockDim.x) {
        cd Y = mk(0.0);
        if (k >= 1 && k <= nbins) Y = g[k - 1] * S[k];
        if (k == kN / 2) Y.im = 0.0;
        buf[0][k] = mk(Y.re, -Y.im);
        if (k > 0 && k < kN / 2) buf[0][kN - k] = Y;
    }
    __syncthreads();
    const cd* y = fft_pow2(buf[0], buf[1], kN, tw);  // 10 stages: the result is in buf[0]
    // y_t = Re / n e^{w_I t}; keep y as the real input of the second transform
    double pk = 0.0;
    for (int t = tid; t < kN; t += blockDim.x) {
        const double yt = y[t].re * (1.0 / kN) * exp(wi * t / fs);
        pk = fmax(pk, fabs(yt));
        buf[0][t] = mk(yt);
    }
    __syncthreads();
    const cd* Yc = fft_pow2(buf[0], buf[1], kN, tw);
    double num = 0.0, den = 0.0;
    for (int k = k_lo + tid; k <= k_hi; k += blockDim.x) {
        const double a = hypot(Yc[k].re, Yc[k].im);
        num += a * (k * fs / kN);
        den += a;
    }
    red[0][tid] = num;
    red[1][tid] = den;
    __shared__ double pmax[kThreads];
    pmax[tid] = pk;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (tid < w) {
            red[0][tid] += red[0][tid + w];
            red[1][tid] += red[1][tid + w];
            pmax[tid] = fmax(pmax[tid], pmax[tid + w]);
        }
        __syncthreads();
    }
    if (tid == 0) {
        peak[s] = pmax[0];
        centroid[s] = red[1][0] > 0.0 ? red[0][0] / red[1][0] : 0.0;
    }
}

__global__ void __launch_bounds__(kThreads) k_gate(GateArgs a) {
    __shared__ double red[kThreads];
    const int s = blockIdx.x, tid = threadIdx.x;
    double pk = 0.0;
    for (int k = tid; k < a.nbins; k += blockDim.x) {
        cd m = mk(0.0);
        for (int e = 0; e < a.E; e++) m = m + a.members[e][(size_t)s * a.stride + k];
        m = m * (1.0 / a.E);
        a.mean[(size_t)s * a.nbins + k] = m;
        pk = fmax(pk, cabs_(m * a.S[k + 1]));
    }
    red[tid] = pk;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] = fmax(red[tid], red[tid + w]);
        __syncthreads();
    }
    const double peak = red[0];
    __syncthreads();
    double worst = 0.0;
    for (int k = tid; k < a.nbins; k += blockDim.x) {
        const cd m = a.mean[(size_t)s * a.nbins + k];
        double d = 0.0;
        for (int e = 0; e < a.E; e++) d = fmax(d, cabs_(a.members[e][(size_t)s * a.stride + k] - m));
        const double sk = cabs_(a.S[k + 1]);
        const double ratio = peak > 0.0 ? d * sk / peak : 0.0;
        // an energetic row goes to the f-k solve whatever the members say:
        // members that agree can all be wrong, and these rows carry the trace
        const bool loud = a.amp_threshold > 0.0 && cabs_(m) * sk > a.amp_threshold * peak;
        a.flag[(size_t)s * a.nbins + k] = (ratio > a.threshold || loud) ? 1 : 0;
        worst = fmax(worst, ratio);
    }
    red[tid] = worst;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] = fmax(red[tid], red[tid + w]);
        __syncthreads();
    }
    if (tid == 0) a.spread[s] = red[0];
}

__global__ void k_scatter(const cd* src, long long src_stride, const long long* index, long long n, cd* dst) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[index[i]] = src[i * src_stride];
}

void launch_gate(cudaStream_t s, const GateArgs& a) { k_gate<<<a.ns, kThreads, 0, s>>>(a); }

void launch_scatter(cudaStream_t s, const cd* src, long long src_stride, const long long* index, long long n,
                    cd* dst) {
    k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, src_stride, index, n, dst);
}

void launch_metrics(cudaStream_t s, const cd* G, long long stride, int ns, int nbins, const cd* S, const cd* twiddle,
                    double fs, double omega_imag, int k_lo, int k_hi, double* peak, double* centroid) {
    k_metrics<<<ns, kThreads, 0, s>>>(G, stride, nbins, S, twiddle, fs, omega_imag, k_lo, k_hi, peak, centroid);
}

}  // namespace trace
}  // namespace gfk
