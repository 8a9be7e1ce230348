// gfk_disp.cu — Rayleigh dispersion curves on the GPU: the secular function of
// internal/propmat and the bracketing root search of internal/disp, one block
// per frequency.
//
// Secular (propmat.go:82-315), in FP64 per (f, c): for every finite layer the
// dimensionless 4x4 system matrix A (SystemMatrix), its exponential over the
// layer shifted by the largest vertical-P growth so it stays bounded
// (LayerPropagator), that matrix's 6x6 second compound applied to the minor
// vector of the free-surface two-plane and renormalised to max |m| = 1, then
// the generalised Laplace expansion against the half-space's closed-form
// decaying minors. The scale factors are positive and are dropped, as the
// reference does. The exponential is ours: scaling and squaring (halve until
// the 1-norm is <= 1/2) with a degree-16 Taylor polynomial in Horner form
// (Moler and Van Loan, "Nineteen dubious ways", methods 1 and 3), truncation
// below 1e-19 relative before squaring.
//
// Modes (disp.go:62-103, bisect disp.go:194-217): the secular function on
// samples + 1 evenly spaced velocities in [0.85 Vs_min, Vs_halfspace (1 - 1e-9)]
// (all threads), the sign changes between defined neighbours in order (one
// thread), and one bisection per bracket (a group of lanes each, evaluating
// several steps' midpoints at once, below) with the reference's stopping
// rules; a bracket whose bisection meets an undefined value yields no root, as
// in the reference.
#include <cmath>
#include <vector>

#include "../../include/gfk.h"
#include "gfk_ctx.h"
#include "gfk_kernels.cuh"

namespace gfk {
namespace disp {

constexpr int kMaxLayers = 64;
constexpr int kThreads = 128;
constexpr int kSpecDepth = 3;                        // bisection steps per round
constexpr int kSpecNodes = (1 << kSpecDepth) - 1;    // midpoints evaluated per round
constexpr int kSpecLanes = 8;                        // lanes per bracket (a power of two > kSpecNodes)
static_assert(kSpecLanes > kSpecNodes && 32 % kSpecLanes == 0, "bracket groups tile a warp");
constexpr int kMaxModes = 64;
constexpr int kMaxSamples = 16384;

struct Layer4 {
    double h, vp, vs, rho;
};

struct Stack {
    Layer4 l[kMaxLayers];
    int n;          // entries including the half-space
    double mu_ref;  // referenceModulus (propmat.go:109-115)
};

__device__ inline void mat4_mul(const double* a, const double* b, double* c) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 4; k++) s = fma(a[4 * i + k], b[4 * k + j], s);
            c[4 * i + j] = s;
        }
}

// exp(M) of a real 4x4 by scaling and squaring with a Taylor polynomial.
__device__ inline void expm4(double* m, double* out) {
    double nrm = 0.0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 4; i++) s += fabs(m[4 * i + j]);
        nrm = fmax(nrm, s);
    }
    int sq = 0;
    while (nrm > 0.5 && sq < 60) {
        nrm *= 0.5;
        sq++;
    }
    const double sc = ldexp(1.0, -sq);
#pragma unroll
    for (int i = 0; i < 16; i++) m[i] *= sc;
    // Horner: T = I + M/16; T = I + M T / j for j = 15 .. 1
    double t[16], u[16];
#pragma unroll
    for (int i = 0; i < 16; i++) t[i] = m[i] * (1.0 / 16.0) + ((i % 5 == 0) ? 1.0 : 0.0);
    for (int j = 15; j >= 1; j--) {
        mat4_mul(m, t, u);
        const double inv = 1.0 / j;
#pragma unroll
        for (int i = 0; i < 16; i++) t[i] = u[i] * inv + ((i % 5 == 0) ? 1.0 : 0.0);
    }
    for (int s = 0; s < sq; s++) {
        mat4_mul(t, t, u);
#pragma unroll
        for (int i = 0; i < 16; i++) t[i] = u[i];
    }
#pragma unroll
    for (int i = 0; i < 16; i++) out[i] = t[i];
}

__device__ inline double vwave(double k, double omega, double v) {
    return sqrt(fmax(0.0, k * k - omega * omega / (v * v)));
}

// propmat.Secular; false where the reference returns an error.
__device__ bool secular(const Stack& st, double omega, double k, double* out) {
    if (!(k > 0.0) || !(omega > 0.0)) return false;
    const int pi_[6] = {0, 0, 0, 1, 1, 2}, pj_[6] = {1, 2, 3, 2, 3, 3};
    double m[6] = {1, 0, 0, 0, 0, 0};
    const double mu_ref = st.mu_ref;
    for (int li = 0; li + 1 < st.n; li++) {
        const Layer4 L = st.l[li];
        const double mu = L.rho * L.vs * L.vs;
        const double lam = L.rho * L.vp * L.vp - 2.0 * mu;
        const double l2m = lam + 2.0 * mu;
        const double rc2 = L.rho * omega * omega / (k * k);
        const double zeta = k * L.h;
        const double lmax = vwave(k, omega, L.vp) / k;
        double a[16] = {0};
        a[0 * 4 + 1] = -1.0;
        a[0 * 4 + 2] = mu_ref / mu;
        a[1 * 4 + 0] = lam / l2m;
        a[1 * 4 + 3] = mu_ref / l2m;
        a[2 * 4 + 0] = (4.0 * mu * (lam + mu) / l2m - rc2) / mu_ref;
        a[2 * 4 + 3] = -lam / l2m;
        a[3 * 4 + 1] = -rc2 / mu_ref;
        a[3 * 4 + 2] = 1.0;
#pragma unroll
        for (int i = 0; i < 16; i++) a[i] *= zeta;
#pragma unroll
        for (int i = 0; i < 4; i++) a[5 * i] -= lmax * zeta;
        double p[16];
        expm4(a, p);
        double nx[6];
        double norm = 0.0;
#pragma unroll
        for (int r = 0; r < 6; r++) {
            const int i = pi_[r], j = pj_[r];
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < 6; c++) {
                const int kk = pi_[c], ll = pj_[c];
                s += (p[4 * i + kk] * p[4 * j + ll] - p[4 * i + ll] * p[4 * j + kk]) * m[c];
            }
            nx[r] = s;
            norm = fmax(norm, fabs(s));
        }
        if (norm == 0.0) return false;
#pragma unroll
        for (int r = 0; r < 6; r++) m[r] = nx[r] / norm;
    }
    const Layer4 H = st.l[st.n - 1];
    if (omega / k >= H.vs) return false;
    const double a_ = vwave(k, omega, H.vp) / k, b_ = vwave(k, omega, H.vs) / k;
    const double mu = H.rho * H.vs * H.vs;
    const double rc2 = H.rho * omega * omega / (k * k);
    const double pv[4] = {1.0, -a_, -2.0 * (mu / mu_ref) * a_, (2.0 * mu - rc2) / mu_ref};
    const double sv[4] = {b_, -1.0, (rc2 - 2.0 * mu) / mu_ref, 2.0 * (mu / mu_ref) * b_};
    const double sign[6] = {1, -1, 1, 1, -1, 1};
    double f = 0.0;
#pragma unroll
    for (int n = 0; n < 6; n++) {
        const int c = 5 - n;  // complement pair
        const double e = pv[pi_[c]] * sv[pj_[c]] - pv[pj_[c]] * sv[pi_[c]];
        f += sign[n] * m[n] * e;
    }
    *out = f;
    return true;
}

__device__ inline bool secular_c(const Stack& st, double freq, double c, double* out) {
    const double omega = 2.0 * 3.14159265358979323846 * freq;
    double v;
    if (!secular(st, omega, omega / c, &v) || isnan(v) || isinf(v)) return false;
    *out = v;
    return true;
}

__device__ inline bool sign_change(double a, double b) { return (a < 0.0 && b > 0.0) || (a > 0.0 && b < 0.0); }

struct ModeArgs {
    const double* freqs;
    int nf, samples, max_modes;
    double tol, lo, hi;
    double* vel;   // [nf][max_modes]
    int* count;    // [nf]; -1 - found when more than max_modes
};

__global__ void __launch_bounds__(kThreads) k_modes(const __grid_constant__ Stack st, ModeArgs a) {
    extern __shared__ double vals[];  // [samples + 1]
    unsigned char* ok = reinterpret_cast<unsigned char*>(vals + a.samples + 1);
    __shared__ int br[kMaxModes + 1];
    __shared__ double root[kMaxModes];
    __shared__ int nbr;
    const int fi = blockIdx.x;
    const double freq = a.freqs[fi];
    // the scan's velocities with one rounding per operation (no contraction
    // into FMAs), so the host can form the very same doubles: lo + i step
    const double step = __dsub_rn(__dmul_rn(a.hi, 1.0 - 1e-9), a.lo) / a.samples;
    for (int i = threadIdx.x; i <= a.samples; i += blockDim.x) {
        const double c = i == 0 ? a.lo : __dadd_rn(a.lo, __dmul_rn((double)i, step));
        double v = 0.0;
        ok[i] = secular_c(st, freq, c, &v) ? 1 : 0;
        vals[i] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int n = 0;
        for (int i = 1; i <= a.samples; i++)
            if (ok[i] && ok[i - 1] && sign_change(vals[i - 1], vals[i])) {
                if (n < kMaxModes) br[n] = i;
                n++;
            }
        nbr = n;
    }
    __syncthreads();
    const int nb = nbr < kMaxModes ? nbr : kMaxModes;
    // Bisection, kSpecDepth steps per round: the kSpecNodes lanes of a group
    // evaluate every midpoint the next kSpecDepth steps could visit (a complete
    // binary tree of brackets, each computed by the same halvings the
    // sequential search would make), then each lane walks the path the
    // sequential search takes through them. The midpoints, the decisions and
    // the stopping rules are those of the one-thread search, so the roots are
    // the same doubles; the dependent chain is kSpecDepth times shorter.
    const int lane = threadIdx.x & 31, grp = lane / kSpecLanes, node = lane % kSpecLanes;
    const int groups = (blockDim.x / 32) * (32 / kSpecLanes);
    const int gid = (threadIdx.x / 32) * (32 / kSpecLanes) + grp;
    for (int b0 = 0; b0 < nb; b0 += groups) {
        const int b = b0 + gid;
        const bool active = b < nb;
        double lo = 0.0, hi = 0.0, flo = 0.0, r = -1.0;
        bool done = !active;
        if (active) {
            const int i = br[b];
            lo = i - 1 == 0 ? a.lo : __dadd_rn(a.lo, __dmul_rn((double)(i - 1), step));
            hi = __dadd_rn(a.lo, __dmul_rn((double)i, step));
            flo = vals[i - 1];  // the scan's value at this very velocity (defined: a bracket end)
        }
        int it = 0;
        while (__any_sync(0xffffffffu, !done)) {
            // this lane's tree node: heap index h = node + 1 at depth floor(log2 h)
            double v = 0.0;
            int vok = 0;
            if (!done && node < kSpecNodes) {
                const int h = node + 1, d = 31 - __clz(h);
                double nlo = lo, nhi = hi;
                for (int sh = d - 1; sh >= 0; sh--) {
                    const double mid = 0.5 * (nlo + nhi);
                    if ((h >> sh) & 1) nlo = mid; else nhi = mid;
                }
                vok = secular_c(st, freq, 0.5 * (nlo + nhi), &v) ? 1 : 0;
            }
            int h = 1;
            for (int step_ = 0; step_ < kSpecDepth; step_++) {
                const int src = (lane & ~(kSpecLanes - 1)) + (h - 1);
                const double hv = __shfl_sync(0xffffffffu, v, src);
                const int hok = __shfl_sync(0xffffffffu, vok, src);
                if (done) continue;
                if (it >= 200) {
                    r = 0.5 * (lo + hi);
                    done = true;
                    continue;
                }
                const double mid = 0.5 * (lo + hi);
                if (mid == lo || mid == hi || (hi - lo) < a.tol * mid) {
                    r = mid;
                    done = true;
                    continue;
                }
                it++;
                if (!hok) {
                    done = true;  // undefined inside the bracket: no root
                    continue;
                }
                if (sign_change(flo, hv)) {
                    hi = mid;
                    h = 2 * h;
                } else {
                    lo = mid;
                    flo = hv;
                    h = 2 * h + 1;
                }
            }
        }
        if (active && node == 0) root[b] = r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int n = 0;
        for (int b = 0; b < nb; b++)
            if (root[b] > 0.0) {
                if (n < a.max_modes) a.vel[(size_t)fi * a.max_modes + n] = root[b];
                n++;
            }
        a.count[fi] = (nbr > kMaxModes || n > a.max_modes) ? -1 - n : n;
    }
}

__global__ void k_secular(const __grid_constant__ Stack st, const double* f, const double* c, long long n,
                          double* out, int* ok) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    ok[i] = secular_c(st, f[i], c[i], &v) ? 1 : 0;
    out[i] = v;
}

}  // namespace disp
}  // namespace gfk

namespace {

int dfail(gfk_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

#define DS_CUDA(ctx, call)                                                                         \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return dfail(ctx, e_ == cudaErrorMemoryAllocation ? GFK_ENOMEM : GFK_ECUDA,            \
                         std::string(#call ": ") + cudaGetErrorString(e_));                        \
    } while (0)

int make_stack(gfk_ctx* ctx, const gfk_medium* m, gfk::disp::Stack* st) {
    if (!m || !m->layers || m->count < 1) return dfail(ctx, GFK_ESTACK, "layer: empty stack");
    const int v = gfk_stack_validate(m);
    if (v != GFK_OK) return dfail(ctx, v, "layer: stack failed validation");
    if (m->count > gfk::disp::kMaxLayers) return dfail(ctx, GFK_ELIMIT, "disp: more than 64 stack entries");
    st->n = m->count;
    st->mu_ref = 0.0;
    for (int i = 0; i < m->count; i++) {
        const gfk_layer& l = m->layers[i];
        st->l[i] = gfk::disp::Layer4{l.thickness_m, l.vp_mps, l.vs_mps, l.density_kgm3};
        st->mu_ref = std::max(st->mu_ref, l.density_kgm3 * l.vs_mps * l.vs_mps);
    }
    return GFK_OK;
}

struct DBuf {
    gfk_ctx* ctx;
    void* p = nullptr;
    ~DBuf() {
        if (p) cudaFreeAsync(p, ctx->stream);
    }
};

}  // namespace

extern "C" {

int gfk_dispersion_modes(gfk_ctx* ctx, const gfk_medium* m, const double* freqs, int32_t nf, gfk_search opt,
                         int32_t max_modes, double* velocities, int32_t* counts) {
    if (!ctx || !m || !freqs || !velocities || !counts) return GFK_EARG;
    if (nf < 0 || max_modes < 1 || max_modes > gfk::disp::kMaxModes)
        return dfail(ctx, GFK_EARG, "disp: max_modes must lie in [1, 64]");
    gfk::disp::Stack st;
    int s0 = make_stack(ctx, m, &st);
    if (s0) return s0;
    for (int i = 0; i < nf; i++)
        if (!(freqs[i] > 0)) {
            char buf[96];
            snprintf(buf, sizeof buf, "disp: frequency must be positive, got %g Hz", freqs[i]);
            return dfail(ctx, GFK_EARG, buf);
        }
    const int samples = opt.samples > 0 ? opt.samples : 2000;
    const double tol = opt.tolerance > 0 ? opt.tolerance : 1e-10;
    if (samples > gfk::disp::kMaxSamples) return dfail(ctx, GFK_ELIMIT, "disp: at most 16384 samples");
    if (nf == 0) return GFK_OK;
    double vmin = m->layers[0].vs_mps;
    for (int i = 0; i < m->count; i++) vmin = std::min(vmin, m->layers[i].vs_mps);
    const double lo = 0.85 * vmin, hi = m->layers[m->count - 1].vs_mps;  // disp.go:62-65
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    DBuf d_f{ctx}, d_v{ctx}, d_c{ctx};
    DS_CUDA(ctx, cudaMallocAsync(&d_f.p, sizeof(double) * nf, s));
    DS_CUDA(ctx, cudaMallocAsync(&d_v.p, sizeof(double) * nf * max_modes, s));
    DS_CUDA(ctx, cudaMallocAsync(&d_c.p, sizeof(int) * nf, s));
    DS_CUDA(ctx, cudaMemcpyAsync(d_f.p, freqs, sizeof(double) * nf, cudaMemcpyHostToDevice, s));
    const size_t smem = sizeof(double) * (samples + 1) + (samples + 1);
    if (smem > 48 * 1024)
        DS_CUDA(ctx, cudaFuncSetAttribute(gfk::disp::k_modes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    gfk::disp::ModeArgs a{static_cast<const double*>(d_f.p), nf, samples, max_modes, tol, lo, hi,
                          static_cast<double*>(d_v.p), static_cast<int*>(d_c.p)};
    gfk::disp::k_modes<<<nf, gfk::disp::kThreads, smem, s>>>(st, a);
    ctx->launches++;
    DS_CUDA(ctx, cudaGetLastError());
    std::vector<int> cnt(nf);
    DS_CUDA(ctx, cudaMemcpyAsync(velocities, d_v.p, sizeof(double) * nf * max_modes, cudaMemcpyDeviceToHost, s));
    DS_CUDA(ctx, cudaMemcpyAsync(cnt.data(), d_c.p, sizeof(int) * nf, cudaMemcpyDeviceToHost, s));
    DS_CUDA(ctx, cudaStreamSynchronize(s));
    int status = GFK_OK;
    for (int i = 0; i < nf; i++) {
        counts[i] = cnt[i] < 0 ? -1 - cnt[i] : cnt[i];
        if (cnt[i] < 0) status = GFK_ELIMIT;
    }
    if (status) dfail(ctx, status, "disp: more modes than max_modes at some frequency");
    return status;
}

int gfk_secular(gfk_ctx* ctx, const gfk_medium* m, const double* freqs, const double* velocities, int64_t n,
                double* out, int32_t* ok) {
    if (!ctx || !m || !freqs || !velocities || !out || !ok || n < 0) return GFK_EARG;
    gfk::disp::Stack st;
    int s0 = make_stack(ctx, m, &st);
    if (s0) return s0;
    if (n == 0) return GFK_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    DBuf d_f{ctx}, d_c{ctx}, d_o{ctx}, d_k{ctx};
    DS_CUDA(ctx, cudaMallocAsync(&d_f.p, sizeof(double) * n, s));
    DS_CUDA(ctx, cudaMallocAsync(&d_c.p, sizeof(double) * n, s));
    DS_CUDA(ctx, cudaMallocAsync(&d_o.p, sizeof(double) * n, s));
    DS_CUDA(ctx, cudaMallocAsync(&d_k.p, sizeof(int) * n, s));
    DS_CUDA(ctx, cudaMemcpyAsync(d_f.p, freqs, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    DS_CUDA(ctx, cudaMemcpyAsync(d_c.p, velocities, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    gfk::disp::k_secular<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(
        st, static_cast<const double*>(d_f.p), static_cast<const double*>(d_c.p), n, static_cast<double*>(d_o.p),
        static_cast<int*>(d_k.p));
    ctx->launches++;
    DS_CUDA(ctx, cudaGetLastError());
    DS_CUDA(ctx, cudaMemcpyAsync(out, d_o.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    DS_CUDA(ctx, cudaMemcpyAsync(ok, d_k.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    DS_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

}  // extern "C"
