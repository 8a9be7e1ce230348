// gfk_consume.cu — bank consumption on the GPU: the interpolation tables of
// Bank.prepare, Bank.Response between grid ranges, and the causal impulse
// responses a sensor engine builds from them.
//
//   tables     internal/bank/interp.go:66-102 — per bin, walking the range
//              axis: log|v| (-1e308 for an exact zero) and the phase unwrapped
//              by folding each step into (-pi, pi]; FP64 from the FP32 payload.
//   response   internal/bank/interp.go:29-54 with format.go:295-309's bracket:
//              linear in log-magnitude and in unwrapped phase between the two
//              bracketing ranges; zero where either end is an exact zero.
//   impulse    internal/dsp/dsp.go:232-261 (CausalImpulseResponseAt) at the
//              bank's own transform size, fed as internal/sensing does
//              (sensing.go:196-204, propagation.go:84-104): velocity i w u(r, f)
//              times the sensor's response, tapered above 0.8 Nyquist,
//              inverse-transformed (1/n), the first `length` samples kept.
//
// One thread per bin builds the tables (the unwrap is sequential in range);
// one block per query range builds its half spectrum in shared memory and runs
// the inverse real transform there as an n/2-point complex FFT (gfk_fft.cuh),
// n = the bank's Samples <= 4096.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/gfk.h"
#include "gfk_ctx.h"
#include "gfk_fft.cuh"
#include "gfk_kernels.cuh"

namespace gfk {
namespace consume {

constexpr double kNegInf = -1e308;  // interp.go:56
constexpr int kThreads = 256;
constexpr int kMaxSamples = 4096;

__global__ void k_tables(const float* __restrict__ data, int count, int bins, double* __restrict__ logmag,
                         double* __restrict__ phase) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= bins) return;
    const double two_pi = 2.0 * 3.14159265358979323846;
    double prev = 0.0, unwrapped = 0.0;
    for (int i = 0; i < count; i++) {
        const size_t j = (size_t)i * bins + k;
        const double re = data[2 * j], im = data[2 * j + 1];
        const double mag = hypot(re, im);
        if (mag == 0.0) {
            logmag[j] = kNegInf;
            phase[j] = unwrapped;
            continue;
        }
        logmag[j] = log(mag);
        const double w = atan2(im, re);
        if (i == 0) {
            unwrapped = w;
        } else {
            double d = w - prev;
            d -= two_pi * round(d / two_pi);  // halves away from zero, as Go's math.Round
            unwrapped += d;
        }
        prev = w;
        phase[j] = unwrapped;
    }
}

struct ImpulseArgs {
    const double* logmag;
    const double* phase;
    int count, bins, n, length;
    const int* lo;          // [nq] lower bracketing range index
    const double* frac;     // [nq]
    const cd* sensor;       // [bins] or null
    int velocity;
    double fs;
    const cd* tw;           // [n/2]
    double* out;            // [nq][length]
};

// The inverse real transform of the half spectrum H_0..H_m (m = n/2) as one
// complex transform of size m (the even/odd split of the output): with
// w = e^{2 pi i / n},
//   Z_k = (H_k + conj(H_{m-k})) + i w^k (H_k - conj(H_{m-k})),  k < m,
//   z = IDFT_m(Z) / n  gives  y_2j = Re z_j,  y_2j+1 = Im z_j,
// and IDFT_m(Z) = conj(DFT_m(conj Z)). Shared memory: m + 1 values.
__global__ void __launch_bounds__(kThreads) k_impulse(ImpulseArgs a) {
    extern __shared__ cd x[];  // [m + 1]: H, then conj(Z) (bit-reversed), then its transform
    const int q = blockIdx.x;
    const int n = a.n, m = n / 2;
    const int logm = 31 - __clz(m);
    const int lo = a.lo[q];
    const int hi = a.count == 1 ? lo : lo + 1;
    const double frac = a.frac[q];
    const double nyq = a.fs / 2, taper_from = 0.8 * nyq;
    const double pi = 3.14159265358979323846;
    for (int k = threadIdx.x; k <= m; k += blockDim.x) {
        cd h = mk(0.0);
        const double f = k * a.fs / n;
        if (k > 0 && k < a.bins) {
            const size_t i0 = (size_t)lo * a.bins + k, i1 = (size_t)hi * a.bins + k;
            if (a.logmag[i0] != kNegInf && a.logmag[i1] != kNegInf) {
                const double lm = a.logmag[i0] + frac * (a.logmag[i1] - a.logmag[i0]);
                const double ph = a.phase[i0] + frac * (a.phase[i1] - a.phase[i0]);
                double sn, cs;
                sincos(ph, &sn, &cs);
                const double mg = exp(lm);
                h = mk(mg * cs, mg * sn);
                if (a.velocity) h = mk(0.0, 2.0 * pi * f) * h;
                if (a.sensor) h = h * a.sensor[k];
            }
            if (f > taper_from) h = h * (0.5 * (1.0 + cos(pi * (f - taper_from) / (nyq - taper_from))));
        }
        if (k == 0 || k == m) h.im = 0.0;  // the real transform reads only their real parts
        x[k] = h;
    }
    __syncthreads();
    // conj(Z_k) and conj(Z_{m-k}) by the thread that owns the pair (k, m - k)
    for (int k = threadIdx.x; k <= m / 2; k += blockDim.x) {
        const int k2 = m - k;
        const cd hk = x[k], hk2 = x[k2];
        const cd wk = mk(a.tw[k].re, -a.tw[k].im);  // e^{2 pi i k / n}
        const cd zk = (hk + mk(hk2.re, -hk2.im)) + cmul_i(wk * (hk - mk(hk2.re, -hk2.im)));
        x[k] = mk(zk.re, -zk.im);
        if (k > 0 && k < m / 2) {
            const cd wk2 = mk(a.tw[k2].re, -a.tw[k2].im);
            const cd zk2 = (hk2 + mk(hk.re, -hk.im)) + cmul_i(wk2 * (hk2 - mk(hk.re, -hk.im)));
            x[k2] = mk(zk2.re, -zk2.im);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; logm > 0 && i < m; i += blockDim.x) {  // into bit-reversed order
        const int r = bitrev(i, logm);
        if (i < r) {
            const cd t = x[i];
            x[i] = x[r];
            x[r] = t;
        }
    }
    __syncthreads();
    fft_pow2_dit_inplace(x, m, a.tw, n);
    const double inv = 1.0 / n;
    for (int t = threadIdx.x; t < a.length; t += blockDim.x) {
        const cd w = x[t >> 1];
        a.out[(size_t)q * a.length + t] = ((t & 1) ? -w.im : w.re) * inv;
    }
}

}  // namespace consume
}  // namespace gfk

namespace {

int cfail(gfk_ctx* ctx, int status, const char* msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

#define CS_CUDA(ctx, call)                                                                         \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            if (ctx) (ctx)->last_error = std::string(#call ": ") + cudaGetErrorString(e_);         \
            return e_ == cudaErrorMemoryAllocation ? GFK_ENOMEM : GFK_ECUDA;                        \
        }                                                                                          \
    } while (0)

// format.go:295-309: the lower bracketing range index and the fraction
// between it and the next, on the host; a range outside the grid is GFK_EARG.
int bracket(gfk_ctx* ctx, int count, double min_m, double max_m, const double* ranges, int nq, std::vector<int>& lo,
            std::vector<double>& frac) {
    const double spacing = count > 1 ? (max_m - min_m) / (count - 1) : 0.0;
    for (int q = 0; q < nq; q++) {
        const double r = ranges[q];
        if (!(r >= min_m && r <= max_m)) {
            char buf[160];
            snprintf(buf, sizeof buf, "bank: range %g m is outside the bank's %g to %g m", r, min_m, max_m);
            return cfail(ctx, GFK_EARG, buf);
        }
        if (count == 1) {
            lo[q] = 0;
            frac[q] = 0.0;
            continue;
        }
        const double x = (r - min_m) / spacing;
        int l = (int)std::floor(x);
        if (l >= count - 1) {
            lo[q] = count - 2;
            frac[q] = 1.0;
        } else {
            lo[q] = l;
            frac[q] = x - l;
        }
    }
    return GFK_OK;
}

// Device copies of a payload and its tables, freed together.
struct Tables {
    gfk_ctx* ctx = nullptr;
    float* data = nullptr;
    double *logmag = nullptr, *phase = nullptr;
    ~Tables() {
        if (!ctx) return;
        if (data) cudaFreeAsync(data, ctx->stream);
        if (logmag) cudaFreeAsync(logmag, ctx->stream);
        if (phase) cudaFreeAsync(phase, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
    }
};

int build_tables(gfk_ctx* ctx, const float* payload, int count, int bins, Tables& t) {
    const size_t cells = (size_t)count * bins;
    t.ctx = ctx;
    CS_CUDA(ctx, cudaMallocAsync((void**)&t.data, cells * 2 * sizeof(float), ctx->stream));
    CS_CUDA(ctx, cudaMallocAsync((void**)&t.logmag, cells * sizeof(double), ctx->stream));
    CS_CUDA(ctx, cudaMallocAsync((void**)&t.phase, cells * sizeof(double), ctx->stream));
    CS_CUDA(ctx, cudaMemcpyAsync(t.data, payload, cells * 2 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    gfk::consume::k_tables<<<(bins + 127) / 128, 128, 0, ctx->stream>>>(t.data, count, bins, t.logmag, t.phase);
    ctx->launches++;
    CS_CUDA(ctx, cudaGetLastError());
    return GFK_OK;
}

}  // namespace

extern "C" {

int gfk_bank_tables(gfk_ctx* ctx, const float* payload, int32_t count, int32_t bins, double* logmag,
                    double* phase) {
    if (!ctx || !payload || !logmag || !phase) return GFK_EARG;
    if (count < 1 || bins < 1) return cfail(ctx, GFK_EARG, "bank: empty payload");
    cudaSetDevice(ctx->device);
    Tables t;
    const int st = build_tables(ctx, payload, count, bins, t);
    if (st) return st;
    const size_t cells = (size_t)count * bins;
    CS_CUDA(ctx, cudaMemcpyAsync(logmag, t.logmag, cells * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CS_CUDA(ctx, cudaMemcpyAsync(phase, t.phase, cells * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CS_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return GFK_OK;
}

int gfk_bank_impulse_responses(gfk_ctx* ctx, const float* payload, int32_t count, int32_t bins, double min_m,
                               double max_m, double fs_hz, int32_t samples, const double* ranges, int32_t nq,
                               const double* sensor, int32_t velocity, int32_t length, double* out) {
    if (!ctx || !payload || !ranges || !out) return GFK_EARG;
    if (count < 1 || nq < 0) return cfail(ctx, GFK_EARG, "bank: empty payload");
    if (samples < 2 || (samples & (samples - 1)) || bins != samples / 2 + 1)
        return cfail(ctx, GFK_EARG, "bank: samples must be a power of two with bins = samples/2 + 1");
    if (samples > gfk::consume::kMaxSamples)
        return cfail(ctx, GFK_ELIMIT, "bank: impulse responses are built for samples <= 4096");
    if (length <= 0) return cfail(ctx, GFK_EARG, "dsp: impulse response length must be positive");
    if (!(fs_hz > 0)) return cfail(ctx, GFK_EARG, "dsp: sample rate must be positive");
    if (samples < length) return cfail(ctx, GFK_EARG, "dsp: transform size is shorter than the samples to keep");
    if (nq == 0) return GFK_OK;
    std::vector<int> lo(nq);
    std::vector<double> frac(nq);
    if (int st = bracket(ctx, count, min_m, max_m, ranges, nq, lo, frac)) return st;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    Tables t;
    int st = build_tables(ctx, payload, count, bins, t);
    if (st) return st;
    std::vector<double> tw(samples);
    for (int m = 0; m < samples / 2; m++) {
        const double a = -2.0 * M_PI * m / samples;
        tw[2 * m] = std::cos(a);
        tw[2 * m + 1] = std::sin(a);
    }
    struct Buf {
        gfk_ctx* ctx;
        void* p = nullptr;
        ~Buf() {
            if (p) cudaFreeAsync(p, ctx->stream);
        }
    } d_lo{ctx}, d_frac{ctx}, d_tw{ctx}, d_sensor{ctx}, d_out{ctx};
    CS_CUDA(ctx, cudaMallocAsync(&d_lo.p, nq * sizeof(int), s));
    CS_CUDA(ctx, cudaMallocAsync(&d_frac.p, nq * sizeof(double), s));
    CS_CUDA(ctx, cudaMallocAsync(&d_tw.p, samples * sizeof(double), s));
    CS_CUDA(ctx, cudaMallocAsync(&d_out.p, (size_t)nq * length * sizeof(double), s));
    CS_CUDA(ctx, cudaMemcpyAsync(d_lo.p, lo.data(), nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CS_CUDA(ctx, cudaMemcpyAsync(d_frac.p, frac.data(), nq * sizeof(double), cudaMemcpyHostToDevice, s));
    CS_CUDA(ctx, cudaMemcpyAsync(d_tw.p, tw.data(), samples * sizeof(double), cudaMemcpyHostToDevice, s));
    if (sensor) {
        CS_CUDA(ctx, cudaMallocAsync(&d_sensor.p, (size_t)bins * 2 * sizeof(double), s));
        CS_CUDA(ctx, cudaMemcpyAsync(d_sensor.p, sensor, (size_t)bins * 2 * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    const size_t smem = (size_t)(samples / 2 + 1) * sizeof(cd);
    if (smem > 48 * 1024)
        CS_CUDA(ctx, cudaFuncSetAttribute(gfk::consume::k_impulse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    gfk::consume::ImpulseArgs a{t.logmag, t.phase, count, bins, samples, length,
                                static_cast<const int*>(d_lo.p), static_cast<const double*>(d_frac.p),
                                static_cast<const cd*>(d_sensor.p), velocity, fs_hz,
                                static_cast<const cd*>(d_tw.p), static_cast<double*>(d_out.p)};
    gfk::consume::k_impulse<<<nq, gfk::consume::kThreads, smem, s>>>(a);
    ctx->launches++;
    CS_CUDA(ctx, cudaGetLastError());
    CS_CUDA(ctx, cudaMemcpyAsync(out, d_out.p, (size_t)nq * length * sizeof(double), cudaMemcpyDeviceToHost, s));
    CS_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

}  // extern "C"

// ------------------------------------------------- device-resident bank --

struct gfk_bank_dev {
    gfk_ctx* ctx = nullptr;
    int count = 0, bins = 0, samples = 0;
    double min_m = 0, max_m = 0, fs = 0;
    Tables t;                      // payload and Bank.prepare tables
    double* d_tw = nullptr;        // e^{-2 pi i m / samples}, m < samples/2
    int* d_lo = nullptr;           // per-query scratch, grown on demand
    double* d_frac = nullptr;
    size_t q_cap = 0;
    double* d_sensor = nullptr;    // bins complex
    double* d_out = nullptr;       // host-output staging
    size_t out_cap = 0;
};

namespace {

void bank_dev_free(gfk_bank_dev* b) {
    cudaStream_t s = b->ctx->stream;
    void* ptrs[] = {b->d_tw, b->d_lo, b->d_frac, b->d_sensor, b->d_out};
    for (void* p : ptrs)
        if (p) cudaFreeAsync(p, s);
    // b->t frees the payload and the tables when b is deleted
}

template <typename T>
int grow(gfk_ctx* ctx, T** p, size_t* cap, size_t n) {
    if (n <= *cap) return GFK_OK;
    if (*p) cudaFreeAsync(*p, ctx->stream);
    *p = nullptr;
    *cap = 0;
    CS_CUDA(ctx, cudaMallocAsync((void**)p, n * sizeof(T), ctx->stream));
    *cap = n;
    return GFK_OK;
}

}  // namespace

void gfk_release_banks(gfk_ctx* ctx) {
    for (gfk_bank_dev* b : ctx->banks) {
        bank_dev_free(b);
        delete b;
    }
    ctx->banks.clear();
}

extern "C" {

int gfk_bank_device_open(gfk_ctx* ctx, const float* payload, int32_t count, int32_t bins, double min_m,
                         double max_m, double fs_hz, int32_t samples, gfk_bank_dev** out) {
    if (!ctx || !payload || !out) return GFK_EARG;
    *out = nullptr;
    if (count < 1) return cfail(ctx, GFK_EARG, "bank: empty payload");
    if (samples < 2 || (samples & (samples - 1)) || bins != samples / 2 + 1)
        return cfail(ctx, GFK_EARG, "bank: samples must be a power of two with bins = samples/2 + 1");
    if (samples > gfk::consume::kMaxSamples)
        return cfail(ctx, GFK_ELIMIT, "bank: impulse responses are built for samples <= 4096");
    if (!(fs_hz > 0)) return cfail(ctx, GFK_EARG, "dsp: sample rate must be positive");
    if (!(min_m <= max_m)) return cfail(ctx, GFK_EARG, "bank: range grid max is below its min");
    cudaSetDevice(ctx->device);
    gfk_bank_dev* b = new gfk_bank_dev();
    b->ctx = ctx;
    b->count = count;
    b->bins = bins;
    b->samples = samples;
    b->min_m = min_m;
    b->max_m = max_m;
    b->fs = fs_hz;
    std::vector<double> tw(samples);
    for (int m = 0; m < samples / 2; m++) {
        const double a = -2.0 * M_PI * m / samples;
        tw[2 * m] = std::cos(a);
        tw[2 * m + 1] = std::sin(a);
    }
    int st = build_tables(ctx, payload, count, bins, b->t);
    size_t cap = 0;
    if (!st) st = grow(ctx, &b->d_tw, &cap, (size_t)samples);
    if (!st && cudaMemcpyAsync(b->d_tw, tw.data(), samples * sizeof(double), cudaMemcpyHostToDevice, ctx->stream) !=
                   cudaSuccess)
        st = cfail(ctx, GFK_ECUDA, "bank: twiddle upload failed");
    if (!st && cudaStreamSynchronize(ctx->stream) != cudaSuccess)  // the caller may free its payload now
        st = cfail(ctx, GFK_ECUDA, "bank: upload or table build failed");
    if (st) {
        bank_dev_free(b);
        delete b;
        return st;
    }
    ctx->banks.push_back(b);
    *out = b;
    return GFK_OK;
}

int gfk_bank_device_impulse_responses(gfk_bank_dev* b, const double* ranges, int32_t nq, const double* sensor,
                                      int32_t velocity, int32_t length, double* out, int32_t out_on_device) {
    if (!b || !ranges || !out) return GFK_EARG;
    gfk_ctx* ctx = b->ctx;
    if (nq < 0) return cfail(ctx, GFK_EARG, "bank: negative query count");
    if (length <= 0) return cfail(ctx, GFK_EARG, "dsp: impulse response length must be positive");
    if (b->samples < length) return cfail(ctx, GFK_EARG, "dsp: transform size is shorter than the samples to keep");
    if (nq == 0) return GFK_OK;
    std::vector<int> lo(nq);
    std::vector<double> frac(nq);
    if (int st = bracket(ctx, b->count, b->min_m, b->max_m, ranges, nq, lo, frac)) return st;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    size_t qcap = b->q_cap, fcap = b->q_cap;
    if (int st = grow(ctx, &b->d_lo, &qcap, (size_t)nq)) return st;
    if (int st = grow(ctx, &b->d_frac, &fcap, (size_t)nq)) return st;
    b->q_cap = std::min(qcap, fcap);
    // the host vectors are synchronised below before they go out of scope
    CS_CUDA(ctx, cudaMemcpyAsync(b->d_lo, lo.data(), nq * sizeof(int), cudaMemcpyHostToDevice, s));
    CS_CUDA(ctx, cudaMemcpyAsync(b->d_frac, frac.data(), nq * sizeof(double), cudaMemcpyHostToDevice, s));
    const cd* d_sensor = nullptr;
    if (sensor) {
        size_t scap = b->d_sensor ? (size_t)2 * b->bins : 0;
        if (int st = grow(ctx, &b->d_sensor, &scap, (size_t)2 * b->bins)) return st;
        CS_CUDA(ctx, cudaMemcpyAsync(b->d_sensor, sensor, (size_t)b->bins * 2 * sizeof(double),
                                     cudaMemcpyHostToDevice, s));
        d_sensor = reinterpret_cast<const cd*>(b->d_sensor);
    }
    double* dst = out;
    if (!out_on_device) {
        if (int st = grow(ctx, &b->d_out, &b->out_cap, (size_t)nq * length)) return st;
        dst = b->d_out;
    }
    const size_t smem = (size_t)(b->samples / 2 + 1) * sizeof(cd);
    if (smem > 48 * 1024)
        CS_CUDA(ctx, cudaFuncSetAttribute(gfk::consume::k_impulse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    gfk::consume::ImpulseArgs a{b->t.logmag, b->t.phase, b->count, b->bins, b->samples, length, b->d_lo, b->d_frac,
                                d_sensor, velocity, b->fs, reinterpret_cast<const cd*>(b->d_tw), dst};
    gfk::consume::k_impulse<<<nq, gfk::consume::kThreads, smem, s>>>(a);
    ctx->launches++;
    CS_CUDA(ctx, cudaGetLastError());
    if (!out_on_device)
        CS_CUDA(ctx, cudaMemcpyAsync(out, b->d_out, (size_t)nq * length * sizeof(double), cudaMemcpyDeviceToHost, s));
    // the query uploads read host vectors local to this call: wait for them
    // (and, for host output, for the responses)
    CS_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

int gfk_bank_device_close(gfk_bank_dev* b) {
    if (!b) return GFK_OK;
    gfk_ctx* ctx = b->ctx;
    cudaSetDevice(ctx->device);
    auto& v = ctx->banks;
    v.erase(std::remove(v.begin(), v.end(), b), v.end());
    bank_dev_free(b);
    delete b;
    return GFK_OK;
}

}  // extern "C"
