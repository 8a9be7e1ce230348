// gfk_surrogate.cu — host runtime of the surrogate network and the sweep
// metrics: label data sets in device memory, the network's parameters and
// working buffers, the training step captured as one CUDA graph, chunked
// inference, held-out evaluation.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/gfk.h"
#include "gfk_ctx.h"
#include "gfk_kernels.cuh"
#include "gfk_mlp.cuh"

using gfk::mlp::bf16;
namespace M = gfk::mlp;

namespace {

int sfail(gfk_ctx* ctx, int status, const char* fmt, ...) {
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return status;
}

#define SG_CUDA(ctx, call)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return sfail((ctx), e_ == cudaErrorMemoryAllocation ? GFK_ENOMEM : GFK_ECUDA, "%s: %s", \
                         #call, cudaGetErrorString(e_));                                            \
    } while (0)

#define SG_TRY(call)              \
    do {                          \
        int st_ = (call);         \
        if (st_ != GFK_OK) return st_; \
    } while (0)

template <class T>
int salloc(gfk_ctx* ctx, T** p, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), bytes, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return sfail(ctx, GFK_ENOMEM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return GFK_OK;
}

template <class T>
void sfree(gfk_ctx* ctx, T*& p) {
    if (p) cudaFreeAsync(p, ctx->stream);
    p = nullptr;
}

// Round to nearest even, FP32 -> BF16 bits.
uint16_t to_bf16(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return static_cast<uint16_t>((u >> 16) | ((u & 0xffff) ? 0x40 : 0));
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return static_cast<uint16_t>(u >> 16);
}

constexpr int kLayers = 5;                 // GEMM layers (input + four hidden)
constexpr int kW = M::kWidth;
constexpr long long kChunkRows = 1 << 20;  // inference rows per pass
constexpr int kHistCap = 4096;             // loss history slots per graph replay block

}  // namespace

// ---------------------------------------------------------------- dataset --

struct gfk_dataset {
    gfk_ctx* ctx = nullptr;
    int nparam = 0, nsoil = 0, nr = 0, nf = 0;
    double floor_rel = 0;
    std::vector<double> ranges, freqs;
    std::vector<float> soilfeat;  // [nsoil][kSoilStride]
    float* d_labels = nullptr;
    float* d_lmax = nullptr;      // [nsoil][nr] log max_f |G|
    float* d_soilfeat = nullptr;
    double *d_ranges = nullptr, *d_freqs = nullptr, *d_stats = nullptr;
    std::vector<char> filled;
};

// ---------------------------------------------------------------- network --

struct NetLayer {
    int in = 0, out = 0, splits = 1;
    long long woff = 0, boff = 0;
    bf16 *wb = nullptr, *wt = nullptr;
    float* part = nullptr;
};

struct gfk_net {
    gfk_ctx* ctx = nullptr;
    gfk_net_config cfg{};
    int B = 0;
    long long nparam = 0, w6off = 0, b6off = 0;
    NetLayer L[kLayers];
    float *d_p = nullptr, *d_m = nullptr, *d_v = nullptr;
    M::TrainScalars* d_ts = nullptr;
    std::vector<float> four;
    float* d_four = nullptr;
    M::FeatureDomain dom{1, 2, 1, 2};
    float ms[4] = {0, 1, 0, 1};
    bool scales = false;
    // training
    bf16 *X = nullptr, *XT = nullptr;
    float* Y = nullptr;
    bf16 *Z[kLayers] = {}, *H[kLayers] = {}, *HT[kLayers] = {}, *dZ[kLayers] = {}, *dZT[kLayers] = {};
    M::AdamSeg* d_seg = nullptr;
    float *Cw = nullptr, *gpart = nullptr, *lpart = nullptr, *gb = nullptr, *hist = nullptr, *gflat = nullptr;
    int* d_status = nullptr;
    int* d_train = nullptr;
    int ntrain = 0;
    int ir0 = 0, nir = 0;  // range window of the captured step
    const gfk_dataset* graph_ds = nullptr;
    std::vector<int> graph_train;
    cudaGraphExec_t gexec = nullptr;
    M::AdamArgs adam{};
    // weight-gradient GEMMs run on a second stream, each as soon as its dZ^T
    // exists, beside the backward-data chain (forked and joined by events, so
    // a captured step holds them as parallel branches)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_dz[kLayers] = {}, ev_join = nullptr;
    // inference
    bf16 *iX = nullptr, *iH0 = nullptr, *iH1 = nullptr;
    float* iT = nullptr;
    double* d_acc = nullptr;
};

namespace {

void dataset_free(gfk_dataset* d) {
    gfk_ctx* c = d->ctx;
    sfree(c, d->d_labels);
    sfree(c, d->d_lmax);
    sfree(c, d->d_soilfeat);
    sfree(c, d->d_ranges);
    sfree(c, d->d_freqs);
    sfree(c, d->d_stats);
    cudaStreamSynchronize(c->stream);
}

void net_free(gfk_net* n) {
    gfk_ctx* c = n->ctx;
    if (n->gexec) cudaGraphExecDestroy(n->gexec);
    n->gexec = nullptr;
    if (n->side) cudaStreamSynchronize(n->side);
    for (cudaEvent_t& e : n->ev_dz)
        if (e) cudaEventDestroy(e);
    if (n->ev_join) cudaEventDestroy(n->ev_join);
    if (n->side) cudaStreamDestroy(n->side);
    n->side = nullptr;
    for (auto& l : n->L) {
        sfree(c, l.wb);
        sfree(c, l.wt);
        sfree(c, l.part);
    }
    for (int l = 0; l < kLayers; l++) {
        sfree(c, n->Z[l]);
        sfree(c, n->H[l]);
        sfree(c, n->HT[l]);
        sfree(c, n->dZ[l]);
        sfree(c, n->dZT[l]);
    }
    float** fl[] = {&n->d_p, &n->d_m, &n->d_v, &n->d_four, &n->Y, &n->Cw, &n->gpart, &n->lpart, &n->gb,
                    &n->hist, &n->gflat, &n->iT};
    for (float** q : fl) sfree(c, *q);
    sfree(c, n->d_ts);
    sfree(c, n->d_seg);
    sfree(c, n->X);
    sfree(c, n->XT);
    sfree(c, n->iX);
    sfree(c, n->iH0);
    sfree(c, n->iH1);
    sfree(c, n->d_status);
    sfree(c, n->d_train);
    sfree(c, n->d_acc);
    cudaStreamSynchronize(c->stream);
}

int check_status(gfk_net* n) {
    int st = 0;
    SG_CUDA(n->ctx, cudaMemcpyAsync(&st, n->d_status, sizeof(int), cudaMemcpyDeviceToHost, n->ctx->stream));
    SG_CUDA(n->ctx, cudaStreamSynchronize(n->ctx->stream));
    if (st & gfk::kStTimeout) return sfail(n->ctx, GFK_ETIMEOUT, "a tensor-core GEMM wait ran out");
    return GFK_OK;
}

int gemm(gfk_net* n, int mode, const bf16* A, const bf16* Bm, int rowsA, int rowsB, int K, int splits,
         const M::GemmArgs& g, cudaStream_t on = nullptr) {
    const int r = M::launch_gemm(on ? on : n->ctx->stream, mode, A, Bm, rowsA, rowsB, K, splits, g);
    if (r) return sfail(n->ctx, r == 1 ? GFK_EARG : GFK_ECUDA, "GEMM launch refused (mode %d, %d x %d x %d): %d",
                        mode, rowsA, rowsB, K, r);
    n->ctx->launches++;
    return GFK_OK;
}

// Forward and backward of one batch already in X, XT, Y; gradient partials
// in L[].part, gb, gpart; loss partials in lpart.
int enqueue_fwd_bwd(gfk_net* n, bool train_step) {
    cudaStream_t s = n->ctx->stream;
    const int B = n->B;
    for (int l = 0; l < kLayers; l++) {
        M::GemmArgs g{};
        g.bias = n->d_p + n->L[l].boff;
        g.out = n->H[l];
        g.outT = l + 1 < kLayers ? n->HT[l] : nullptr;
        g.zout = n->Z[l];
        g.status = n->d_status;
        SG_TRY(gemm(n, M::kFwdTrain, l ? n->H[l - 1] : n->X, n->L[l].wb, B, kW, n->L[l].in, 1, g));
    }
    M::launch_head_train(s, n->H[kLayers - 1], n->Z[kLayers - 1], n->d_p + n->w6off, n->d_p + n->b6off, n->Y,
                         n->Cw, B, n->dZ[kLayers - 1], n->dZT[kLayers - 1], n->gpart, n->lpart);
    n->ctx->launches++;
    auto wgrad = [&](int l) -> int {  // on the side stream once dZ^T[l] is written
        SG_CUDA(n->ctx, cudaEventRecord(n->ev_dz[l], s));
        SG_CUDA(n->ctx, cudaStreamWaitEvent(n->side, n->ev_dz[l], 0));
        M::GemmArgs g{};
        g.part = n->L[l].part;
        g.status = n->d_status;
        return gemm(n, M::kWgrad, n->dZT[l], l ? n->HT[l - 1] : n->XT, kW, n->L[l].in, B, n->L[l].splits, g,
                    n->side);
    };
    SG_TRY(wgrad(kLayers - 1));
    for (int l = kLayers - 1; l >= 1; l--) {
        M::GemmArgs g{};
        g.zin = n->Z[l - 1];
        g.out = n->dZ[l - 1];
        g.outT = n->dZT[l - 1];
        g.status = n->d_status;
        SG_TRY(gemm(n, M::kBwdData, n->dZ[l], n->L[l].wt, B, n->L[l].in, kW, 1, g));
        SG_TRY(wgrad(l - 1));
    }
    // the bias gradients need only dZ^T and the loss history only the head's
    // loss partials, all written on this stream by now: they run beside the
    // side stream's last weight-gradient GEMMs. The history slot is the step
    // counter's, so only a training step (after k_step_begin) records one.
    const bf16* dzt[kLayers];
    for (int l = 0; l < kLayers; l++) dzt[l] = n->dZT[l];
    M::launch_bias_grad(s, dzt, kLayers, B, n->gb);
    n->ctx->launches++;
    if (train_step) {
        M::launch_loss_hist(s, n->lpart, n->B / M::kHeadRows, n->B, n->d_ts, n->hist, kHistCap);
        n->ctx->launches++;
    }
    SG_CUDA(n->ctx, cudaEventRecord(n->ev_join, n->side));
    SG_CUDA(n->ctx, cudaStreamWaitEvent(s, n->ev_join, 0));
    return GFK_OK;
}

int enqueue_step(gfk_net* n, const gfk_dataset* d) {
    cudaStream_t s = n->ctx->stream;
    M::launch_step_begin(s, n->d_ts);
    M::BatchArgs b{};
    b.labels = d->d_labels;
    b.lmax = d->d_lmax;
    b.soilfeat = d->d_soilfeat;
    b.train = n->d_train;
    b.ntrain = n->ntrain;
    b.nr = d->nr;
    b.nf = d->nf;
    b.ir0 = n->ir0;
    b.nir = n->nir;
    b.B = n->B;
    b.ranges = d->d_ranges;
    b.freqs = d->d_freqs;
    b.dom = n->dom;
    b.fourier = n->d_four;
    b.y_mean0 = n->ms[0];
    b.y_std0 = n->ms[1];
    b.y_mean1 = n->ms[2];
    b.y_std1 = n->ms[3];
    b.loss_mode = n->cfg.loss_mode;
    b.phase_weight = n->cfg.phase_weight;
    b.weight_floor = n->cfg.weight_floor;
    b.phase_cap = n->cfg.phase_cap > 0 ? n->cfg.phase_cap : 3.0e38f;
    b.seed = n->cfg.seed * 0x9e3779b97f4a7c15ULL + 17;
    b.ts = n->d_ts;
    b.X = n->X;
    b.XT = n->XT;
    b.Y = n->Y;
    b.C = n->Cw;
    M::launch_batch(s, b);
    n->ctx->launches += 2;
    SG_TRY(enqueue_fwd_bwd(n, true));
    M::launch_adam(s, n->adam, n->nparam);
    n->ctx->launches += 2;
    return GFK_OK;
}

int ensure_inference(gfk_net* n) {
    if (n->iX) return GFK_OK;
    SG_TRY(salloc(n->ctx, &n->iX, (size_t)kChunkRows * M::kIn));
    SG_TRY(salloc(n->ctx, &n->iH0, (size_t)kChunkRows * kW));
    SG_TRY(salloc(n->ctx, &n->iH1, (size_t)kChunkRows * kW));
    SG_TRY(salloc(n->ctx, &n->iT, (size_t)kChunkRows * 2));
    SG_TRY(salloc(n->ctx, &n->d_acc, (size_t)592 * 6));
    return GFK_OK;
}

// Soil table rows: scalars at [0, np), travel times at [kScalars, kScalars + kTimes).
std::vector<float> soil_table(const double* scalars, const double* times, int ns, int np) {
    std::vector<float> t((size_t)ns * M::kSoilStride, 0.0f);
    for (int s = 0; s < ns; s++) {
        for (int j = 0; j < np; j++) t[(size_t)s * M::kSoilStride + j] = static_cast<float>(scalars[(size_t)s * np + j]);
        if (times)
            for (int q = 0; q < M::kTimes; q++)
                t[(size_t)s * M::kSoilStride + M::kScalars + q] = static_cast<float>(times[(size_t)s * M::kTimes + q]);
    }
    return t;
}

// Rows [0, ns nf nr) of the inference layout through the network; G to d_G
// (device, may be null) and, per chunk, T and an evaluation callback.
template <class OnChunk>
int run_inference(gfk_net* n, const float* d_soil, int ns, const double* d_r, int nr, const double* d_f, int nf,
                  cd* d_G, OnChunk on_chunk) {
    SG_TRY(ensure_inference(n));
    cudaStream_t s = n->ctx->stream;
    const long long total = (long long)ns * nf * nr;
    for (long long p0 = 0; p0 < total; p0 += kChunkRows) {
        const long long rows = std::min(kChunkRows, total - p0);
        const long long rp = (rows + 127) / 128 * 128;
        M::FeatureArgs fa{d_soil, ns, nr, nf, p0, rows, d_r, d_f, n->dom, n->d_four, n->iX};
        M::launch_features(s, fa, rp);
        n->ctx->launches++;
        bf16* in = n->iX;
        bf16* bufs[2] = {n->iH0, n->iH1};
        for (int l = 0; l < kLayers; l++) {
            M::GemmArgs g{};
            g.bias = n->d_p + n->L[l].boff;
            g.out = bufs[l & 1];
            g.status = n->d_status;
            SG_TRY(gemm(n, M::kFwdInfer, in, n->L[l].wb, (int)rp, kW, n->L[l].in, 1, g));
            in = bufs[l & 1];
        }
        M::HeadInferArgs ha{in, n->d_p + n->w6off, n->d_p + n->b6off, p0, rows, nr, nf, d_r, d_f,
                            n->ms[0], n->ms[1], n->ms[2], n->ms[3], d_G, n->iT};
        M::launch_head_infer(s, ha);
        n->ctx->launches++;
        SG_TRY(on_chunk(p0, rows));
    }
    return check_status(n);
}

}  // namespace

void gfk_release_surrogates(gfk_ctx* ctx) {
    for (gfk_net* n : ctx->nets) {
        net_free(n);
        delete n;
    }
    ctx->nets.clear();
    for (gfk_dataset* d : ctx->datasets) {
        dataset_free(d);
        delete d;
    }
    ctx->datasets.clear();
}

extern "C" {

int gfk_trace_metrics(gfk_ctx* ctx, const double* d_G, int64_t stride, int32_t ns, int32_t nbins,
                      const double* shaping, int32_t n, double fs_hz, double omega_imag, int32_t k_lo, int32_t k_hi,
                      double* peak, double* centroid) {
    if (!ctx || !d_G || !shaping || !peak || !centroid) return GFK_EARG;
    if (n != gfk::trace::kN) return sfail(ctx, GFK_ELIMIT, "trace length %d: only %d is built", n, gfk::trace::kN);
    if (ns < 0 || nbins < 1 || nbins > n / 2 || stride < nbins || k_lo < 0 || k_hi > n / 2 || k_lo > k_hi ||
        !(fs_hz > 0))
        return sfail(ctx, GFK_EARG, "trace metrics: bad sizes");
    if (ns == 0) return GFK_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    std::vector<double> tw(n);  // e^{-2 pi i k / n}, k < n/2
    for (int k = 0; k < n / 2; k++) {
        const double a = -2.0 * M_PI * k / n;
        tw[2 * k] = std::cos(a);
        tw[2 * k + 1] = std::sin(a);
    }
    double *d_S = nullptr, *d_tw = nullptr, *d_out = nullptr;
    SG_TRY(salloc(ctx, &d_S, (size_t)(n / 2 + 1) * 2));
    SG_TRY(salloc(ctx, &d_tw, (size_t)n));
    SG_TRY(salloc(ctx, &d_out, (size_t)ns * 2));
    SG_CUDA(ctx, cudaMemcpyAsync(d_S, shaping, sizeof(double) * (n / 2 + 1) * 2, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(d_tw, tw.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    gfk::trace::launch_metrics(s, reinterpret_cast<const cd*>(d_G), stride, ns, nbins,
                               reinterpret_cast<const cd*>(d_S), reinterpret_cast<const cd*>(d_tw), fs_hz,
                               omega_imag, k_lo, k_hi, d_out, d_out + ns);
    ctx->launches++;
    SG_CUDA(ctx, cudaGetLastError());
    SG_CUDA(ctx, cudaMemcpyAsync(peak, d_out, sizeof(double) * ns, cudaMemcpyDeviceToHost, s));
    SG_CUDA(ctx, cudaMemcpyAsync(centroid, d_out + ns, sizeof(double) * ns, cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(d_S, s);
    cudaFreeAsync(d_tw, s);
    cudaFreeAsync(d_out, s);
    SG_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

int gfk_ensemble_gate(gfk_ctx* ctx, const double* const* d_members, int32_t E, int64_t stride, int32_t ns,
                      int32_t nbins, const double* shaping, double threshold, double amp_threshold, double* d_mean,
                      uint8_t* flags, double* spread) {
    if (!ctx || !d_members || !shaping || !d_mean || !flags || !spread) return GFK_EARG;
    if (E < 1 || E > gfk::trace::kMaxMembers || ns < 0 || nbins < 1 || stride < nbins)
        return sfail(ctx, GFK_EARG, "ensemble gate: bad sizes");
    if (ns == 0) return GFK_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    gfk::trace::GateArgs a{};
    for (int e = 0; e < E; e++) a.members[e] = reinterpret_cast<const cd*>(d_members[e]);
    a.E = E;
    a.stride = stride;
    a.ns = ns;
    a.nbins = nbins;
    a.threshold = threshold;
    a.amp_threshold = amp_threshold;
    a.mean = reinterpret_cast<cd*>(d_mean);
    cd* d_S = nullptr;
    unsigned char* d_flag = nullptr;
    double* d_spread = nullptr;
    SG_TRY(salloc(ctx, &d_S, (size_t)nbins + 1));
    SG_TRY(salloc(ctx, &d_flag, (size_t)ns * nbins));
    SG_TRY(salloc(ctx, &d_spread, (size_t)ns));
    SG_CUDA(ctx, cudaMemcpyAsync(d_S, shaping, sizeof(cd) * (nbins + 1), cudaMemcpyHostToDevice, s));
    a.S = d_S;
    a.flag = d_flag;
    a.spread = d_spread;
    gfk::trace::launch_gate(s, a);
    ctx->launches++;
    SG_CUDA(ctx, cudaGetLastError());
    SG_CUDA(ctx, cudaMemcpyAsync(flags, d_flag, (size_t)ns * nbins, cudaMemcpyDeviceToHost, s));
    SG_CUDA(ctx, cudaMemcpyAsync(spread, d_spread, sizeof(double) * ns, cudaMemcpyDeviceToHost, s));
    cudaFreeAsync(d_S, s);
    cudaFreeAsync(d_flag, s);
    cudaFreeAsync(d_spread, s);
    SG_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

int gfk_scatter_rows(gfk_ctx* ctx, const double* d_src, int64_t src_stride, const int64_t* index, int64_t n,
                     double* d_dst) {
    if (!ctx || !d_src || !index || !d_dst || n < 0 || src_stride < 1) return GFK_EARG;
    if (n == 0) return GFK_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    long long* d_idx = nullptr;
    SG_TRY(salloc(ctx, &d_idx, (size_t)n));
    SG_CUDA(ctx, cudaMemcpyAsync(d_idx, index, sizeof(long long) * n, cudaMemcpyHostToDevice, s));
    gfk::trace::launch_scatter(s, reinterpret_cast<const cd*>(d_src), src_stride, d_idx, n, reinterpret_cast<cd*>(d_dst));
    ctx->launches++;
    SG_CUDA(ctx, cudaGetLastError());
    cudaFreeAsync(d_idx, s);
    SG_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

int gfk_dataset_create(gfk_ctx* ctx, int32_t np, int32_t nsoil, const double* scalars, const double* times,
                       const double* ranges, int32_t nr, const double* freqs, int32_t nf, double floor_rel,
                       gfk_dataset** out) {
    if (!ctx || !out || !scalars || !ranges || !freqs) return GFK_EARG;
    *out = nullptr;
    if (np < 1 || np > M::kMaxSoil || nsoil < 1 || nr < 1 || nr > 128 || nf < 1 || !(floor_rel > 0 && floor_rel < 1))
        return sfail(ctx, GFK_EARG, "data set: bad sizes");
    for (int i = 0; i < nr; i++)
        if (!(ranges[i] > 0)) return sfail(ctx, GFK_EARG, "data set: range %d is not positive", i);
    for (int j = 0; j < nf; j++)
        if (!(freqs[j] > 0)) return sfail(ctx, GFK_EARG, "data set: frequency %d is not positive", j);
    if ((size_t)nr * nf * 2 > 200 * 1024) return sfail(ctx, GFK_ELIMIT, "data set: nr x nf above 102400");
    cudaSetDevice(ctx->device);
    gfk_dataset* d = new gfk_dataset();
    d->ctx = ctx;
    d->nparam = np;
    d->nsoil = nsoil;
    d->nr = nr;
    d->nf = nf;
    d->floor_rel = floor_rel;
    d->ranges.assign(ranges, ranges + nr);
    d->freqs.assign(freqs, freqs + nf);
    if (times)
        for (size_t i = 0; i < (size_t)nsoil * M::kTimes; i++)
            if (!(times[i] >= 0) || times[i] > 1.0) {
                delete d;
                return sfail(ctx, GFK_EARG, "data set: travel times must lie in [0, 1] s");
            }
    d->soilfeat = soil_table(scalars, times, nsoil, np);
    d->filled.assign(nsoil, 0);
    int st = GFK_OK;
    if ((st = salloc(ctx, &d->d_labels, (size_t)nsoil * nr * nf * 2)) || (st = salloc(ctx, &d->d_lmax, (size_t)nsoil * nr)) ||
        (st = salloc(ctx, &d->d_soilfeat, d->soilfeat.size())) ||
        (st = salloc(ctx, &d->d_ranges, nr)) || (st = salloc(ctx, &d->d_freqs, nf)) ||
        (st = salloc(ctx, &d->d_stats, (size_t)nsoil * 6))) {
        dataset_free(d);
        delete d;
        return st;
    }
    cudaStream_t s = ctx->stream;
    cudaMemcpyAsync(d->d_soilfeat, d->soilfeat.data(), d->soilfeat.size() * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d->d_ranges, ranges, nr * 8, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d->d_freqs, freqs, nf * 8, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d->d_stats, 0, (size_t)nsoil * 6 * 8, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        dataset_free(d);
        delete d;
        return sfail(ctx, GFK_ECUDA, "data set upload failed");
    }
    ctx->datasets.push_back(d);
    *out = d;
    return GFK_OK;
}

int gfk_dataset_fill(gfk_dataset* d, const double* d_G, int32_t first, int32_t ns) {
    if (!d || !d_G) return GFK_EARG;
    gfk_ctx* ctx = d->ctx;
    if (first < 0 || ns < 1 || first + ns > d->nsoil) return sfail(ctx, GFK_EARG, "data set fill: soils out of range");
    cudaSetDevice(ctx->device);
    M::LabelArgs a{reinterpret_cast<const cd*>(d_G), ns, d->nr, d->nf, d->d_ranges, d->d_freqs, d->floor_rel,
                   d->d_labels + (size_t)first * d->nr * d->nf * 2, d->d_lmax + (size_t)first * d->nr,
                   d->d_stats + (size_t)first * 6};
    if (M::launch_labels(ctx->stream, a)) return sfail(ctx, GFK_ECUDA, "label kernel refused");
    ctx->launches++;
    SG_CUDA(ctx, cudaGetLastError());
    SG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::fill(d->filled.begin() + first, d->filled.begin() + first + ns, 1);
    return GFK_OK;
}

int gfk_dataset_stats(gfk_dataset* d, double out[6]) {
    if (!d || !out) return GFK_EARG;
    std::vector<double> st((size_t)d->nsoil * 6);
    SG_CUDA(d->ctx, cudaMemcpyAsync(st.data(), d->d_stats, st.size() * 8, cudaMemcpyDeviceToHost, d->ctx->stream));
    SG_CUDA(d->ctx, cudaStreamSynchronize(d->ctx->stream));
    for (int q = 0; q < 6; q++) out[q] = 0.0;
    for (int s = 0; s < d->nsoil; s++)
        if (d->filled[s])
            for (int q = 0; q < 6; q++) out[q] += st[(size_t)s * 6 + q];
    return GFK_OK;
}

int gfk_dataset_labels(gfk_dataset* d, int32_t soil, float* out) {
    if (!d || !out || soil < 0 || soil >= d->nsoil) return GFK_EARG;
    const size_t n = (size_t)d->nr * d->nf * 2;
    SG_CUDA(d->ctx, cudaMemcpyAsync(out, d->d_labels + (size_t)soil * n, n * 4, cudaMemcpyDeviceToHost,
                                    d->ctx->stream));
    SG_CUDA(d->ctx, cudaStreamSynchronize(d->ctx->stream));
    return GFK_OK;
}

int gfk_dataset_destroy(gfk_dataset* d) {
    if (!d) return GFK_OK;
    gfk_ctx* ctx = d->ctx;
    for (gfk_net* n : ctx->nets)
        if (n->graph_ds == d) {  // a graph that reads these labels is stale now
            if (n->gexec) cudaGraphExecDestroy(n->gexec);
            n->gexec = nullptr;
            n->graph_ds = nullptr;
        }
    auto& v = ctx->datasets;
    v.erase(std::remove(v.begin(), v.end(), d), v.end());
    dataset_free(d);
    delete d;
    return GFK_OK;
}

int gfk_net_create(gfk_ctx* ctx, const gfk_net_config* cfg, gfk_net** out) {
    if (!ctx || !cfg || !out) return GFK_EARG;
    *out = nullptr;
    if (cfg->nsoil_scalars < 1 || cfg->nsoil_scalars > M::kMaxSoil || cfg->batch < 128 || cfg->batch % 128 ||
        cfg->batch > (1 << 20))
        return sfail(ctx, GFK_EARG, "network: batch must be a positive multiple of 128 (<= 2^20)");
    if (cfg->loss_mode != GFK_LOSS_PLAIN && cfg->loss_mode != GFK_LOSS_COMPLEX && cfg->loss_mode != GFK_LOSS_AMPLITUDE)
        return sfail(ctx, GFK_EARG, "network: unknown loss mode %d", cfg->loss_mode);
    cudaSetDevice(ctx->device);
    if (M::prepare_gemm()) return sfail(ctx, GFK_ECUDA, "tensor-core GEMM kernels could not be configured");
    gfk_net* n = new gfk_net();
    n->ctx = ctx;
    n->cfg = *cfg;
    n->B = cfg->batch;
    long long off = 0;
    for (int l = 0; l < kLayers; l++) {
        NetLayer& L = n->L[l];
        L.in = l ? kW : M::kIn;
        L.out = kW;
        L.woff = off;
        off += (long long)L.out * L.in;
        L.boff = off;
        off += L.out;
        // split the batch so that the weight-gradient GEMM fills the GPU
        const int tiles = (L.out / 128) * (L.in / 128);
        int sp = 1;
        while (tiles * sp < 128 && n->B % (64 * sp * 2) == 0) sp *= 2;
        L.splits = sp;
    }
    n->w6off = off;
    off += 2 * kW;
    n->b6off = off;
    off += 2;
    n->nparam = off;

    // initial parameters: U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases
    std::mt19937_64 rng(cfg->seed);
    std::vector<float> p(n->nparam);
    for (int l = 0; l <= kLayers; l++) {
        const int fan_in = l < kLayers ? n->L[l].in : kW;
        const long long a = l < kLayers ? n->L[l].woff : n->w6off;
        const long long e = l < kLayers ? n->L[l].boff + n->L[l].out : n->nparam;
        std::uniform_real_distribution<float> u(-1.0f / std::sqrt((float)fan_in), 1.0f / std::sqrt((float)fan_in));
        for (long long i = a; i < e; i++) p[i] = u(rng);
    }
    std::normal_distribution<float> nd(0.0f, cfg->fourier_sigma > 0 ? cfg->fourier_sigma : 1.0f);
    n->four.resize(2 * M::kFourier);
    for (auto& x : n->four) x = nd(rng);

    int st = GFK_OK;
    auto A = [&](auto** ptr, size_t cnt) {
        if (st == GFK_OK) st = salloc(ctx, ptr, cnt);
    };
    A(&n->d_p, n->nparam);
    A(&n->d_m, n->nparam);
    A(&n->d_v, n->nparam);
    A(&n->d_ts, 1);
    A(&n->d_four, n->four.size());
    A(&n->X, (size_t)n->B * M::kIn);
    A(&n->XT, (size_t)n->B * M::kIn);
    A(&n->Y, (size_t)n->B * 2);
    A(&n->Cw, (size_t)n->B * 2);
    for (int l = 0; l < kLayers; l++) {
        NetLayer& L = n->L[l];
        A(&L.wb, (size_t)L.out * L.in);
        A(&L.wt, (size_t)L.out * L.in);
        A(&L.part, (size_t)L.splits * L.out * L.in);
        A(&n->Z[l], (size_t)n->B * kW);
        A(&n->H[l], (size_t)n->B * kW);
        if (l + 1 < kLayers) A(&n->HT[l], (size_t)n->B * kW);
        A(&n->dZ[l], (size_t)n->B * kW);
        A(&n->dZT[l], (size_t)n->B * kW);
    }
    A(&n->gpart, (size_t)(n->B / M::kHeadRows) * M::kHeadStride);
    A(&n->lpart, (size_t)(n->B / M::kHeadRows) * 4);
    A(&n->gb, (size_t)kLayers * kW);
    A(&n->hist, (size_t)kHistCap * 2);
    A(&n->gflat, n->nparam);
    A(&n->d_status, 1);
    if (st == GFK_OK && cudaStreamCreateWithFlags(&n->side, cudaStreamNonBlocking) != cudaSuccess)
        st = sfail(ctx, GFK_ECUDA, "side stream creation failed");
    for (int l = 0; l < kLayers && st == GFK_OK; l++)
        if (cudaEventCreateWithFlags(&n->ev_dz[l], cudaEventDisableTiming) != cudaSuccess)
            st = sfail(ctx, GFK_ECUDA, "event creation failed");
    if (st == GFK_OK && cudaEventCreateWithFlags(&n->ev_join, cudaEventDisableTiming) != cudaSuccess)
        st = sfail(ctx, GFK_ECUDA, "event creation failed");
    if (st != GFK_OK) {
        net_free(n);
        delete n;
        return st;
    }
    // optimiser segments, in parameter order
    M::AdamArgs& ad = n->adam;
    ad.nseg = 0;
    for (int l = 0; l < kLayers; l++) {
        NetLayer& L = n->L[l];
        ad.seg[ad.nseg++] = M::AdamSeg{L.woff, (long long)L.out * L.in, L.part, (long long)L.out * L.in, L.splits,
                                       L.out, L.in, L.wb, L.wt};
        ad.seg[ad.nseg++] = M::AdamSeg{L.boff, L.out, n->gb + (size_t)l * kW, 0, 1, 0, 0, nullptr, nullptr};
    }
    ad.seg[ad.nseg++] = M::AdamSeg{n->w6off, 2 * kW + 2, n->gpart, M::kHeadStride, n->B / M::kHeadRows, 0, 0,
                                   nullptr, nullptr};
    ad.p = n->d_p;
    ad.m = n->d_m;
    ad.v = n->d_v;
    ad.eps = cfg->eps;
    ad.weight_decay = cfg->weight_decay;
    ad.ts = n->d_ts;
    if (salloc(ctx, &n->d_seg, (size_t)M::kMaxSegs) != GFK_OK) {
        net_free(n);
        delete n;
        return GFK_ENOMEM;
    }
    ad.dseg = n->d_seg;

    M::TrainScalars ts{};
    ts.step = 0;
    ts.lr_max = cfg->lr_max;
    ts.lr_min = cfg->lr_min;
    ts.warmup = cfg->warmup_steps;
    ts.total = cfg->total_steps;
    ts.beta1 = cfg->beta1;
    ts.beta2 = cfg->beta2;
    cudaStream_t s = ctx->stream;
    cudaMemcpyAsync(n->d_p, p.data(), p.size() * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(n->d_m, 0, n->nparam * 4, s);
    cudaMemsetAsync(n->d_v, 0, n->nparam * 4, s);
    cudaMemsetAsync(n->d_status, 0, 4, s);
    cudaMemcpyAsync(n->d_ts, &ts, sizeof ts, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(n->d_four, n->four.data(), n->four.size() * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(n->d_seg, ad.seg, sizeof(M::AdamSeg) * ad.nseg, cudaMemcpyHostToDevice, s);
    M::launch_sync_weights(s, n->adam, n->nparam);
    ctx->launches += 2;
    if (cudaStreamSynchronize(s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        net_free(n);
        delete n;
        return sfail(ctx, GFK_ECUDA, "network initialisation failed");
    }
    ctx->nets.push_back(n);
    *out = n;
    return GFK_OK;
}

int gfk_net_set_scales(gfk_net* n, double r_lo, double r_hi, double f_lo, double f_hi, const float ms[4]) {
    if (!n || !ms) return GFK_EARG;
    if (!(r_lo > 0 && r_hi > r_lo && f_lo > 0 && f_hi > f_lo && ms[1] > 0 && ms[3] > 0))
        return sfail(n->ctx, GFK_EARG, "network scales: need 0 < lo < hi and positive deviations");
    n->dom = M::FeatureDomain{(float)r_lo, (float)r_hi, (float)f_lo, (float)f_hi};
    std::memcpy(n->ms, ms, sizeof n->ms);
    n->scales = true;
    if (n->gexec) cudaGraphExecDestroy(n->gexec);  // the scales are baked into the graph
    n->gexec = nullptr;
    return GFK_OK;
}

int gfk_net_train_ranges(gfk_net* n, gfk_dataset* d, const int32_t* train, int32_t ntrain, int32_t first_range,
                         int32_t nranges, int32_t steps, float* loss) {
    if (!n || !d || !train || ntrain < 1 || steps < 0) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    if (d->ctx != ctx) return sfail(ctx, GFK_EARG, "network and data set belong to different contexts");
    if (!n->scales) return sfail(ctx, GFK_EARG, "network scales are not set");
    if (d->nparam != n->cfg.nsoil_scalars) return sfail(ctx, GFK_EARG, "data set has a different soil scalar count");
    if (first_range < 0 || nranges < 1 || first_range + nranges > d->nr)
        return sfail(ctx, GFK_EARG, "training ranges [%d, %d) outside the data set's %d", first_range,
                     first_range + nranges, d->nr);
    for (int i = 0; i < ntrain; i++)
        if (train[i] < 0 || train[i] >= d->nsoil || !d->filled[train[i]])
            return sfail(ctx, GFK_EARG, "training soil %d is not a filled soil of the data set", train[i]);
    if (n->gexec && (n->ir0 != first_range || n->nir != nranges)) {  // the window is baked into the graph
        cudaGraphExecDestroy(n->gexec);
        n->gexec = nullptr;
    }
    n->ir0 = first_range;
    n->nir = nranges;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const bool same = n->gexec && n->graph_ds == d && n->graph_train.size() == (size_t)ntrain &&
                      std::equal(train, train + ntrain, n->graph_train.begin());
    if (!same) {
        if (n->gexec) cudaGraphExecDestroy(n->gexec);
        n->gexec = nullptr;
        if (ntrain > n->ntrain) {
            sfree(ctx, n->d_train);
            SG_TRY(salloc(ctx, &n->d_train, ntrain));
        }
        n->ntrain = ntrain;
        SG_CUDA(ctx, cudaMemcpyAsync(n->d_train, train, ntrain * 4, cudaMemcpyHostToDevice, s));
        SG_CUDA(ctx, cudaStreamSynchronize(s));
        // capture one step; the step counter lives on the device
        const int64_t before = ctx->launches;
        SG_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st = enqueue_step(n, d);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &g);
        ctx->launches = before;
        if (st != GFK_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return sfail(ctx, GFK_ECUDA, "training step capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&n->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            n->gexec = nullptr;
            return sfail(ctx, GFK_ECUDA, "training graph instantiation failed: %s", cudaGetErrorString(e));
        }
        n->graph_ds = d;
        n->graph_train.assign(train, train + ntrain);
    }
    // launches per replayed step, counted from the step's own enqueue
    const int64_t per_step = 2 + kLayers + 1 + (kLayers - 1) + kLayers + 1 + 3;
    std::vector<float> h(kHistCap * 2);
    for (int done = 0; done < steps;) {
        const int blk = std::min(kHistCap, steps - done);
        for (int i = 0; i < blk; i++) SG_CUDA(ctx, cudaGraphLaunch(n->gexec, s));
        ctx->launches += per_step * blk;
        if (loss) {
            // slots follow (step - 1) % cap; this block's steps fill blk slots ending at the current step
            long long step_now = 0;
            SG_CUDA(ctx, cudaMemcpyAsync(&step_now, &n->d_ts->step, 8, cudaMemcpyDeviceToHost, s));
            SG_CUDA(ctx, cudaMemcpyAsync(h.data(), n->hist, h.size() * 4, cudaMemcpyDeviceToHost, s));
            SG_CUDA(ctx, cudaStreamSynchronize(s));
            for (int i = 0; i < blk; i++) {
                const long long stp = step_now - blk + 1 + i;
                const long long slot = (stp - 1) % kHistCap;
                loss[2 * (size_t)(done + i)] = h[2 * slot];
                loss[2 * (size_t)(done + i) + 1] = h[2 * slot + 1];
            }
        }
        done += blk;
    }
    SG_CUDA(ctx, cudaGetLastError());
    return check_status(n);
}

int gfk_net_train(gfk_net* n, gfk_dataset* d, const int32_t* train, int32_t ntrain, int32_t steps, float* loss) {
    if (!d) return GFK_EARG;
    return gfk_net_train_ranges(n, d, train, ntrain, 0, d->nr, steps, loss);
}

int gfk_net_predict(gfk_net* n, const double* scalars, const double* times, int32_t ns, const double* ranges,
                    int32_t nr, const double* freqs, int32_t nf, double* out, int32_t on_device) {
    if (!n || !scalars || !ranges || !freqs || !out || ns < 0 || nr < 1 || nf < 1) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    if (!n->scales) return sfail(ctx, GFK_EARG, "network scales are not set");
    if (ns == 0) return GFK_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const std::vector<float> tab = soil_table(scalars, times, ns, n->cfg.nsoil_scalars);
    float* d_soil = nullptr;
    double *d_r = nullptr, *d_f = nullptr;
    cd* d_G = nullptr;
    const size_t total = (size_t)ns * nf * nr;
    SG_TRY(salloc(ctx, &d_soil, tab.size()));
    SG_TRY(salloc(ctx, &d_r, nr));
    SG_TRY(salloc(ctx, &d_f, nf));
    if (!on_device) SG_TRY(salloc(ctx, &d_G, total));
    SG_CUDA(ctx, cudaMemcpyAsync(d_soil, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(d_r, ranges, nr * 8, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(d_f, freqs, nf * 8, cudaMemcpyHostToDevice, s));
    cd* G = on_device ? reinterpret_cast<cd*>(out) : d_G;
    int st = run_inference(n, d_soil, ns, d_r, nr, d_f, nf, G, [](long long, long long) { return (int)GFK_OK; });
    if (st == GFK_OK && !on_device) {
        cudaError_t e = cudaMemcpyAsync(out, d_G, total * sizeof(cd), cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) st = sfail(ctx, GFK_ECUDA, "prediction download: %s", cudaGetErrorString(e));
    }
    cudaFreeAsync(d_soil, s);
    cudaFreeAsync(d_r, s);
    cudaFreeAsync(d_f, s);
    if (d_G) cudaFreeAsync(d_G, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && st == GFK_OK) st = sfail(ctx, GFK_ECUDA, "prediction failed");
    return st;
}

int gfk_net_evaluate(gfk_net* n, gfk_dataset* d, const int32_t* soils, int32_t ns, double out[7]) {
    if (!n || !d || !soils || !out || ns < 1) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    if (!n->scales) return sfail(ctx, GFK_EARG, "network scales are not set");
    for (int i = 0; i < ns; i++)
        if (soils[i] < 0 || soils[i] >= d->nsoil || !d->filled[soils[i]])
            return sfail(ctx, GFK_EARG, "evaluation soil %d is not a filled soil", soils[i]);
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    std::vector<float> tab((size_t)ns * M::kSoilStride);
    for (int i = 0; i < ns; i++)
        std::copy_n(d->soilfeat.begin() + (size_t)soils[i] * M::kSoilStride, M::kSoilStride,
                    tab.begin() + (size_t)i * M::kSoilStride);
    float* d_soil = nullptr;
    int* d_ids = nullptr;
    cd* d_G = nullptr;
    SG_TRY(salloc(ctx, &d_soil, tab.size()));
    SG_TRY(salloc(ctx, &d_ids, ns));
    SG_TRY(salloc(ctx, &d_G, (size_t)ns * d->nf * d->nr));
    SG_CUDA(ctx, cudaMemcpyAsync(d_soil, tab.data(), tab.size() * 4, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(d_ids, soils, ns * 4, cudaMemcpyHostToDevice, s));
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const int nblk = 592;
    std::vector<double> part((size_t)nblk * 6);
    auto on_chunk = [&](long long p0, long long rows) -> int {
        M::launch_eval(s, n->iT, d->d_labels, d_ids, p0, rows, d->nr, d->nf, d->d_ranges, d->d_freqs, n->d_acc,
                       nblk);
        ctx->launches++;
        SG_CUDA(ctx, cudaMemcpyAsync(part.data(), n->d_acc, part.size() * 8, cudaMemcpyDeviceToHost, s));
        SG_CUDA(ctx, cudaStreamSynchronize(s));
        for (int b = 0; b < nblk; b++)
            for (int q = 0; q < 6; q++) acc[q] += part[(size_t)b * 6 + q];
        return GFK_OK;
    };
    int st = run_inference(n, d_soil, ns, d->d_ranges, d->nr, d->d_freqs, d->nf, d_G, on_chunk);
    cudaFreeAsync(d_soil, s);
    cudaFreeAsync(d_ids, s);
    cudaFreeAsync(d_G, s);
    cudaStreamSynchronize(s);
    if (st != GFK_OK) return st;
    out[0] = (double)ns * d->nf * d->nr;
    for (int q = 0; q < 6; q++) out[q + 1] = acc[q];
    return GFK_OK;
}

int64_t gfk_net_param_count(const gfk_net* n) { return n ? n->nparam : 0; }

int gfk_net_params(gfk_net* n, float* host, int64_t cnt, int32_t set) {
    if (!n || !host || cnt != n->nparam) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    if (set) {
        SG_CUDA(ctx, cudaMemcpyAsync(n->d_p, host, cnt * 4, cudaMemcpyHostToDevice, s));
        M::launch_sync_weights(s, n->adam, n->nparam);
        ctx->launches += 2;
    } else {
        SG_CUDA(ctx, cudaMemcpyAsync(host, n->d_p, cnt * 4, cudaMemcpyDeviceToHost, s));
    }
    SG_CUDA(ctx, cudaStreamSynchronize(s));
    return GFK_OK;
}

int gfk_net_fourier(gfk_net* n, float* host, int32_t set) {
    if (!n || !host) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    cudaSetDevice(ctx->device);
    if (set) {
        std::copy_n(host, n->four.size(), n->four.begin());
        SG_CUDA(ctx, cudaMemcpyAsync(n->d_four, host, n->four.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        SG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    } else {
        std::copy(n->four.begin(), n->four.end(), host);
    }
    return GFK_OK;
}

int gfk_net_probe(gfk_net* n, const float* X, const float* Y, const float* coeffs, float* grad, float loss[2]) {
    if (!n || !X || !Y || !grad || !loss) return GFK_EARG;
    gfk_ctx* ctx = n->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const int B = n->B;
    std::vector<uint16_t> xb((size_t)B * M::kIn), xt((size_t)B * M::kIn);
    for (int b = 0; b < B; b++)
        for (int j = 0; j < M::kIn; j++) {
            const uint16_t v = to_bf16(X[(size_t)b * M::kIn + j]);
            xb[(size_t)b * M::kIn + j] = v;
            xt[(size_t)j * B + b] = v;
        }
    SG_CUDA(ctx, cudaMemcpyAsync(n->X, xb.data(), xb.size() * 2, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(n->XT, xt.data(), xt.size() * 2, cudaMemcpyHostToDevice, s));
    SG_CUDA(ctx, cudaMemcpyAsync(n->Y, Y, (size_t)B * 2 * 4, cudaMemcpyHostToDevice, s));
    std::vector<float> cw((size_t)B * 2);
    for (int b = 0; b < B; b++) {
        cw[2 * b] = coeffs ? coeffs[2 * b] : 1.0f;
        cw[2 * b + 1] = coeffs ? coeffs[2 * b + 1] : (std::isnan(Y[2 * b + 1]) ? 0.0f : n->cfg.phase_weight);
    }
    SG_CUDA(ctx, cudaMemcpyAsync(n->Cw, cw.data(), cw.size() * 4, cudaMemcpyHostToDevice, s));
    SG_TRY(enqueue_fwd_bwd(n, false));
    M::launch_grad_flat(s, n->adam, n->nparam, n->gflat);
    ctx->launches++;
    SG_CUDA(ctx, cudaGetLastError());
    const int nblk = B / M::kHeadRows;
    std::vector<float> lp((size_t)nblk * 4);
    SG_CUDA(ctx, cudaMemcpyAsync(grad, n->gflat, n->nparam * 4, cudaMemcpyDeviceToHost, s));
    SG_CUDA(ctx, cudaMemcpyAsync(lp.data(), n->lpart, lp.size() * 4, cudaMemcpyDeviceToHost, s));
    SG_CUDA(ctx, cudaStreamSynchronize(s));
    double sm[4] = {0, 0, 0, 0};
    for (int b = 0; b < nblk; b++)
        for (int q = 0; q < 4; q++) sm[q] += lp[4 * b + q];
    loss[0] = (float)(sm[2] > 0 ? sm[0] / sm[2] : 0.0);
    loss[1] = (float)(sm[3] > 0 ? sm[1] / sm[3] : 0.0);
    return check_status(n);
}

int gfk_net_destroy(gfk_net* n) {
    if (!n) return GFK_OK;
    auto& v = n->ctx->nets;
    v.erase(std::remove(v.begin(), v.end(), n), v.end());
    net_free(n);
    delete n;
    return GFK_OK;
}

}  // extern "C"
