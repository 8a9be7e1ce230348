// gfk_host.cu — the C ABI of libgfk (include/gfk.h): contexts, plans, the
// reference's host-side rules (validation, guard, GridFor) and the bank file.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gfk.h"
#include "gfk_ctx.h"
#include "gfk_kernels.cuh"



// ------------------------------------------------------------------ ctx --


namespace {

int fail(gfk_ctx* ctx, int status, const char* fmt, ...) {
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

#define GFK_CUDA(ctx, call)                                                                        \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail((ctx), e_ == cudaErrorMemoryAllocation ? GFK_ENOMEM : GFK_ECUDA, "%s: %s", \
                        #call, cudaGetErrorString(e_));                                            \
    } while (0)

constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kMaxLayerPhase = 16.0;  // internal/fk/fk.go:242

double q_of(const gfk_medium* m, const gfk_layer& l) {  // fk.go:67-75
    if (l.qs > 0) return l.qs;
    if (m->default_q > 0) return m->default_q;
    return 30.0;
}

bool has_sls(const gfk_medium* m) { return m->sls_tau_sigma > 0 && m->sls_tau_eps > 0; }

double slowest_vs(const gfk_medium* m) {  // layer.go:93-100
    double s = m->layers[0].vs_mps;
    for (int i = 0; i < m->count; i++) s = std::min(s, m->layers[i].vs_mps);
    return s;
}

double reference_modulus(const gfk_medium* m) {  // fk.go:216-222
    const gfk_layer& l0 = m->layers[0];
    double r = l0.density_kgm3 * l0.vs_mps * l0.vs_mps;
    for (int i = 0; i < m->count; i++) {
        const gfk_layer& l = m->layers[i];
        r = std::max(r, l.density_kgm3 * l.vs_mps * l.vs_mps);
    }
    return r;
}

// visco.SLS.Q (visco.go:84-90) at real f.
double sls_q(const gfk_medium* m, double f) {
    const double w = kTwoPi * f;
    // M = (1 + i w te)/(1 + i w ts); Q = Re M / Im M
    const double a = 1.0, b = w * m->sls_tau_eps, c = 1.0, d = w * m->sls_tau_sigma;
    const double den = c * c + d * d;
    const double re = (a * c + b * d) / den, im = (b * c - a * d) / den;
    if (im == 0) return INFINITY;
    return re / im;
}

double pole_q(const gfk_medium* m, double f) {  // fk.go:83-88
    if (has_sls(m)) return sls_q(m, f);
    return q_of(m, m->layers[m->count - 1]);
}

int validate(gfk_ctx* ctx, const gfk_medium* m) {  // layer.go:53-73
    if (!m || !m->layers || m->count <= 0)
        return fail(ctx, GFK_ESTACK, "layer: a stack needs at least a half-space");
    if (m->count > gfk::kMaxLayers)
        return fail(ctx, GFK_ELIMIT, "layer: %d layers, this build handles at most %d", m->count, gfk::kMaxLayers);
    for (int i = 0; i < m->count; i++) {
        const gfk_layer& l = m->layers[i];
        const bool fin = std::isfinite(l.vs_mps) && std::isfinite(l.vp_mps) && std::isfinite(l.density_kgm3) &&
                         std::isfinite(l.qs) && std::isfinite(l.qp) &&
                         (i == m->count - 1 || std::isfinite(l.thickness_m));
        if (!fin) return fail(ctx, GFK_ESTACK, "layer %d: parameters must be finite", i);
        if (l.vs_mps <= 0) return fail(ctx, GFK_ESTACK, "layer %d: Vs must be positive, got %g m/s", i, l.vs_mps);
        if (l.vp_mps <= 0) return fail(ctx, GFK_ESTACK, "layer %d: Vp must be positive, got %g m/s", i, l.vp_mps);
        if (l.density_kgm3 <= 0)
            return fail(ctx, GFK_ESTACK, "layer %d: density must be positive, got %g kg/m^3", i, l.density_kgm3);
        if (l.vp_mps <= M_SQRT2 * l.vs_mps)
            return fail(ctx, GFK_ESTACK, "layer %d: Vp=%g must exceed sqrt(2)*Vs=%g for a non-negative Poisson ratio",
                        i, l.vp_mps, M_SQRT2 * l.vs_mps);
        if (i < m->count - 1 && l.thickness_m <= 0)
            return fail(ctx, GFK_ESTACK, "layer %d: thickness must be positive, got %g m", i, l.thickness_m);
    }
    return GFK_OK;
}

int check_layer_phase(gfk_ctx* ctx, const gfk_medium* m, double f) {  // fk.go:251-266
    if (!m || !m->layers || m->count <= 0) return fail(ctx, GFK_ESTACK, "layer: a stack needs at least a half-space");
    const double slowest = slowest_vs(m);
    const double k = kTwoPi * f / (0.87 * slowest);
    for (int i = 0; i < m->count - 1; i++) {
        const double h = m->layers[i].thickness_m;
        const double kh = k * h;
        if (kh > kMaxLayerPhase)
            return fail(ctx, GFK_EGUARD,
                        "fk: layer %d is %g m thick, which is k*h = %.1f at %g Hz and past the %.0f this propagator "
                        "stays accurate to; it would return a plausible wrong number rather than fail. Band-limit to "
                        "%.0f Hz for this stack, or reformulate the solve with compound matrices as internal/propmat does",
                        i, h, kh, f, kMaxLayerPhase, kMaxLayerPhase * 0.87 * slowest / (kTwoPi * h));
    }
    return GFK_OK;
}

int grid_for_bounds(const gfk_medium* m, double slowest, double rmin, double rmax, double f, gfk_integration opt,
                    gfk_grid* out);

int grid_for(gfk_ctx* ctx, const gfk_medium* m, const double* ranges, int nr, double f, gfk_integration opt,
             gfk_grid* out) {  // fk.go:464-495
    if (nr <= 0 || !ranges) return fail(ctx, GFK_EARG, "fk: no ranges given");
    if (!m || !m->layers || m->count <= 0) return fail(ctx, GFK_ESTACK, "layer: a stack needs at least a half-space");
    double rmin = INFINITY, rmax = 0;
    for (int i = 0; i < nr; i++) {
        if (!(ranges[i] > 0)) return fail(ctx, GFK_EARG, "fk: range must be positive, got %g m", ranges[i]);
        rmin = std::min(rmin, ranges[i]);
        rmax = std::max(rmax, ranges[i]);
    }
    return grid_for_bounds(m, slowest_vs(m), rmin, rmax, f, opt, out);
}

// GridFor's rule once the range bounds and the medium's slowest shear velocity
// are known (a plan computes them once per medium, not per frequency). With a
// fixed sample count the step, and with it the pole Q, does not matter.
int grid_for_bounds(const gfk_medium* m, double slowest, double rmin, double rmax, double f, gfk_integration opt,
                    gfk_grid* out) {
    const double kbody = kTwoPi * f / slowest;
    const double kmf = opt.kmax_factor > 0 ? opt.kmax_factor : 30;
    const double kmax = std::max(opt.kmax > 0 ? opt.kmax : kmf * kbody, 40 / rmin);
    int n = opt.samples;
    if (n <= 0) {
        double dk = kTwoPi / (8 * rmax);
        const double q = pole_q(m, f);
        if (kbody > 0 && q > 0) dk = std::min(dk, kbody / (2 * q) / 4);
        const double nn = std::ceil(kmax / dk);
        n = nn > 2.0e9 ? 2000000000 : (int)nn;
    }
    if (n < 64) n = 64;
    out->kmax = kmax;
    out->samples = n;
    out->_pad = 0;
    return GFK_OK;
}

gfk::MediumP medium_params(const gfk_medium* m) {
    gfk::MediumP p{};
    p.ref_freq = m->ref_freq_hz;
    p.default_q = m->default_q;
    p.tau_sigma = m->sls_tau_sigma;
    p.tau_eps = m->sls_tau_eps;
    p.count = m->count;
    p.sls = has_sls(m) ? 1 : 0;
    return p;
}

}  // namespace

// ---------------------------------------------------------------- plans --
//
// A plan is a fixed set of bank rows — (medium, frequency) pairs, one or many
// media — over one range list, with its device buffers. Rows are ordered
// medium by medium, each medium's frequencies in the caller's order.

// How a plan sets its wavenumber grid per frequency.
enum GridMode { kGridMulti = 0, kGridSingle = 1 };

struct TimedSeg {
    int kind;  // 0 prop, 1 quad, 2 other, 3 whole graph
    cudaEvent_t a, b;
    bool pending;
};

struct gfk_plan {
    gfk_ctx* ctx = nullptr;
    gfk_solve solve{};
    std::vector<double> ranges;
    int nsoil = 0, nf = 0, nr = 0, max_nk = 0, max_nl = 0;
    // host tables
    std::vector<gfk::LayerP> lp;
    std::vector<gfk::MediumP> media;
    std::vector<gfk::FreqDesc> fd;  // integrand offsets relative to each row's chunk
    std::vector<double> freqs;
    std::vector<int32_t> host_status;  // per row, set on the host (guard, arguments, stack)
    bool shared = false;
    double g_kmax = 0;
    int g_n = 0;
    std::vector<int> chunk_begin;  // row chunks [chunk_begin[c], chunk_begin[c+1])
    std::vector<int> chunk_max_nk;
    int64_t rem_capacity = 0;  // complex values
    // device
    gfk::LayerP* d_lp = nullptr;
    gfk::MediumP* d_media = nullptr;
    gfk::FreqDesc* d_fd = nullptr;
    double *d_ranges = nullptr, *d_W = nullptr;
    gfk::LayerC* d_lc = nullptr;
    cd *d_wc2 = nullptr, *d_C = nullptr, *d_rem = nullptr, *d_G = nullptr;
    int* d_status = nullptr;
    unsigned int* d_queue = nullptr;  // the persistent propagator's work queue (zeroed before each launch)
    // fused propagator + sum for a few ranges (no integrand in HBM)
    bool fused = false;
    cd* d_partial = nullptr;
    // split (tensor-core) quadrature
    bool tc = false;
    int Mp = 0, Np = 0, Kp = 0, col_exp = 0;
    int8_t *d_A = nullptr, *d_B = nullptr;
    int* d_rowexp = nullptr;
    unsigned long long* d_rowmax = nullptr;
    // split-K wavenumber sums for chunks too small to fill the SMs
    int ksplit = 1;
    cd* d_ksum = nullptr;  // [ksplit][rows of a chunk][nr] partial sums
    int32_t launches_per_exec = 0;  // after the first execute (which may also build the Hankel weights)
    std::shared_ptr<gfk_weights> wts;  // d_W or d_B, shared with other plans on the same grid and ranges
    int prop_variant = -1;       // Dunkin launch shape; -1 until the first execute tunes it
    std::vector<float> tune_ms;  // per variant, from the tuning run
    int tc_variant = -1;            // tensor-core sum tile shape; -1 until the first execute tunes it
    std::vector<float> tc_tune_ms;  // per shape, from the tuning run
    // end-to-end call into pinned host memory: each chunk's rows are copied
    // out on the context's copy stream while the next chunk computes
    double* async_out = nullptr;
    cudaEvent_t ev_chunk = nullptr;
    // CUDA graph of one whole execute
    bool use_graph = false;
    cudaGraphExec_t gexec = nullptr;
    // timing
    std::vector<TimedSeg> segs;
    size_t seg_next = 0;
    double acc_ms[4] = {0, 0, 0, 0};
    int acc_execs = 0;
    bool executed = false;
};

namespace {

const int64_t kDefaultRemBudget = int64_t(4) << 30;  // bytes of integrand per chunk
const int kMaxChunkRows = 65535;                       // grid.y of the per-row kernels

void plan_free(gfk_plan* p) {
    if (!p) return;
    cudaStream_t s = p->ctx ? p->ctx->stream : nullptr;
    if (p->gexec) cudaGraphExecDestroy(p->gexec);
    if (p->ev_chunk) cudaEventDestroy(p->ev_chunk);
    void* ptrs[] = {p->d_lp, p->d_media,  p->d_fd, p->d_ranges, p->d_lc,     p->d_wc2,    p->d_C,
                    p->d_rem, p->d_G,     p->d_status, p->d_A, p->d_rowexp, p->d_rowmax, p->d_partial,
                    p->d_ksum, p->d_queue};
    for (void* q : ptrs)
        if (q) cudaFreeAsync(q, s);
    p->wts.reset();  // the weights go with their last plan (or stay in the context's cache)
    for (auto& sg : p->segs) {
        cudaEventDestroy(sg.a);
        cudaEventDestroy(sg.b);
    }
    if (s) cudaStreamSynchronize(s);
}

template <class T>
int dalloc(gfk_ctx* ctx, T** ptr, size_t count) {
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMallocAsync((void**)ptr, bytes, ctx->stream);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return fail(ctx, GFK_ENOMEM, "device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    return GFK_OK;
}

// The plan's Hankel weights: the context's cached copy when the grid and the
// ranges match, else a new device buffer that becomes the cached one.
int plan_weights(gfk_plan* p, bool tc, int n, double dk, size_t bytes) {
    gfk_ctx* ctx = p->ctx;
    const int nr = (int)p->ranges.size();
    if (ctx->weights && ctx->weights->same(tc, n, dk, p->ranges.data(), nr)) {
        p->wts = ctx->weights;
        return GFK_OK;
    }
    auto w = std::make_shared<gfk_weights>();
    w->ctx = ctx;
    w->tc = tc;
    w->n = n;
    w->dk = dk;
    w->ranges = p->ranges;
    if (cudaMallocAsync(&w->d, std::max<size_t>(bytes, 1), ctx->stream) != cudaSuccess) {
        w->d = nullptr;
        return fail(ctx, GFK_ENOMEM, "device allocation of %zu bytes of Hankel weights failed", bytes);
    }
    ctx->weights = w;
    p->wts = std::move(w);
    return GFK_OK;
}

template <class T>
int h2d(gfk_ctx* ctx, T* dst, const T* src, size_t count) {
    if (count == 0) return GFK_OK;
    GFK_CUDA(ctx, cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return GFK_OK;
}

int begin_seg(gfk_plan* p, int kind, size_t* slot) {
    gfk_ctx* ctx = p->ctx;
    if (p->segs.size() < 256) {
        TimedSeg sg{kind, nullptr, nullptr, false};
        GFK_CUDA(ctx, cudaEventCreate(&sg.a));
        GFK_CUDA(ctx, cudaEventCreate(&sg.b));
        p->segs.push_back(sg);
        *slot = p->segs.size() - 1;
    } else {
        *slot = p->seg_next % p->segs.size();
        TimedSeg& old = p->segs[*slot];
        if (old.pending) {
            GFK_CUDA(ctx, cudaEventSynchronize(old.b));
            float ms = 0;
            cudaEventElapsedTime(&ms, old.a, old.b);
            p->acc_ms[old.kind] += ms;
            old.pending = false;
        }
    }
    p->seg_next++;
    p->segs[*slot].kind = kind;
    GFK_CUDA(ctx, cudaEventRecord(p->segs[*slot].a, ctx->stream));
    return GFK_OK;
}

int end_seg(gfk_plan* p, size_t slot) {
    GFK_CUDA(p->ctx, cudaEventRecord(p->segs[slot].b, p->ctx->stream));
    p->segs[slot].pending = true;
    return GFK_OK;
}

int flush_segs(gfk_plan* p) {
    for (auto& sg : p->segs) {
        if (!sg.pending) continue;
        GFK_CUDA(p->ctx, cudaEventSynchronize(sg.b));
        float ms = 0;
        cudaEventElapsedTime(&ms, sg.a, sg.b);
        p->acc_ms[sg.kind] += ms;
        sg.pending = false;
    }
    return GFK_OK;
}

struct SoilIn {
    const gfk_medium* m;
    const double* freqs;
    int nf;
};

int plan_build(gfk_ctx* ctx, const SoilIn* soils, int nsoil, const gfk_solve* s, const double* ranges, int32_t nr,
               gfk_integration opt, GridMode mode, gfk_plan** out, int chunk_rows = 0) {
    const int max_rows = chunk_rows > 0 ? std::min(chunk_rows, kMaxChunkRows) : kMaxChunkRows;
    *out = nullptr;
    if (!ctx) return GFK_EARG;
    if (!s) return fail(ctx, GFK_EARG, "solve options missing");
    if (s->formulation != GFK_REFERENCE_DIRECT && s->formulation != GFK_DUNKIN)
        return fail(ctx, GFK_EARG, "unknown formulation %d", s->formulation);
    if (s->quadrature != GFK_PLAIN_FP64 && s->quadrature != GFK_SPLIT_INT8)
        return fail(ctx, GFK_EARG, "unknown quadrature %d", s->quadrature);
    if (s->formulation == GFK_REFERENCE_DIRECT && s->omega_imag != 0)
        return fail(ctx, GFK_EARG, "the reference formulation evaluates at real frequencies; omega_imag must be 0");
    if (!(s->omega_imag >= 0) || !std::isfinite(s->omega_imag))
        return fail(ctx, GFK_EARG, "omega_imag must be finite and non-negative, got %g", s->omega_imag);
    if (nsoil <= 0 || !soils) return fail(ctx, GFK_EARG, "no media given");
    if (nr <= 0 || !ranges) return fail(ctx, GFK_EARG, "fk: no ranges given");
    for (int j = 0; j < nr; j++)
        if (!(ranges[j] > 0)) return fail(ctx, GFK_EARG, "fk: range must be positive, got %g m", ranges[j]);
    int64_t nf_total = 0;
    for (int i = 0; i < nsoil; i++) {
        if (soils[i].nf < 0 || (soils[i].nf > 0 && !soils[i].freqs)) return fail(ctx, GFK_EARG, "fk: bad frequency list");
        nf_total += soils[i].nf;
    }
    if (nf_total > INT32_MAX / 2) return fail(ctx, GFK_ELIMIT, "too many bank rows (%lld)", (long long)nf_total);
    if (nsoil == 1) {  // a single medium's stack errors fail the call, as the Go calls do
        const gfk_medium* m = soils[0].m;
        if (!m || !m->layers || m->count <= 0)
            return fail(ctx, GFK_ESTACK, "layer: a stack needs at least a half-space");
        if (m->count > gfk::kMaxLayers)
            return fail(ctx, GFK_ELIMIT, "layer: %d layers, this build handles at most %d", m->count, gfk::kMaxLayers);
    }

    gfk_plan* p = new gfk_plan();
    p->ctx = ctx;
    p->solve = *s;
    p->ranges.assign(ranges, ranges + nr);
    p->nsoil = nsoil;
    p->nf = (int)nf_total;
    p->nr = nr;
    const bool guard = s->guard || s->formulation == GFK_REFERENCE_DIRECT;
    double rmin = INFINITY, rmax = 0;
    for (double r : p->ranges) {
        rmin = std::min(rmin, r);
        rmax = std::max(rmax, r);
    }
    p->host_status.assign(p->nf, GFK_OK);
    p->fd.assign(p->nf, gfk::FreqDesc{});
    p->freqs.assign(p->nf, 0.0);
    std::string first_msg;
    int64_t lc_total = 0;
    double g_kmax = -1;
    int g_n = -1;
    bool shared = true;
    int row = 0;
    for (int si = 0; si < nsoil; si++) {
        const gfk_medium* m = soils[si].m;
        gfk::MediumP mp{};
        int stack_status = GFK_OK;
        std::string stack_msg;
        if (!m || !m->layers || m->count <= 0) {
            stack_status = fail(ctx, GFK_ESTACK, "layer: a stack needs at least a half-space");
        } else if (m->count > gfk::kMaxLayers) {
            stack_status = fail(ctx, GFK_ELIMIT, "layer: %d layers, this build handles at most %d", m->count,
                                gfk::kMaxLayers);
        } else {
            stack_status = validate(ctx, m);
        }
        stack_msg = ctx->last_error;
        double slowest = 1.0;
        if (stack_status == GFK_OK) {
            mp = medium_params(m);
            mp.mu_ref = reference_modulus(m);
            mp.lp_off = (int)p->lp.size();
            for (int i = 0; i < m->count; i++) {
                const gfk_layer& l = m->layers[i];
                p->lp.push_back(gfk::LayerP{l.thickness_m, l.vp_mps, l.vs_mps, l.density_kgm3, l.qs, l.qp});
            }
            slowest = slowest_vs(m);
            p->max_nl = std::max(p->max_nl, m->count);
        } else {
            mp.count = 0;  // an invalid medium never reaches the device
        }
        p->media.push_back(mp);
        for (int fi = 0; fi < soils[si].nf; fi++, row++) {
            const double fr = soils[si].freqs[fi];
            p->freqs[row] = fr;
            gfk::FreqDesc& d = p->fd[row];
            d.freq = fr;
            d.soil = si;
            d.lc_off = lc_total;
            int st = GFK_OK;
            if (stack_status != GFK_OK && stack_status != GFK_ESTACK) {
                st = stack_status;
                ctx->last_error = stack_msg;
            }
            if (!st && guard && m && m->layers && m->count > 0) st = check_layer_phase(ctx, m, fr);
            gfk_grid g{0, 0, 0};
            if (!st && m && m->layers && m->count > 0) {
                if (mode == kGridMulti) {
                    st = grid_for_bounds(m, slowest, rmin, rmax, fr, opt, &g);  // ranges validated above
                } else {  // Medium.VerticalDisplacement's own rule (fk.go:407-421)
                    const double kbody = kTwoPi * fr / slowest;
                    const double kmf = opt.kmax_factor > 0 ? opt.kmax_factor : 30;
                    g.kmax = std::max(opt.kmax > 0 ? opt.kmax : kmf * kbody, 40 / p->ranges[0]);
                    g.samples = opt.samples > 0 ? opt.samples : 20000;
                }
            }
            if (!st && !(fr > 0))
                st = fail(ctx, GFK_EARG, "fk: wavenumber and frequency must be positive, got %g and %g",
                          std::max(200 * kTwoPi * fr / slowest, 400 / rmin), fr);
            if (!st && stack_status) {
                st = stack_status;
                ctx->last_error = stack_msg;
            }
            if (st) {
                p->host_status[row] = st;
                if (first_msg.empty()) first_msg = ctx->last_error;
                continue;  // kfar = 0: no device work for this row
            }
            lc_total += m->count;
            const double kbody = kTwoPi * fr / slowest;
            d.kfar = std::max(200 * kbody, 400 / rmin);
            d.nk = g.samples;
            d.dk = g.kmax / g.samples;
            p->max_nk = std::max(p->max_nk, g.samples);
            if (g_n < 0) {
                g_n = g.samples;
                g_kmax = g.kmax;
            } else if (g_n != g.samples || g_kmax != g.kmax) {
                shared = false;
            }
        }
    }
    ctx->last_error = first_msg;
    p->shared = shared && g_n > 0;
    p->g_n = std::max(g_n, 0);
    p->g_kmax = g_kmax;
    if (s->quadrature == GFK_SPLIT_INT8) {
        if (p->nf > 0 && g_n > 0 && !p->shared) {
            plan_free(p);
            delete p;
            return fail(ctx, GFK_EARG, "the split quadrature needs one wavenumber grid for every frequency "
                                       "(a fixed Integration.kmax and samples)");
        }
        if (g_n > 65536) {
            plan_free(p);
            delete p;
            return fail(ctx, GFK_ELIMIT, "the split quadrature's exact s32 sums allow at most 65536 wavenumbers, got %d",
                        g_n);
        }
        p->tc = p->shared;
    }
    // a few ranges on a shared grid: fuse the sum into the Dunkin propagator
    if (p->shared && s->formulation == GFK_DUNKIN && nr <= gfk::fused_max_ranges() && mode == kGridMulti) {
        p->fused = true;
        p->tc = false;
    }
    // row chunks bounded by the integrand budget and the grid limit; on a shared
    // grid every row keeps its dense slot (row x Nk), failed rows included
    const int64_t budget = kDefaultRemBudget / (int64_t)sizeof(cd);
    int64_t acc = 0, cap = 0;
    int rows_in = 0, cmax = 0;
    p->chunk_begin.push_back(0);
    for (int f = 0; f < p->nf; f++) {
        const int nk = p->shared ? p->g_n : (p->fd[f].kfar > 0 ? p->fd[f].nk : 0);
        if (rows_in > 0 && (acc + nk > budget || rows_in >= max_rows)) {
            p->chunk_begin.push_back(f);
            p->chunk_max_nk.push_back(cmax);
            cap = std::max(cap, acc);
            acc = 0;
            rows_in = 0;
            cmax = 0;
        }
        p->fd[f].off = acc;
        acc += nk;
        rows_in++;
        cmax = std::max(cmax, nk);
    }
    cap = std::max(cap, acc);
    p->chunk_begin.push_back(p->nf);
    p->chunk_max_nk.push_back(cmax);
    p->rem_capacity = cap;

    // device buffers
    int st = GFK_OK;
    const size_t nfa = std::max(p->nf, 1);
    if (!st) st = dalloc(ctx, &p->d_lp, std::max<size_t>(p->lp.size(), 1));
    if (!st) st = dalloc(ctx, &p->d_media, (size_t)nsoil);
    if (!st) st = dalloc(ctx, &p->d_fd, nfa);
    if (!st) st = dalloc(ctx, &p->d_ranges, nr);
    if (!st) st = dalloc(ctx, &p->d_lc, (size_t)std::max<int64_t>(lc_total, 1));
    if (!st) st = dalloc(ctx, &p->d_wc2, nfa);
    if (!st) st = dalloc(ctx, &p->d_C, nfa);
    if (!st) st = dalloc(ctx, &p->d_G, nfa * nr);
    if (!st) st = dalloc(ctx, &p->d_status, nfa);
    if (!st) st = dalloc(ctx, &p->d_queue, 1);
    if (p->fused) {
        int max_cnf = 0;
        for (size_t c = 0; c + 1 < p->chunk_begin.size(); c++)
            max_cnf = std::max(max_cnf, p->chunk_begin[c + 1] - p->chunk_begin[c]);
        const int nkb = (g_n + 127) / 128;
        if (!st) st = dalloc(ctx, &p->d_partial, (size_t)max_cnf * nkb * nr);
    } else if (!st) {
        st = dalloc(ctx, &p->d_rem, (size_t)std::max<int64_t>(cap, 1));
    }
    if (!st && p->shared && !p->tc) {
        if (!(st = plan_weights(p, false, g_n, g_kmax / g_n, sizeof(double) * (size_t)g_n * nr)))
            p->d_W = static_cast<double*>(p->wts->d);
    }
    if (!st && p->tc) {
        int max_cnf = 0;
        for (size_t c = 0; c + 1 < p->chunk_begin.size(); c++)
            max_cnf = std::max(max_cnf, p->chunk_begin[c + 1] - p->chunk_begin[c]);
        p->Mp = (2 * max_cnf + 127) / 128 * 128;
        p->Np = (nr + 127) / 128 * 128;
        p->Kp = (g_n + 63) / 64 * 64;
        p->col_exp = gfk::tc_col_exp(g_kmax / g_n);
        // the propagator writes every digit of a chunk's rows up to Kp; rows
        // past a chunk's 2 cnf are computed by the sum but never stored, so
        // the planes need no clearing
        st = dalloc(ctx, &p->d_A, (size_t)4 * p->Mp * p->Kp);
        if (!st && !(st = plan_weights(p, true, g_n, g_kmax / g_n, (size_t)4 * p->Np * p->Kp)))
            p->d_B = static_cast<int8_t*>(p->wts->d);
        if (!st) st = dalloc(ctx, &p->d_rowexp, (size_t)p->Mp);
        if (!st) st = dalloc(ctx, &p->d_rowmax, (size_t)3 * max_cnf);  // row maxima, then finished-block counts
    }
    if (!st && p->shared && !p->fused) {
        int max_cnf = 0;
        for (size_t c = 0; c + 1 < p->chunk_begin.size(); c++)
            max_cnf = std::max(max_cnf, p->chunk_begin[c + 1] - p->chunk_begin[c]);
        int ks = p->tc ? gfk::quad_tc_splits(2 * max_cnf, nr, p->Kp) : gfk::quad_gemm_splits(max_cnf, g_n, nr);
        const int64_t per_split = (int64_t)max_cnf * nr;
        while (ks > 1 && ks * per_split * (int64_t)sizeof(cd) > (int64_t(512) << 20)) ks--;
        p->ksplit = ks;
        if (ks > 1) st = dalloc(ctx, &p->d_ksum, (size_t)(ks * per_split));
    }
    if (!st) st = h2d(ctx, p->d_lp, p->lp.data(), p->lp.size());
    if (!st) st = h2d(ctx, p->d_media, p->media.data(), p->media.size());
    if (!st) st = h2d(ctx, p->d_fd, p->fd.data(), p->fd.size());
    if (!st) st = h2d(ctx, p->d_ranges, p->ranges.data(), nr);
    if (!st && cudaStreamSynchronize(ctx->stream) != cudaSuccess)  // host tables may be freed by the caller
        st = fail(ctx, GFK_ECUDA, "plan upload failed");
    if (st) {
        plan_free(p);
        delete p;
        return st;
    }
    int nchunks = 0;
    for (size_t c = 0; c + 1 < p->chunk_begin.size(); c++)
        if (p->chunk_begin[c + 1] > p->chunk_begin[c]) nchunks++;
    p->launches_per_exec = p->nf > 0 ? 2 + 2 * nchunks : 0;
    if (p->nf > 0 && p->ksplit > 1) p->launches_per_exec += nchunks;
    if (p->fused) p->prop_variant = 0;  // one launch shape; nothing to tune
    *out = p;
    return GFK_OK;
}

// Where the propagator cuts the digit planes of a chunk of `rows` rows: its
// maxima in d_rowmax[0, 2 rows), its finished-block counts after them.
gfk::SliceOut slice_out(const gfk_plan* p, int rows) {
    return gfk::SliceOut{p->d_rowmax, p->d_rowmax + 2 * (size_t)rows, p->d_rowexp, p->d_A, p->Mp, p->Kp};
}

// Times every Dunkin launch shape on a window of up to 1024 rows of the first
// chunk (its middle) and keeps the fastest. Small windows rank the shapes
// by their launch tails: 64 rows could not tell shapes 4% apart at full size,
// and 256 rows ranked the shapes with several wavenumber runs per block last
// although they are the fastest on the graded soil's 2048 rows. The window's
// integrand rows are recomputed by the real launch afterwards.
int tune_prop(gfk_plan* p) {
    gfk_ctx* ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    const int nv = gfk::prop_variant_count();
    p->prop_variant = 0;
    if (const char* env = getenv("GFK_PROP_VARIANT")) {
        p->prop_variant = std::max(0, std::min(nv - 1, atoi(env)));
        return GFK_OK;
    }
    if (p->solve.formulation != GFK_DUNKIN || p->nf == 0) return GFK_OK;
    for (const auto& t : ctx->tuned)
        if (t.nl == p->max_nl && t.nk == p->max_nk) {
            p->prop_variant = t.variant;
            return GFK_OK;
        }
    const int c0 = p->chunk_begin[0], c1 = p->chunk_begin[1];
    const int win = std::min(1024, c1 - c0);
    if (win <= 0) return GFK_OK;
    const int fb = c0 + (c1 - c0 - win) / 2;
    int cmax = 0;
    for (int f = fb; f < fb + win; f++) cmax = std::max(cmax, p->fd[f].kfar > 0 ? p->fd[f].nk : 0);
    if ((int64_t)win * cmax < 4096) return GFK_OK;  // too little work to tell shapes apart
    // with the tensor-core sum the shapes are timed with their slicing (the
    // window's digit planes are cut again by the real launch)
    const gfk::SliceOut so = slice_out(p, win);
    if (p->tc) GFK_CUDA(ctx, cudaMemsetAsync(p->d_rowmax, 0, sizeof(unsigned long long) * 3 * win, s));
    cudaEvent_t a, b;
    GFK_CUDA(ctx, cudaEventCreate(&a));
    GFK_CUDA(ctx, cudaEventCreate(&b));
    p->tune_ms.assign(nv, INFINITY);
    for (int rep = 0; rep < 2; rep++)
        for (int v = 0; v < nv; v++) {
            cudaMemsetAsync(p->d_queue, 0, sizeof(unsigned int), s);
            cudaEventRecord(a, s);
            gfk::launch_prop(s, p->d_lc, p->d_media, p->d_fd + fb, p->d_wc2 + fb, win, cmax, p->d_C + fb,
                             GFK_DUNKIN, p->d_rem, p->d_status + fb, v, p->tc ? &so : nullptr, p->d_queue);
            cudaEventRecord(b, s);
            ctx->launches++;
            cudaError_t e = cudaEventSynchronize(b);
            if (e != cudaSuccess) {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
                return fail(ctx, GFK_ECUDA, "propagator tuning: %s", cudaGetErrorString(e));
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            p->tune_ms[v] = std::min(p->tune_ms[v], ms);
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    int best = 0;
    for (int v = 1; v < nv; v++)
        if (p->tune_ms[v] < p->tune_ms[best]) best = v;
    p->prop_variant = best;
    ctx->tuned.push_back({p->max_nl, p->max_nk, best});
    return GFK_OK;
}

// Times every tile shape of the tensor-core sum on the first row chunk (its
// slices are in place) and keeps the fastest; the context remembers the
// choice per padded (rows, ranges, wavenumbers). The timed launches write the
// chunk's result rows, which the real launch then recomputes.
// GFK_QUAD_TC_VARIANT=<index> forces a shape.
int tune_tc(gfk_plan* p, int fb, int cnf, double dk) {
    gfk_ctx* ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    const int nv = gfk::quad_tc_variant_count();
    p->tc_variant = 0;
    if (const char* env = getenv("GFK_QUAD_TC_VARIANT")) {
        p->tc_variant = std::max(0, std::min(nv - 1, atoi(env)));
        return GFK_OK;
    }
    for (const auto& t : ctx->tuned_tc)
        if (t.Mp == p->Mp && t.Np == p->Np && t.Kp == p->Kp) {
            p->tc_variant = t.variant;
            return GFK_OK;
        }
    cudaEvent_t a, b;
    GFK_CUDA(ctx, cudaEventCreate(&a));
    GFK_CUDA(ctx, cudaEventCreate(&b));
    p->tc_tune_ms.assign(nv, INFINITY);
    for (int rep = 0; rep < 2; rep++)
        for (int v = 0; v < nv; v++) {
            cudaEventRecord(a, s);
            const int rc = gfk::launch_quad_tc(s, p->d_A, p->d_B, 2 * cnf, p->nr, p->Mp, p->Np, p->Kp, p->d_rowexp,
                                               p->col_exp, p->d_C + fb, p->d_ranges, dk, p->d_G + (size_t)fb * p->nr,
                                               p->d_status + fb, p->ksplit, p->d_ksum, v);
            cudaEventRecord(b, s);
            ctx->launches += 1 + (p->ksplit > 1 ? 1 : 0);
            cudaError_t e = rc ? cudaErrorInvalidValue : cudaEventSynchronize(b);
            if (e != cudaSuccess) {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
                return fail(ctx, GFK_ECUDA, "tensor-core sum tuning (shape %d): %s", v, cudaGetErrorString(e));
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            p->tc_tune_ms[v] = std::min(p->tc_tune_ms[v], ms);
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    int best = 0;
    for (int v = 1; v < nv; v++)
        if (p->tc_tune_ms[v] < p->tc_tune_ms[best]) best = v;
    p->tc_variant = best;
    ctx->tuned_tc.push_back({p->Mp, p->Np, p->Kp, best});
    return GFK_OK;
}

// With async_out set, queues the download of rows [fb, fb + n) on the copy
// stream once the compute stream has finished them.
int copy_chunk_out(gfk_plan* p, int fb, int n) {
    if (!p->async_out || n <= 0) return GFK_OK;
    gfk_ctx* ctx = p->ctx;
    GFK_CUDA(ctx, cudaEventRecord(p->ev_chunk, ctx->stream));
    GFK_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, p->ev_chunk, 0));
    GFK_CUDA(ctx, cudaMemcpyAsync(p->async_out + (size_t)2 * fb * p->nr, p->d_G + (size_t)fb * p->nr,
                                  sizeof(cd) * (size_t)n * p->nr, cudaMemcpyDeviceToHost, ctx->copy_stream));
    return GFK_OK;
}

// Enqueues one whole execute on the context's stream. `timed` records the
// per-kernel-class event segments (not inside a graph capture).
int plan_enqueue(gfk_plan* p, bool timed) {
    gfk_ctx* ctx = p->ctx;
    cudaStream_t s = ctx->stream;
    const int nf = p->nf;
    const int form = p->solve.formulation;
    int st = GFK_OK;
    size_t seg = 0;
    GFK_CUDA(ctx, cudaMemsetAsync(p->d_status, 0, sizeof(int) * nf, s));
    if (timed && (st = begin_seg(p, 2, &seg))) return st;
    gfk::launch_layer_consts_fl(s, p->d_lp, p->d_media, p->d_fd, nf, p->max_nl, p->solve.omega_imag, form, p->d_lc,
                                p->d_wc2);
    gfk::launch_static(s, p->d_lc, p->d_media, p->d_fd, p->d_wc2, nf, form, p->d_C, p->d_status);
    // the Hankel weights depend only on the plan's grid and ranges: built by
    // the first execute of the first plan that holds them, kept for later
    // executes and plans (and out of a captured graph)
    if (p->shared && p->wts && !p->wts->built) {
        if (p->tc)
            gfk::launch_j0_slices(s, p->d_ranges, p->nr, p->g_n, p->Kp, p->Np, p->g_kmax / p->g_n, p->col_exp,
                                  p->d_B);
        else
            gfk::launch_j0_table(s, p->d_ranges, p->nr, p->g_n, p->g_kmax / p->g_n, p->d_W);
        ctx->launches++;
        p->wts->built = true;
    }
    if (timed && (st = end_seg(p, seg))) return st;
    ctx->launches += 2;
    if (timed && p->prop_variant < 0 && (st = tune_prop(p))) return st;
    const double dk = p->shared ? p->g_kmax / p->g_n : 0.0;
    for (size_t c = 0; c + 1 < p->chunk_begin.size(); c++) {
        const int fb = p->chunk_begin[c], fe = p->chunk_begin[c + 1];
        const int cnf = fe - fb;
        if (cnf <= 0) continue;
        const int cmax = p->chunk_max_nk[c];
        if (p->fused) {
            if (timed && (st = begin_seg(p, 0, &seg))) return st;
            gfk::launch_prop_fused(s, p->d_lc, p->d_media, p->d_fd + fb, p->d_wc2 + fb, cnf, p->g_n, p->d_C + fb,
                                   p->d_W, p->d_ranges, p->nr, p->d_partial, p->d_status + fb,
                                   p->d_G + (size_t)fb * p->nr);
            if (timed && (st = end_seg(p, seg))) return st;
            ctx->launches += 2;
            if ((st = copy_chunk_out(p, fb, cnf))) return st;
            continue;
        }
        // the tensor-core sum's digit planes are cut by the propagator itself
        const gfk::SliceOut so = slice_out(p, cnf);
        if (p->tc) GFK_CUDA(ctx, cudaMemsetAsync(p->d_rowmax, 0, sizeof(unsigned long long) * 3 * cnf, s));
        if (gfk::prop_variant_persistent(p->prop_variant))
            GFK_CUDA(ctx, cudaMemsetAsync(p->d_queue, 0, sizeof(unsigned int), s));
        if (timed && (st = begin_seg(p, 0, &seg))) return st;
        gfk::launch_prop(s, p->d_lc, p->d_media, p->d_fd + fb, p->d_wc2 + fb, cnf, cmax, p->d_C + fb, form, p->d_rem,
                         p->d_status + fb, std::max(p->prop_variant, 0), p->tc ? &so : nullptr, p->d_queue);
        if (timed && (st = end_seg(p, seg))) return st;
        if (timed && (st = begin_seg(p, 1, &seg))) return st;
        if (p->tc) {
            if (timed && p->tc_variant < 0 && (st = tune_tc(p, fb, cnf, dk))) return st;
            if (gfk::launch_quad_tc(s, p->d_A, p->d_B, 2 * cnf, p->nr, p->Mp, p->Np, p->Kp, p->d_rowexp, p->col_exp,
                                    p->d_C + fb, p->d_ranges, dk, p->d_G + (size_t)fb * p->nr, p->d_status + fb,
                                    p->ksplit, p->d_ksum, std::max(p->tc_variant, 0)))
                return fail(ctx, GFK_ECUDA, "tensor-core quadrature launch setup failed");
            ctx->launches += 1 + (p->ksplit > 1 ? 1 : 0);
        } else if (p->shared) {
            gfk::launch_quad_gemm(s, p->d_rem, p->d_W, p->d_C + fb, p->d_ranges, cnf, p->g_n, p->nr, dk,
                                  p->d_G + (size_t)fb * p->nr, p->ksplit, p->d_ksum);
            ctx->launches += p->ksplit > 1 ? 1 : 0;
        } else {
            gfk::launch_quad_ragged(s, p->d_rem, p->d_C + fb, p->d_ranges, cnf, p->nr, p->d_fd + fb,
                                    p->d_G + (size_t)fb * p->nr);
        }
        if (timed && (st = end_seg(p, seg))) return st;
        ctx->launches += p->tc ? 1 : 2;
        if ((st = copy_chunk_out(p, fb, cnf))) return st;
    }
    GFK_CUDA(ctx, cudaGetLastError());
    return GFK_OK;
}

int plan_exec(gfk_plan* p) {
    gfk_ctx* ctx = p->ctx;
    if (p->nf == 0) {
        p->executed = true;
        return GFK_OK;
    }
    int st = GFK_OK;
    if (p->use_graph && p->executed && p->prop_variant >= 0 && (!p->tc || p->tc_variant >= 0)) {
        if (!p->gexec) {  // capture one whole execute, once
            const int64_t before = ctx->launches;
            cudaGraph_t g = nullptr;
            GFK_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            st = plan_enqueue(p, false);
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (!st && e != cudaSuccess) st = fail(ctx, GFK_ECUDA, "graph capture: %s", cudaGetErrorString(e));
            if (!st && cudaGraphInstantiate(&p->gexec, g, 0) != cudaSuccess)
                st = fail(ctx, GFK_ECUDA, "graph instantiation failed");
            if (g) cudaGraphDestroy(g);
            ctx->launches = before;  // capturing launches nothing
            if (st) return st;
        }
        size_t seg;
        if ((st = begin_seg(p, 3, &seg))) return st;
        GFK_CUDA(ctx, cudaGraphLaunch(p->gexec, ctx->stream));
        if ((st = end_seg(p, seg))) return st;
        ctx->launches += p->launches_per_exec;
    } else {
        if ((st = plan_enqueue(p, true))) return st;
    }
    p->acc_execs++;
    p->executed = true;
    return GFK_OK;
}

int plan_download(gfk_plan* p, double* out, int32_t* status) {
    gfk_ctx* ctx = p->ctx;
    const int nf = p->nf, nr = p->nr;
    if (nf == 0) return GFK_OK;
    std::vector<int> dst(nf);
    if (out)
        GFK_CUDA(ctx, cudaMemcpyAsync(out, p->d_G, sizeof(cd) * (size_t)nf * nr, cudaMemcpyDeviceToHost, ctx->stream));
    GFK_CUDA(ctx, cudaMemcpyAsync(dst.data(), p->d_status, sizeof(int) * nf, cudaMemcpyDeviceToHost, ctx->stream));
    GFK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    int first = GFK_OK;
    std::string msg = ctx->last_error;
    for (int f = 0; f < nf; f++) {
        int st = p->host_status[f];
        if (!st && (dst[f] & gfk::kStSingular)) {
            st = GFK_ESINGULAR;
            if (first == GFK_OK)
                msg = "fk: layer propagator or surface system is singular at f=" + std::to_string(p->freqs[f]);
        } else if (!st && (dst[f] & gfk::kStTimeout)) {
            st = GFK_ETIMEOUT;
            if (first == GFK_OK) msg = "a device-side wait in the tensor-core quadrature timed out";
        } else if (!st && (dst[f] & gfk::kStNonfinite)) {
            st = GFK_ENONFINITE;
            if (first == GFK_OK) msg = "fk: non-finite response at f=" + std::to_string(p->freqs[f]);
        }
        if (st && out) std::memset(out + (size_t)2 * nr * f, 0, sizeof(double) * 2 * nr);
        if (status) status[f] = st;
        if (st && first == GFK_OK) first = st;
    }
    if (first) ctx->last_error = msg;
    return first;
}

int plan_one(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* ranges, int32_t nr,
             const double* freqs, int32_t nf, gfk_integration opt, GridMode mode, gfk_plan** out,
             int chunk_rows = 0) {
    SoilIn si{m, freqs, nf};
    return plan_build(ctx, &si, 1, s, ranges, nr, opt, mode, out, chunk_rows);
}

}  // namespace

// ------------------------------------------------------------------ ABI --

extern "C" {

const char* gfk_status_string(int status) {
    switch (status) {
        case GFK_OK: return "ok";
        case GFK_EARG: return "invalid argument";
        case GFK_ESTACK: return "invalid layer stack";
        case GFK_EGUARD: return "layer phase past MaxLayerPhase";
        case GFK_ESINGULAR: return "singular propagator or surface system";
        case GFK_ENONFINITE: return "non-finite result";
        case GFK_ETIMEOUT: return "device wait timed out";
        case GFK_ECUDA: return "CUDA error";
        case GFK_ENOMEM: return "out of memory";
        case GFK_EIO: return "bank file I/O error";
        case GFK_ELIMIT: return "size beyond limit";
        default: return "unknown status";
    }
}

int gfk_open(int device, gfk_ctx** out) {
    if (!out) return GFK_EARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return GFK_ECUDA;
    if (device < 0 || device >= n) return GFK_EARG;
    gfk_ctx* c = new gfk_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return GFK_ECUDA;
    }
    // keep freed stream-ordered allocations cached for the next call
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = c;
    return GFK_OK;
}

gfk_weights::~gfk_weights() {
    if (d) cudaFreeAsync(d, ctx->stream);
}

int gfk_close(gfk_ctx* ctx) {
    if (!ctx) return GFK_OK;
    cudaSetDevice(ctx->device);
    for (gfk_plan* p : ctx->plans) {  // plans still open become invalid here
        plan_free(p);
        delete p;
    }
    ctx->plans.clear();
    ctx->weights.reset();
    gfk_release_surrogates(ctx);
    gfk_release_banks(ctx);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return GFK_OK;
}

const char* gfk_last_error(const gfk_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int64_t gfk_kernel_launches(const gfk_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* gfk_stream(const gfk_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int gfk_selftest_wait_timeout(gfk_ctx* ctx, int64_t wait_cycles, int32_t* rows_timed_out) {
    if (!ctx || !rows_timed_out || wait_cycles <= 0) return GFK_EARG;
    *rows_timed_out = 0;
    cudaSetDevice(ctx->device);
    int rows = 0;
    const int rc = gfk::quad_tc_selftest_timeout(ctx->stream, wait_cycles, &rows);
    ctx->launches++;
    if (rc) return fail(ctx, GFK_ECUDA, "wait self-test: CUDA failure (step %d): %s", rc,
                        cudaGetErrorString(cudaGetLastError()));
    *rows_timed_out = rows;
    if (rows == 0) {
        ctx->last_error.clear();
        return GFK_OK;
    }
    return fail(ctx, GFK_ETIMEOUT, "a device-side wait in the tensor-core quadrature timed out (self-test)");
}

int gfk_stack_validate(const gfk_medium* m) { return validate(nullptr, m); }

int gfk_check_layer_phase(const gfk_medium* m, double freq_hz) { return check_layer_phase(nullptr, m, freq_hz); }

int gfk_grid_for(const gfk_medium* m, const double* ranges, int32_t nr, double freq_hz, gfk_integration opt,
                 gfk_grid* out) {
    if (!out) return GFK_EARG;
    return grid_for(nullptr, m, ranges, nr, freq_hz, opt, out);
}

int gfk_plan_create(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* ranges, int32_t nr,
                    const double* freqs, int32_t nf, gfk_integration opt, gfk_plan** out) {
    if (!out) return GFK_EARG;
    if (!ctx) return GFK_EARG;
    cudaSetDevice(ctx->device);
    int st = plan_one(ctx, m, s, ranges, nr, freqs, nf, opt, kGridMulti, out);
    if (!st) ctx->plans.push_back(*out);
    return st;
}

int gfk_plan_execute(gfk_plan* p) {
    if (!p) return GFK_EARG;
    cudaSetDevice(p->ctx->device);
    return plan_exec(p);
}

int gfk_plan_result_device(gfk_plan* p, const double** d_out) {
    if (!p || !d_out) return GFK_EARG;
    *d_out = reinterpret_cast<const double*>(p->d_G);
    return GFK_OK;
}

int gfk_plan_download(gfk_plan* p, double* out, int32_t* status_per_f) {
    if (!p) return GFK_EARG;
    if (!p->executed) return fail(p->ctx, GFK_EARG, "plan has not been executed");
    return plan_download(p, out, status_per_f);
}

int32_t gfk_plan_launches_per_execute(const gfk_plan* p) { return p ? p->launches_per_exec : 0; }

int gfk_plan_tuning(const gfk_plan* p, int32_t* variant, float* ms_per_variant, int32_t capacity) {
    if (!p || !variant) return GFK_EARG;
    *variant = p->prop_variant;
    const int n = (int)p->tune_ms.size();
    for (int i = 0; ms_per_variant && i < std::min(n, (int)capacity); i++) ms_per_variant[i] = p->tune_ms[i];
    return n;
}

int gfk_prop_shape(int32_t variant, int32_t* threads, int32_t* blocks_per_sm, int32_t* wavenumbers_per_thread,
                   int32_t* runs_per_item, int32_t* persistent) {
    if (!threads || !blocks_per_sm || !wavenumbers_per_thread || !runs_per_item || !persistent) return GFK_EARG;
    int t, b, i, r, q;
    if (!gfk::prop_variant_shape(variant, &t, &b, &i, &r, &q)) return GFK_EARG;
    *threads = t;
    *blocks_per_sm = b;
    *wavenumbers_per_thread = i;
    *runs_per_item = r;
    *persistent = q;
    return GFK_OK;
}

int gfk_plan_quad_shape(const gfk_plan* p, int32_t* tile_n, int32_t* stages, float* ms_per_shape, int32_t capacity) {
    if (!p || !tile_n || !stages) return GFK_EARG;
    int tn = 0, ns = 0;
    if (p->tc && p->tc_variant >= 0) gfk::quad_tc_variant_shape(p->tc_variant, &tn, &ns);
    *tile_n = tn;
    *stages = ns;
    const int n = (int)p->tc_tune_ms.size();
    for (int i = 0; ms_per_shape && i < std::min(n, (int)capacity); i++) ms_per_shape[i] = p->tc_tune_ms[i];
    return n;
}

int gfk_plan_kernel_times(gfk_plan* p, double* prop_ms, double* quad_ms, double* other_ms, int32_t reset) {
    if (!p) return GFK_EARG;
    int st = flush_segs(p);
    if (st) return st;
    const double n = p->acc_execs > 0 ? p->acc_execs : 1;
    if (prop_ms) *prop_ms = p->acc_ms[0] / n;
    if (quad_ms) *quad_ms = p->acc_ms[1] / n;
    if (other_ms) *other_ms = (p->acc_ms[2] + p->acc_ms[3]) / n;
    if (reset) {
        p->acc_ms[0] = p->acc_ms[1] = p->acc_ms[2] = p->acc_ms[3] = 0;
        p->acc_execs = 0;
    }
    return GFK_OK;
}

int gfk_plan_use_graph(gfk_plan* p, int32_t enable) {
    if (!p) return GFK_EARG;
    p->use_graph = enable != 0;
    if (!p->use_graph && p->gexec) {
        cudaGraphExecDestroy(p->gexec);
        p->gexec = nullptr;
    }
    return GFK_OK;
}

int gfk_batch_create(gfk_ctx* ctx, const gfk_medium* media, int32_t nsoil, const double* const* freqs_hz,
                     const int32_t* nf, const gfk_solve* s, const double* ranges_m, int32_t nr, gfk_integration opt,
                     gfk_plan** out) {
    if (!ctx || !out) return GFK_EARG;
    if (nsoil <= 0 || !media || !freqs_hz || !nf) return fail(ctx, GFK_EARG, "no media given");
    cudaSetDevice(ctx->device);
    std::vector<SoilIn> soils(nsoil);
    for (int i = 0; i < nsoil; i++) soils[i] = SoilIn{&media[i], freqs_hz[i], nf[i]};
    int st = plan_build(ctx, soils.data(), nsoil, s, ranges_m, nr, opt, kGridMulti, out);
    if (!st) ctx->plans.push_back(*out);
    return st;
}

static int exec_download_overlapped(gfk_plan* p, double* out, int32_t* status_per_f);

int gfk_plan_execute_download(gfk_plan* p, double* out, int32_t* status_per_f) {
    if (!p) return GFK_EARG;
    cudaSetDevice(p->ctx->device);
    return exec_download_overlapped(p, out, status_per_f);
}

int gfk_plan_destroy(gfk_plan* p) {
    if (!p) return GFK_OK;
    cudaSetDevice(p->ctx->device);
    auto& v = p->ctx->plans;
    v.erase(std::remove(v.begin(), v.end(), p), v.end());
    plan_free(p);
    delete p;
    return GFK_OK;
}

// True when `out` is page-locked host memory and the context's copy stream
// exists (created here on first use).
static bool pinned_with_copy_stream(gfk_ctx* ctx, const void* out) {
    if (!out) return false;
    cudaPointerAttributes pa{};
    const bool pinned = cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a pageable pointer is not an error
    if (!pinned) return false;
    if (!ctx->copy_stream && cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        ctx->copy_stream = nullptr;
        return false;
    }
    return true;
}

// One execute with each row chunk copied into `out` (page-locked) on the copy
// stream as soon as it is computed, then the statuses, failed rows zeroed, as
// plan_download gives them. Runs the execute as separate launches (a captured
// graph carries no copies). Plans of one chunk execute, then download.
static int exec_download_overlapped(gfk_plan* p, double* out, int32_t* status_per_f) {
    gfk_ctx* ctx = p->ctx;
    if (p->chunk_begin.size() <= 2 || !pinned_with_copy_stream(ctx, out)) {
        const int st = plan_exec(p);
        return st ? st : plan_download(p, out, status_per_f);
    }
    if (!p->ev_chunk && cudaEventCreateWithFlags(&p->ev_chunk, cudaEventDisableTiming) != cudaSuccess)
        return fail(ctx, GFK_ECUDA, "bank download: event creation failed");
    const bool graph = p->use_graph;
    p->use_graph = false;
    p->async_out = out;
    int st = plan_exec(p);
    p->async_out = nullptr;
    p->use_graph = graph;
    if (cudaStreamSynchronize(ctx->copy_stream) != cudaSuccess && !st) st = fail(ctx, GFK_ECUDA, "bank download failed");
    if (st) return st;
    std::vector<int32_t> stv(std::max(p->nf, 1));
    st = plan_download(p, nullptr, stv.data());
    for (int f = 0; f < p->nf; f++) {
        if (stv[f]) std::memset(out + (size_t)2 * p->nr * f, 0, sizeof(double) * 2 * p->nr);
        if (status_per_f) status_per_f[f] = stv[f];
    }
    return st;
}

int gfk_bank_spectra(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* ranges, int32_t nr,
                     const double* freqs, int32_t nf, gfk_integration opt, double* out, int32_t* status_per_f) {
    if (!ctx) return GFK_EARG;
    cudaSetDevice(ctx->device);
    // Into page-locked host memory a large bank (>= 8 MB) is computed in two
    // row chunks, the first downloaded on a second stream while the second
    // computes (smaller banks lose more to the extra launches than they hide).
    const bool overlap = out && nf >= 256 && nr >= 1 && (int64_t)nf * nr * 16 >= (int64_t(8) << 20) &&
                         pinned_with_copy_stream(ctx, out);
    gfk_plan* p = nullptr;
    int st = plan_one(ctx, m, s, ranges, nr, freqs, nf, opt, kGridMulti, &p, overlap ? (nf + 1) / 2 : 0);
    if (st) return st;
    st = exec_download_overlapped(p, out, status_per_f);
    std::string msg = ctx->last_error;
    plan_free(p);
    delete p;
    ctx->last_error = msg;
    return st;
}

int gfk_bank_payload(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* ranges, int32_t nr,
                     const double* freqs, int32_t nf, gfk_integration opt, int32_t first_bin, int32_t bins,
                     float* payload, int32_t* status_per_f) {
    if (!ctx) return GFK_EARG;
    if (!payload || bins <= 0 || first_bin < 0 || nf < 0 || (int64_t)first_bin + nf > bins)
        return fail(ctx, GFK_EARG, "bank: bins [%d, %d) do not fit a payload of %d bins", first_bin, first_bin + nf,
                    bins);
    cudaSetDevice(ctx->device);
    gfk_plan* p = nullptr;
    int st = plan_one(ctx, m, s, ranges, nr, freqs, nf, opt, kGridMulti, &p);
    if (st) return st;
    st = plan_exec(p);
    std::vector<int32_t> stv(std::max(p->nf, 1), GFK_OK);
    int first = GFK_OK;
    if (!st) first = plan_download(p, nullptr, stv.data());  // statuses only; the first failure in order
    std::string msg = ctx->last_error;
    cudaStream_t cs = ctx->stream;
    float* d_pay = nullptr;
    const size_t nfloat = (size_t)2 * nr * bins;
    if (!st) {
        // failed rows pack as zeros, as the FP64 call returns them
        for (int f = 0; f < p->nf && !st; f++)
            if (stv[f] && cudaMemsetAsync(p->d_G + (size_t)f * nr, 0, sizeof(cd) * nr, cs) != cudaSuccess)
                st = fail(ctx, GFK_ECUDA, "bank: clearing a failed row failed");
        if (!st && cudaMallocAsync((void**)&d_pay, sizeof(float) * nfloat, cs) != cudaSuccess) {
            d_pay = nullptr;
            st = fail(ctx, GFK_ENOMEM, "bank: device payload of %zu bytes", sizeof(float) * nfloat);
        }
        if (!st && cudaMemsetAsync(d_pay, 0, sizeof(float) * nfloat, cs) != cudaSuccess)
            st = fail(ctx, GFK_ECUDA, "bank: clearing the payload failed");
        if (!st && p->nf > 0) {
            gfk::launch_bank_pack(cs, p->d_G, p->nf, nr, first_bin, bins, d_pay);
            ctx->launches++;
            if (cudaGetLastError() != cudaSuccess) st = fail(ctx, GFK_ECUDA, "bank: packing kernel failed");
        }
        if (!st && cudaMemcpyAsync(payload, d_pay, sizeof(float) * nfloat, cudaMemcpyDeviceToHost, cs) != cudaSuccess)
            st = fail(ctx, GFK_ECUDA, "bank: payload download failed");
        if (d_pay) cudaFreeAsync(d_pay, cs);
        if (cudaStreamSynchronize(cs) != cudaSuccess && !st) st = fail(ctx, GFK_ECUDA, "bank: payload download failed");
    }
    if (status_per_f)
        for (int f = 0; f < p->nf; f++) status_per_f[f] = stv[f];
    if (!st) {
        st = first;
        ctx->last_error = msg;
    }
    msg = ctx->last_error;
    plan_free(p);
    delete p;
    ctx->last_error = msg;
    return st;
}

int gfk_vertical_displacement_multi(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* ranges,
                                    int32_t nr, double freq_hz, gfk_integration opt, double* out) {
    int32_t status = 0;
    return gfk_bank_spectra(ctx, m, s, ranges, nr, &freq_hz, 1, opt, out, &status);
}

int gfk_vertical_displacement(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, double range_m, double freq_hz,
                              gfk_integration opt, double* out) {
    if (!ctx) return GFK_EARG;
    if (!(range_m > 0)) return fail(ctx, GFK_EARG, "fk: range must be positive, got %g m", range_m);
    if (!(freq_hz > 0)) return fail(ctx, GFK_EARG, "fk: frequency must be positive, got %g Hz", freq_hz);
    cudaSetDevice(ctx->device);
    gfk_plan* p = nullptr;
    int st = plan_one(ctx, m, s, &range_m, 1, &freq_hz, 1, opt, kGridSingle, &p);
    if (st) return st;
    // a single range always takes the per-frequency (sequential-sum) quadrature
    p->shared = false;
    p->tc = false;
    st = plan_exec(p);
    int32_t fst = 0;
    if (!st) st = plan_download(p, out, &fst);
    std::string msg = ctx->last_error;
    plan_free(p);
    delete p;
    ctx->last_error = msg;
    return st;
}

// (k, f) pairs: the pairs are grouped by frequency into one single-range
// plan each would be wasteful; instead a plan over the unique frequencies
// supplies the layer constants and a pair kernel evaluates each k.
}  // extern "C"

namespace gfk {
__global__ void k_pairs(const LayerC* __restrict__ lc, int nl, const double* __restrict__ freqs,
                        const cd* __restrict__ wc2, const int* __restrict__ fidx, const double* __restrict__ k,
                        int64_t n, double mu_ref, int formulation, cd* __restrict__ out, int* __restrict__ status) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int f = fidx[i];
    cd u;
    if (formulation == 0) {
        bool ok;
        u = direct_u(lc + (size_t)f * nl, nl, kTwoPi * freqs[f], k[i], mu_ref, ok);
        if (!ok) {
            atomicOr(status, kStSingular);
            u = mk(0.0);
        }
    } else {
        u = dunkin_u(lc + (size_t)f * nl, nl, wc2[f], k[i], mu_ref);
    }
    if (!(isfinite(u.re) && isfinite(u.im))) atomicOr(status, kStNonfinite);
    out[i] = u;
}
}  // namespace gfk

extern "C" int gfk_surface_response(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, const double* k,
                                    const double* freq_hz, int64_t n, double* out) {
    if (!ctx) return GFK_EARG;
    if (n < 0 || (n > 0 && (!k || !freq_hz || !out))) return fail(ctx, GFK_EARG, "fk: bad (k, f) arrays");
    if (n == 0) return GFK_OK;
    if (!s) return fail(ctx, GFK_EARG, "solve options missing");
    if (s->formulation == GFK_REFERENCE_DIRECT && s->omega_imag != 0)
        return fail(ctx, GFK_EARG, "the reference formulation evaluates at real frequencies; omega_imag must be 0");
    for (int64_t i = 0; i < n; i++)
        if (!(k[i] > 0) || !(freq_hz[i] > 0))
            return fail(ctx, GFK_EARG, "fk: wavenumber and frequency must be positive, got %g and %g", k[i],
                        freq_hz[i]);
    int st = validate(ctx, m);
    if (st) return st;
    cudaSetDevice(ctx->device);
    std::vector<double> uf(freq_hz, freq_hz + n);
    std::sort(uf.begin(), uf.end());
    uf.erase(std::unique(uf.begin(), uf.end()), uf.end());
    std::vector<int> fidx(n);
    for (int64_t i = 0; i < n; i++)
        fidx[i] = (int)(std::lower_bound(uf.begin(), uf.end(), freq_hz[i]) - uf.begin());
    const int nf = (int)uf.size(), nl = m->count;
    const double mu_ref = reference_modulus(m);
    std::vector<gfk::LayerP> lp(nl);
    for (int i = 0; i < nl; i++) {
        const gfk_layer& l = m->layers[i];
        lp[i] = gfk::LayerP{l.thickness_m, l.vp_mps, l.vs_mps, l.density_kgm3, l.qs, l.qp};
    }
    gfk::MediumP mp = medium_params(m);
    mp.mu_ref = mu_ref;
    mp.lp_off = 0;
    std::vector<gfk::FreqDesc> fds(nf);
    for (int f = 0; f < nf; f++) {
        fds[f] = gfk::FreqDesc{};
        fds[f].freq = uf[f];
        fds[f].lc_off = (int64_t)f * nl;
    }
    gfk::LayerP* d_layers = nullptr;
    gfk::MediumP* d_media = nullptr;
    gfk::FreqDesc* d_fd = nullptr;
    double *d_f = nullptr, *d_k = nullptr;
    int *d_fidx = nullptr, *d_status = nullptr;
    gfk::LayerC* d_lc = nullptr;
    cd *d_wc2 = nullptr, *d_out = nullptr;
    st = dalloc(ctx, &d_layers, nl);
    if (!st) st = dalloc(ctx, &d_media, 1);
    if (!st) st = dalloc(ctx, &d_fd, nf);
    if (!st) st = dalloc(ctx, &d_f, nf);
    if (!st) st = dalloc(ctx, &d_k, n);
    if (!st) st = dalloc(ctx, &d_fidx, n);
    if (!st) st = dalloc(ctx, &d_status, 1);
    if (!st) st = dalloc(ctx, &d_lc, (size_t)nf * nl);
    if (!st) st = dalloc(ctx, &d_wc2, nf);
    if (!st) st = dalloc(ctx, &d_out, n);
    if (!st) st = h2d(ctx, d_layers, lp.data(), nl);
    if (!st) st = h2d(ctx, d_media, &mp, 1);
    if (!st) st = h2d(ctx, d_fd, fds.data(), nf);
    if (!st) st = h2d(ctx, d_f, uf.data(), nf);
    if (!st) st = h2d(ctx, d_k, k, n);
    if (!st) st = h2d(ctx, d_fidx, fidx.data(), n);
    int hstat = 0;
    if (!st) {
        cudaMemsetAsync(d_status, 0, sizeof(int), ctx->stream);
        gfk::launch_layer_consts(ctx->stream, d_layers, d_media, d_fd, nf, s->omega_imag, s->formulation, d_lc, d_wc2);
        gfk::k_pairs<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
            d_lc, nl, d_f, d_wc2, d_fidx, d_k, n, mu_ref, s->formulation, d_out, d_status);
        ctx->launches += 2;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = fail(ctx, GFK_ECUDA, "k_pairs launch: %s", cudaGetErrorString(e));
    }
    if (!st) {
        cudaMemcpyAsync(out, d_out, sizeof(cd) * n, cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemcpyAsync(&hstat, d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = fail(ctx, GFK_ECUDA, "surface response: %s", cudaGetErrorString(e));
    }
    void* ptrs[] = {d_layers, d_media, d_fd, d_f, d_k, d_fidx, d_status, d_lc, d_wc2, d_out};
    for (void* q : ptrs)
        if (q) cudaFreeAsync(q, ctx->stream);
    cudaStreamSynchronize(ctx->stream);  // the host tables above are freed on return
    if (st) return st;
    if (hstat & gfk::kStSingular)
        return fail(ctx, GFK_ESINGULAR, "fk: layer propagator or surface system is singular");
    if (hstat & gfk::kStNonfinite) return fail(ctx, GFK_ENONFINITE, "fk: non-finite surface response");
    return GFK_OK;
}

extern "C" int gfk_static_coefficient(gfk_ctx* ctx, const gfk_medium* m, const gfk_solve* s, double freq_hz,
                                      double k_far, double* out) {
    double u[2];
    int st = gfk_surface_response(ctx, m, s, &k_far, &freq_hz, 1, u);
    if (st) return st;
    out[0] = k_far * u[0];
    out[1] = k_far * u[1];
    return GFK_OK;
}

// ------------------------------------------------------------ bank file --

extern "C" int gfk_bank_pack(const double* spectra, int32_t nf, int32_t nr, int32_t first_bin, int32_t bins,
                             float* payload) {
    if (nf < 0 || nr <= 0 || bins <= 0 || !payload || (nf > 0 && !spectra)) return GFK_EARG;
    std::memset(payload, 0, sizeof(float) * 2 * (size_t)nr * bins);
    for (int f = 0; f < nf; f++) {
        const int bin = first_bin + f;
        if (bin < 0 || bin >= bins) continue;
        for (int j = 0; j < nr; j++) {
            const size_t o = 2 * ((size_t)j * bins + bin);
            payload[o] = (float)spectra[2 * ((size_t)f * nr + j)];
            payload[o + 1] = (float)spectra[2 * ((size_t)f * nr + j) + 1];
        }
    }
    return GFK_OK;
}

extern "C" int gfk_bank_write(const char* path, const char* header_json, const float* payload, int64_t nfloats) {
    // internal/bank/format.go:215-240
    if (!path || !header_json || nfloats < 0 || (nfloats > 0 && !payload)) return GFK_EARG;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return GFK_EIO;
    static const unsigned char magic[8] = {'G', 'E', 'O', 'B', 'A', 'N', 'K', 0};
    const size_t hlen = std::strlen(header_json);
    auto le32 = [](uint32_t v, unsigned char* b) {
        b[0] = v & 0xff; b[1] = (v >> 8) & 0xff; b[2] = (v >> 16) & 0xff; b[3] = (v >> 24) & 0xff;
    };
    unsigned char hdr[16];
    std::memcpy(hdr, magic, 8);
    le32(1u, hdr + 8);
    le32((uint32_t)hlen, hdr + 12);
    bool ok = std::fwrite(hdr, 1, 16, fp) == 16 && std::fwrite(header_json, 1, hlen, fp) == hlen;
    size_t pos = 16 + hlen;
    static const unsigned char zeros[4096] = {0};
    const size_t pad = (4096 - pos % 4096) % 4096;
    if (ok && pad) ok = std::fwrite(zeros, 1, pad, fp) == pad;
    // payload: little-endian float32 (this library targets little-endian hosts)
    if (ok && nfloats > 0) ok = std::fwrite(payload, sizeof(float), (size_t)nfloats, fp) == (size_t)nfloats;
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? GFK_OK : GFK_EIO;
}
