// gfk_kernels.cu — FP64 kernels of the Green's-function bank path.
//
//   k_layer_consts  per (frequency, layer): complex velocities -> solver constants
//                   (fk.go:96-128 hoisted out of the wavenumber loop)
//   k_static        per frequency: C = k_far u(k_far) (fk.go:365-371, 521)
//   k_prop          per (frequency, wavenumber): the layered solve and the
//                   static-subtracted integrand k u - C (fk.go:534-544)
//   k_j0_table      the shared-grid Hankel weights w_i J0(k_i r_j) dk (fk.go:540-546)
//   k_quad_gemm     the shared-grid wavenumber sum as an FP64 complex x real GEMM
//   k_quad_ragged   per-frequency grids: the same sum with J0 in the loop
//   k_bank_pack     FP64 [f][r] -> float32 range-major bank payload
//                   (internal/bank/format.go:185-193)
#include "gfk_kernels.cuh"

#include <algorithm>
#include <atomic>

namespace gfk {

// ------------------------------------------------------------ constants --

// One layer's constants at one frequency.
__device__ __forceinline__ LayerC layer_const(const MediumP& med, const LayerP& L, double fr, double wi,
                                              int formulation) {
    const double q = q_of(med, L);
    LayerC out;
    if (formulation == 0) {
        // Medium.propsOf (fk.go:119-128): Qp = 2.25 Qs, real frequency
        const cd a = complex_velocity(med, L.vp, 2.25 * q, fr, 0.0);
        const cd b = complex_velocity(med, L.vs, q, fr, 0.0);
        out.c[0] = a;
        out.c[1] = b;
        out.c[2] = (L.rho * b) * b;
        out.c[3] = mk(L.rho);
    } else {
        const double qp = L.qp > 0 ? L.qp : 2.25 * q;
        const cd a = complex_velocity(med, L.vp, qp, fr, wi);
        const cd b = complex_velocity(med, L.vs, q, fr, wi);
        const cd a2 = a * a, b2 = b * b;
        out.c[0] = 1.0 / a2;
        out.c[1] = 1.0 / b2;
        out.c[2] = b2 / a2;
        out.c[3] = (L.rho * b2) / med.mu_ref;
    }
    out.h = L.h;
    out.pad = 0.0;
    return out;
}

__global__ void k_layer_consts(const LayerP* __restrict__ lp, const MediumP* __restrict__ media,
                               const FreqDesc* __restrict__ fd, int nf, double wi, int formulation,
                               LayerC* __restrict__ lc, cd* __restrict__ wc2) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const FreqDesc d = fd[f];
    const MediumP med = media[d.soil];
    const double fr = d.freq;
    for (int l = 0; l < med.count; l++) lc[d.lc_off + l] = layer_const(med, lp[med.lp_off + l], fr, wi, formulation);
    const cd wc = mk(kTwoPi * fr, -wi);
    wc2[f] = wc * wc;
}

void launch_layer_consts(cudaStream_t s, const LayerP* lp, const MediumP* media, const FreqDesc* fd, int nf,
                         double wi, int formulation, LayerC* lc, cd* wc2) {
    if (nf <= 0) return;
    k_layer_consts<<<(nf + 127) / 128, 128, 0, s>>>(lp, media, fd, nf, wi, formulation, lc, wc2);
}

// The same constants with one thread per (frequency, layer): a few hundred
// frequencies of a thin stack otherwise leave most SMs idle while each thread
// walks its layers' transcendental functions in sequence.
__global__ void k_layer_consts_fl(const LayerP* __restrict__ lp, const MediumP* __restrict__ media,
                                  const FreqDesc* __restrict__ fd, int nf, double wi, int formulation,
                                  LayerC* __restrict__ lc, cd* __restrict__ wc2) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (f >= nf) return;
    const FreqDesc d = fd[f];
    const MediumP med = media[d.soil];
    if (l < med.count) lc[d.lc_off + l] = layer_const(med, lp[med.lp_off + l], d.freq, wi, formulation);
    if (l == 0) {
        const cd wc = mk(kTwoPi * d.freq, -wi);
        wc2[f] = wc * wc;
    }
}

void launch_layer_consts_fl(cudaStream_t s, const LayerP* lp, const MediumP* media, const FreqDesc* fd, int nf,
                            int max_layers, double wi, int formulation, LayerC* lc, cd* wc2) {
    if (nf <= 0 || max_layers <= 0) return;
    dim3 grid((nf + 63) / 64, max_layers);
    k_layer_consts_fl<<<grid, 64, 0, s>>>(lp, media, fd, nf, wi, formulation, lc, wc2);
}

__device__ __forceinline__ bool finite_cd(cd a) { return isfinite(a.re) && isfinite(a.im); }

// ------------------------------------------------------ static coefficient --

__global__ void k_static(const LayerC* __restrict__ lc, const MediumP* __restrict__ media,
                         const FreqDesc* __restrict__ fd, const cd* __restrict__ wc2, int nf, int formulation,
                         cd* __restrict__ C, int* __restrict__ status) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const FreqDesc d = fd[f];
    const double k = d.kfar;
    if (!(k > 0)) {
        C[f] = mk(0.0);
        return;
    }
    const MediumP med = media[d.soil];
    cd u;
    if (formulation == 0) {
        bool ok;
        u = direct_u(lc + d.lc_off, med.count, kTwoPi * d.freq, k, med.mu_ref, ok);
        if (!ok) atomicOr(status + f, kStSingular);
    } else {
        u = dunkin_u(lc + d.lc_off, med.count, wc2[f], k, med.mu_ref);
    }
    cd c = k * u;
    if (!finite_cd(c)) {
        atomicOr(status + f, kStNonfinite);
        c = mk(0.0);
    }
    C[f] = c;
}

void launch_static(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2, int nf,
                   int formulation, cd* C, int* status) {
    if (nf <= 0) return;
    k_static<<<(nf + 63) / 64, 64, 0, s>>>(lc, media, fd, wc2, nf, formulation, C, status);
}

// ------------------------------------------------------------ propagator --
//
// The work item is (row f, run): one thread per (f, k) (ILP = 1) or per
// (f, k, k + THREADS) pair (ILP = 2, two wavenumbers in lockstep), SWEEPS
// times over consecutive stretches of THREADS x ILP wavenumbers; a row has
// `runs` items. k_prop serves one item per block (blockIdx = (run, f));
// k_prop_q is persistent: each resident block takes items from a device
// queue in row order until none are left. The row's layer constants are
// staged in shared memory. Launch shapes are template parameters; the plan
// times them once and keeps the fastest.

// Shared memory of one propagator block.
template <int THREADS, bool SLICE>
struct PropSmem {
    LayerC lc[kMaxLayers];
    cd tile[SLICE ? THREADS * 8 : 1];
    int last, item;
};

// `stage`: the block's staged layer constants are not row f's (uniform).
template <int FORM, int THREADS, int ILP, int SWEEPS, bool SLICE>
__device__ __forceinline__ void prop_item(const LayerC* __restrict__ lc, const MediumP* __restrict__ media,
                                          const FreqDesc* __restrict__ fd, const cd* __restrict__ wc2,
                                          const cd* __restrict__ C, cd* __restrict__ rem, int* __restrict__ status,
                                          const SliceOut& so, int f, int run, int runs, bool stage,
                                          PropSmem<THREADS, SLICE>& sm) {
    LayerC* const s_lc = sm.lc;
    const FreqDesc fdesc = fd[f];
    const MediumP med = media[fdesc.soil];
    const int nl = med.count;
    const double mu_ref = med.mu_ref;
    if (stage) {
        for (int l = threadIdx.x; l < nl; l += blockDim.x) s_lc[l] = lc[fdesc.lc_off + l];
        __syncthreads();
    }
    const int n = fdesc.kfar > 0 ? fdesc.nk : 0;
    const double d = fdesc.dk;
    const cd c = C[f];
    const cd w2 = wc2[f];
    cd* row = rem + fdesc.off;
    int bad = 0;
    double mre = 0.0, mim = 0.0;
#pragma unroll 1
    for (int sw = 0; sw < SWEEPS; sw++) {
        const int i0 = (run * SWEEPS + sw) * (THREADS * ILP) + threadIdx.x + 1;
        if (i0 > n) break;
        if (FORM == 0) {
            bool ok;
            const double k = (double)i0 * d;
            cd u = direct_u(s_lc, nl, kTwoPi * fdesc.freq, k, mu_ref, ok);
            if (!ok) bad |= kStSingular;
            cd r = k * u - c;
            if (!finite_cd(r)) { bad |= kStNonfinite; r = mk(0.0); }
            row[i0 - 1] = r;
            mre = fmax(mre, fabs(r.re)); mim = fmax(mim, fabs(r.im));
        } else if (ILP == 1) {
            const double k = (double)i0 * d;
            const cd u = dunkin_u(s_lc, nl, w2, k, mu_ref);
            cd r = k * u - c;
            if (!finite_cd(r)) { bad |= kStNonfinite; r = mk(0.0); }
            row[i0 - 1] = r;
            mre = fmax(mre, fabs(r.re)); mim = fmax(mim, fabs(r.im));
        } else {
            const int i1 = i0 + THREADS;
            const bool has1 = i1 <= n;
            const double k0 = (double)i0 * d;
            const double k1 = has1 ? (double)i1 * d : k0;
            cd u0, u1;
            dunkin_u2(s_lc, nl, w2, k0, k1, mu_ref, u0, u1);
            cd r0 = k0 * u0 - c;
            if (!finite_cd(r0)) { bad |= kStNonfinite; r0 = mk(0.0); }
            row[i0 - 1] = r0;
            mre = fmax(mre, fabs(r0.re)); mim = fmax(mim, fabs(r0.im));
            if (has1) {
                cd r1 = k1 * u1 - c;
                if (!finite_cd(r1)) { bad |= kStNonfinite; r1 = mk(0.0); }
                row[i1 - 1] = r1;
                mre = fmax(mre, fabs(r1.re)); mim = fmax(mim, fabs(r1.im));
            }
        }
    }
    if (bad) atomicOr(status + f, bad);
    if constexpr (SLICE) {
        // The tensor-core sum's integer slicing, by the row's last block: the
        // row's maxima (the bits of a non-negative double order like the value),
        // then a device-scope fence and the row's count of finished blocks; the
        // block that finishes the row slices it while it is still in L2. No block
        // waits for another. (The pattern of a grid barrier's arrival: block
        // barrier, one thread's fence, the atomic count.)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mre = fmax(mre, __shfl_xor_sync(0xffffffffu, mre, o));
            mim = fmax(mim, __shfl_xor_sync(0xffffffffu, mim, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(so.rowmax + 2 * f, (unsigned long long)__double_as_longlong(mre));
            atomicMax(so.rowmax + 2 * f + 1, (unsigned long long)__double_as_longlong(mim));
        }
        // the barrier orders every thread's stores before thread 0's fence
        // (cumulative), which orders them before the count
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const bool last = atomicAdd(so.done + f, 1ull) == (unsigned long long)(runs - 1);
            if (last) __threadfence();
            sm.last = last;
        }
        __syncthreads();
        if (!sm.last) return;
        const unsigned long long b0 = __ldcg(so.rowmax + 2 * f), b1 = __ldcg(so.rowmax + 2 * f + 1);
        const int e[2] = {slice_exp(__longlong_as_double((long long)b0)), slice_exp(__longlong_as_double((long long)b1))};
        if (threadIdx.x == 0) {
            so.row_exp[2 * f] = e[0];
            so.row_exp[2 * f + 1] = e[1];
            so.done[f] = 0;  // every block of the row has counted: ready for the next launch
        }
        // a row with no device work (both maxima 0) slices to zeros without
        // reading its integrand slot
        slice_row<THREADS>(row, n, b0 != 0 || b1 != 0, e, so, f, sm.tile);
    }
}

template <int FORM, int THREADS, int MINB, int ILP, int SWEEPS, bool SLICE>
__global__ __launch_bounds__(THREADS, MINB) void k_prop(const LayerC* __restrict__ lc,
                                                       const MediumP* __restrict__ media,
                                                       const FreqDesc* __restrict__ fd, const cd* __restrict__ wc2,
                                                       const cd* __restrict__ C, cd* __restrict__ rem,
                                                       int* __restrict__ status, SliceOut so, PropQueue) {
    __shared__ PropSmem<THREADS, SLICE> sm;
    prop_item<FORM, THREADS, ILP, SWEEPS, SLICE>(lc, media, fd, wc2, C, rem, status, so, blockIdx.y, blockIdx.x,
                                                 gridDim.x, true, sm);
}

// Persistent: items (f, run) in row order from q.next (zero at launch), so a
// row's items run together and the row is sliced while it is in L2. Blocks
// never wait for one another; each leaves when the queue is empty.
template <int FORM, int THREADS, int MINB, int ILP, int SWEEPS, bool SLICE>
__global__ __launch_bounds__(THREADS, MINB) void k_prop_q(const LayerC* __restrict__ lc,
                                                         const MediumP* __restrict__ media,
                                                         const FreqDesc* __restrict__ fd, const cd* __restrict__ wc2,
                                                         const cd* __restrict__ C, cd* __restrict__ rem,
                                                         int* __restrict__ status, SliceOut so, PropQueue q) {
    __shared__ PropSmem<THREADS, SLICE> sm;
    int cur = -1;
    for (;;) {
        __syncthreads();  // every thread is done with the previous item's shared memory
        if (threadIdx.x == 0) sm.item = (int)atomicAdd(q.next, 1u);
        __syncthreads();
        const int item = sm.item;
        if (item >= q.items) return;
        const int f = item / q.runs, run = item - f * q.runs;
        prop_item<FORM, THREADS, ILP, SWEEPS, SLICE>(lc, media, fd, wc2, C, rem, status, so, f, run, q.runs, f != cur,
                                                     sm);
        cur = f;
    }
}

namespace {
using PropFn = void (*)(const LayerC*, const MediumP*, const FreqDesc*, const cd*, const cd*, cd*, int*, SliceOut,
                        PropQueue);
struct PropVariant {
    PropFn fn, fn_slice;  // without and with the fused slicing
    int threads, minb, ilp, sweeps;
    bool persistent;  // k_prop_q: one block per resident slot, items from a queue
};
#define GFK_PROP_SHAPE(T, B, I, S) {k_prop<1, T, B, I, S, false>, k_prop<1, T, B, I, S, true>, T, B, I, S, false}
#define GFK_PROP_QUEUE(T, B, I, S) {k_prop_q<1, T, B, I, S, false>, k_prop_q<1, T, B, I, S, true>, T, B, I, S, true}
const PropVariant kDunkinVariants[] = {
    GFK_PROP_SHAPE(128, 4, 1, 1),  // <= 128 registers, 16 warps/SM
    GFK_PROP_SHAPE(128, 5, 1, 1),  // <= 96 registers, 20 warps/SM
    GFK_PROP_SHAPE(128, 6, 1, 1),  // <= 80 registers, 24 warps/SM
    GFK_PROP_SHAPE(128, 2, 2, 1),  // two wavenumbers in lockstep, 8 warps/SM
    GFK_PROP_SHAPE(64, 4, 2, 1),
    GFK_PROP_SHAPE(256, 2, 1, 1),
    GFK_PROP_SHAPE(128, 5, 1, 4),  // four runs of 128 wavenumbers per block
    GFK_PROP_SHAPE(128, 5, 1, 8),
    GFK_PROP_SHAPE(128, 4, 1, 4),
    GFK_PROP_SHAPE(128, 4, 1, 8),
    GFK_PROP_QUEUE(128, 5, 1, 1),  // persistent, items of 128, 256 and 512 wavenumbers
    GFK_PROP_QUEUE(128, 5, 1, 2),
    GFK_PROP_QUEUE(128, 5, 1, 4),
};
constexpr int kPropVariants = sizeof(kDunkinVariants) / sizeof(kDunkinVariants[0]);
#undef GFK_PROP_SHAPE
#undef GFK_PROP_QUEUE

// Resident blocks of a persistent shape on the whole device (queried once per
// kernel; concurrent first calls compute the same value).
int persistent_grid(int variant, bool slice) {
    static std::atomic<int> cache[kPropVariants][2] = {};
    std::atomic<int>& slot = cache[variant][slice ? 1 : 0];
    int g = slot.load(std::memory_order_relaxed);
    if (g == 0) {
        const PropVariant& v = kDunkinVariants[variant];
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)(slice ? v.fn_slice : v.fn), v.threads,
                                                      0);
        g = std::max(1, sms * std::max(per_sm, 1));
        slot.store(g, std::memory_order_relaxed);
    }
    return g;
}
}  // namespace

int prop_variant_count() { return kPropVariants; }

bool prop_variant_persistent(int variant) {
    return variant >= 0 && variant < kPropVariants && kDunkinVariants[variant].persistent;
}

bool prop_variant_shape(int variant, int* threads, int* blocks_per_sm, int* ilp, int* sweeps, int* persistent) {
    if (variant < 0 || variant >= kPropVariants) return false;
    const PropVariant& v = kDunkinVariants[variant];
    *threads = v.threads;
    *blocks_per_sm = v.minb;
    *ilp = v.ilp;
    *sweeps = v.sweeps;
    *persistent = v.persistent ? 1 : 0;
    return true;
}

void launch_prop(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2, int nf,
                 int max_nk, const cd* C, int formulation, cd* rem, int* status, int variant, const SliceOut* slice,
                 unsigned int* queue) {
    if (nf <= 0 || max_nk <= 0) return;
    const SliceOut so = slice ? *slice : SliceOut{};
    if (formulation == 0) {
        dim3 grid((max_nk + 127) / 128, nf);
        if (slice)
            k_prop<0, 128, 1, 1, 1, true><<<grid, 128, 0, s>>>(lc, media, fd, wc2, C, rem, status, so, PropQueue{});
        else
            k_prop<0, 128, 1, 1, 1, false><<<grid, 128, 0, s>>>(lc, media, fd, wc2, C, rem, status, so, PropQueue{});
        return;
    }
    if (variant < 0 || variant >= kPropVariants) variant = 0;
    if (kDunkinVariants[variant].persistent && !queue) variant = 1;  // no queue: the same block shape, one item each
    const PropVariant& v = kDunkinVariants[variant];
    const int per_item = v.threads * v.ilp * v.sweeps;
    const int runs = (max_nk + per_item - 1) / per_item;
    const PropFn fn = slice ? v.fn_slice : v.fn;
    if (v.persistent) {
        const PropQueue q{queue, nf * runs, runs};
        fn<<<std::min(persistent_grid(variant, slice != nullptr), nf * runs), v.threads, 0, s>>>(lc, media, fd, wc2, C,
                                                                                              rem, status, so, q);
    } else {
        fn<<<dim3(runs, nf), v.threads, 0, s>>>(lc, media, fd, wc2, C, rem, status, so, PropQueue{});
    }
}

// ------------------------------------------------- fused propagator + sum --
//
// For a handful of ranges the wavenumber sum is a dot product per range: each
// thread accumulates its integrand values k u - C times the Hankel weights
// W[k][0..nr) over kFuseSweeps wavenumbers, the block reduces over its
// kFuseSweeps x 128 wavenumbers in a fixed order (warp tree, then warps), and
// one partial per (row, k block, range) is written. The
// integrand never reaches HBM; k_fused_finish adds the partials in block
// order (deterministic) and the closed k = 0 panel (fk.go:529-532).

constexpr int kFuseThreads = 128;
constexpr int kFuseSweeps = 8;  // a block covers kFuseSweeps x 128 wavenumbers of its row

template <int NR>
__global__ __launch_bounds__(kFuseThreads, 4) void k_prop_fused(const LayerC* __restrict__ lc,
                                                                const MediumP* __restrict__ media,
                                                                const FreqDesc* __restrict__ fd,
                                                                const cd* __restrict__ wc2, const cd* __restrict__ C,
                                                                const double* __restrict__ W, int nr, int nkb,
                                                                cd* __restrict__ partial, int* __restrict__ status) {
    __shared__ LayerC s_lc[kMaxLayers];
    __shared__ double s_red[2 * NR][kFuseThreads / 32];
    const int f = blockIdx.y;
    const FreqDesc fdesc = fd[f];
    const MediumP med = media[fdesc.soil];
    const int nl = med.count;
    for (int l = threadIdx.x; l < nl; l += blockDim.x) s_lc[l] = lc[fdesc.lc_off + l];
    __syncthreads();
    const int n = fdesc.kfar > 0 ? fdesc.nk : 0;
    const cd wc2f = wc2[f], cf = C[f];
    double acc[2 * NR];
#pragma unroll
    for (int q = 0; q < 2 * NR; q++) acc[q] = 0.0;
    // kFuseSweeps wavenumbers per thread, 128 apart, summed in order: one
    // layer-table load and one block reduction per 512 wavenumbers
#pragma unroll 1
    for (int sweep = 0; sweep < kFuseSweeps; sweep++) {
        const int i = (blockIdx.x * kFuseSweeps + sweep) * kFuseThreads + threadIdx.x + 1;
        if (i > n) break;
        const double k = (double)i * fdesc.dk;
        cd r = k * dunkin_u(s_lc, nl, wc2f, k, med.mu_ref) - cf;
        if (!finite_cd(r)) {
            atomicOr(status + f, kStNonfinite);
            r = mk(0.0);
        }
#pragma unroll
        for (int j = 0; j < NR; j++) {
            const double w = j < nr ? W[(size_t)(i - 1) * nr + j] : 0.0;
            acc[2 * j] = fma(r.re, w, acc[2 * j]);
            acc[2 * j + 1] = fma(r.im, w, acc[2 * j + 1]);
        }
    }
    // warp tree, then the block's warps in order: a fixed summation order
#pragma unroll
    for (int q = 0; q < 2 * NR; q++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_down_sync(0xffffffffu, acc[q], o);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < 2 * NR; q++) s_red[q][warp] = acc[q];
    __syncthreads();
    if (threadIdx.x < nr) {
        const int j = threadIdx.x;
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int w = 0; w < kFuseThreads / 32; w++) {
            re += s_red[2 * j][w];
            im += s_red[2 * j + 1][w];
        }
        partial[((size_t)f * nkb + blockIdx.x) * nr + j] = mk(re, im);
    }
}

__global__ void k_fused_finish(const cd* __restrict__ partial, const cd* __restrict__ C,
                               const double* __restrict__ ranges, const FreqDesc* __restrict__ fd, int nf, int nr,
                               int nkb, cd* __restrict__ G) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nf * nr) return;
    const int f = (int)(t / nr), j = (int)(t - (int64_t)f * nr);
    const cd c = C[f];
    const double d = fd[f].dk;
    cd acc = c / ranges[j] - (0.5 * d) * c;
    for (int b = 0; b < nkb; b++) acc += partial[((size_t)f * nkb + b) * nr + j];
    G[(size_t)f * nr + j] = acc;
}

int fused_max_ranges() { return 8; }

void launch_prop_fused(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2,
                       int nf, int nk, const cd* C, const double* W, const double* ranges, int nr, cd* partial,
                       int* status, cd* G) {
    if (nf <= 0 || nk <= 0 || nr <= 0 || nr > 8) return;
    const int nkb = (nk + kFuseThreads * kFuseSweeps - 1) / (kFuseThreads * kFuseSweeps);
    dim3 grid(nkb, nf);
    if (nr <= 1)
        k_prop_fused<1><<<grid, kFuseThreads, 0, s>>>(lc, media, fd, wc2, C, W, nr, nkb, partial, status);
    else if (nr <= 2)
        k_prop_fused<2><<<grid, kFuseThreads, 0, s>>>(lc, media, fd, wc2, C, W, nr, nkb, partial, status);
    else if (nr <= 4)
        k_prop_fused<4><<<grid, kFuseThreads, 0, s>>>(lc, media, fd, wc2, C, W, nr, nkb, partial, status);
    else
        k_prop_fused<8><<<grid, kFuseThreads, 0, s>>>(lc, media, fd, wc2, C, W, nr, nkb, partial, status);
    const int64_t nt = (int64_t)nf * nr;
    k_fused_finish<<<(unsigned)((nt + 255) / 256), 256, 0, s>>>(partial, C, ranges, fd, nf, nr, nkb, G);
}

// -------------------------------------------------------------- J0 table --

__global__ void k_j0_table(const double* __restrict__ ranges, int nr, int nk, double dk, double* __restrict__ W) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nk * nr) return;
    const int i = (int)(idx / nr) + 1;
    const int j = (int)(idx - (int64_t)(i - 1) * nr);
    const double k = (double)i * dk;
    const double w = i == nk ? 0.5 : 1.0;
    W[idx] = (w * j0(k * ranges[j])) * dk;
}

void launch_j0_table(cudaStream_t s, const double* ranges, int nr, int nk, double dk, double* W) {
    const int64_t n = (int64_t)nk * nr;
    k_j0_table<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ranges, nr, nk, dk, W);
}

// ----------------------------------------------------- FP64 quadrature --
//
// G[f][j] = C_f/r_j - (dk/2) C_f + sum_i rem[f][i] W[i][j]:
// a complex (nf x nk) by real (nk x nr) product, computed as the real GEMM of
// the 2 nf rows (re, im) of the integrand on the FP64 tensor cores:
// mma.sync m8n8k4 f64 (A 8x4 row-major, B 4x8 column-major, FP64 accumulate;
// lane t holds A[t/4][t%4], B[t%4][t/4] and C[t/4][2(t%4) + {0,1}]). Block
// tile 128 real rows (64 frequencies) x 16 TNW ranges x 16 wavenumbers, 8
// warps as 4 (rows) x 2 (ranges), a warp owning 32 x 8 TNW of the output
// (4 x TNW 8x8 accumulator tiles). The tiles move global -> shared with
// cp.async in a 3-stage ring; a stage holds the integrand as [k][2f + part]
// and the weights as [k][r], both with a row stride of 8 mod 16 doubles, so
// each fragment load (4 wavenumber rows x 8 consecutive doubles) takes the
// minimum two shared-memory wavefronts.

namespace qd {
constexpr int BM = 128, BK = 16, STAGES = 3, THREADS = 256;  // real rows, wavenumbers per stage
constexpr int ASTR = BM + 8;
template <int TNW>
__host__ __device__ constexpr int bstr() { return 16 * TNW + 8; }
template <int TNW>
constexpr int smem_bytes() { return STAGES * (BK * ASTR + BK * bstr<TNW>()) * (int)sizeof(double); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(src), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
}  // namespace qd

// Not volatile: the result is used, and the compiler may move the next
// step's fragment loads ahead of these MMAs.
__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

template <int TNW>
__global__ __launch_bounds__(qd::THREADS, TNW == 8 ? 1 : 2) void k_quad_gemm(const cd* __restrict__ rem,
                                                              const double* __restrict__ W,
                                                              const cd* __restrict__ C,
                                                              const double* __restrict__ ranges, int nf, int nk,
                                                              int nr, double dk, cd* __restrict__ G,
                                                              cd* __restrict__ part) {
    using namespace qd;
    constexpr int BN = 16 * TNW, BSTR = bstr<TNW>();
    extern __shared__ __align__(16) double d_smem[];
    double* const sA = d_smem;                       // [STAGES][BK][ASTR]
    double* const sB = d_smem + STAGES * BK * ASTR;  // [STAGES][BK][BSTR]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int f0 = blockIdx.y * (BM / 2);
    const int n0 = blockIdx.x * BN;
    const int ntiles = (nk + BK - 1) / BK;
    const int kt0 = (int)((long long)blockIdx.z * ntiles / gridDim.z);
    const int nt = (int)((long long)(blockIdx.z + 1) * ntiles / gridDim.z) - kt0;

    auto load = [&](int stage, int kt) {
        const int kb = kt * BK;
        double* a = sA + stage * BK * ASTR;
        double* b = sB + stage * BK * BSTR;
        const int fr = tid >> 2, kq = (tid & 3) * 4;
        const int gf = f0 + fr;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int k = kb + kq + q;
            const bool ok = gf < nf && k < nk;
            qd::cp_async16(a + (kq + q) * ASTR + 2 * fr,
                           ok ? (const void*)(rem + (size_t)gf * nk + k) : (const void*)rem, ok);
        }
        const int kr = tid >> 4, c0 = (tid & 15) * 2;
        const int k = kb + kr;
#pragma unroll
        for (int q = 0; q < BN / 32; q++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int col = c0 + 32 * q + e, gc = n0 + col;
                const bool ok = k < nk && gc < nr;
                qd::cp_async8(b + kr * BSTR + col, ok ? (const void*)(W + (size_t)k * nr + gc) : (const void*)W, ok);
            }
    };

    double acc[4][TNW][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < TNW; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < nt) load(s, kt0 + s);
        qd::cp_commit();
    }
    const int fa = (lane & 3) * ASTR + wm * 32 + (lane >> 2);       // this lane's A fragment element
    const int fb = (lane & 3) * BSTR + wn * 8 * TNW + (lane >> 2);  // and B fragment element
    for (int t = 0; t < nt; t++) {
        qd::cp_wait<STAGES - 2>();
        __syncthreads();
        if (t + STAGES - 1 < nt) load((t + STAGES - 1) % STAGES, kt0 + t + STAGES - 1);
        qd::cp_commit();
        const double* a = sA + (t % STAGES) * BK * ASTR + fa;
        const double* b = sB + (t % STAGES) * BK * BSTR + fb;
        // fragments of step k4 + 1 are loaded while step k4's MMAs issue
        double av[2][4], bv[2][TNW];
#pragma unroll
        for (int i = 0; i < 4; i++) av[0][i] = a[8 * i];
#pragma unroll
        for (int j = 0; j < TNW; j++) bv[0][j] = b[8 * j];
#pragma unroll
        for (int k4 = 0; k4 < BK / 4; k4++) {
            const int c = k4 & 1;
            if (k4 + 1 < BK / 4) {
#pragma unroll
                for (int i = 0; i < 4; i++) av[c ^ 1][i] = a[4 * (k4 + 1) * ASTR + 8 * i];
#pragma unroll
                for (int j = 0; j < TNW; j++) bv[c ^ 1][j] = b[4 * (k4 + 1) * BSTR + 8 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < TNW; j++) dmma(acc[i][j][0], acc[i][j][1], av[c][i], bv[c][j]);
        }
    }
    qd::cp_wait<0>();

    // lane holds real row wm*32 + 8i + lane/4 (frequency f0 + row/2, part row&1)
    // and ranges wn*8 TNW + 8j + 2(lane%4) + {0,1}
    double* const dst = reinterpret_cast<double*>(part ? part + (size_t)blockIdx.z * nf * nr : G);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int row = wm * 32 + 8 * i + (lane >> 2);
        const int f = f0 + (row >> 1), pr = row & 1;
        if (f >= nf) continue;
        const double cp = pr ? C[f].im : C[f].re;
#pragma unroll
        for (int j = 0; j < TNW; j++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int jj = n0 + wn * 8 * TNW + 8 * j + 2 * (lane & 3) + e;
                if (jj >= nr) continue;
                double v = acc[i][j][e];
                if (!part) v = (cp / ranges[jj] - (0.5 * dk) * cp) + v;  // fk.go:529-532
                dst[2 * ((size_t)f * nr + jj) + pr] = v;
            }
    }
}

int quad_gemm_splits(int nf, int nk, int nr) {
    // one block per SM of 148: the smallest split count (<= 64, each split
    // >= 8 wavenumber tiles) whose blocks fill the waves within 2% of the best
    // count's (more splits only add partial sums); banks of many waves keep one
    const int bn = nr > 64 ? 128 : 64;
    const long long tiles = (long long)((nr + bn - 1) / bn) * ((2 * nf + qd::BM - 1) / qd::BM);
    const int ntiles = (nk + qd::BK - 1) / qd::BK;
    if (tiles >= 8 * 148) return 1;
    const int smax = std::min(64, std::max(1, ntiles / 8));
    auto eff = [&](int s) {
        const long long blocks = tiles * s;
        return (double)blocks / ((double)((blocks + 147) / 148) * 148.0);
    };
    double best = 0.0;
    for (int s = 1; s <= smax; s++) best = std::max(best, eff(s));
    for (int s = 1; s <= smax; s++)
        if (eff(s) >= best - 0.02) return s;
    return 1;
}

namespace {
template <class K>
void set_smem_once(K kernel, int bytes, std::atomic<bool>* done) {
    if (!done->load(std::memory_order_relaxed) &&
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess)
        done->store(true, std::memory_order_relaxed);
}
}  // namespace

void launch_quad_gemm(cudaStream_t s, const cd* rem, const double* W, const cd* C, const double* ranges, int nf,
                      int nk, int nr, double dk, cd* G, int splits, cd* part) {
    if (nf <= 0 || nr <= 0) return;
    if (splits < 1 || !part) splits = 1;
    cd* const p = splits > 1 ? part : nullptr;
    // a failed attribute call leaves the launch to fail, and the caller's
    // cudaGetLastError to report it
    static std::atomic<bool> a8{false}, a4{false};
    if (nr > 64) {
        set_smem_once(k_quad_gemm<8>, qd::smem_bytes<8>(), &a8);
        dim3 grid((nr + 127) / 128, (2 * nf + qd::BM - 1) / qd::BM, splits);
        k_quad_gemm<8><<<grid, qd::THREADS, qd::smem_bytes<8>(), s>>>(rem, W, C, ranges, nf, nk, nr, dk, G, p);
    } else {
        set_smem_once(k_quad_gemm<4>, qd::smem_bytes<4>(), &a4);
        dim3 grid((nr + 63) / 64, (2 * nf + qd::BM - 1) / qd::BM, splits);
        k_quad_gemm<4><<<grid, qd::THREADS, qd::smem_bytes<4>(), s>>>(rem, W, C, ranges, nf, nk, nr, dk, G, p);
    }
    if (splits > 1) launch_quad_finish(s, part, splits, C, ranges, nf, nr, dk, G);
}

__global__ void k_quad_finish(const cd* __restrict__ part, int splits, const cd* __restrict__ C,
                              const double* __restrict__ ranges, int nf, int nr, double dk, cd* __restrict__ G) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nf * nr) return;
    const int f = (int)(i / nr), j = (int)(i % nr);
    cd acc = part[i];
    for (int z = 1; z < splits; z++) acc = acc + part[(size_t)z * nf * nr + i];
    const cd c = C[f];
    G[i] = (c / ranges[j] - (0.5 * dk) * c) + acc;  // fk.go:529-532
}

void launch_quad_finish(cudaStream_t s, const cd* part, int splits, const cd* C, const double* ranges, int nf,
                        int nr, double dk, cd* G) {
    const long long n = (long long)nf * nr;
    if (n <= 0) return;
    k_quad_finish<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, splits, C, ranges, nf, nr, dk, G);
}

// ---------------------------------------------- per-frequency-grid sum --
// The reference's own order: the boundary term, then i = 1..n in sequence
// (fk.go:529-548), one range per thread.

__global__ __launch_bounds__(128) void k_quad_ragged(const cd* __restrict__ rem, const cd* __restrict__ C,
                                                     const double* __restrict__ ranges, int nf, int nr,
                                                     const FreqDesc* __restrict__ fd, cd* __restrict__ G) {
    const int f = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nr) return;
    const FreqDesc fdesc = fd[f];
    const int n = fdesc.kfar > 0 ? fdesc.nk : 0;
    const double d = fdesc.dk;
    const double r = ranges[j];
    const cd c = C[f];
    cd acc = c / r - (0.5 * d) * c;
    const cd* row = rem + fdesc.off;
    for (int i = 1; i <= n; i++) {
        const double k = (double)i * d;
        const double w = i == n ? 0.5 : 1.0;
        const double wt = (w * j0(k * r)) * d;
        const cd v = row[i - 1];
        acc.re = fma(wt, v.re, acc.re);
        acc.im = fma(wt, v.im, acc.im);
    }
    G[(size_t)f * nr + j] = acc;
}

void launch_quad_ragged(cudaStream_t s, const cd* rem, const cd* C, const double* ranges, int nf, int nr,
                        const FreqDesc* fd, cd* G) {
    if (nf <= 0) return;
    dim3 grid((nr + 127) / 128, nf);
    k_quad_ragged<<<grid, 128, 0, s>>>(rem, C, ranges, nf, nr, fd, G);
}

// ------------------------------------------------------------ bank pack --

__global__ void k_bank_pack(const cd* __restrict__ G, int nf, int nr, int first_bin, int bins,
                            float* __restrict__ payload) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nf * nr) return;
    const int j = (int)(idx / nf);
    const int f = (int)(idx - (int64_t)j * nf);
    const int bin = first_bin + f;
    if (bin < 0 || bin >= bins) return;
    const cd v = G[(size_t)f * nr + j];
    const size_t o = 2 * ((size_t)j * bins + bin);
    payload[o] = (float)v.re;
    payload[o + 1] = (float)v.im;
}

void launch_bank_pack(cudaStream_t s, const cd* G, int nf, int nr, int first_bin, int bins, float* payload) {
    const int64_t n = (int64_t)nf * nr;
    k_bank_pack<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(G, nf, nr, first_bin, bins, payload);
}

}  // namespace gfk
