// gfk_mlp.cu — the surrogate network's kernels.
//
// The network maps (soil scalars, range, frequency) to the vertical Green's
// spectrum as t0 = log|G| and t1 = -phi/(w r), phi the unwrapped phase: an
// input layer 128 -> 512, four hidden layers 512 -> 512 (all SiLU) and an
// FP32 output layer 512 -> 2. Weights and activations are BF16, accumulation
// FP32 in TMEM, master weights and Adam moments FP32.
//
// Every 512-wide layer runs on one BF16 tcgen05 GEMM kernel with the layer's
// elementwise work fused into its epilogue:
//   forward   Z = X W^T + b, H = silu(Z)       (A = X [B][K], B = W [N][K])
//   backward  dZ' = (dZ W) silu'(Z')          (A = dZ [B][N], B = W^T [K][N])
//   weights   dW = dZ^T X, split over the batch (A = dZ^T, B = X^T)
// so every operand is K-major and is fed by plain TMA tiles: the epilogues
// write the transposed copies (X^T, dZ^T) the weight gradients read, and Adam
// writes W and W^T. The kernel shape is the wavenumber-sum kernel's: one
// 128 x 128 tile per CTA, warp 0 TMA, warp 1 TMEM + MMA issue, warps 2-5
// epilogue, SWIZZLE_64B tiles (32 BF16 = 64 bytes per row), 3-stage ring,
// bounded waits. No cluster multicast.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <math_constants.h>

#include <atomic>
#include <utility>

#include "gfk_kernels.cuh"
#include "gfk_mlp.cuh"
#include "gfk_tc.cuh"

namespace gfk {
namespace mlp {

using namespace gfk::tc;

constexpr int BM = 128, BN = 128;
constexpr int BKE = 32;                        // BF16 elements per 64-byte swizzled row (one TMA box)
constexpr int BOX = 2;                         // boxes per operand per stage
constexpr int BK = BKE * BOX;                  // 64 elements of K per stage
constexpr int TILE = BM * 64;                  // bytes per box: 128 rows x 64 bytes
constexpr int STAGE_BYTES = 2 * BOX * TILE;    // 32768
constexpr int STAGES = 3;
constexpr int THREADS = 192;
constexpr int TMEM_COLS = BN;                  // 128 FP32 accumulator columns
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256 + BN * 4;
constexpr int kTileLd = BN + 8;  // BF16 row pitch of the epilogue's staging tiles (272 bytes)
static_assert(2 * BM * kTileLd * 2 <= STAGES * STAGE_BYTES, "staging tiles alias the pipeline stages");

// Instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = 128.
__host__ __device__ inline uint32_t idesc_bf16_128x128() {
    cute::UMMA::InstrDescriptor id;
    id.desc_ = 0;
    id.c_format_ = 1;  // F32
    id.a_format_ = 1;  // BF16
    id.b_format_ = 1;
    id.a_major_ = 0;   // K-major
    id.b_major_ = 0;
    id.n_dim_ = BN >> 3;
    id.m_dim_ = BM >> 4;
    return id.desc_;
}

// Programmatic dependent launch. The network's kernels are launched so that
// the next one may be scheduled while the previous one finishes: each calls
// dep_wait() before its first global-memory access (it returns once the
// previous kernel in the stream has completed and its writes are visible; a
// no-op for an ordinary launch) and dep_release() to let its successor start
// its own set-up early.
__device__ __forceinline__ void dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void dep_release() { asm volatile("griddepcontrol.launch_dependents;" :::); }

template <typename... P, typename... A>
void launch_dep(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// Hardware exponential and approximate reciprocal (no IEEE division): the
// results are rounded to BF16 (8-bit mantissa) right after.
__device__ __forceinline__ float sigmoid_(float z) { return __fdividef(1.0f, 1.0f + __expf(-z)); }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void unpack8(const uint4& u, float* f) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __bfloat1622float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
}

template <int MODE>
__global__ void __launch_bounds__(THREADS, 2)
    k_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* accf = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
    float* bias_s = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES + 256);  // [BN]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kbase = blockIdx.z * a.K;
    const int nkb = a.K / BK;

    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(accf, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    dep_wait();  // the set-up above overlaps the previous kernel's tail
    dep_release();

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < nkb; kb++) {
                const int st = kb % STAGES;
                const uint32_t ph = (kb / STAGES) & 1;
                if (!mbar_wait(&empty[st], ph ^ 1)) {
                    *abort_flag = 1;
                    break;
                }
                if (*(volatile int*)abort_flag) break;
                mbar_expect_tx(&full[st], STAGE_BYTES);
                uint8_t* base = smem + st * STAGE_BYTES;
                const int kx = kbase + kb * BK;
#pragma unroll
                for (int b = 0; b < BOX; b++) tma_load_2d(base + b * TILE, &tmA, &full[st], kx + b * BKE, m0);
#pragma unroll
                for (int b = 0; b < BOX; b++)
                    tma_load_2d(base + (BOX + b) * TILE, &tmB, &full[st], kx + b * BKE, n0);
                issued = kb + 1;
            }
            for (int kb = issued - 1; kb >= 0 && kb >= issued - STAGES; kb--)
                if (!mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1)) *abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_128x128();
            uint32_t acc = 0;
            for (int kb = 0; kb < nkb; kb++) {
                const int st = kb % STAGES;
                if (!mbar_wait(&full[st], (kb / STAGES) & 1)) {
                    *abort_flag = 1;
                    break;
                }
                if (*(volatile int*)abort_flag) break;
                tc_fence_after();
                const uint32_t base = smem_u32(smem + st * STAGE_BYTES);
#pragma unroll
                for (int b = 0; b < BOX; b++) {
#pragma unroll
                    for (int kk = 0; kk < BKE / 16; kk++) {  // K = 16 per instruction = 32 bytes
                        const uint64_t da = sdesc_k_sw64(base + b * TILE + kk * 32);
                        const uint64_t db = sdesc_k_sw64(base + (BOX + b) * TILE + kk * 32);
                        tc_mma_f16(tmem, da, db, idesc, acc);
                        acc = 1;
                    }
                }
                tc_commit(&empty[st]);
            }
            tc_commit(accf);
        }
    } else {
        // epilogue, phase 1 (warps 2-5): TMEM -> registers -> elementwise work;
        // BF16 results go to a shared-memory tile (the pipeline stages are free
        // once every MMA has completed), FP32 gradient partials straight out
        // the tile's bias columns, read once while the MMAs run
        if (MODE == kFwdTrain || MODE == kFwdInfer) {
            bias_s[threadIdx.x - 64] = a.bias[n0 + threadIdx.x - 64];
            asm volatile("bar.sync 1, 128;" ::: "memory");
        }
        const int q = warp & 3;
        const int rl = q * 32 + lane;
        const int row = m0 + rl;
        // backward-data: this row's pre-activations, one 32-column chunk ahead
        // (the first chunk is in flight while the MMAs run)
        uint4 zcur[4], znext[4];
        if (MODE == kBwdData) {
            const uint4* zs = reinterpret_cast<const uint4*>(a.zin + (size_t)row * a.N + n0);
#pragma unroll
            for (int c = 0; c < 4; c++) zcur[c] = zs[c];
        }
        const bool ok = mbar_wait(accf, 0);
        if (!ok) *(volatile int*)abort_flag = 1;  // the tile stays unwritten: no stores below
        tc_fence_after();
        const bool row_ok = ok && !*(volatile int*)abort_flag;
        bf16* tileO = reinterpret_cast<bf16*>(smem);
        bf16* tileZ = tileO + BM * kTileLd;
#pragma unroll 1
        for (int j = 0; j < BN / 32; j++) {
            uint32_t v[32];
            tmem_ld32(tmem + (static_cast<uint32_t>(q * 32) << 16) + j * 32, v);
            if (MODE == kBwdData && j + 1 < BN / 32) {
                const uint4* zs = reinterpret_cast<const uint4*>(a.zin + (size_t)row * a.N + n0 + (j + 1) * 32);
#pragma unroll
                for (int c = 0; c < 4; c++) znext[c] = zs[c];
            }
            tmem_wait_ld();
            if (!row_ok) continue;
            const int nb = n0 + j * 32;
            if (MODE == kWgrad) {
                float4* dst = reinterpret_cast<float4*>(a.part + ((size_t)blockIdx.z * a.M + row) * a.N + nb);
#pragma unroll
                for (int c = 0; c < 8; c++)
                    dst[c] = make_float4(__uint_as_float(v[4 * c]), __uint_as_float(v[4 * c + 1]),
                                         __uint_as_float(v[4 * c + 2]), __uint_as_float(v[4 * c + 3]));
                continue;
            }
            float y[32];
            if (MODE == kFwdTrain || MODE == kFwdInfer) {
                float zv[32];
#pragma unroll
                for (int c = 0; c < 32; c++) {
                    zv[c] = __uint_as_float(v[c]) + bias_s[j * 32 + c];
                    y[c] = zv[c] * sigmoid_(zv[c]);
                }
                if (MODE == kFwdTrain) {
                    uint4* zd = reinterpret_cast<uint4*>(tileZ + rl * kTileLd + j * 32);
#pragma unroll
                    for (int c = 0; c < 4; c++)
                        zd[c] = make_uint4(pack2(zv[8 * c], zv[8 * c + 1]), pack2(zv[8 * c + 2], zv[8 * c + 3]),
                                           pack2(zv[8 * c + 4], zv[8 * c + 5]), pack2(zv[8 * c + 6], zv[8 * c + 7]));
                }
            } else {  // kBwdData
                float zv[32];
#pragma unroll
                for (int c = 0; c < 4; c++) unpack8(zcur[c], zv + 8 * c);
#pragma unroll
                for (int c = 0; c < 32; c++) {
                    const float sg = sigmoid_(zv[c]);
                    y[c] = __uint_as_float(v[c]) * (sg * (1.0f + zv[c] * (1.0f - sg)));
                }
#pragma unroll
                for (int c = 0; c < 4; c++) zcur[c] = znext[c];
            }
            uint4* od = reinterpret_cast<uint4*>(tileO + rl * kTileLd + j * 32);
#pragma unroll
            for (int c = 0; c < 4; c++)
                od[c] = make_uint4(pack2(y[8 * c], y[8 * c + 1]), pack2(y[8 * c + 2], y[8 * c + 3]),
                                   pack2(y[8 * c + 4], y[8 * c + 5]), pack2(y[8 * c + 6], y[8 * c + 7]));
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // phase 2 (all warps): coalesced stores of the tile, its transpose and Z
    if (MODE != kWgrad && !*(volatile int*)abort_flag) {
        const bf16* tileO = reinterpret_cast<const bf16*>(smem);
        const bf16* tileZ = tileO + BM * kTileLd;
        for (int c = threadIdx.x; c < BM * (BN / 8); c += THREADS) {
            const int r = c / (BN / 8), c8 = (c % (BN / 8)) * 8;
            const size_t g = (size_t)(m0 + r) * a.N + n0 + c8;
            *reinterpret_cast<uint4*>(a.out + g) = *reinterpret_cast<const uint4*>(tileO + r * kTileLd + c8);
            if (MODE == kFwdTrain)
                *reinterpret_cast<uint4*>(a.zout + g) = *reinterpret_cast<const uint4*>(tileZ + r * kTileLd + c8);
        }
        if (MODE != kFwdInfer && a.outT) {
            // 32 bytes (16 rows) of one transposed row per thread; lanes run
            // over columns, so the shared-memory column reads do not conflict
            for (int c = threadIdx.x; c < BN * (BM / 16); c += THREADS) {
                const int n = c % BN, r16 = (c / BN) * 16;
                uint32_t w[8];
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    __nv_bfloat162 v2;
                    v2.x = tileO[(r16 + 2 * e) * kTileLd + n];
                    v2.y = tileO[(r16 + 2 * e + 1) * kTileLd + n];
                    w[e] = *reinterpret_cast<uint32_t*>(&v2);
                }
                uint4* d = reinterpret_cast<uint4*>(a.outT + (size_t)(n0 + n) * a.M + m0 + r16);
                d[0] = make_uint4(w[0], w[1], w[2], w[3]);
                d[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
        }
    }
    if (threadIdx.x == 0 && *(volatile int*)abort_flag && a.status) atomicOr(a.status, kStTimeout);
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ----------------------------------------------------------------- batch --

// splitmix64 finaliser (Steele, Lea, Flood 2014) as a counter-based generator.
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

__device__ __forceinline__ int pick(unsigned long long h32, int n) {
    return static_cast<int>(((h32 & 0xffffffffULL) * static_cast<unsigned long long>(n)) >> 32);
}

struct PointScalars {
    float ur, uf, lr, lf, f;
};

__device__ __forceinline__ PointScalars point_scalars(double r, double f, const FeatureDomain& d) {
    PointScalars p;
    p.ur = static_cast<float>((r - d.r_lo) / (d.r_hi - d.r_lo));
    p.uf = static_cast<float>((f - d.f_lo) / (d.f_hi - d.f_lo));
    p.lr = static_cast<float>(2.0 * log(r / d.r_lo) / log(d.r_hi / d.r_lo) - 1.0);
    p.lf = static_cast<float>(2.0 * log(f / d.f_lo) / log(d.f_hi / d.f_lo) - 1.0);
    p.f = static_cast<float>(f);
    return p;
}

// sf: one soil table row (scalars at [0, 11), travel times at [16, 22)).
__device__ __forceinline__ float feature(int j, const float* sf, const PointScalars& p, const float* four) {
    if (j < kMaxSoil) return sf[j];
    if (j < kScalars) {
        switch (j) {
            case 11: return 2.0f * p.ur - 1.0f;
            case 12: return 2.0f * p.uf - 1.0f;
            case 13: return p.lr;
            case 14: return p.lf;
            default: return 0.0f;
        }
    }
    if (j < kLogTimeFeat) {
        const int q = (j - kTimeFeat) >> 1;
        float sn, cs;
        sincospif(2.0f * (p.f * sf[kScalars + q]), &sn, &cs);
        return (j & 1) ? cs : sn;
    }
    if (j < kFourierFeat) {
        const float x = p.f * sf[kScalars + (j - kLogTimeFeat)];
        return x > 0.0f ? fminf(fmaxf((logf(x) + 2.0f) / 3.0f, -2.0f), 2.0f) : -2.0f;
    }
    const int q = (j - kFourierFeat) >> 1;
    float sn, cs;
    sincospif(2.0f * (four[2 * q] * p.ur + four[2 * q + 1] * p.uf), &sn, &cs);
    return (j & 1) ? cs : sn;
}

__global__ void k_step_begin(TrainScalars* ts) {
    dep_wait();
    dep_release();
    const long long t = ++ts->step;
    float lr;
    if (t <= ts->warmup) {
        lr = ts->lr_max * static_cast<float>(t) / static_cast<float>(ts->warmup > 0 ? ts->warmup : 1);
    } else {
        const double span = ts->total > ts->warmup ? static_cast<double>(ts->total - ts->warmup) : 1.0;
        const double p = fmin(1.0, static_cast<double>(t - ts->warmup) / span);
        lr = static_cast<float>(ts->lr_min + 0.5 * (ts->lr_max - ts->lr_min) * (1.0 + cospi(p)));
    }
    ts->lr = lr;
    ts->bc1 = static_cast<float>(1.0 - pow(static_cast<double>(ts->beta1), static_cast<double>(t)));
    ts->bc2 = static_cast<float>(1.0 - pow(static_cast<double>(ts->beta2), static_cast<double>(t)));
}

// kBatchRows samples per block: one thread per sample draws the cell and builds
// its scalars and targets, then one thread per feature fills the rows. Small
// blocks keep many of them resident, so the dependent gathers (soil, cell,
// label) of different blocks overlap.
constexpr int kBatchRows = 16;
__global__ void __launch_bounds__(kIn) k_batch(BatchArgs a) {
    dep_wait();
    dep_release();
    __shared__ bf16 tile[kBatchRows][kIn + 2];
    __shared__ PointScalars ps[kBatchRows];
    __shared__ int soil_of[kBatchRows];
    const long long t = a.ts->step;
    const int b0 = blockIdx.x * kBatchRows;
    const int j = threadIdx.x;
    if (j < kBatchRows) {
        const int b = b0 + j;
        const unsigned long long h = mix64(a.seed ^ mix64(static_cast<unsigned long long>(t) * a.B + b));
        const int soil = a.train[pick(h, a.ntrain)];
        const unsigned long long h2 = mix64(h);
        const int ir = a.ir0 + pick(h2, a.nir), jf = pick(h2 >> 32, a.nf);
        ps[j] = point_scalars(a.ranges[ir], a.freqs[jf], a.dom);
        soil_of[j] = soil;
        const float* L = a.labels + (((size_t)soil * a.nr + ir) * a.nf + jf) * 2;
        const bool ph = !isnan(L[1]);
        a.Y[2 * b] = (L[0] - a.y_mean0) / a.y_std0;
        a.Y[2 * b + 1] = (L[1] - a.y_mean1) / a.y_std1;  // NaN stays NaN
        float c0 = 1.0f, c1 = ph ? a.phase_weight : 0.0f;
        if (a.loss_mode == 2) {
            const float w = fmaxf(__expf(L[0] - a.lmax[(size_t)soil * a.nr + ir]), a.weight_floor);
            c0 = w;
            c1 = ph ? a.phase_weight * w : 0.0f;
        } else if (a.loss_mode == 1) {
            const float w = fmaxf(__expf(2.0f * (L[0] - a.lmax[(size_t)soil * a.nr + ir])), a.weight_floor);
            const float wr = static_cast<float>(2.0 * 3.14159265358979323846 * a.freqs[jf] * a.ranges[ir]) *
                             (a.y_std1 / a.y_std0);
            c0 = w;
            c1 = ph ? a.phase_weight * w * fminf(wr * wr, a.phase_cap) : 0.0f;
        }
        a.C[2 * b] = c0;
        a.C[2 * b + 1] = c1;
    }
    __syncthreads();
    for (int i = 0; i < kBatchRows; i++)
        tile[i][j] = __float2bfloat16_rn(feature(j, a.soilfeat + (size_t)soil_of[i] * kSoilStride, ps[i], a.fourier));
    __syncthreads();
    for (int i = 0; i < kBatchRows; i++) a.X[(size_t)(b0 + i) * kIn + j] = tile[i][j];
    // X^T: thread j writes its feature's kBatchRows consecutive samples
    uint32_t w[kBatchRows / 2];
#pragma unroll
    for (int i = 0; i < kBatchRows / 2; i++) {
        __nv_bfloat162 v;
        v.x = tile[2 * i][j];
        v.y = tile[2 * i + 1][j];
        w[i] = *reinterpret_cast<uint32_t*>(&v);
    }
    uint4* d = reinterpret_cast<uint4*>(a.XT + (size_t)j * a.B + b0);
#pragma unroll
    for (int i = 0; i < kBatchRows / 8; i++) d[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}

// ------------------------------------------------------------------ head --

// 8 warps x 4 rows; lane owns columns u*256 + lane*8 + e (u = 0, 1; e < 8).
__global__ void __launch_bounds__(256) k_head_train(const bf16* __restrict__ H, const bf16* __restrict__ Z,
                                                    const float* __restrict__ W6, const float* __restrict__ b6,
                                                    const float* __restrict__ Y, const float* __restrict__ Cw, int B,
                                                    bf16* __restrict__ dZ, bf16* __restrict__ dZT,
                                                    float* __restrict__ gpart, float* __restrict__ lpart) {
    dep_wait();
    dep_release();
    __shared__ __align__(16) bf16 tile[kHeadRows][kWidth + 8];
    __shared__ float red[2 * kWidth + 2];
    __shared__ float lred[8][4];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = blockIdx.x * kHeadRows;
    float w0[16], w1[16], g0[16], g1[16];
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int c = u * 256 + lane * 8 + e;
            w0[u * 8 + e] = W6[c];
            w1[u * 8 + e] = W6[kWidth + c];
            g0[u * 8 + e] = 0.0f;
            g1[u * 8 + e] = 0.0f;
        }
    float l0 = 0.0f, l1 = 0.0f, sc0 = 0.0f, sc1 = 0.0f, ds0 = 0.0f, ds1 = 0.0f;
    for (int t = 0; t < 4; t++) {
        const int rl = warp * 4 + t, row = r0 + rl;
        float h[16], z[16];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            unpack8(*reinterpret_cast<const uint4*>(H + (size_t)row * kWidth + u * 256 + lane * 8), h + 8 * u);
            unpack8(*reinterpret_cast<const uint4*>(Z + (size_t)row * kWidth + u * 256 + lane * 8), z + 8 * u);
        }
        float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            y0 = fmaf(h[i], w0[i], y0);
            y1 = fmaf(h[i], w1[i], y1);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            y0 += __shfl_xor_sync(0xffffffffu, y0, o);
            y1 += __shfl_xor_sync(0xffffffffu, y1, o);
        }
        y0 += b6[0];
        y1 += b6[1];
        const float t0 = Y[2 * row], t1 = Y[2 * row + 1];
        const float c0 = Cw[2 * row], c1 = Cw[2 * row + 1];
        const bool ph = !isnan(t1) && c1 > 0.0f;
        const float e0 = y0 - t0, e1 = ph ? y1 - t1 : 0.0f;
        const float d0 = 2.0f * c0 * e0 / B, d1 = ph ? 2.0f * c1 * e1 / B : 0.0f;
        l0 += c0 * e0 * e0;
        l1 += ph ? c1 * e1 * e1 : 0.0f;
        sc0 += c0;
        sc1 += ph ? c1 : 0.0f;
        ds0 += d0;
        ds1 += d1;
        float dz[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            g0[i] = fmaf(d0, h[i], g0[i]);
            g1[i] = fmaf(d1, h[i], g1[i]);
            const float dh = d0 * w0[i] + d1 * w1[i];
            const float sg = sigmoid_(z[i]);
            dz[i] = dh * (sg * (1.0f + z[i] * (1.0f - sg)));
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint4 pk = make_uint4(pack2(dz[8 * u], dz[8 * u + 1]), pack2(dz[8 * u + 2], dz[8 * u + 3]),
                                        pack2(dz[8 * u + 4], dz[8 * u + 5]), pack2(dz[8 * u + 6], dz[8 * u + 7]));
            *reinterpret_cast<uint4*>(dZ + (size_t)row * kWidth + u * 256 + lane * 8) = pk;
            *reinterpret_cast<uint4*>(&tile[rl][u * 256 + lane * 8]) = pk;
        }
    }
    // deterministic cross-warp sum of the dW6 / db6 contributions
    for (int w = 0; w < 8; w++) {
        if (warp == w) {
#pragma unroll
            for (int u = 0; u < 2; u++)
#pragma unroll
                for (int e = 0; e < 8; e++) {
                    const int c = u * 256 + lane * 8 + e;
                    red[c] = (w ? red[c] : 0.0f) + g0[u * 8 + e];
                    red[kWidth + c] = (w ? red[kWidth + c] : 0.0f) + g1[u * 8 + e];
                }
            if (lane == 0) {
                red[2 * kWidth] = (w ? red[2 * kWidth] : 0.0f) + ds0;
                red[2 * kWidth + 1] = (w ? red[2 * kWidth + 1] : 0.0f) + ds1;
                lred[w][0] = l0;
                lred[w][1] = l1;
                lred[w][2] = sc0;
                lred[w][3] = sc1;
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < kHeadStride; i += blockDim.x)
        gpart[(size_t)blockIdx.x * kHeadStride + i] = i < 2 * kWidth + 2 ? red[i] : 0.0f;
    if (threadIdx.x == 0) {
        float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int w = 0; w < 8; w++)
            for (int q = 0; q < 4; q++) s[q] += lred[w][q];
        for (int q = 0; q < 4; q++) lpart[blockIdx.x * 4 + q] = s[q];
    }
    // dZ^T: 32 consecutive rows of column c, 64 bytes per store group
    for (int c = threadIdx.x; c < kWidth; c += blockDim.x) {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            __nv_bfloat162 v;
            v.x = tile[2 * i][c];
            v.y = tile[2 * i + 1][c];
            w[i] = *reinterpret_cast<uint32_t*>(&v);
        }
        uint4* d = reinterpret_cast<uint4*>(dZT + (size_t)c * B + r0);
#pragma unroll
        for (int i = 0; i < 4; i++) d[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
    }
}

struct BiasPtrs {
    const bf16* p[8];
};

// One block per (output unit, layer): tree sum of that dz^T row.
__global__ void __launch_bounds__(256) k_bias_grad(BiasPtrs d, int B, float* gb) {
    dep_wait();
    dep_release();
    __shared__ float sm[256];
    const int o = blockIdx.x, l = blockIdx.y;
    const bf16* row = d.p[l] + (size_t)o * B;
    float s = 0.0f;
    for (int b = threadIdx.x * 8; b < B; b += blockDim.x * 8) {
        float v[8];
        unpack8(*reinterpret_cast<const uint4*>(row + b), v);
#pragma unroll
        for (int i = 0; i < 8; i++) s += v[i];
    }
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) gb[l * kWidth + o] = sm[0];
}

// ------------------------------------------------------------------ adam --

// Grids are (blocks over the largest segment, segments): a block works inside
// one segment, whose descriptor it reads from device memory.
// The partials are loaded 32 or 8 at a time before they are added (in the same
// order as one at a time), so a thread has that many loads in flight instead of
// one dependent load per partial (the head's segment sums 256 partials).
__device__ __forceinline__ float seg_grad(const AdamSeg& g, long long j) {
    const float* __restrict__ src = g.src + j;
    float grad = 0.0f;
    int q = 0;
    for (; q + 32 <= g.nsrc; q += 32) {
        float t[32];
#pragma unroll
        for (int u = 0; u < 32; u++) t[u] = __ldg(src + (long long)(q + u) * g.stride);
#pragma unroll
        for (int u = 0; u < 32; u++) grad += t[u];
    }
    for (; q + 8 <= g.nsrc; q += 8) {
        float t[8];
#pragma unroll
        for (int u = 0; u < 8; u++) t[u] = __ldg(src + (long long)(q + u) * g.stride);
#pragma unroll
        for (int u = 0; u < 8; u++) grad += t[u];
    }
    for (; q < g.nsrc; q++) grad += __ldg(src + (long long)q * g.stride);
    return grad;
}

// AdamW (Loshchilov & Hutter 2019) on the FP32 master copy, gradients summed
// from their partials in a fixed order; refreshes the BF16 copy W.
__global__ void k_adam(AdamArgs a) {
    dep_wait();
    dep_release();
    const AdamSeg g = a.dseg[blockIdx.y];
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (j >= g.n) return;
    const long long i = g.off + j;
    const float m0 = a.m[i], v0 = a.v[i];
    float p = a.p[i];
    const float grad = seg_grad(g, j);
    const TrainScalars* ts = a.ts;
    const float b1 = ts->beta1, b2 = ts->beta2;
    const float m = b1 * m0 + (1.0f - b1) * grad;
    const float v = b2 * v0 + (1.0f - b2) * grad * grad;
    a.m[i] = m;
    a.v[i] = v;
    p -= ts->lr * ((m / ts->bc1) / (sqrtf(v / ts->bc2) + a.eps) + a.weight_decay * p);
    a.p[i] = p;
    if (g.wb) g.wb[j] = __float2bfloat16_rn(p);
}

// W^T from W for every weight segment, 32 x 32 tiles through shared memory.
__global__ void k_transpose_w(AdamArgs a) {
    dep_wait();
    dep_release();
    __shared__ bf16 t[32][33];
    const AdamSeg g = a.dseg[blockIdx.z];
    if (!g.wb) return;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    if (c0 >= g.cols || r0 >= g.rows) return;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) t[y][threadIdx.x] = g.wb[(size_t)(r0 + y) * g.cols + c0 + threadIdx.x];
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) g.wt[(size_t)(c0 + y) * g.rows + r0 + threadIdx.x] = t[threadIdx.x][y];
}

__global__ void k_sync_weights(AdamArgs a) {
    const AdamSeg g = a.dseg[blockIdx.y];
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (j >= g.n || !g.wb) return;
    g.wb[j] = __float2bfloat16_rn(a.p[g.off + j]);
}

__global__ void k_grad_flat(AdamArgs a, float* out) {
    const AdamSeg g = a.dseg[blockIdx.y];
    const long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
    if (j >= g.n) return;
    out[g.off + j] = seg_grad(g, j);
}

// One warp: fixed-order sums of the head kernel's loss partials; each slot
// holds the step's two coefficient-weighted mean squared errors.
__global__ void k_loss_hist(const float* lpart, int nblk, int B, const TrainScalars* ts, float* hist, int cap) {
    dep_wait();
    dep_release();
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int b = threadIdx.x; b < nblk; b += 32)
        for (int q = 0; q < 4; q++) s[q] += lpart[4 * b + q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        for (int q = 0; q < 4; q++) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
    if (threadIdx.x == 0) {
        const long long slot = (ts->step - 1) % cap;
        hist[2 * slot] = s[2] > 0.0f ? s[0] / s[2] : 0.0f;
        hist[2 * slot + 1] = s[3] > 0.0f ? s[1] / s[3] : 0.0f;
    }
}

// ------------------------------------------------------------- inference --

__global__ void __launch_bounds__(kIn) k_features(FeatureArgs a, long long rows_padded) {
    dep_wait();
    dep_release();
    const long long q0 = blockIdx.x * 32LL;
    const int j = threadIdx.x;
    for (int i = 0; i < 32; i++) {
        const long long q = q0 + i;
        if (q >= rows_padded) return;
        float v = 0.0f;
        if (q < a.rows) {
            const long long p = a.p0 + q;
            const int ir = static_cast<int>(p % a.nr);
            const long long t = p / a.nr;
            const int jf = static_cast<int>(t % a.nf);
            const long long s = t / a.nf;
            const PointScalars ps = point_scalars(a.ranges[ir], a.freqs[jf], a.dom);
            v = feature(j, a.soilfeat + s * kSoilStride, ps, a.fourier);
        }
        a.X[q * kIn + j] = __float2bfloat16_rn(v);
    }
}

__global__ void __launch_bounds__(256) k_head_infer(HeadInferArgs a) {
    dep_wait();
    dep_release();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long q = blockIdx.x * 8LL + warp;
    if (q >= a.rows) return;
    float h[16];
#pragma unroll
    for (int u = 0; u < 2; u++)
        unpack8(*reinterpret_cast<const uint4*>(a.H + q * kWidth + u * 256 + lane * 8), h + 8 * u);
    float y0 = 0.0f, y1 = 0.0f;
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int c = u * 256 + lane * 8 + e;
            y0 = fmaf(h[8 * u + e], a.W6[c], y0);
            y1 = fmaf(h[8 * u + e], a.W6[kWidth + c], y1);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        y0 += __shfl_xor_sync(0xffffffffu, y0, o);
        y1 += __shfl_xor_sync(0xffffffffu, y1, o);
    }
    if (lane) return;
    const double t0 = static_cast<double>(y0 + a.b6[0]) * a.y_std0 + a.y_mean0;
    const double t1 = static_cast<double>(y1 + a.b6[1]) * a.y_std1 + a.y_mean1;
    const long long p = a.p0 + q;
    const int ir = static_cast<int>(p % a.nr);
    const int jf = static_cast<int>((p / a.nr) % a.nf);
    const double phi = -t1 * (2.0 * CUDART_PI * a.freqs[jf]) * a.ranges[ir];
    double sn, cs;
    sincos(phi, &sn, &cs);
    const double amp = exp(t0);
    a.G[p] = mk(amp * cs, amp * sn);
    if (a.T) {
        a.T[2 * q] = static_cast<float>(t0);
        a.T[2 * q + 1] = static_cast<float>(t1);
    }
}

// ---------------------------------------------------------------- labels --

constexpr int kLabelThreads = 128;
constexpr int16_t kBroken = INT16_MIN;

__device__ __forceinline__ double amp_of(cd g) { return hypot(g.re, g.im); }

// One block per soil. Phase unwrapping follows bank.prepare
// (internal/bank/interp.go:66-102): along range, each step folded into
// (-pi, pi]. A 1 m range step spans many cycles at high frequency for slow
// soils, so the fold is taken about a prediction instead of about zero: the
// same range step one frequency bin lower, scaled by f_j / f_{j-1} (the
// step is -k(f) dr and k grows about linearly in f). The first range is
// unwrapped along frequency the same way. Whole-cycle counts are kept as
// integers, so phi = principal value + 2 pi n exactly. A chain stops (the
// phase label becomes NaN) at the first cell below the amplitude floor.
__global__ void __launch_bounds__(kLabelThreads) k_labels(LabelArgs a) {
    extern __shared__ int16_t cyc[];  // [nr][nf]
    __shared__ double red[kLabelThreads];
    const int s = blockIdx.x, tid = threadIdx.x;
    const cd* G = a.G + (size_t)s * a.nf * a.nr;
    const int cells = a.nf * a.nr;
    double mx = 0.0;
    for (int c = tid; c < cells; c += blockDim.x) mx = fmax(mx, amp_of(G[c]));
    red[tid] = mx;
    __syncthreads();
    for (int w = kLabelThreads / 2; w > 0; w >>= 1) {
        if (tid < w) red[tid] = fmax(red[tid], red[tid + w]);
        __syncthreads();
    }
    const double floor_amp = red[0] * a.floor_rel;
    __syncthreads();
    const double two_pi = 2.0 * CUDART_PI;
    if (tid < a.nr) {
        const int i = tid;
        double dprev = 0.0, wprev = 0.0, rmax = 0.0;
        int n = 0;
        bool ok = true;
        for (int j = 0; j < a.nf; j++) {
            const cd g = G[(size_t)j * a.nr + i];
            rmax = fmax(rmax, amp_of(g));
            const double w = atan2(g.im, g.re);
            if (i == 0) {
                if (j > 0) {
                    const double dw = w - wprev;
                    const double m = rint((dprev - dw) / two_pi);
                    dprev = dw + two_pi * m;
                    n += static_cast<int>(m);
                }
                ok = ok && amp_of(g) > floor_amp;
                cyc[j] = ok ? static_cast<int16_t>(n) : kBroken;
                wprev = w;
            } else {
                const cd gp = G[(size_t)j * a.nr + i - 1];
                const double dw = w - atan2(gp.im, gp.re);
                const double pred = j > 0 ? dprev * (a.freqs[j] / a.freqs[j - 1]) : 0.0;
                const double m = rint((pred - dw) / two_pi);
                dprev = dw + two_pi * m;
                ok = ok && amp_of(g) > floor_amp && amp_of(gp) > floor_amp;
                cyc[(size_t)i * a.nf + j] = ok ? static_cast<int16_t>(m) : kBroken;
            }
        }
        a.lmax[(size_t)s * a.nr + i] = static_cast<float>(log(fmax(rmax, 1e-300)));
    }
    __syncthreads();
    double st[6] = {0, 0, 0, 0, 0, 0};
    const float qnan = __int_as_float(0x7fc00000);
    for (int j = tid; j < a.nf; j += blockDim.x) {
        int n = cyc[j];
        bool valid = n != kBroken;
        const double w_r = two_pi * a.freqs[j];
        for (int i = 0; i < a.nr; i++) {
            if (i > 0) {
                const int m = cyc[(size_t)i * a.nf + j];
                if (m == kBroken) valid = false;
                if (valid) n += m;
            }
            const cd g = G[(size_t)j * a.nr + i];
            const double t0 = log(fmax(amp_of(g), floor_amp));
            float* L = a.labels + (((size_t)s * a.nr + i) * a.nf + j) * 2;
            L[0] = static_cast<float>(t0);
            st[0] += 1.0;
            st[1] += t0;
            st[2] += t0 * t0;
            if (valid) {
                const double phi = atan2(g.im, g.re) + two_pi * n;
                const double t1 = -phi / (w_r * a.ranges[i]);
                L[1] = static_cast<float>(t1);
                st[3] += 1.0;
                st[4] += t1;
                st[5] += t1 * t1;
            } else {
                L[1] = qnan;
            }
        }
    }
    for (int q = 0; q < 6; q++) {
        __syncthreads();
        red[tid] = st[q];
        __syncthreads();
        for (int w = kLabelThreads / 2; w > 0; w >>= 1) {
            if (tid < w) red[tid] += red[tid + w];
            __syncthreads();
        }
        if (tid == 0) a.stats[(size_t)s * 6 + q] = red[0];
    }
}

// ------------------------------------------------------------------ eval --

__global__ void __launch_bounds__(256) k_eval(const float* T, const float* labels, const int* soil_ids,
                                              long long p0, long long rows, int nr, int nf, const double* ranges,
                                              const double* freqs, double* acc) {
    __shared__ double sm[6][256];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (long long q = blockIdx.x * 256LL + threadIdx.x; q < rows; q += (long long)gridDim.x * 256) {
        const long long p = p0 + q;
        const int ir = static_cast<int>(p % nr);
        const int jf = static_cast<int>((p / nr) % nf);
        const long long sl = p / ((long long)nr * nf);
        const float* L = labels + (((size_t)soil_ids[sl] * nr + ir) * nf + jf) * 2;
        const double wr = 2.0 * CUDART_PI * freqs[jf] * ranges[ir];
        const double e0 = (double)T[2 * q] - L[0];
        a[0] += e0 * e0;
        const double al = exp((double)L[0]), ap = exp((double)T[2 * q]);
        if (!isnan(L[1])) {
            const double e1 = (double)T[2 * q + 1] - L[1];
            a[1] += 1.0;
            a[2] += e1 * e1;
            a[3] += (e1 * wr) * (e1 * wr);
            // |ap e^{-i t1p wr} - al e^{-i t1l wr}|^2
            a[4] += ap * ap + al * al - 2.0 * ap * al * cos(e1 * wr);
        } else {
            a[4] += (ap - al) * (ap - al);
        }
        a[5] += al * al;
    }
    for (int k = 0; k < 6; k++) sm[k][threadIdx.x] = a[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; k++) sm[k][threadIdx.x] += sm[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 6) acc[blockIdx.x * 6 + threadIdx.x] = sm[threadIdx.x][0];
}

// ------------------------------------------------------------------ host --

namespace {
bool make_map_bf16(CUtensorMap* map, const bf16* base, int rows, int K) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    cuuint32_t box[2] = {(cuuint32_t)BKE, (cuuint32_t)BM};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int MODE>
bool set_attr() {
    return cudaFuncSetAttribute(k_gemm<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) ==
           cudaSuccess;
}

template <int MODE>
void launch_mode(cudaStream_t s, const CUtensorMap& ta, const CUtensorMap& tb, dim3 grid, const GemmArgs& a) {
    // weight gradients run on a second stream behind an event: an ordinary
    // launch, so that event stays a full dependency
    if (MODE == kWgrad)
        k_gemm<MODE><<<grid, THREADS, SMEM_BYTES, s>>>(ta, tb, a);
    else
        launch_dep(k_gemm<MODE>, grid, dim3(THREADS), SMEM_BYTES, s, ta, tb, a);
}
}  // namespace

int prepare_gemm() {
    static std::atomic<bool> done{false};
    if (!done.load(std::memory_order_relaxed) && set_attr<kFwdTrain>() && set_attr<kFwdInfer>() &&
        set_attr<kBwdData>() && set_attr<kWgrad>())
        done.store(true, std::memory_order_relaxed);
    return done.load(std::memory_order_relaxed) ? 0 : 3;
}

int launch_gemm(cudaStream_t s, int mode, const bf16* A, const bf16* B, int rowsA, int rowsB, int ktotal, int splits,
                const GemmArgs& a0) {
    if (rowsA <= 0 || rowsB <= 0 || splits <= 0 || rowsA % BM || rowsB % BN || ktotal % (BK * splits)) return 1;
    if (prepare_gemm()) return 3;
    CUtensorMap ta, tb;
    if (!make_map_bf16(&ta, A, rowsA, ktotal) || !make_map_bf16(&tb, B, rowsB, ktotal)) return 2;
    GemmArgs a = a0;
    a.M = rowsA;
    a.N = rowsB;
    a.K = ktotal / splits;
    const dim3 grid(rowsB / BN, rowsA / BM, splits);
    switch (mode) {
        case kFwdTrain: launch_mode<kFwdTrain>(s, ta, tb, grid, a); return 0;
        case kFwdInfer: launch_mode<kFwdInfer>(s, ta, tb, grid, a); return 0;
        case kBwdData: launch_mode<kBwdData>(s, ta, tb, grid, a); return 0;
        case kWgrad: launch_mode<kWgrad>(s, ta, tb, grid, a); return 0;
    }
    return 1;
}

void launch_step_begin(cudaStream_t s, TrainScalars* ts) { launch_dep(k_step_begin, dim3(1), dim3(1), 0, s, ts); }

void launch_batch(cudaStream_t s, const BatchArgs& a) {
    launch_dep(k_batch, dim3(a.B / kBatchRows), dim3(kIn), 0, s, a);
}

void launch_head_train(cudaStream_t s, const bf16* H, const bf16* Z, const float* W6, const float* b6, const float* Y,
                       const float* C, int B, bf16* dZ, bf16* dZT, float* gpart, float* lpart) {
    launch_dep(k_head_train, dim3(B / kHeadRows), dim3(256), 0, s, H, Z, W6, b6, Y, C, B, dZ, dZT, gpart, lpart);
}

void launch_bias_grad(cudaStream_t s, const bf16* const* dZT, int layers, int B, float* gb) {
    BiasPtrs d{};
    for (int l = 0; l < layers && l < 8; l++) d.p[l] = dZT[l];
    k_bias_grad<<<dim3(kWidth, layers), 256, 0, s>>>(d, B, gb);  // follows the join of the two streams
}

namespace {
long long max_seg(const AdamArgs& a) {
    long long m = 1;
    for (int s = 0; s < a.nseg; s++) m = a.seg[s].n > m ? a.seg[s].n : m;
    return m;
}
void launch_transposes(cudaStream_t s, const AdamArgs& a) {
    int rows = 32, cols = 32;
    for (int q = 0; q < a.nseg; q++)
        if (a.seg[q].wb) {
            rows = a.seg[q].rows > rows ? a.seg[q].rows : rows;
            cols = a.seg[q].cols > cols ? a.seg[q].cols : cols;
        }
    launch_dep(k_transpose_w, dim3(cols / 32, rows / 32, a.nseg), dim3(32, 8), 0, s, a);
}
}  // namespace

void launch_adam(cudaStream_t s, const AdamArgs& a, long long) {
    launch_dep(k_adam, dim3((unsigned)((max_seg(a) + 255) / 256), a.nseg), dim3(256), 0, s, a);
    launch_transposes(s, a);
}

void launch_sync_weights(cudaStream_t s, const AdamArgs& a, long long) {
    k_sync_weights<<<dim3((unsigned)((max_seg(a) + 255) / 256), a.nseg), 256, 0, s>>>(a);
    launch_transposes(s, a);
}

void launch_grad_flat(cudaStream_t s, const AdamArgs& a, long long, float* out) {
    k_grad_flat<<<dim3((unsigned)((max_seg(a) + 255) / 256), a.nseg), 256, 0, s>>>(a, out);
}

void launch_loss_hist(cudaStream_t s, const float* lpart, int nblk, int B, const TrainScalars* ts, float* hist,
                      int cap) {
    launch_dep(k_loss_hist, dim3(1), dim3(32), 0, s, lpart, nblk, B, ts, hist, cap);
}

void launch_features(cudaStream_t s, const FeatureArgs& a, long long rows_padded) {
    launch_dep(k_features, dim3((unsigned)((rows_padded + 31) / 32)), dim3(kIn), 0, s, a, rows_padded);
}

void launch_head_infer(cudaStream_t s, const HeadInferArgs& a) {
    launch_dep(k_head_infer, dim3((unsigned)((a.rows + 7) / 8)), dim3(256), 0, s, a);
}

int launch_labels(cudaStream_t s, const LabelArgs& a) {
    if (a.nr > kLabelThreads || a.nr < 1 || a.nf < 1) return 1;
    const size_t smem = (size_t)a.nr * a.nf * sizeof(int16_t);
    if (smem > 200 * 1024) return 1;
    static size_t attr = 0;
    if (smem > 48 * 1024 && smem > attr) {
        if (cudaFuncSetAttribute(k_labels, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return 3;
        attr = smem;
    }
    k_labels<<<a.ns, kLabelThreads, smem, s>>>(a);
    return 0;
}

void launch_eval(cudaStream_t s, const float* T, const float* labels, const int* soil_ids, long long p0,
                 long long rows, int nr, int nf, const double* ranges, const double* freqs, double* acc, int nblk) {
    k_eval<<<nblk, 256, 0, s>>>(T, labels, soil_ids, p0, rows, nr, nf, ranges, freqs, acc);
}

}  // namespace mlp
}  // namespace gfk
