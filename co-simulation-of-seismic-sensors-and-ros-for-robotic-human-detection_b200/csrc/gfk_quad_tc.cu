// gfk_quad_tc.cu — the shared-grid wavenumber sum on the tcgen05 tensor cores.
//
// G[f][r] = head + sum_k REM[f][k] W[k][r] is a complex-by-real GEMM
// (M = 2 nf real rows, N = nr ranges, K = nk wavenumbers). The sum cancels
// heavily (|G| is 40-400x below sum |terms| typically, 1e5x at worst on the
// graded-soil workload), so it needs ~28 significant bits end to end. It is
// computed with exact integer slices (the Ozaki splitting): each operand row
// (REM) / column (W) is scaled by a power of two into (-1, 1) and written as
// four signed 7-bit digits (gfk_slice.cuh),
//     a = 2^e_a sum_s a_s 2^-7(s+1),   b = 2^e_b sum_t b_t 2^-7(t+1),
// the ten digit products with s + t <= 3 run as int8 x int8 -> s32 tensor-core
// MMAs (tcgen05.mma kind::i8), accumulated EXACTLY in TMEM per level s + t, and
// the four level sums are recombined in FP64 in the epilogue:
//     sum_k a b = 2^(e_a+e_b) sum_l acc_l 2^-7(l+2) + O(2^-28) relative.
// No FP32 rounding enters, so no compensated summation is needed.
//
// Kernel shape: one CTA per 128 x 128 output tile, 6 warps:
//   warp 0  TMA producer (one lane): per 64-byte K block, 4 A-slice and 4
//           B-slice tiles (SWIZZLE_64B, 8 KB each) into a 3-stage ring;
//   warp 1  allocates 512 TMEM columns (4 levels x 128 s32 columns) and one
//           lane issues the MMAs (M = 128, N = 128, K = 32 per instruction);
//   warps 2-5 epilogue: tcgen05.ld the 4 levels, recombine, add the static
//           head term, write FP64.
// Every mbarrier wait is bounded (~1 s of SM clock); a timeout sets a status
// bit, stops issuing, drains what is in flight and frees TMEM before exit.
// No TMA multicast is used anywhere.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "gfk_kernels.cuh"
#include "gfk_tc.cuh"

namespace gfk {
namespace tc {

constexpr int BM = 128, BK = 64;  // BK in int8 elements (bytes)
constexpr int S = 4;              // slices per operand
constexpr int TILE_A = BM * BK;   // 8192 bytes per A slice tile
constexpr int THREADS = 192;

// Tile shapes the plan's tuner chooses among: TN output ranges per CTA (64 or
// 128; four TN-column s32 accumulators in TMEM) and NST pipeline stages.
template <int TN, int NST>
struct Shape {
    static constexpr int TILE_B = TN * BK;
    static constexpr int STAGE_BYTES = S * (TILE_A + TILE_B);
    static constexpr int TMEM_COLS = S * TN;
    static constexpr int SMEM_BYTES = NST * STAGE_BYTES + 1024 + 256;
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
    static_assert(TMEM_COLS == 256 || TMEM_COLS == 512, "TMEM allocation");
};

// Instruction descriptor: s8 x s8 -> s32, both K-major, M = 128, N = TN.
template <int TN>
__host__ __device__ inline uint32_t idesc_i8() {
    cute::UMMA::InstrDescriptor id;
    id.desc_ = 0;
    id.c_format_ = 2;  // S32
    id.a_format_ = 1;  // signed 8-bit
    id.b_format_ = 1;
    id.a_major_ = 0;   // K-major
    id.b_major_ = 0;
    id.n_dim_ = TN >> 3;
    id.m_dim_ = BM >> 4;
    return id.desc_;
}

struct Args {
    int M, N;           // valid real rows (2 nf) and ranges
    int Mp, Np, Kp;     // padded extents of the slice planes
    const int* row_exp; // [M] power-of-two exponent of each real row
    int col_exp;        // exponent shared by every W column
    const cd* C;        // [nf] static coefficients
    const double* ranges;
    double dk;
    cd* G;              // [nf][N]
    int* status;        // [nf] status bits
    cd* part;           // split partial sums [gridDim.z][M/2][N], or null (one split)
    long long wait_cycles;  // bound on each mbarrier wait (kWaitCycles)
    int starve;         // self-test only: the producer issues no loads, so the first wait runs out
};

template <int TN, int NST>
__global__ void __launch_bounds__(THREADS, 1)
    k_quad_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Args a) {
    using Sh = Shape<TN, NST>;
    constexpr int STAGES = NST, STAGE_BYTES = Sh::STAGE_BYTES, TMEM_COLS = Sh::TMEM_COLS;
    constexpr int BN = TN, TILE_B = Sh::TILE_B;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
    uint64_t* empty = full + STAGES;
    uint64_t* accf = empty + STAGES;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);
    int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // this CTA's K blocks [kb0, kb0 + nkb): all of them, or split z of gridDim.z
    const int nkb_all = a.Kp / BK;
    const int kb0 = (int)((long long)blockIdx.z * nkb_all / gridDim.z);
    const int nkb = (int)((long long)(blockIdx.z + 1) * nkb_all / gridDim.z) - kb0;

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

    if (warp == 0) {
        if (lane == 0) {
            int issued = 0;
            for (int kb = 0; kb < (a.starve ? 0 : nkb); kb++) {
                const int st = kb % STAGES;
                const uint32_t ph = (kb / STAGES) & 1;
                if (!mbar_wait(&empty[st], ph ^ 1, a.wait_cycles)) {
                    *abort_flag = 1;
                    break;
                }
                if (*(volatile int*)abort_flag) break;
                mbar_expect_tx(&full[st], STAGE_BYTES);
                uint8_t* base = smem + st * STAGE_BYTES;
#pragma unroll
                for (int s = 0; s < S; s++)
                    tma_load_2d(base + s * TILE_A, &tmA, &full[st], (kb0 + kb) * BK, s * a.Mp + m0);
#pragma unroll
                for (int t = 0; t < S; t++)
                    tma_load_2d(base + S * TILE_A + t * TILE_B, &tmB, &full[st], (kb0 + kb) * BK, t * a.Np + n0);
                issued = kb + 1;
            }
            // drain: the last loads of each stage land before the CTA may exit
            for (int kb = issued - 1; kb >= 0 && kb >= issued - STAGES; kb--)
                if (!mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, a.wait_cycles)) *abort_flag = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = idesc_i8<TN>();
            bool init[S] = {false, false, false, false};
            for (int kb = 0; kb < nkb; kb++) {
                const int st = kb % STAGES;
                if (!mbar_wait(&full[st], (kb / STAGES) & 1, a.wait_cycles)) {
                    *abort_flag = 1;
                    break;
                }
                if (*(volatile int*)abort_flag) break;
                tc_fence_after();
                const uint32_t base = smem_u32(smem + st * STAGE_BYTES);
#pragma unroll
                for (int lvl = 0; lvl < S; lvl++) {
#pragma unroll
                    for (int s = 0; s <= lvl; s++) {
                        const int t = lvl - s;
#pragma unroll
                        for (int kk = 0; kk < BK / 32; kk++) {
                            const uint64_t da = sdesc_k_sw64(base + s * TILE_A + kk * 32);
                            const uint64_t db = sdesc_k_sw64(base + S * TILE_A + t * TILE_B + kk * 32);
                            tc_mma_i8(tmem + lvl * BN, da, db, idesc, init[lvl] ? 1u : 0u);
                            init[lvl] = true;
                        }
                    }
                }
                tc_commit(&empty[st]);  // frees the stage once these MMAs have read it
            }
            tc_commit(accf);  // arrives when every MMA issued above has completed
        }
    } else {
        // epilogue: warps 2..5 cover TMEM lane quarters 2, 3, 0, 1
        const bool ok = mbar_wait(accf, 0, a.wait_cycles);
        tc_fence_after();
        const int q = warp & 3;
        const int row = m0 + q * 32 + lane;
        const bool row_ok = ok && row < a.M && !*(volatile int*)abort_flag;
        const int f = row >> 1, part = row & 1;
        double rscale = 0.0;
        cd c = mk(0.0);
        if (row_ok) {
            rscale = ldexp(1.0, a.row_exp[row] + a.col_exp);
            c = a.C[f];
        }
        const double cpart = part ? c.im : c.re;
        cd* const dst = a.part ? a.part + (size_t)blockIdx.z * (a.M >> 1) * a.N : a.G;
#pragma unroll 1
        for (int j = 0; j < BN / 32; j++) {
            uint32_t v0[32], v1[32], v2[32], v3[32];
            const uint32_t lane_addr = tmem + (static_cast<uint32_t>(q * 32) << 16) + j * 32;
            tmem_ld32(lane_addr + 0 * BN, v0);
            tmem_ld32(lane_addr + 1 * BN, v1);
            tmem_ld32(lane_addr + 2 * BN, v2);
            tmem_ld32(lane_addr + 3 * BN, v3);
            tmem_wait_ld();
            if (row_ok) {
#pragma unroll
                for (int cc = 0; cc < 32; cc++) {
                    const int n = n0 + j * 32 + cc;
                    if (n < a.N) {
                        const double acc = (double)(int)v0[cc] * 0x1p-14 + (double)(int)v1[cc] * 0x1p-21 +
                                           (double)(int)v2[cc] * 0x1p-28 + (double)(int)v3[cc] * 0x1p-35;
                        double* out = reinterpret_cast<double*>(dst + (size_t)f * a.N + n);
                        if (a.part) {
                            out[part] = acc * rscale;
                        } else {
                            const double head = cpart / a.ranges[n] - (0.5 * a.dk) * cpart;  // fk.go:529-532
                            out[part] = head + acc * rscale;
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0 && *(volatile int*)abort_flag) {
        const int r0 = m0 >> 1;
        for (int f = r0; f < r0 + BM / 2 && 2 * f < a.M; f++) atomicOr(a.status + f, kStTimeout);
    }
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ------------------------------------------------------------- slicing --

// Hankel weights w_i J0(k_i r_j) dk (fk.go:540-546), transposed to [range][k]
// and sliced with the shared column exponent: |w J0 dk| <= dk always.
__global__ void k_j0_slices(const double* __restrict__ ranges, int nr, int nk, int Kp, int Np, double dk,
                            int col_exp, int8_t* __restrict__ B) {
    const int n = blockIdx.y;
    const int k0 = (blockIdx.x * blockDim.x + threadIdx.x) * 16;
    if (n >= Np || k0 >= Kp) return;
    const double sc = ldexp(1.0, 28 - col_exp);
    const double r = n < nr ? ranges[n] : 0.0;
    alignas(16) int8_t out[4][16];
#pragma unroll 4
    for (int q = 0; q < 16; q++) {
        const int i = k0 + q + 1;  // wavenumber index, k_i = i dk
        double wv = 0.0;
        if (n < nr && i <= nk) {
            const double k = (double)i * dk;
            const double w = i == nk ? 0.5 : 1.0;
            wv = (w * j0(k * r)) * dk;
        }
        const uint32_t d = digits4(scaled_int(wv, sc));
#pragma unroll
        for (int s = 0; s < 4; s++) out[s][q] = (int8_t)(d >> (8 * s));
    }
#pragma unroll
    for (int s = 0; s < 4; s++)
        *reinterpret_cast<int4*>(B + ((size_t)s * Np + n) * Kp + k0) = *reinterpret_cast<const int4*>(out[s]);
}

}  // namespace tc

// ------------------------------------------------------------------ host --

namespace {
// A [planes*rows_p][Kp] int8 plane stack; box = box_rows x 64 bytes, SWIZZLE_64B.
bool make_map(CUtensorMap* map, const int8_t* base, int rows_total, int Kp, int box_rows) {
    auto fn = tc::encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows_total};
    cuuint64_t strides[1] = {(cuuint64_t)Kp};
    cuuint32_t box[2] = {(cuuint32_t)tc::BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<int8_t*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The tile shapes a plan's tuner times: (ranges per CTA, pipeline stages).
struct TcVariant {
    void (*fn)(const CUtensorMap, const CUtensorMap, tc::Args);
    int tn, stages, smem;
    std::atomic<bool> attr;  // the shared-memory attribute is set (once per process)
};
TcVariant g_tc_variants[] = {
    {tc::k_quad_tc<128, 3>, 128, 3, tc::Shape<128, 3>::SMEM_BYTES, false},
    {tc::k_quad_tc<128, 2>, 128, 2, tc::Shape<128, 2>::SMEM_BYTES, false},
    {tc::k_quad_tc<64, 4>, 64, 4, tc::Shape<64, 4>::SMEM_BYTES, false},
    {tc::k_quad_tc<64, 3>, 64, 3, tc::Shape<64, 3>::SMEM_BYTES, false},
};
constexpr int kTcVariants = sizeof(g_tc_variants) / sizeof(g_tc_variants[0]);
}  // namespace

int quad_tc_variant_count() { return kTcVariants; }

void quad_tc_variant_shape(int variant, int* tile_n, int* stages) {
    const TcVariant& v = g_tc_variants[(variant >= 0 && variant < kTcVariants) ? variant : 0];
    *tile_n = v.tn;
    *stages = v.stages;
}

int tc_col_exp(double dk) { return ilogb(dk * (128.0 / 127.0)) + 1; }

void launch_j0_slices(cudaStream_t s, const double* ranges, int nr, int nk, int Kp, int Np, double dk, int col_exp,
                      int8_t* B) {
    dim3 grid((Kp / 16 + 127) / 128, Np);
    tc::k_j0_slices<<<grid, 128, 0, s>>>(ranges, nr, nk, Kp, Np, dk, col_exp, B);
}

int quad_tc_splits(int M, int N, int Kp) {
    // one CTA per SM (its shared memory); each split keeps at least 4 K blocks.
    // Counted with the widest tile, so every shape's splits fit the plan's workspace.
    const long long tiles = (long long)((M + tc::BM - 1) / tc::BM) * ((N + 127) / 128);
    const int nkb = Kp / tc::BK;
    if (tiles >= 74 || nkb < 8) return 1;
    const int want = (int)((148 + tiles - 1) / tiles);
    return std::max(1, std::min({want, nkb / 4, 32}));
}

int launch_quad_tc(cudaStream_t s, const int8_t* A, const int8_t* B, int M, int N, int Mp, int Np, int Kp,
                   const int* row_exp, int col_exp, const cd* C, const double* ranges, double dk, cd* G, int* status,
                   int splits, cd* part, int variant, long long wait_cycles, int starve) {
    if (variant < 0 || variant >= kTcVariants) variant = 0;
    TcVariant& v = g_tc_variants[variant];
    if (Mp % tc::BM || Np % v.tn || Kp % tc::BK || M > Mp || N > Np) return 1;
    if (splits < 1 || !part) splits = 1;
    if (splits > Kp / tc::BK) return 1;
    CUtensorMap ta, tb;
    if (!make_map(&ta, A, tc::S * Mp, Kp, tc::BM) || !make_map(&tb, B, tc::S * Np, Kp, v.tn)) return 2;
    if (!v.attr.load(std::memory_order_relaxed)) {
        if (cudaFuncSetAttribute(v.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, v.smem) != cudaSuccess) return 3;
        v.attr.store(true, std::memory_order_relaxed);
    }
    tc::Args a{M, N, Mp, Np, Kp, row_exp, col_exp, C, ranges, dk, G, status, splits > 1 ? part : nullptr,
               wait_cycles > 0 ? wait_cycles : tc::kWaitCycles, starve};
    // row tiles over this launch's M valid rows only: a chunk smaller than the
    // plan's largest (Mp) would otherwise multiply padding rows it never stores
    dim3 grid((N + v.tn - 1) / v.tn, (M + tc::BM - 1) / tc::BM, splits);
    v.fn<<<grid, tc::THREADS, v.smem, s>>>(ta, tb, a);
    if (splits > 1) launch_quad_finish(s, part, splits, C, ranges, M >> 1, N, dk, G);
    return 0;
}

// A starved launch of the tensor-core sum on one 128 x 128 x 64 tile: the
// producer issues no loads, so the MMA issuer's first wait runs out after
// wait_cycles, the kernel drains, frees its TMEM and marks the tile's rows
// timed out. Returns 0 with *timed_out the number of the 64 rows so marked,
// or a nonzero launch/CUDA error code.
int quad_tc_selftest_timeout(cudaStream_t s, long long wait_cycles, int* timed_out) {
    *timed_out = 0;
    const int M = 128, N = 128, Kp = 64, nf = M / 2;
    int8_t *A = nullptr, *B = nullptr;
    int *row_exp = nullptr, *status = nullptr;
    cd *C = nullptr, *G = nullptr;
    double* ranges = nullptr;
    int rc = 0;
    auto alloc = [&](void** p, size_t bytes) {
        if (!rc && cudaMallocAsync(p, bytes, s) != cudaSuccess) rc = 10;
        if (!rc && cudaMemsetAsync(*p, 0, bytes, s) != cudaSuccess) rc = 11;
    };
    alloc((void**)&A, (size_t)tc::S * M * Kp);
    alloc((void**)&B, (size_t)tc::S * N * Kp);
    alloc((void**)&row_exp, sizeof(int) * M);
    alloc((void**)&status, sizeof(int) * nf);
    alloc((void**)&C, sizeof(cd) * nf);
    alloc((void**)&G, sizeof(cd) * nf * N);
    alloc((void**)&ranges, sizeof(double) * N);
    if (!rc) rc = launch_quad_tc(s, A, B, M, N, M, N, Kp, row_exp, 0, C, ranges, 1.0, G, status, 1, nullptr, 0,
                                 wait_cycles, 1);
    if (!rc && cudaGetLastError() != cudaSuccess) rc = 12;
    int host[64] = {0};
    if (!rc && cudaMemcpyAsync(host, status, sizeof(int) * nf, cudaMemcpyDeviceToHost, s) != cudaSuccess) rc = 13;
    void* bufs[] = {A, B, row_exp, status, C, G, ranges};
    for (void* p : bufs)
        if (p) cudaFreeAsync(p, s);
    if (cudaStreamSynchronize(s) != cudaSuccess && !rc) rc = 14;
    for (int f = 0; f < nf && !rc; f++)
        if (host[f] & kStTimeout) (*timed_out)++;
    return rc;
}

}  // namespace gfk
