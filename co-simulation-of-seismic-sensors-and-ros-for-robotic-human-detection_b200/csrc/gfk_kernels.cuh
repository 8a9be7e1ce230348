// gfk_kernels.cuh — kernel declarations shared by the host code.
#pragma once
#include <stdint.h>
#include "gfk_slice.cuh"
#include "gfk_solver.cuh"

namespace gfk {

// Device status bits, mapped to gfk_status by the host.
enum : int { kStSingular = 1, kStNonfinite = 2, kStTimeout = 4 };

// Every kernel below serves nf rows described by fd[0..nf); a row's medium is
// media[fd[f].soil], whose layers are lp[media[..].lp_off ..].

// lc[fd[f].lc_off + l] for every layer of the row's medium, and wc2[f].
void launch_layer_consts(cudaStream_t s, const LayerP* lp, const MediumP* media, const FreqDesc* fd, int nf,
                         double wi, int formulation, LayerC* lc, cd* wc2);
// One thread per (frequency, layer); max_layers >= every medium's count.
void launch_layer_consts_fl(cudaStream_t s, const LayerP* lp, const MediumP* media, const FreqDesc* fd, int nf,
                            int max_layers, double wi, int formulation, LayerC* lc, cd* wc2);

void launch_static(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2, int nf,
                   int formulation, cd* C, int* status);

// The work queue of the persistent propagator shapes: next (zero at launch)
// counts the items taken; a row has `runs` items.
struct PropQueue {
    unsigned int* next;
    int items, runs;
};

// rem[fd[f].off + i - 1] = k_i u(k_i, f) - C_f for i = 1..nk, k_i = i dk.
// `variant` picks one of prop_variant_count() launch shapes of the Dunkin
// kernel; the persistent ones (prop_variant_persistent) take their items from
// `queue`, one zeroed word (without one they run as one item per block).
// With `slice` (a shared grid, rows fd[f].off = f nk) each row is also cut into
// the tensor-core sum's int8 digit planes by the block that finishes it;
// slice->rowmax and slice->done must be zero for the launch's rows (the
// launch leaves done at zero again).
void launch_prop(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2, int nf,
                 int max_nk, const cd* C, int formulation, cd* rem, int* status, int variant = 0,
                 const SliceOut* slice = nullptr, unsigned int* queue = nullptr);
int prop_variant_count();
bool prop_variant_persistent(int variant);
// threads per block, blocks per SM it is compiled for, wavenumbers per thread
// at a time, 128-wavenumber runs per item, persistent or one item per block
bool prop_variant_shape(int variant, int* threads, int* blocks_per_sm, int* ilp, int* sweeps, int* persistent);

// Tensor-core quadrature (gfk_quad_tc.cu): exact int8 slices of the integrand
// rows (cut by launch_prop) and of the Hankel weights, tcgen05 kind::i8 GEMM,
// FP64 recombination.
int tc_col_exp(double dk);
void launch_j0_slices(cudaStream_t s, const double* ranges, int nr, int nk, int Kp, int Np, double dk, int col_exp,
                      int8_t* B);
// splits > 1 divides the K blocks among blockIdx.z and writes the head-free
// partial sums to part [splits][M/2][N]; launch_quad_finish then adds them.
// variant picks the tile shape (quad_tc_variant_shape: ranges per CTA and
// pipeline stages); wait_cycles bounds each mbarrier wait (<= 0: the default
// ~1 s); starve is the self-test's: the producer issues nothing, so the waits
// run out.
int launch_quad_tc(cudaStream_t s, const int8_t* A, const int8_t* B, int M, int N, int Mp, int Np, int Kp,
                   const int* row_exp, int col_exp, const cd* C, const double* ranges, double dk, cd* G, int* status,
                   int splits, cd* part, int variant = 0, long long wait_cycles = 0, int starve = 0);
int quad_tc_variant_count();
void quad_tc_variant_shape(int variant, int* tile_n, int* stages);
int quad_tc_selftest_timeout(cudaStream_t s, long long wait_cycles, int* timed_out);
int quad_tc_splits(int M, int N, int Kp);  // split count filling the SMs for one chunk shape

// Shared grid, nr <= fused_max_ranges(): propagator and wavenumber sum in one
// pass (the integrand stays on chip); partial holds nf x ceil(nk/128) x nr.
int fused_max_ranges();
void launch_prop_fused(cudaStream_t s, const LayerC* lc, const MediumP* media, const FreqDesc* fd, const cd* wc2,
                       int nf, int nk, const cd* C, const double* W, const double* ranges, int nr, cd* partial,
                       int* status, cd* G);

// W[(i-1) nr + j] = w_i J0(k_i r_j) dk, w = 1/2 at i = nk.
void launch_j0_table(cudaStream_t s, const double* ranges, int nr, int nk, double dk, double* W);

// G[f][j] = C_f/r_j - dk C_f/2 + sum_i rem[f][i] W[i][j]; rem is [nf][nk].
// splits > 1: the wavenumber tiles are divided among blockIdx.z, partial sums
// go to part [splits][nf][nr] and launch_quad_finish completes G.
void launch_quad_gemm(cudaStream_t s, const cd* rem, const double* W, const cd* C, const double* ranges,
                      int nf, int nk, int nr, double dk, cd* G, int splits, cd* part);
int quad_gemm_splits(int nf, int nk, int nr);

// G[f][j] = C_f/r_j - dk C_f/2 + sum_z part[z][f][j], z in order (deterministic).
void launch_quad_finish(cudaStream_t s, const cd* part, int splits, const cd* C, const double* ranges, int nf,
                        int nr, double dk, cd* G);

// Per-frequency grids: the same sum with J0 evaluated in the loop.
void launch_quad_ragged(cudaStream_t s, const cd* rem, const cd* C, const double* ranges, int nf, int nr,
                        const FreqDesc* fd, cd* G);

void launch_bank_pack(cudaStream_t s, const cd* G, int nf, int nr, int first_bin, int bins, float* payload);

}  // namespace gfk
