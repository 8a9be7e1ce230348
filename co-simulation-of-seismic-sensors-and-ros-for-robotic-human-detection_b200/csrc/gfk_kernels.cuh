// gfk_kernels.cuh — kernel declarations shared by the host code.
#pragma once
#include <stdint.h>
#include "gfk_solver.cuh"

namespace gfk {

// Device status bits, mapped to gfk_status by the host.
enum : int { kStSingular = 1, kStNonfinite = 2 };

void launch_layer_consts(cudaStream_t s, const LayerP* layers, MediumP med, const double* freqs, int nf,
                         double wi, double mu_ref, int formulation, LayerC* lc, cd* wc2);

void launch_static(cudaStream_t s, const LayerC* lc, int nl, const double* freqs, const cd* wc2,
                   const double* kfar, int nf, double mu_ref, int formulation, cd* C, int* status);

// rem[off[f] + i - 1] = k_i u(k_i, f) - C_f for i = 1..nk[f], k_i = i dk[f].
// `variant` picks one of prop_variant_count() launch shapes of the Dunkin kernel.
void launch_prop(cudaStream_t s, const LayerC* lc, int nl, const double* freqs, const cd* wc2, int nf,
                 const int* nk, const double* dk, const int64_t* off, int max_nk, const cd* C,
                 double mu_ref, int formulation, cd* rem, int* status, int variant = 0);
int prop_variant_count();

// W[(i-1) nr + j] = w_i J0(k_i r_j) dk, w = 1/2 at i = nk.
void launch_j0_table(cudaStream_t s, const double* ranges, int nr, int nk, double dk, double* W);

// G[f][j] = C_f/r_j - dk C_f/2 + sum_i rem[f][i] W[i][j]; rem is [nf][nk].
void launch_quad_gemm(cudaStream_t s, const cd* rem, const double* W, const cd* C, const double* ranges,
                      int nf, int nk, int nr, double dk, cd* G);

// Per-frequency grids: the same sum with J0 evaluated in the loop.
void launch_quad_ragged(cudaStream_t s, const cd* rem, const cd* C, const double* ranges, int nf, int nr,
                        const int* nk, const double* dk, const int64_t* off, cd* G);

void launch_bank_pack(cudaStream_t s, const cd* G, int nf, int nr, int first_bin, int bins, float* payload);

}  // namespace gfk
