// gfk_mlp.cuh — kernels of the surrogate network (BF16 MLP on tcgen05) and of
// the device-side Sobol trace metrics.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "gfk_solver.cuh"

namespace gfk {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kWidth = 512;    // hidden width
constexpr int kIn = 128;       // input features
constexpr int kScalars = 16;   // soil scalars (<= 11 used), range/frequency scalars
constexpr int kMaxSoil = 11;   // soil parameters a network may take
constexpr int kTimes = 6;      // vertical travel times per soil (h/Vs, h/Vp of up to 3 layers)
constexpr int kTimeFeat = kScalars;                  // sin, cos(2 pi f T_q): [16, 28)
constexpr int kLogTimeFeat = kTimeFeat + 2 * kTimes; // log-scaled f T_q: [28, 34)
constexpr int kFourierFeat = kLogTimeFeat + kTimes;  // Fourier pairs of (range, frequency): [34, 128)
constexpr int kFourier = (kIn - kFourierFeat) / 2;   // 47
constexpr int kSoilStride = 32;  // soil table row: scalars [0, 11), travel times [16, 22)
constexpr int kHeadRows = 32;  // rows per block of the head kernels
constexpr int kHeadStride = 2 * kWidth + 2 + 2;  // head partial: dW6 [2][W], db6 [2], pad

enum GemmMode { kFwdTrain = 0, kFwdInfer = 1, kBwdData = 2, kWgrad = 3 };

// C[M][N] = A[M][K] . B[N][K]^T over the K slice [z K, (z+1) K) of CTA layer z,
// BF16 operands, FP32 accumulation in TMEM; M, N multiples of 128, K of 64.
//   kFwdTrain: z = C + bias -> zout (bf16), h = silu(z) -> out, h^T -> outT
//   kFwdInfer: h = silu(C + bias) -> out
//   kBwdData:  dz = C * silu'(zin) -> out, dz^T -> outT (outT may be null)
//   kWgrad:    C -> part[z][M][N] (fp32), z = 0..splits-1
struct GemmArgs {
    int M, N, K;
    const float* bias;
    const bf16* zin;
    bf16* out;
    bf16* outT;
    bf16* zout;
    float* part;
    int* status;
};

// Sets the kernels' shared-memory limits; call once before any stream capture.
int prepare_gemm();
// Returns 0 on success, nonzero if the shapes or the tensor maps are refused.
int launch_gemm(cudaStream_t s, int mode, const bf16* A, const bf16* B, int rowsA, int rowsB, int ktotal,
                int splits, const GemmArgs& a);

// Per-step scalars kept on the device so that one captured graph replays
// every step: the step counter, the scheduled learning rate and the Adam
// bias corrections.
struct TrainScalars {
    long long step;
    float lr, bc1, bc2;
    float lr_max, lr_min;
    int warmup, total;
    float beta1, beta2;
};

struct FeatureDomain {
    float r_lo, r_hi, f_lo, f_hi;
};

// The input row of one (soil, range, frequency) point:
//   [0, 11)   soil scalars, mapped to [-1, 1]
//   11, 12    range and frequency, linear on the domain, in [-1, 1]
//   13, 14    their logarithms, in [-1, 1]
//   16 + 2q, 17 + 2q   sin, cos(2 pi f T_q), T_q the soil's vertical travel times
//   28 + q    (ln(f T_q) + 2) / 3, clamped to [-2, 2]
//   34 + 2q, 35 + 2q   sin, cos(2 pi (B_q0 u_r + B_q1 u_f)), u in [0, 1]
// The travel-time phases give the network the layer resonances (f T = 1/4,
// 3/4, ...) directly instead of leaving it to synthesise oscillations whose
// period depends on the soil.
//
// Loss per sample: c0 e0^2 + c1 e1^2 on the standardised errors, with
//   mode 0: c0 = 1, c1 = phase_weight (0 where the phase is not learnt);
//   mode 1 (complex): c0 = w, c1 = phase_weight w min((w_f r s1/s0)^2, cap),
//   w = max(|G|^2 / max_f |G(r, .)|^2, weight_floor): the squared error of G
//   relative to the soil's spectral peak at that range, phase in radians;
//   mode 2 (amplitude-weighted): c0 = v, c1 = phase_weight v,
//   v = max(|G| / max_f |G(r, .)|, weight_floor).
struct BatchArgs {
    const float* labels;   // [nsoil][nr][nf][2]: log|G|, -phi/(w r) (NaN: phase not learnt)
    const float* lmax;     // [nsoil][nr]: log max_f |G|
    const float* soilfeat; // [nsoil][kSoilStride]
    const int* train;      // soils the batch draws from
    int ntrain, nr, nf, B;
    int ir0, nir;          // ranges the batch draws from: [ir0, ir0 + nir)
    const double* ranges;  // [nr]
    const double* freqs;   // [nf]
    FeatureDomain dom;
    const float* fourier;  // [kFourier][2]
    float y_mean0, y_std0, y_mean1, y_std1;
    int loss_mode;
    float phase_weight, weight_floor, phase_cap;
    unsigned long long seed;
    const TrainScalars* ts;
    bf16* X;               // [B][kIn]
    bf16* XT;              // [kIn][B]
    float* Y;              // [B][2] standardised targets (NaN phase kept)
    float* C;              // [B][2] loss coefficients
};
void launch_step_begin(cudaStream_t s, TrainScalars* ts);
void launch_batch(cudaStream_t s, const BatchArgs& a);

// The output layer (512 -> 2, FP32) and the loss (1/B) sum c0 e0^2 + c1 e1^2;
// writes dz of the last hidden layer (and its transpose), and per-block
// partials of dW6, db6 [kHeadStride] and of the loss [4]: sum c0 e0^2,
// sum c1 e1^2, sum c0, sum c1.
void launch_head_train(cudaStream_t s, const bf16* H, const bf16* Z, const float* W6, const float* b6,
                       const float* Y, const float* C, int B, bf16* dZ, bf16* dZT, float* gpart, float* lpart);
// Column sums of dz^T rows: gb[l][o] = sum_b dZT_l[o][b] for `layers` layers.
void launch_bias_grad(cudaStream_t s, const bf16* const* dZT, int layers, int B, float* gb);

struct AdamSeg {
    long long off;        // first parameter of the segment in the flat vector
    long long n;          // parameters in the segment
    const float* src;     // gradient partials
    long long stride;     // distance between partials
    int nsrc;             // partials summed
    int rows, cols;       // weight shape (bf16 copies), 0 for none
    bf16* wb;             // [rows][cols] copy
    bf16* wt;             // [cols][rows] copy
};
constexpr int kMaxSegs = 16;
struct AdamArgs {
    int nseg;
    AdamSeg seg[kMaxSegs];  // host copy
    const AdamSeg* dseg;    // the same table in device memory, read by the kernels
    float* p;             // FP32 master parameters
    float* m;
    float* v;
    float eps, weight_decay;
    const TrainScalars* ts;
};
// AdamW over every segment (one grid row per segment), then the BF16
// transposes W^T of the weight segments (32 x 32 shared-memory tiles).
void launch_adam(cudaStream_t s, const AdamArgs& a, long long nparam);
// bf16 copies of every weight segment from the master parameters.
void launch_sync_weights(cudaStream_t s, const AdamArgs& a, long long nparam);
// The summed gradient of every parameter (no update), for gradient checks.
void launch_grad_flat(cudaStream_t s, const AdamArgs& a, long long nparam, float* out);
// hist[(step - 1) % cap] = the step's two mean squared errors.
void launch_loss_hist(cudaStream_t s, const float* lpart, int nblk, int B, const TrainScalars* ts, float* hist,
                      int cap);

// Inference rows: row p = (soil * nf + jf) * nr + ir for soils [s0, s0 + ns).
struct FeatureArgs {
    const float* soilfeat;  // [ns][kSoilStride] of the soils being evaluated
    int ns, nr, nf;
    long long p0, rows;     // first row and rows in this chunk
    const double* ranges;
    const double* freqs;
    FeatureDomain dom;
    const float* fourier;
    bf16* X;                // [rows_padded][kIn]
};
void launch_features(cudaStream_t s, const FeatureArgs& a, long long rows_padded);

// Output layer for inference, mapped back to G = exp(t0) exp(-i t1 w r).
struct HeadInferArgs {
    const bf16* H;
    const float* W6;
    const float* b6;
    long long p0, rows;
    int nr, nf;
    const double* ranges;
    const double* freqs;
    float y_mean0, y_std0, y_mean1, y_std1;
    cd* G;                  // [ns * nf * nr]
    float* T;               // optional [rows][2] de-standardised (t0, t1)
};
void launch_head_infer(cudaStream_t s, const HeadInferArgs& a);

// Labels of one soil block from a bank [soil][nf][nr] of complex128 rows.
struct LabelArgs {
    const cd* G;            // [ns][nf][nr]
    int ns, nr, nf;
    const double* ranges;
    const double* freqs;
    double floor_rel;       // amplitude floor relative to the soil's maximum
    float* labels;          // [ns][nr][nf][2]
    float* lmax;            // [ns][nr]: log max_f |G|
    double* stats;          // [ns][6]: n0, sum t0, sum t0^2, n1, sum t1, sum t1^2
};
int launch_labels(cudaStream_t s, const LabelArgs& a);

// Held-out comparison of predicted (t0, t1) [rows][2] (rows p0.. of the
// inference layout over soils soil_ids[]) against the labels. acc[nblk][6]:
// sum e0^2, phase cells, sum e1^2, sum (e1 w r)^2, sum |G_pred - G|^2, sum |G|^2.
void launch_eval(cudaStream_t s, const float* T, const float* labels, const int* soil_ids, long long p0,
                 long long rows, int nr, int nf, const double* ranges, const double* freqs, double* acc, int nblk);

}  // namespace mlp

namespace trace {
// Per soil: y = irfft(G[k-1] S[k], n) e^{w_I t}; peak = max |y|; centroid =
// sum a f / sum a over the band, a = |rfft(y, n)|. n = 1024.
constexpr int kN = 1024;
void launch_metrics(cudaStream_t s, const cd* G, long long stride, int ns, int nbins, const cd* S,
                    const cd* twiddle, double fs, double omega_imag, int k_lo, int k_hi, double* peak,
                    double* centroid);

// Ensemble gate, one block per soil: mean[s][k] = mean over members of
// G_e[s stride + k]; flag[s][k] = 1 where max_e |G_e - mean| |S[k+1]| exceeds
// threshold * max_k |mean S[k+1]| (the ensemble's disagreement on that row's
// share of the recorded trace, relative to the trace spectrum's peak);
// spread[s] = max_k of that ratio.
constexpr int kMaxMembers = 16;
struct GateArgs {
    const cd* members[kMaxMembers];
    int E;
    long long stride;
    int ns, nbins;
    const cd* S;
    double threshold;
    double amp_threshold;  // > 0: also flag rows whose |mean S| exceeds it times the peak
    cd* mean;
    unsigned char* flag;
    double* spread;
};
void launch_gate(cudaStream_t s, const GateArgs& a);
// dst[index[i]] = src[i * src_stride] for i < n.
void launch_scatter(cudaStream_t s, const cd* src, long long src_stride, const long long* index, long long n,
                    cd* dst);
}  // namespace trace
}  // namespace gfk
