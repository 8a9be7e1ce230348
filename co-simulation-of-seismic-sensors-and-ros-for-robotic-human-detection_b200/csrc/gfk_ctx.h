// gfk_ctx.h — the context object behind the C ABI's gfk_ctx handle, shared
// by the translation units of libgfk.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

struct gfk_plan;
struct gfk_dataset;
struct gfk_net;
struct gfk_bank_dev;

// The Hankel weights of a shared-grid wavenumber sum (the tensor-core sum's
// int8 digit planes, or the plain sum's FP64 table). They depend only on the
// grid and the ranges, so plans with the same ones share one device copy; it
// is freed, ordered on the context's stream, when its last holder lets go.
struct gfk_weights {
    gfk_ctx* ctx = nullptr;
    bool tc = false;
    int n = 0;         // wavenumbers
    double dk = 0.0;   // wavenumber step
    std::vector<double> ranges;
    void* d = nullptr;
    bool built = false;  // its build has been enqueued on the context's stream
    bool same(bool tc_, int n_, double dk_, const double* r, int nr) const {
        return tc == tc_ && n == n_ && dk == dk_ && (int)ranges.size() == nr &&
               std::equal(ranges.begin(), ranges.end(), r);
    }
    ~gfk_weights();
};

struct gfk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // device-to-host copies beside the compute (created on first use)
    std::string last_error;
    int64_t launches = 0;
    std::vector<gfk_plan*> plans;        // live plans, destroyed by gfk_close
    std::vector<gfk_dataset*> datasets;  // live surrogate data sets and networks,
    std::vector<gfk_net*> nets;          // destroyed by gfk_close as well
    std::vector<gfk_bank_dev*> banks;    // device-resident banks (gfk_consume.cu)
    // propagator launch shape chosen by tuning, per (layer count, wavenumber count)
    struct Tuned {
        int nl, nk, variant;
    };
    std::vector<Tuned> tuned;
    // tensor-core sum tile shape chosen by tuning, per padded (rows, ranges, wavenumbers)
    struct TunedTc {
        int Mp, Np, Kp, variant;
    };
    std::vector<TunedTc> tuned_tc;
    // the most recent plan's Hankel weights, kept for the next plan
    std::shared_ptr<gfk_weights> weights;
};

// Frees every surrogate object the context still holds (gfk_surrogate.cu).
void gfk_release_surrogates(gfk_ctx* ctx);
// Frees every device-resident bank the context still holds (gfk_consume.cu).
void gfk_release_banks(gfk_ctx* ctx);
