// gfk_ctx.h — the context object behind the C ABI's gfk_ctx handle, shared
// by the translation units of libgfk.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

struct gfk_plan;
struct gfk_dataset;
struct gfk_net;
struct gfk_bank_dev;

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
};

// Frees every surrogate object the context still holds (gfk_surrogate.cu).
void gfk_release_surrogates(gfk_ctx* ctx);
// Frees every device-resident bank the context still holds (gfk_consume.cu).
void gfk_release_banks(gfk_ctx* ctx);
