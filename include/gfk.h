/*
 * gfk.h — C ABI of libgfk, the B200 (sm_100a) Green's-function bank engine.
 *
 * libgfk computes what the reference's Go package internal/fk computes: the
 * vertical surface displacement of a layered viscoelastic half-space per newton
 * of vertical surface point force, integrated over horizontal wavenumber with a
 * static-asymptote-subtracted trapezoid Hankel (J0) rule, for many ranges and
 * frequencies at once. It also assembles the float32 range-major payload of an
 * internal/bank file and writes the file.
 *
 * Every entry point takes plain C types: pointers, sizes and the structs below.
 * Host pointers are host memory owned by the caller (pinned memory is faster but
 * not required); device pointers are named d_* and live on the context's device.
 * A context serialises its calls on one CUDA stream and is not thread-safe:
 * concurrent callers either share one context behind a lock or use one each.
 *
 * Each function documents the reference interface it replaces as
 * path:line within the reference project.
 */
#ifndef GFK_H
#define GFK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
/* Each mirrors one class of Go error value returned by the reference. */
enum gfk_status {
    GFK_OK = 0,
    GFK_EARG = 1,       /* non-positive k, f or r; empty range set
                           (internal/fk/fk.go:277-279, 397-402, 465-474) */
    GFK_ESTACK = 2,     /* layer.Stack.Validate failed (internal/layer/layer.go:53-73) */
    GFK_EGUARD = 3,     /* k*h past MaxLayerPhase at the pole wavenumber
                           (internal/fk/fk.go:242, 251-266); GFK_REFERENCE_DIRECT only */
    GFK_ESINGULAR = 4,  /* singular layer propagator or surface system
                           (internal/fk/fk.go:293-295, 322-324) */
    GFK_ENONFINITE = 5, /* a result was NaN or Inf */
    GFK_ETIMEOUT = 6,   /* a bounded device-side wait ran out */
    GFK_ECUDA = 7,      /* CUDA runtime error; the message names the call */
    GFK_ENOMEM = 8,     /* device or host allocation failed */
    GFK_EIO = 9,        /* bank file could not be written or read */
    GFK_ELIMIT = 10     /* a size beyond a documented maximum */
};

/* ---- how the boundary-value problem is solved --------------------------- */
enum gfk_formulation {
    /* The reference algorithm restated: direct 4x4 complex propagators
     * exp(A k h) = E diag(e^(lambda k h)) E^-1, pivoted 4x4 surface solve,
     * Qp = 2.25*Qs, real frequency, MaxLayerPhase guard on
     * (internal/fk/fk.go:119-327, internal/fk/cmat.go:12-96). */
    GFK_REFERENCE_DIRECT = 0,
    /* Complex Dunkin second-compound (minor) propagation of the half-space's
     * decaying 2-plane up to the surface, with closed-form, cancellation-free
     * layer compounds; no k*h limit. Honours per-layer Qp and a complex
     * frequency offset omega_imag. Design source internal/propmat/propmat.go:168-315. */
    GFK_DUNKIN = 1
};

enum gfk_quadrature {
    GFK_PLAIN_FP64 = 0,    /* FP64 wavenumber sum on the FP64 pipe */
    GFK_SPLIT_INT8 = 1     /* shared-grid sum as an exact-integer-sliced tensor-core GEMM:
                              each integrand row and Hankel-weight column is scaled by a
                              power of two and cut into four signed 7-bit digits; the ten
                              digit products of weight >= 2^-28 run as tcgen05 kind::i8
                              MMAs with exact s32 accumulation and are recombined in FP64.
                              Needs one wavenumber grid for all frequencies, <= 65536
                              wavenumbers. */
};

/* ---- medium --------------------------------------------------------------- */
/* One homogeneous layer: internal/layer/layer.go:24-36 (layer.Layer). */
typedef struct gfk_layer {
    double thickness_m;   /* ignored for the last entry, the half-space */
    double vp_mps;
    double vs_mps;
    double density_kgm3;
    double qs;            /* <= 0: the medium's default_q, then 30 (fk.go:67-75) */
    double qp;            /* <= 0: 2.25*Qs. Ignored by GFK_REFERENCE_DIRECT (fk.go:121-122) */
} gfk_layer;

/* fk.Medium (internal/fk/fk.go:37-53): layers[0..count-1], last = half-space. */
typedef struct gfk_medium {
    const gfk_layer *layers;
    int32_t count;
    int32_t _pad;
    double ref_freq_hz;   /* Medium.RefFreq; <= 0 uses 30 Hz (fk.go:60-65) */
    double default_q;     /* Medium.DefaultQ; <= 0 uses 30 (fk.go:67-75) */
    double sls_tau_sigma; /* Medium.Relax (visco.SLS, internal/visco/visco.go:42-47):  */
    double sls_tau_eps;   /* both > 0 replaces Kjartansson constant Q with one SLS    */
} gfk_medium;

/* fk.Integration (internal/fk/fk.go:330-341). */
typedef struct gfk_integration {
    int32_t samples;      /* <= 0: GridFor's own count (single-range calls: 20000) */
    int32_t _pad;
    double kmax_factor;   /* <= 0: 30 */
    double kmax;          /* > 0: use this in place of kmax_factor*k_body at every
                             frequency, i.e. k_max = max(kmax, 40/r_min). It is what
                             Integration{KMaxFactor: kmax/k_body(f)} expresses per
                             frequency, made exact so one grid serves all of them. */
} gfk_integration;

/* fk.Grid (internal/fk/fk.go:446-449). */
typedef struct gfk_grid {
    double kmax;
    int32_t samples;
    int32_t _pad;
} gfk_grid;

typedef struct gfk_solve {
    int32_t formulation;  /* enum gfk_formulation */
    int32_t quadrature;   /* enum gfk_quadrature */
    int32_t guard;        /* nonzero applies the MaxLayerPhase refusal; forced on by
                             GFK_REFERENCE_DIRECT */
    int32_t _pad;
    double omega_imag;    /* complex-frequency offset w_I (rad/s): every frequency is
                             evaluated at w - i*w_I. Must be 0 for GFK_REFERENCE_DIRECT. */
} gfk_solve;

/* ---- context -------------------------------------------------------------- */
typedef struct gfk_ctx gfk_ctx;

/* Creates a context on CUDA device `device`: one stream; device buffers come
 * from the device's stream-ordered memory pool, kept cached between calls. */
int gfk_open(int device, gfk_ctx **out);
/* Destroys the context and any of its plans still open (their handles
 * become invalid). */
int gfk_close(gfk_ctx *ctx);
/* Short name of a status code. */
const char *gfk_status_string(int status);
/* Full message of the context's last failure, worded like the Go error. */
const char *gfk_last_error(const gfk_ctx *ctx);
/* Number of libgfk kernels launched by this context since it was opened. */
int64_t gfk_kernel_launches(const gfk_ctx *ctx);
/* No counterpart in the reference (Go calls are synchronous): the CUDA stream
 * (a cudaStream_t, non-blocking) every call of this context is queued on, so
 * a caller can order its own device work and timing events with libgfk's. */
void *gfk_stream(const gfk_ctx *ctx);
/* No counterpart in the reference: a self-test of the bounded device waits.
 * Launches the tensor-core wavenumber sum on one 128 x 128 x 64 tile with its
 * producer told to issue no loads, so the MMA issuer's wait runs out after
 * wait_cycles SM clocks (use a few million: ~1-2 ms). The kernel then drains,
 * frees its tensor memory, exits and marks the tile's 64 rows timed out, as a
 * real stall would. Returns GFK_ETIMEOUT with *rows_timed_out = 64 when the
 * timeout was detected and reported; GFK_OK (0 rows) would mean the wait did
 * not run out. The context stays usable afterwards. */
int gfk_selftest_wait_timeout(gfk_ctx *ctx, int64_t wait_cycles, int32_t *rows_timed_out);

/* ---- host-only helpers (no device work) ---------------------------------- */
/* layer.Stack.Validate (internal/layer/layer.go:53-73). */
int gfk_stack_validate(const gfk_medium *m);
/* Medium.checkLayerPhase (internal/fk/fk.go:251-266): GFK_EGUARD past the limit. */
int gfk_check_layer_phase(const gfk_medium *m, double freq_hz);
/* Medium.GridFor (internal/fk/fk.go:464-495). */
int gfk_grid_for(const gfk_medium *m, const double *ranges_m, int32_t nr,
                 double freq_hz, gfk_integration opt, gfk_grid *out);

/* ---- the path ------------------------------------------------------------- */
/* Medium.SurfaceResponse (internal/fk/fk.go:276-327), batched over n (k, f)
 * pairs. out holds n complex values as (re, im) pairs. */
int gfk_surface_response(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                         const double *k, const double *freq_hz, int64_t n,
                         double *out);

/* Medium.StaticCoefficient (internal/fk/fk.go:365-371). out: one (re, im). */
int gfk_static_coefficient(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                           double freq_hz, double k_far, double *out);

/* Medium.VerticalDisplacement (internal/fk/fk.go:396-443). out: one (re, im). */
int gfk_vertical_displacement(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                              double range_m, double freq_hz, gfk_integration opt,
                              double *out);

/* Medium.VerticalDisplacementMulti (internal/fk/fk.go:506-550): one frequency,
 * nr ranges. out: nr (re, im) pairs. */
int gfk_vertical_displacement_multi(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                                    const double *ranges_m, int32_t nr, double freq_hz,
                                    gfk_integration opt, double *out);

/* The bank build's per-bin loop (cmd/geobank/main.go:133-167) as one call:
 * VerticalDisplacementMulti at nf frequencies. out: [nf][nr] (re, im) pairs.
 * status_per_f (may be NULL): per-frequency status; the call returns the first
 * non-OK one in frequency order, as geobank aborts on its first error
 * (cmd/geobank/main.go:143-150,168-170). Results of failed frequencies are 0. */
int gfk_bank_spectra(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                     const double *ranges_m, int32_t nr,
                     const double *freqs_hz, int32_t nf, gfk_integration opt,
                     double *out, int32_t *status_per_f);

/* The same build ending in the bank file's payload (cmd/geobank/main.go:116-121,
 * 133-167; internal/bank/format.go:185-193): the
 * spectra of bins first_bin .. first_bin + nf - 1 (frequencies freqs_hz) are
 * packed on the device into the float32 range-major payload, [nr][bins]
 * (re, im) pairs, and only that is downloaded: half the bytes of the FP64
 * result and no host-side packing. Other bins and failed frequencies hold
 * zeros. payload: host, 2 * nr * bins floats. Statuses as gfk_bank_spectra. */
int gfk_bank_payload(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                     const double *ranges_m, int32_t nr, const double *freqs_hz, int32_t nf,
                     gfk_integration opt, int32_t first_bin, int32_t bins, float *payload,
                     int32_t *status_per_f);

/* ---- plans: device-resident repeated builds ------------------------------ */
/* A plan fixes (medium, solve, ranges, frequencies, integration) and owns the
 * device buffers; executing it recomputes everything (layer constants, static
 * coefficients, propagators, J0 table, quadrature) on the context's stream with
 * no host transfers. Used by the benchmark and by callers that keep results in
 * device memory. */
typedef struct gfk_plan gfk_plan;
int gfk_plan_create(gfk_ctx *ctx, const gfk_medium *m, const gfk_solve *s,
                    const double *ranges_m, int32_t nr,
                    const double *freqs_hz, int32_t nf, gfk_integration opt,
                    gfk_plan **out);
int gfk_plan_execute(gfk_plan *p);
/* Device pointer to the [nf][nr] complex128 result of the last execute. */
int gfk_plan_result_device(gfk_plan *p, const double **d_out);
/* Copies the result (and per-frequency status) of the last execute to the host. */
int gfk_plan_download(gfk_plan *p, double *out, int32_t *status_per_f);
/* Execute, then download, as the two calls above, except that into
 * page-locked `out` a plan of several row chunks copies each chunk's rows out
 * on a second stream while the next chunk computes (the execute then runs as
 * separate launches, not as the plan's CUDA graph). Same results, statuses
 * and zeroed failed rows as gfk_plan_execute + gfk_plan_download. */
int gfk_plan_execute_download(gfk_plan *p, double *out, int32_t *status_per_f);
/* Number of kernel launches one execute performs (after the first, which
 * also runs the propagator tuning below). */
int32_t gfk_plan_launches_per_execute(const gfk_plan *p);
/* The plan's first execute times each launch shape of the Dunkin propagator
 * (gfk_prop_shape) on a window of up to 1024 of its own frequencies and keeps
 * the fastest; the context remembers the choice
 * per (layer count, wavenumber count) for later plans and calls. The
 * environment variable GFK_PROP_VARIANT=<index> forces one instead. Writes the chosen index and up
 * to `capacity` measured times (ms); returns the number of shapes. */
int gfk_plan_tuning(const gfk_plan *p, int32_t *variant, float *ms_per_variant, int32_t capacity);
/* Launch shape `variant` of the Dunkin propagator: threads per block, the
 * blocks per SM it is compiled for, wavenumbers per thread at a time, runs of
 * `threads` wavenumbers per work item, and whether it is persistent (one
 * block per resident slot taking (row, run) items from a device queue in row
 * order; otherwise one item per block). GFK_EARG for an unknown index. */
int gfk_prop_shape(int32_t variant, int32_t *threads, int32_t *blocks_per_sm, int32_t *wavenumbers_per_thread,
                   int32_t *runs_per_item, int32_t *persistent);
/* The tensor-core sum's tile shape (GFK_SPLIT_INT8 on a shared grid): the
 * plan's first execute times each shape (ranges per CTA: 128 or 64; pipeline
 * stages: 2-4) on its first row chunk and keeps the fastest; the context
 * remembers the choice per padded (rows, ranges, wavenumbers).
 * GFK_QUAD_TC_VARIANT=<index> forces one. Writes the chosen shape (0 and 0
 * before the first execute or for other sums) and up to `capacity` measured
 * times (ms); returns the number of shapes timed. */
int gfk_plan_quad_shape(const gfk_plan *p, int32_t *tile_n, int32_t *stages, float *ms_per_shape,
                        int32_t capacity);
/* Average duration in ms of the dominant kernel (the quadrature or the
 * propagator, whichever took longer) over the executes since the last reset,
 * timed with CUDA events on the plan's stream; name receives its label. */
int gfk_plan_kernel_times(gfk_plan *p, double *prop_ms, double *quad_ms,
                          double *other_ms, int32_t reset);
int gfk_plan_destroy(gfk_plan *p);
/* enable != 0: from the second execute on, the whole execute (every launch of
 * every row chunk) is one CUDA graph, captured once and relaunched. */
int gfk_plan_use_graph(gfk_plan *p, int32_t enable);

/* A plan over many media at once — the batched form of cmd/geobank's loop
 * (cmd/geobank/main.go:133-167) across soils: medium i contributes the rows
 * (medium i, freqs_hz[i][0..nf[i])). Rows are ordered medium by medium; the
 * result of gfk_plan_download is [sum nf][nr] (re, im) pairs in that order,
 * with per-row status. A medium that fails validation marks its rows and
 * takes no device work. All media share the ranges and the integration. */
int gfk_batch_create(gfk_ctx *ctx, const gfk_medium *media, int32_t nsoil,
                     const double *const *freqs_hz, const int32_t *nf,
                     const gfk_solve *s, const double *ranges_m, int32_t nr,
                     gfk_integration opt, gfk_plan **out);

/* ---- allocation-free variant --------------------------------------------- */
/* No counterpart in the reference: a gfk_vertical_displacement_multi for
 * callers that cannot allocate device memory when they need a response — a
 * process whose device memory another framework's caching allocator has
 * already claimed, or a deadline-bound loop (a sensor node emitting fixed
 * chunks) where cudaMalloc/cudaFree can synchronise the device. It performs no
 * device, stream-ordered or host heap allocation: its device working memory is
 * one 4 MiB array compiled into libgfk, which every GPU that loads the library
 * holds until exit. Limits: nr <= GFK_NOALLOC_MAX_RANGES ranges and a grid of
 * at most GFK_NOALLOC_MAX_SAMPLES wavenumbers; larger requests return
 * GFK_ELIMIT. Inputs and the output (nr (re, im) pairs) are host memory; the
 * work runs on `stream` (a cudaStream_t, NULL for the default stream) of the
 * current device and the call returns after it completes. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that
 * device current; make it before any stream capture begins. The address is
 * kept per device together with the ID of the CUDA context it belongs to, so
 * after a cudaDeviceReset (a new primary context) the next call looks it up
 * again and is a first call in that respect too. All calls share the array,
 * so calls whose GPU work overlaps race and must be serialised by the caller.
 * Statuses as gfk_vertical_displacement_multi; on any failure after the
 * device work, out holds zeros, as a failed frequency does there. No message
 * is kept. */
#define GFK_NOALLOC_MAX_RANGES 16384
#define GFK_NOALLOC_MAX_SAMPLES 196608
int gfk_vertical_displacement_multi_noalloc(const gfk_medium *m, const gfk_solve *s,
                                            const double *ranges_m, int32_t nr, double freq_hz,
                                            gfk_integration opt, double *out, void *stream);

/* ---- bank file (internal/bank/format.go:32-46, 215-240) ------------------ */
/* Packs an FP64 [nf][nr] result into the bank's float32 payload: range-major
 * [count][bins] (re, im) pairs with bin = first_bin + f index; bins outside
 * [first_bin, first_bin+nf) stay zero (cmd/geobank/main.go:116-121,161-165).
 * Host memory in and out; payload has 2*count*bins floats. */
int gfk_bank_pack(const double *spectra, int32_t nf, int32_t nr,
                  int32_t first_bin, int32_t bins, float *payload);
/* Writes magic "GEOBANK\0", uint32 version 1, uint32 header length, the JSON
 * header, zero padding to a 4096-byte boundary, then the little-endian payload. */
int gfk_bank_write(const char *path, const char *header_json,
                   const float *payload, int64_t nfloats);

/* ---- finite-difference validator (internal/fdtd) ------------------------ */
/* fdtd.Model (internal/fdtd/model.go:30-100): the stack (medium.layers), the
 * optional standard linear solid (medium.sls_tau_sigma/eps; zero: elastic),
 * its reference frequency (medium.ref_freq_hz, <= 0: 30 Hz), the domain and
 * the grid; pml_cells <= 0: 20, pml_reflection <= 0: 1e-4, dominant_freq_hz
 * <= 0: from the slowest velocity, courant <= 0: 0.5. */
typedef struct gfk_fdtd_model {
    gfk_medium medium;
    double max_range_m;
    double depth_m;
    double spacing_m;
    int32_t pml_cells;
    int32_t _pad;
    double pml_reflection;
    double dominant_freq_hz;
    double courant;
} gfk_fdtd_model;
/* New's grid (fdtd.go:45-64): the time step and the cell counts including
 * the absorbing layers. Host only. */
int gfk_fdtd_grid(const gfk_fdtd_model *m, double *dt, int32_t *nr, int32_t *nz);
/* fdtd.Run (internal/fdtd/run.go:78-127): `steps` steps of the axisymmetric
 * velocity-stress scheme driven by a vertical surface force (force[n] newtons
 * at step n, zero past nforce), recording the free-surface vertical velocity
 * (fdtd.go:330-345) at the grid columns nearest `ranges` into traces
 * [nrcv][steps] (host). snapped (host, nrcv, may be NULL) receives the column
 * ranges; meta (host, 5): dt, t0 (= dt/2, the velocities' time offset), the
 * largest particle speed seen, nr, nz. GFK_ENONFINITE with the reference's
 * message when the run diverges; GFK_EARG for a receiver outside the
 * interior or non-positive steps, spacing or domain. */
int gfk_fdtd_run(gfk_ctx *ctx, const gfk_fdtd_model *m, const double *force, int32_t nforce,
                 const double *ranges_m, int32_t nrcv, int32_t steps, double *traces, double *snapped,
                 double *meta);

/* ---- Rayleigh dispersion (internal/propmat, internal/disp) ---------------- */
/* disp.Search (internal/disp/disp.go:30-54): samples <= 0 uses 2000 (at most
 * 16384), tolerance <= 0 uses 1e-10. */
typedef struct gfk_search {
    int32_t samples;
    int32_t _pad;
    double tolerance;
} gfk_search;
/* disp.Modes (internal/disp/disp.go:68-103) at nf frequencies: every Rayleigh
 * phase velocity of the lossless stack (Vp, Vs, density and thicknesses; Q is
 * ignored, as propmat's secular function is real), slowest first, found by
 * scanning propmat.SecularAtVelocity (internal/propmat/propmat.go:265-320) on
 * the disp.Bounds interval and bisecting each sign change. velocities:
 * [nf][max_modes] host doubles, counts: [nf] modes found. GFK_ESTACK for a
 * stack layer.Stack.Validate refuses, GFK_EARG for a non-positive frequency,
 * GFK_ELIMIT (counts still filled, velocities truncated) when a frequency has
 * more than max_modes (<= 64) modes. */
int gfk_dispersion_modes(gfk_ctx *ctx, const gfk_medium *m, const double *freqs_hz, int32_t nf,
                         gfk_search opt, int32_t max_modes, double *velocities, int32_t *counts);
/* propmat.SecularAtVelocity at n (frequency, phase velocity) pairs: out[i] the
 * normalised secular value, ok[i] 0 where the reference returns an error or a
 * non-finite value (phase velocity not below the half-space's Vs). */
int gfk_secular(gfk_ctx *ctx, const gfk_medium *m, const double *freqs_hz, const double *velocities,
                int64_t n, double *out, int32_t *ok);

/* ---- bank consumption (internal/bank/interp.go, internal/dsp/dsp.go) ----- */
/* Bank.prepare (internal/bank/interp.go:66-102): the FP64 log-magnitude and
 * range-unwrapped phase tables of a bank payload, float32 (re, im) pairs
 * [count][bins] (range-major, as in the file). An exact zero has
 * log-magnitude -1e308 and keeps the running phase. Host arrays in and out,
 * count*bins doubles each. */
int gfk_bank_tables(gfk_ctx *ctx, const float *payload, int32_t count, int32_t bins,
                    double *logmag, double *phase);
/* The causal impulse responses a sensor engine builds from a bank
 * (internal/sensing/sensing.go:196-204 with propagation.go:84-104): at each of
 * nq ranges, Bank.Response (interp.go:29-54, bracket format.go:295-309) on
 * every bin k = 1..samples/2, times i 2 pi f_k when velocity is nonzero, times
 * sensor[k] (host, bins complex (re, im) pairs) when sensor is not NULL, fed to
 * dsp.CausalImpulseResponseAt (dsp.go:232-261) with the transform size
 * `samples` (the bank's): tapered above 0.8 Nyquist, inverse real transform
 * scaled 1/samples, first `length` samples kept. The grid is
 * [min_m, max_m] with `count` ranges; bins must be samples/2 + 1, samples a
 * power of two <= 4096 (GFK_ELIMIT above). A range outside the grid is
 * GFK_EARG with the reference's message. out: host [nq][length] doubles. */
int gfk_bank_impulse_responses(gfk_ctx *ctx, const float *payload, int32_t count, int32_t bins,
                               double min_m, double max_m, double fs_hz, int32_t samples,
                               const double *ranges_m, int32_t nq, const double *sensor,
                               int32_t velocity, int32_t length, double *out);

/* A bank kept on the device for repeated queries: internal/sensing loads a
 * bank once and asks it for responses contact after contact
 * (sensing.go:196-204 over bank.Open, format.go:249-286), so the payload is
 * uploaded and Bank.prepare's tables built once here (same argument rules as
 * gfk_bank_impulse_responses), and each query call moves only its ranges in
 * and its responses out. The handle belongs to ctx (freed by gfk_close if not
 * closed before). */
typedef struct gfk_bank_dev gfk_bank_dev;
int gfk_bank_device_open(gfk_ctx *ctx, const float *payload, int32_t count, int32_t bins, double min_m,
                         double max_m, double fs_hz, int32_t samples, gfk_bank_dev **out);
/* gfk_bank_impulse_responses against an open bank. out_on_device nonzero: out
 * is a device pointer of nq * length doubles on the context's device; zero: out
 * is host memory (pinned is fastest). Either way the call returns with the
 * responses written. */
int gfk_bank_device_impulse_responses(gfk_bank_dev *b, const double *ranges, int32_t nq, const double *sensor,
                                      int32_t velocity, int32_t length, double *out, int32_t out_on_device);
int gfk_bank_device_close(gfk_bank_dev *b);

/* ---- sweep metrics of geophone traces ------------------------------------ */
/* For each of ns soils, the geophone trace synthesised from its displacement
 * spectrum and its two sweep metrics (internal/sweep/sweep.go:128-169 Measure:
 * peak |y| and the |Y|-weighted spectral centroid over the band). d_G is a
 * device array of (re, im) pairs: soil s's bins k = 1..nbins at
 * d_G[2 (s stride + k - 1)]. shaping holds the n/2+1 complex factors S_k the
 * spectrum is multiplied by (velocity per newton, sensor response, taper
 * above 0.8 Nyquist and the footstep's spectrum; internal/geophone/
 * geophone.go:175-203, internal/dsp/dsp.go:232-261, internal/grf/grf.go:
 * 280-330), computed by the caller at w_c = 2 pi f - i omega_imag; the trace
 * is irfft(G S, n) e^(omega_imag t). n must be 1024. Band bins are
 * [k_lo, k_hi]. peak and centroid are host arrays of ns doubles. */
int gfk_trace_metrics(gfk_ctx *ctx, const double *d_G, int64_t stride, int32_t ns, int32_t nbins,
                      const double *shaping, int32_t n, double fs_hz, double omega_imag,
                      int32_t k_lo, int32_t k_hi, double *peak, double *centroid);

/* ---- ensemble gate for surrogate answers ---------------------------------- */
/* No counterpart in the reference. For E predicted spectra of ns soils
 * (device arrays of (re, im) pairs, soil s's bins k = 1..nbins at
 * d_members[e][2 (s stride + k - 1)]): d_mean (device, [ns][nbins] pairs)
 * receives their mean; flags (host, [ns][nbins] bytes) marks the rows whose
 * ensemble disagreement, weighted by the trace shaping |S_k| (the factors of
 * gfk_trace_metrics, n/2 + 1 = nbins + 1 pairs, host), exceeds threshold times
 * the peak of |mean S| over the soil's bins, and, when amp_threshold > 0, the
 * rows whose |mean S_k| itself exceeds amp_threshold times that peak (the
 * energetic rows, re-solved even where the members agree); spread (host, ns)
 * receives each soil's largest disagreement ratio. E <= 16. */
int gfk_ensemble_gate(gfk_ctx *ctx, const double *const *d_members, int32_t E, int64_t stride,
                      int32_t ns, int32_t nbins, const double *shaping, double threshold, double amp_threshold,
                      double *d_mean, uint8_t *flags, double *spread);
/* d_dst[2 index[i]] <- d_src[2 i src_stride] (re, im pairs), i < n; index host,
 * the pointers device memory. Puts solved rows back into a spectrum buffer. */
int gfk_scatter_rows(gfk_ctx *ctx, const double *d_src, int64_t src_stride, const int64_t *index,
                     int64_t n, double *d_dst);

/* ---- surrogate network ---------------------------------------------------- */
/* No counterpart in the reference (it has no learned component). A small
 * network maps (soil, range, frequency) to the vertical displacement spectrum
 * as t0 = log|G| and t1 = -phi/(w r), phi the phase unwrapped along range like
 * internal/bank/interp.go:66-102: 128 input features, five SiLU layers of
 * width 512 and a 2-wide FP32 output layer. BF16 weights and activations,
 * FP32 accumulation, FP32 master weights and AdamW moments; every step runs
 * libgfk's own forward, backward and optimiser kernels and is replayed as
 * one CUDA graph.
 *
 * A soil is given as up to GFK_NET_MAX_SOIL scalars, already mapped to
 * [-1, 1] by the caller, plus GFK_NET_TIMES vertical travel times in seconds
 * (thickness / Vs and thickness / Vp of up to three layers; 0 where unused):
 * the features carry sin, cos(2 pi f T) and log(f T) of each, which place the
 * layer resonances. The other features are range and frequency and 47
 * Fourier pairs of them.
 *
 * A data set holds the labels of nsoil soils over one range and frequency
 * grid in device memory, filled from device banks the solver produced. */
typedef struct gfk_dataset gfk_dataset;
typedef struct gfk_net gfk_net;

#define GFK_NET_MAX_SOIL 11
#define GFK_NET_TIMES 6
#define GFK_NET_WIDTH 512
#define GFK_NET_INPUTS 128

/* Loss per sample, on the standardised errors e0 (log-amplitude) and e1
 * (phase slowness): c0 e0^2 + c1 e1^2 with
 *   GFK_LOSS_PLAIN:   c0 = 1, c1 = phase_weight;
 *   GFK_LOSS_COMPLEX: c0 = w, c1 = phase_weight w min((w_f r std1/std0)^2,
 *                     phase_cap), w = max(|G|^2 / max_f |G(r, .)|^2,
 *                     weight_floor) — the squared error of G itself relative
 *                     to the spectral peak at that range, phase in radians;
 *   GFK_LOSS_AMPLITUDE: c0 = v, c1 = phase_weight v, v = max(|G| / max_f
 *                     |G(r, .)|, weight_floor).
 * c1 = 0 where the phase is not learnt. */
enum gfk_loss_mode { GFK_LOSS_PLAIN = 0, GFK_LOSS_COMPLEX = 1, GFK_LOSS_AMPLITUDE = 2 };

typedef struct {
    int32_t nsoil_scalars;  /* soil scalars per soil, <= GFK_NET_MAX_SOIL */
    int32_t batch;          /* rows per step, a multiple of 128 */
    int32_t warmup_steps;   /* linear warm-up, then cosine decay ... */
    int32_t total_steps;    /* ... to lr_min at this step */
    float lr_max, lr_min;
    float beta1, beta2, eps, weight_decay;
    float phase_weight;
    float fourier_sigma;    /* std of the Fourier frequencies, cycles per domain */
    int32_t loss_mode;      /* enum gfk_loss_mode */
    float weight_floor;     /* GFK_LOSS_COMPLEX: smallest amplitude weight */
    float phase_cap;        /* GFK_LOSS_COMPLEX: cap on the phase error's scale */
    int32_t _pad;
    uint64_t seed;          /* initial weights, Fourier frequencies, batches */
} gfk_net_config;

/* Labels are built from banks with an amplitude floor floor_rel times the
 * soil's largest |G|: t0 is clamped at the floor, and a cell's phase is not
 * learnt once its unwrapping chain has met a cell below it. nr <= 128.
 * soil_times: [nsoil][GFK_NET_TIMES] or NULL (all zero). */
int gfk_dataset_create(gfk_ctx *ctx, int32_t nsoil_scalars, int32_t nsoil, const double *soil_scalars,
                       const double *soil_times, const double *ranges_m, int32_t nr, const double *freqs_hz,
                       int32_t nf, double floor_rel, gfk_dataset **out);
/* Labels of soils [first_soil, first_soil + nsoil) from the device bank d_G
 * [nsoil][nf][nr] (re, im) pairs (gfk_plan_result_device of a batch plan). */
int gfk_dataset_fill(gfk_dataset *ds, const double *d_G, int32_t first_soil, int32_t nsoil);
/* Sums over the filled soils: cells, sum t0, sum t0^2, phase cells, sum t1,
 * sum t1^2. */
int gfk_dataset_stats(gfk_dataset *ds, double out[6]);
/* One soil's labels, host [nr][nf][2] floats (NaN where the phase is not learnt). */
int gfk_dataset_labels(gfk_dataset *ds, int32_t soil, float *out);
int gfk_dataset_destroy(gfk_dataset *ds);

int gfk_net_create(gfk_ctx *ctx, const gfk_net_config *cfg, gfk_net **out);
/* The input domain (range and frequency spans the features are scaled on)
 * and the target standardisation y = (t - mean) / std: mean_std =
 * {mean0, std0, mean1, std1}. Set before training or prediction. */
int gfk_net_set_scales(gfk_net *net, double r_lo, double r_hi, double f_lo, double f_hi,
                       const float mean_std[4]);
/* `steps` optimiser steps on batches drawn uniformly from the cells of the
 * listed soils. loss (optional, host [steps][2]) receives each step's
 * coefficient-weighted mean squared errors of the two standardised targets. */
int gfk_net_train(gfk_net *net, gfk_dataset *ds, const int32_t *train_soils, int32_t ntrain,
                  int32_t steps, float *loss);
/* As gfk_net_train, drawing only from the data set's ranges [first_range,
 * first_range + nranges): a network that serves one sensor range (the Sobol
 * workload's 10 m) spends its capacity there. */
int gfk_net_train_ranges(gfk_net *net, gfk_dataset *ds, const int32_t *train_soils, int32_t ntrain,
                         int32_t first_range, int32_t nranges, int32_t steps, float *loss);
/* G for ns soils at every (frequency, range) pair: out[2 ((s nf + j) nr + i)]
 * (re, im). out is device memory when out_on_device is nonzero. soil_times
 * as in gfk_dataset_create. */
int gfk_net_predict(gfk_net *net, const double *soil_scalars, const double *soil_times, int32_t ns,
                    const double *ranges_m, int32_t nr, const double *freqs_hz, int32_t nf, double *out,
                    int32_t out_on_device);
/* Held-out error against the data set's labels for the listed soils, over the
 * data set's grid: out = {cells, sum e0^2, phase cells, sum e1^2,
 * sum (e1 w r)^2, sum |G_pred - G|^2, sum |G|^2}. */
int gfk_net_evaluate(gfk_net *net, gfk_dataset *ds, const int32_t *soils, int32_t ns, double out[7]);
int64_t gfk_net_param_count(const gfk_net *net);
/* Get (set = 0) or set (set != 0) the FP32 master parameters, n floats:
 * W1 [512][128], b1, W2..W5 [512][512] and their biases, W6 [2][512], b6 [2]. */
int gfk_net_params(gfk_net *net, float *host, int64_t n, int32_t set);
/* Get or set the 47 x 2 Fourier frequencies. */
int gfk_net_fourier(gfk_net *net, float *host, int32_t set);
/* One forward and backward pass on a given batch without an update, for
 * gradient checks: X host [batch][128] features, Y host [batch][2]
 * standardised targets (NaN: no phase term), coeffs host [batch][2] loss
 * coefficients (c0, c1) or NULL for (1, phase_weight). grad receives the
 * gradient of (1/batch) sum c0 e0^2 + c1 e1^2 (layout of gfk_net_params),
 * loss the two coefficient-weighted mean squared errors. */
int gfk_net_probe(gfk_net *net, const float *X, const float *Y, const float *coeffs, float *grad,
                  float loss[2]);
int gfk_net_destroy(gfk_net *net);

#ifdef __cplusplus
}
#endif
#endif /* GFK_H */
