// gfk_noalloc.cu — a VerticalDisplacementMulti that allocates nothing.
//
// Some callers cannot allocate device memory at the time they need a
// response: a process whose device memory has been claimed up front by
// another framework's caching allocator (a cudaMalloc there fails or fights
// that pool), and latency-bound loops, such as a sensor node producing fixed
// chunks on a deadline, where cudaMalloc/cudaFree can synchronise the device
// and stall every other stream. This entry point serves them: all the device
// memory it uses is one fixed array compiled into the library, so a call does
// no cudaMalloc, cudaFree or stream-ordered allocation, and no host heap
// allocation either.
//
// The array is a file-scope __device__ buffer of kNoallocScratchBytes (4 MiB).
// Every GPU that loads libgfk holds it until the process exits, and every call
// on a device shares it, so calls whose GPU work overlaps — on two streams, or
// from two host threads — race on it and must be serialised by the caller.
// Host code may not use the array's name as a device address; the address is
// looked up once per device with cudaGetSymbolAddress, with that device
// current, by the first call made on it. Make that first call before any
// stream capture begins. The address belongs to the device's current CUDA
// context: if the caller resets the device (cudaDeviceReset) or otherwise
// replaces its primary context, the next call sees a new context ID and looks
// the address up again, so that call is a first call too.
#include <cuda.h>

#include <cstddef>
#include <cstring>
#include <mutex>

#include "../../include/gfk.h"
#include "gfk_kernels.cuh"

namespace {

constexpr size_t kNoallocScratchBytes = size_t(4) << 20;

// Layout of the scratch array (offsets in bytes, each 256-aligned).
constexpr size_t kOffLayersP = 0;                                                  // LayerP[64]
constexpr size_t kOffLayersC = 4096;                                               // LayerC[64]
constexpr size_t kOffScalars = kOffLayersC + 64 * sizeof(gfk::LayerC);             // medium, row, scalars
constexpr size_t kOffRanges = kOffScalars + 256;                                   // double[nr]
constexpr size_t kOffG = kOffRanges + size_t(GFK_NOALLOC_MAX_RANGES) * 8;          // cd[nr]
constexpr size_t kOffRem = kOffG + size_t(GFK_NOALLOC_MAX_RANGES) * 16;            // cd[nk]
static_assert(kOffRem + size_t(GFK_NOALLOC_MAX_SAMPLES) * 16 <= kNoallocScratchBytes, "scratch too small");
static_assert(64 * sizeof(gfk::LayerP) <= kOffLayersC, "layer block too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Per-call values, copied into the scratch array's scalar block.
struct Scalars {
    gfk::MediumP medium;
    gfk::FreqDesc row;
    int status;
    int pad;
    cd wc2, C;
};
static_assert(sizeof(Scalars) <= 256, "scalar block too small");
static_assert(offsetof(Scalars, row) % 8 == 0 && offsetof(Scalars, wc2) % 8 == 0, "alignment");

std::mutex g_setup_mu;
void* g_scratch_addr[256] = {nullptr};            // device address of the array, per device ordinal
unsigned long long g_scratch_ctx[256] = {0};      // ID of the context that address belongs to

// The current context's unique ID (cuCtxGetId, through the runtime's driver
// entry points, so libgfk needs no -lcuda); 0 when there is none or the
// driver cannot say.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    struct Entry {
        GetCurrent get_current = nullptr;
        GetId get_id = nullptr;
    };
    static const Entry e = [] {  // looked up once, thread-safely (a function-local static)
        Entry r;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            r.get_current = reinterpret_cast<GetCurrent>(p);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            r.get_id = reinterpret_cast<GetId>(p);
        return r;
    }();
    const GetCurrent get_current = e.get_current;
    const GetId get_id = e.get_id;
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// The array's device address on `device` (current): looked up with
// cudaGetSymbolAddress on the first call in a context, then reused while
// that context stays current.
int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= 256) return GFK_ECUDA;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[device] || ctx == 0 || ctx != g_scratch_ctx[device]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return GFK_ECUDA;
        g_scratch_addr[device] = ptr;
        g_scratch_ctx[device] = current_context_id();  // the lookup makes the primary context current
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return GFK_OK;
}

constexpr double kTwoPi = 6.283185307179586476925286766559;

}  // namespace

extern "C" int gfk_vertical_displacement_multi_noalloc(const gfk_medium* m, const gfk_solve* s,
                                                       const double* ranges_m, int32_t nr, double freq_hz,
                                                       gfk_integration opt, double* out, void* stream) {
    if (!m || !s || !out || !ranges_m) return GFK_EARG;
    if (nr <= 0) return GFK_EARG;
    if (nr > GFK_NOALLOC_MAX_RANGES) return GFK_ELIMIT;
    if (s->formulation != GFK_REFERENCE_DIRECT && s->formulation != GFK_DUNKIN) return GFK_EARG;
    if (s->quadrature != GFK_PLAIN_FP64) return GFK_EARG;
    if (s->formulation == GFK_REFERENCE_DIRECT && s->omega_imag != 0) return GFK_EARG;
    if (!(s->omega_imag >= 0) || !(s->omega_imag < INFINITY)) return GFK_EARG;
    if (!m->layers || m->count <= 0) return GFK_ESTACK;
    if (m->count > gfk::kMaxLayers) return GFK_ELIMIT;
    // the reference's order: guard, grid, then the stack (fk.go:507-523, 280)
    if (s->guard || s->formulation == GFK_REFERENCE_DIRECT) {
        int st = gfk_check_layer_phase(m, freq_hz);
        if (st) return st;
    }
    gfk_grid g;
    int st = gfk_grid_for(m, ranges_m, nr, freq_hz, opt, &g);
    if (st) return st;
    if (!(freq_hz > 0)) return GFK_EARG;
    st = gfk_stack_validate(m);
    if (st) return st;
    if (g.samples > GFK_NOALLOC_MAX_SAMPLES) return GFK_ELIMIT;

    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return GFK_ECUDA;
    unsigned char* base = nullptr;
    if ((st = scratch_address(device, &base))) return st;

    gfk::LayerP lp[gfk::kMaxLayers];
    double mu_ref = 0, slowest = m->layers[0].vs_mps, rmin = ranges_m[0];
    for (int i = 0; i < m->count; i++) {
        const gfk_layer& l = m->layers[i];
        lp[i] = gfk::LayerP{l.thickness_m, l.vp_mps, l.vs_mps, l.density_kgm3, l.qs, l.qp};
        mu_ref = fmax(mu_ref, l.density_kgm3 * l.vs_mps * l.vs_mps);
        slowest = fmin(slowest, l.vs_mps);
    }
    for (int j = 0; j < nr; j++) rmin = fmin(rmin, ranges_m[j]);
    Scalars sc{};
    sc.medium.ref_freq = m->ref_freq_hz;
    sc.medium.default_q = m->default_q;
    sc.medium.tau_sigma = m->sls_tau_sigma;
    sc.medium.tau_eps = m->sls_tau_eps;
    sc.medium.mu_ref = mu_ref;
    sc.medium.count = m->count;
    sc.medium.sls = (m->sls_tau_sigma > 0 && m->sls_tau_eps > 0) ? 1 : 0;
    sc.medium.lp_off = 0;
    sc.row.freq = freq_hz;
    sc.row.dk = g.kmax / g.samples;
    sc.row.kfar = fmax(200 * (kTwoPi * freq_hz / slowest), 400 / rmin);  // fk.go:515-521
    sc.row.off = 0;
    sc.row.lc_off = 0;
    sc.row.nk = g.samples;
    sc.row.soil = 0;
    sc.status = 0;  // the array keeps the last call's flags: cleared here

    auto* d_lp = reinterpret_cast<gfk::LayerP*>(base + kOffLayersP);
    auto* d_lc = reinterpret_cast<gfk::LayerC*>(base + kOffLayersC);
    unsigned char* sb = base + kOffScalars;
    auto* d_sc = reinterpret_cast<Scalars*>(sb);
    auto* d_medium = reinterpret_cast<gfk::MediumP*>(sb + offsetof(Scalars, medium));
    auto* d_row = reinterpret_cast<gfk::FreqDesc*>(sb + offsetof(Scalars, row));
    auto* d_status = reinterpret_cast<int*>(sb + offsetof(Scalars, status));
    auto* d_wc2 = reinterpret_cast<cd*>(sb + offsetof(Scalars, wc2));
    auto* d_C = reinterpret_cast<cd*>(sb + offsetof(Scalars, C));
    auto* d_r = reinterpret_cast<double*>(base + kOffRanges);
    auto* d_G = reinterpret_cast<cd*>(base + kOffG);
    auto* d_rem = reinterpret_cast<cd*>(base + kOffRem);

    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    ok(cudaMemcpyAsync(d_lp, lp, sizeof(gfk::LayerP) * m->count, cudaMemcpyHostToDevice, strm));
    ok(cudaMemcpyAsync(d_sc, &sc, sizeof sc, cudaMemcpyHostToDevice, strm));
    ok(cudaMemcpyAsync(d_r, ranges_m, sizeof(double) * nr, cudaMemcpyHostToDevice, strm));
    if (e != cudaSuccess) return GFK_ECUDA;
    const int form = s->formulation;
    gfk::launch_layer_consts(strm, d_lp, d_medium, d_row, 1, s->omega_imag, form, d_lc, d_wc2);
    gfk::launch_static(strm, d_lc, d_medium, d_row, d_wc2, 1, form, d_C, d_status);
    gfk::launch_prop(strm, d_lc, d_medium, d_row, d_wc2, 1, g.samples, d_C, form, d_rem, d_status);
    gfk::launch_quad_ragged(strm, d_rem, d_C, d_r, 1, nr, d_row, d_G);
    ok(cudaGetLastError());
    int flags = 0;
    ok(cudaMemcpyAsync(out, d_G, sizeof(cd) * nr, cudaMemcpyDeviceToHost, strm));
    ok(cudaMemcpyAsync(&flags, d_status, sizeof(int), cudaMemcpyDeviceToHost, strm));
    ok(cudaStreamSynchronize(strm));
    // a failed call leaves zeros in out, as gfk_vertical_displacement_multi
    // does for a failed frequency, never partial or non-finite values
    int result = GFK_OK;
    if (e != cudaSuccess) result = GFK_ECUDA;
    else if (flags & gfk::kStSingular) result = GFK_ESINGULAR;
    else if (flags & gfk::kStNonfinite) result = GFK_ENONFINITE;
    if (result != GFK_OK) std::memset(out, 0, sizeof(double) * 2 * (size_t)nr);
    return result;
}
