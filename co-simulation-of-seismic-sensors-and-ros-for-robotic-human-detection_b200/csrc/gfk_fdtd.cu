// gfk_fdtd.cu — the reference's axisymmetric finite-difference validator
// (internal/fdtd) on the GPU: a vertical point force on the free surface of a
// layered, optionally viscoelastic (one standard linear solid) half-space, in
// cylindrical coordinates, Virieux staggering, C-PML absorbing layers.
//
// What is restated, from internal/fdtd:
//   grid, time step, materials   fdtd.go:45-98, model.go:30-246 (host)
//   C-PML profiles                pml.go:30-70 (host), update pml.go:66-70
//   velocities                    fdtd.go:149-216
//   stresses and memory variables fdtd.go:218-320
//   surface velocity read-out     fdtd.go:330-345, Run's loop run.go:78-127
//
// Every phase of a step is a pure function of the previous phase's fields,
// so each is one kernel over the grid (thread per cell, rows of the grid
// contiguous): the velocity kernel also writes the prescribed surface
// traction for this step, and the stress kernel also records the receivers
// (their velocities are final by then). The arithmetic of every cell is the
// reference's, in the same order, except that divisions by the spacing, the
// radius and the density are multiplications by precomputed reciprocals (the
// same values to a rounding); FP64 throughout. Every 256 steps a max-speed
// reduction checks for divergence, as Run does.
#include <cmath>
#include <complex>
#include <string>
#include <vector>

#include <math_constants.h>

#include "../../include/gfk.h"
#include "gfk_ctx.h"
#include "gfk_kernels.cuh"

namespace gfk {
namespace fdtd {

struct Args {
    int nr, nz;
    double dr, dz, dt, src_area;
    bool lossy;
    double mem_decay, mem_drive;
    // materials per row; the time step over the densities, precomputed
    const double *rho, *lamU, *muU, *rhoZ, *muZ;
    const double *dt_rho, *dt_rhoZ;
    // reciprocal spacings and radii: 1 / dr, 1 / dz, 1 / ((i + 1/2) dr), 1 / (i dr)
    double idr, idz;
    const double *ir_half, *ir_int;
    // C-PML profiles (a, b) and the first damped index of each
    const double *aRi, *bRi, *aRh, *bRh, *aZi, *bZi, *aZh, *bZh;
    int fRi, fRh, fZi, fZh;
    // fields [nz][nr]
    double *vr, *vz, *trr, *tqq, *tzz, *trz;
    double *rrr, *rqq, *rzz, *rrz;
    double *psiTrrR, *psiTrzZ, *psiTrzR, *psiTzzZ, *psiVrR, *psiVzZ, *psiVzR, *psiVrZ;
    // receivers
    const int* cols;
    int nrcv, steps;
    double* traces;  // [nrcv][steps]
};

__device__ __forceinline__ double cpml(double* psi, double a, double b, double deriv) {
    const double p = b * *psi + a * deriv;
    *psi = p;
    return p;
}

__device__ __forceinline__ double relax(const Args& s, double* r, double e) {
    const double next = s.mem_decay * *r - s.mem_drive * e;
    const double avg = 0.5 * (*r + next);
    *r = next;
    return avg;
}

__global__ void k_velocities(Args s, double surface_traction) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= s.nr - 1 || j >= s.nz - 1) return;
    const int nr = s.nr;
    const int k = j * nr + i;
    // radial velocity
    {
        double dtrr = (s.trr[k + 1] - s.trr[k]) * s.idr;
        if (i >= s.fRh) dtrr += cpml(&s.psiTrrR[k], s.aRh[i], s.bRh[i], dtrr);
        double dtrz = j == 0 ? 2 * s.trz[k] * s.idz : (s.trz[k] - s.trz[k - nr]) * s.idz;
        if (j >= s.fZi) dtrz += cpml(&s.psiTrzZ[k], s.aZi[j], s.bZi[j], dtrz);
        const double hoop = 0.5 * ((s.trr[k] - s.tqq[k]) + (s.trr[k + 1] - s.tqq[k + 1])) * s.ir_half[i];
        s.vr[k] += s.dt_rho[j] * (dtrr + dtrz + hoop);
    }
    // vertical velocity
    {
        const double tzz_k = k == 0 ? surface_traction : s.tzz[k];
        if (k == 0) s.tzz[0] = surface_traction;  // fdtd.go:144
        double dtzz = (s.tzz[k + nr] - tzz_k) * s.idz;
        if (j >= s.fZh) dtzz += cpml(&s.psiTzzZ[k], s.aZh[j], s.bZh[j], dtzz);
        double radial;
        if (i == 0) {
            radial = 4 * s.trz[k] * s.idr;
        } else {
            double d = (s.trz[k] - s.trz[k - 1]) * s.idr;
            if (i >= s.fRi) d += cpml(&s.psiTrzR[k], s.aRi[i], s.bRi[i], d);
            radial = d + 0.5 * (s.trz[k] + s.trz[k - 1]) * s.ir_int[i];
        }
        s.vz[k] += s.dt_rhoZ[j] * (dtzz + radial);
    }
}

__device__ double surface_velocity(const Args& s, int i) {
    double dvr, vrr;
    if (i == 0) {
        dvr = 2 * s.vr[0] / s.dr;
        vrr = dvr;
    } else {
        dvr = (s.vr[i] - s.vr[i - 1]) / s.dr;
        vrr = 0.5 * (s.vr[i] + s.vr[i - 1]) / (double(i) * s.dr);
    }
    const double lam = s.lamU[0], mu = s.muU[0];
    const double dvz = -lam / (lam + 2 * mu) * (dvr + vrr);
    return s.vz[i] - 0.5 * s.dz * dvz;
}

__global__ void k_stresses(Args s, double dTdt, int step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.y == 0)
        for (int q = threadIdx.x; q < s.nrcv; q += blockDim.x)
            s.traces[(size_t)q * s.steps + step] = surface_velocity(s, s.cols[q]);
    if (i >= s.nr || j >= s.nz) return;
    const int nr = s.nr;
    const int k = j * nr + i;
    const double lam = s.lamU[j], mu = s.muU[j];
    const double lam2mu = lam + 2 * mu;
    // normal stresses
    double dvr, vrr;
    if (i == 0) {
        dvr = 2 * s.vr[k] * s.idr;
        vrr = dvr;
    } else {
        dvr = (s.vr[k] - s.vr[k - 1]) * s.idr;
        vrr = 0.5 * (s.vr[k] + s.vr[k - 1]) * s.ir_int[i];
    }
    if (i >= s.fRi) dvr += cpml(&s.psiVrR[k], s.aRi[i], s.bRi[i], dvr);
    double dvz;
    if (j == 0) {
        const double applied = i == 0 ? dTdt : 0.0;
        dvz = (applied - lam * (dvr + vrr)) / lam2mu;
    } else {
        dvz = (s.vz[k] - s.vz[k - nr]) * s.idz;
        if (j >= s.fZi) dvz += cpml(&s.psiVzZ[k], s.aZi[j], s.bZi[j], dvz);
    }
    const double err = lam2mu * dvr + lam * (vrr + dvz);
    const double eqq = lam * (dvr + dvz) + lam2mu * vrr;
    if (s.lossy) {
        s.trr[k] += s.dt * (err + relax(s, &s.rrr[k], err));
        s.tqq[k] += s.dt * (eqq + relax(s, &s.rqq[k], eqq));
    } else {
        s.trr[k] += s.dt * err;
        s.tqq[k] += s.dt * eqq;
    }
    if (j != 0) {
        const double ezz = lam * (dvr + vrr) + lam2mu * dvz;
        if (s.lossy)
            s.tzz[k] += s.dt * (ezz + relax(s, &s.rzz[k], ezz));
        else
            s.tzz[k] += s.dt * ezz;
    }
    // shear stress
    if (i < nr - 1 && j < s.nz - 1) {
        double dvzdr = (s.vz[k + 1] - s.vz[k]) * s.idr;
        if (i >= s.fRh) dvzdr += cpml(&s.psiVzR[k], s.aRh[i], s.bRh[i], dvzdr);
        double dvrdz = (s.vr[k + nr] - s.vr[k]) * s.idz;
        if (j >= s.fZh) dvrdz += cpml(&s.psiVrZ[k], s.aZh[j], s.bZh[j], dvrdz);
        const double e = s.muZ[j] * (dvzdr + dvrdz);
        if (s.lossy)
            s.trz[k] += s.dt * (e + relax(s, &s.rrz[k], e));
        else
            s.trz[k] += s.dt * e;
    }
}

// Block maxima of |vz| and |vr| (NaN propagates as NaN).
__global__ void k_maxspeed(const double* vz, const double* vr, long long n, double* out) {
    __shared__ double red[256];
    double m = 0.0;
    bool nan = false;
    for (long long q = blockIdx.x * 256LL + threadIdx.x; q < n; q += (long long)gridDim.x * 256) {
        const double a = fabs(vz[q]), b = fabs(vr[q]);
        nan |= isnan(a) || isnan(b);
        m = fmax(m, fmax(a, b));
    }
    red[threadIdx.x] = nan ? CUDART_NAN : m;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            const double x = red[threadIdx.x], y = red[threadIdx.x + w];
            red[threadIdx.x] = (isnan(x) || isnan(y)) ? CUDART_NAN : fmax(x, y);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

}  // namespace fdtd
}  // namespace gfk

namespace {

using cplx = std::complex<double>;

struct Sls {
    double ts = 0, te = 0;
    bool lossy() const { return te > ts; }
    double delta() const { return te / ts - 1; }
    cplx modulus(double f) const {  // visco.go:78-81
        const cplx w(0, 2 * M_PI * f);
        return (1.0 + w * te) / (1.0 + w * ts);
    }
    double relaxed_velocity(double v, double fref) const {  // visco.go:100-102
        return v * (1.0 / std::sqrt(modulus(fref))).real();
    }
};

struct Grid {
    int nr = 0, nz = 0, pml = 0;
    double h = 0, dt = 0, vmax = 0, dominant = 0, fref = 30, refl = 1e-4;
    Sls sls;
};

int ffail(gfk_ctx* ctx, int st, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return st;
}

const gfk_layer& layer_at(const gfk_medium& m, double z) {  // model.go:206-217
    double top = 0;
    for (int i = 0; i + 1 < m.count; i++) {
        top += m.layers[i].thickness_m;
        if (z < top) return m.layers[i];
    }
    return m.layers[m.count - 1];
}

int setup(gfk_ctx* ctx, const gfk_fdtd_model* md, Grid* g) {
    const gfk_medium& m = md->medium;
    if (!m.layers || m.count < 1) return ffail(ctx, GFK_ESTACK, "layer: empty stack");
    const int v = gfk_stack_validate(&m);
    if (v) return ffail(ctx, v, "layer: stack failed validation");
    if (!(md->spacing_m > 0)) return ffail(ctx, GFK_EARG, "fdtd: spacing must be positive");
    if (!(md->max_range_m > 0) || !(md->depth_m > 0)) return ffail(ctx, GFK_EARG, "fdtd: domain must be positive");
    g->sls.ts = m.sls_tau_sigma;
    g->sls.te = m.sls_tau_eps;
    if (g->sls.te < g->sls.ts)
        return ffail(ctx, GFK_EARG, "fdtd: TauEps must be at least TauSigma for a dissipative solid");
    g->fref = m.ref_freq_hz > 0 ? m.ref_freq_hz : 30.0;
    g->pml = md->pml_cells > 0 ? md->pml_cells : 20;
    g->refl = md->pml_reflection > 0 ? md->pml_reflection : 1e-4;
    const double courant = md->courant > 0 ? md->courant : 0.5;
    g->h = md->spacing_m;
    g->nr = (int)std::lround(md->max_range_m / g->h) + 1 + g->pml;
    g->nz = (int)std::lround(md->depth_m / g->h) + 1 + g->pml;
    double vmax = 0;  // model.go:219-233
    for (int i = 0; i < m.count; i++) {
        double vv = m.layers[i].vp_mps;
        if (g->sls.lossy()) vv = g->sls.relaxed_velocity(vv, g->fref) * std::sqrt(1 + g->sls.delta());
        vmax = std::max(vmax, vv);
    }
    g->vmax = vmax;
    g->dt = courant * (g->h / (vmax * M_SQRT2));
    if (md->dominant_freq_hz > 0) {
        g->dominant = md->dominant_freq_hz;
    } else {  // fdtd.go:106-117
        double slow = m.layers[0].vs_mps;
        for (int i = 0; i < m.count; i++) slow = std::min(slow, m.layers[i].vs_mps);
        if (g->sls.lossy()) slow = g->sls.relaxed_velocity(slow, g->fref);
        g->dominant = slow / (20 * g->h);
    }
    return GFK_OK;
}

struct Profile {
    std::vector<double> a, b;
    int first;
};

Profile profile(int n, double h, double offset, double inner, double thickness, double vmax, double refl,
                double dominant, double dt) {  // pml.go:30-62
    Profile p{std::vector<double>(n, 0.0), std::vector<double>(n, 1.0), n};
    if (thickness <= 0) return p;
    const double d0 = -(2 + 1) * vmax * std::log(refl) / (2 * thickness);
    const double amax = M_PI * dominant;
    for (int i = 0; i < n; i++) {
        const double s = (i + offset) * h - inner;
        if (s <= 0) continue;
        const double x = std::min(s / thickness, 1.0);
        const double d = d0 * std::pow(x, 2);
        const double alpha = amax * (1 - x);
        if (d + alpha <= 0) continue;
        const double b = std::exp(-(d + alpha) * dt);
        p.a[i] = d * (b - 1) / (d + alpha);
        p.b[i] = b;
        p.first = std::min(p.first, i);
    }
    return p;
}

}  // namespace

extern "C" {

int gfk_fdtd_grid(const gfk_fdtd_model* m, double* dt, int32_t* nr, int32_t* nz) {
    if (!m || !dt || !nr || !nz) return GFK_EARG;
    Grid g;
    const int st = setup(nullptr, m, &g);
    if (st) return st;
    *dt = g.dt;
    *nr = g.nr;
    *nz = g.nz;
    return GFK_OK;
}

int gfk_fdtd_run(gfk_ctx* ctx, const gfk_fdtd_model* md, const double* force, int32_t nforce, const double* ranges,
                 int32_t nrcv, int32_t steps, double* traces, double* snapped, double* meta) {
    if (!ctx || !md || (!force && nforce > 0) || (!ranges && nrcv > 0) || (!traces && nrcv > 0) || !meta)
        return GFK_EARG;
    Grid g;
    int st = setup(ctx, md, &g);
    if (st) return st;
    if (steps <= 0) return ffail(ctx, GFK_EARG, "fdtd: a shot needs a positive number of steps");
    const int nr = g.nr, nz = g.nz;
    const double h = g.h;
    std::vector<int> cols(std::max(nrcv, 1));
    for (int q = 0; q < nrcv; q++) {  // fdtd.go:135-139, run.go:90-96
        int c = (int)std::lround(ranges[q] / h);
        c = std::max(0, std::min(c, nr - 2));
        const double sn = c * h;
        if (sn >= md->max_range_m) {
            char buf[160];
            snprintf(buf, sizeof buf, "fdtd: receiver at %g m is outside the interior (%g m)", ranges[q],
                     md->max_range_m);
            return ffail(ctx, GFK_EARG, buf);
        }
        cols[q] = c;
        if (snapped) snapped[q] = sn;
    }
    // materials per row (model.go:150-204)
    const gfk_medium& m = md->medium;
    std::vector<double> rho(nz), lamU(nz), muU(nz), rhoZ(nz), muZ(nz);
    for (int j = 0; j < nz; j++) {
        const gfk_layer& l = layer_at(m, j * h);
        const double r = l.density_kgm3, vp = l.vp_mps, vs = l.vs_mps;
        double mp, ms;
        if (g.sls.lossy()) {
            const double cp = g.sls.relaxed_velocity(vp, g.fref), cs = g.sls.relaxed_velocity(vs, g.fref);
            mp = r * cp * cp * (1 + g.sls.delta());
            ms = r * cs * cs * (1 + g.sls.delta());
        } else {
            mp = r * vp * vp;
            ms = r * vs * vs;
        }
        rho[j] = r;
        muU[j] = ms;
        lamU[j] = mp - 2 * ms;
    }
    for (int j = 0; j < nz; j++) {
        const int k = std::min(j + 1, nz - 1);
        rhoZ[j] = 0.5 * (rho[j] + rho[k]);
        muZ[j] = (muU[j] <= 0 || muU[k] <= 0) ? 0.0 : 2 * muU[j] * muU[k] / (muU[j] + muU[k]);
    }
    const double thick = g.pml * h;
    const Profile pRi = profile(nr, h, 0, md->max_range_m, thick, g.vmax, g.refl, g.dominant, g.dt);
    const Profile pRh = profile(nr, h, 0.5, md->max_range_m, thick, g.vmax, g.refl, g.dominant, g.dt);
    const Profile pZi = profile(nz, h, 0, md->depth_m, thick, g.vmax, g.refl, g.dominant, g.dt);
    const Profile pZh = profile(nz, h, 0.5, md->depth_m, thick, g.vmax, g.refl, g.dominant, g.dt);

    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const size_t n = (size_t)nr * nz;
    std::vector<void*> owned;
    auto dev = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMallocAsync(&p, std::max<size_t>(bytes, 8), s) != cudaSuccess) return nullptr;
        owned.push_back(p);
        cudaMemsetAsync(p, 0, std::max<size_t>(bytes, 8), s);
        return p;
    };
    auto up = [&](const std::vector<double>& v) -> double* {
        double* p = static_cast<double*>(dev(v.size() * 8));
        if (p) cudaMemcpyAsync(p, v.data(), v.size() * 8, cudaMemcpyHostToDevice, s);
        return p;
    };
    auto cleanup = [&]() {
        for (void* p : owned) cudaFreeAsync(p, s);
        cudaStreamSynchronize(s);
    };
    gfk::fdtd::Args a{};
    a.nr = nr;
    a.nz = nz;
    a.dr = h;
    a.dz = h;
    a.dt = g.dt;
    a.src_area = M_PI * h * h / 4;
    a.lossy = g.sls.lossy();
    if (a.lossy) {  // fdtd.go:71-77
        const double tau = g.sls.ts, kappa = g.sls.delta() / (1 + g.sls.delta());
        const double den = 1 + g.dt / (2 * tau);
        a.mem_decay = (1 - g.dt / (2 * tau)) / den;
        a.mem_drive = (g.dt * kappa / tau) / den;
    }
    std::vector<double> dtr(nz), dtrz(nz), irh(nr), iri(nr, 0.0);
    for (int j = 0; j < nz; j++) {
        dtr[j] = g.dt / rho[j];
        dtrz[j] = g.dt / rhoZ[j];
    }
    for (int i = 0; i < nr; i++) {
        irh[i] = 1.0 / ((i + 0.5) * h);
        if (i > 0) iri[i] = 1.0 / (i * h);
    }
    a.idr = 1.0 / h;
    a.idz = 1.0 / h;
    a.dt_rho = up(dtr);
    a.dt_rhoZ = up(dtrz);
    a.ir_half = up(irh);
    a.ir_int = up(iri);
    a.rho = up(rho);
    a.lamU = up(lamU);
    a.muU = up(muU);
    a.rhoZ = up(rhoZ);
    a.muZ = up(muZ);
    a.aRi = up(pRi.a);
    a.bRi = up(pRi.b);
    a.aRh = up(pRh.a);
    a.bRh = up(pRh.b);
    a.aZi = up(pZi.a);
    a.bZi = up(pZi.b);
    a.aZh = up(pZh.a);
    a.bZh = up(pZh.b);
    a.fRi = pRi.first;
    a.fRh = pRh.first;
    a.fZi = pZi.first;
    a.fZh = pZh.first;
    double** fields[] = {&a.vr, &a.vz, &a.trr, &a.tqq, &a.tzz, &a.trz, &a.psiTrrR, &a.psiTrzZ, &a.psiTrzR,
                         &a.psiTzzZ, &a.psiVrR, &a.psiVzZ, &a.psiVzR, &a.psiVrZ};
    for (double** f : fields) *f = static_cast<double*>(dev(n * 8));
    if (a.lossy) {
        double** mem[] = {&a.rrr, &a.rqq, &a.rzz, &a.rrz};
        for (double** f : mem) *f = static_cast<double*>(dev(n * 8));
    }
    int* d_cols = static_cast<int*>(dev(cols.size() * sizeof(int)));
    double* d_traces = static_cast<double*>(dev((size_t)std::max(nrcv, 1) * steps * 8));
    const int nblk = 296;
    double* d_max = static_cast<double*>(dev(nblk * 8));
    for (void* p : owned)
        if (!p) {
            cleanup();
            return ffail(ctx, GFK_ENOMEM, "fdtd: device allocation failed");
        }
    cudaMemcpyAsync(d_cols, cols.data(), cols.size() * sizeof(int), cudaMemcpyHostToDevice, s);
    a.cols = d_cols;
    a.nrcv = nrcv;
    a.steps = steps;
    a.traces = d_traces;

    auto force_at = [&](int i) { return (i < 0 || i >= nforce) ? 0.0 : force[i]; };
    const dim3 blk(32, 8), grd((nr + 31) / 32, (nz + 7) / 8);
    double peak = 0;
    std::vector<double> mx(nblk);
    for (int step = 0; step < steps; step++) {  // fdtd.go:142-147, run.go:98-121
        gfk::fdtd::k_velocities<<<grd, blk, 0, s>>>(a, -force_at(step) / a.src_area);
        gfk::fdtd::k_stresses<<<grd, blk, 0, s>>>(a, (force_at(step + 1) - force_at(step)) / g.dt, step);
        ctx->launches += 2;
        if (step % 256 == 0) {
            gfk::fdtd::k_maxspeed<<<nblk, 256, 0, s>>>(a.vz, a.vr, (long long)n, d_max);
            ctx->launches++;
            if (cudaMemcpyAsync(mx.data(), d_max, nblk * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                cleanup();
                return ffail(ctx, GFK_ECUDA, "fdtd: step kernels failed");
            }
            double p = 0;
            bool bad = false;
            for (double x : mx) {
                bad |= std::isnan(x) || std::isinf(x);
                p = std::max(p, x);
            }
            peak = std::max(peak, p);
            if (bad) {
                cleanup();
                char buf[96];
                snprintf(buf, sizeof buf, "fdtd: diverged at step %d of %d", step, steps);
                return ffail(ctx, GFK_ENONFINITE, buf);
            }
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && nrcv > 0)
        e = cudaMemcpyAsync(traces, d_traces, (size_t)nrcv * steps * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cleanup();
    if (e != cudaSuccess) return ffail(ctx, GFK_ECUDA, std::string("fdtd: ") + cudaGetErrorString(e));
    meta[0] = g.dt;
    meta[1] = 0.5 * g.dt;
    meta[2] = peak;
    meta[3] = nr;
    meta[4] = nz;
    return GFK_OK;
}

}  // extern "C"
