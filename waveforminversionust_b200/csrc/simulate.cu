// RF simulation of Runtime/matlab/wust_simulate.m: the 2-D first-order
// k-space pseudospectral method of k-Wave (linear acoustics, scalar density,
// no absorption, Dirichlet pressure source, pressure sensors, PML outside
// the grid) for every transmitter of a record, batched on one GPU.
//
// The reference runs k-Wave's kspaceFirstOrder2D once per transmitter, or
// the vendored native solver (Runtime/third_party/kspaceFirstOrder-CUDA) over
// the batch.  Here all transmitters of a batch share one set of FFT plans and
// coefficient arrays and march together: the fields of S transmitters are S
// planes [x][y] (y fastest, the column-major layout of c(y, x)), and each
// time step is
//     P   = R2C(p)                                       S planes
//     G   = kappa D+ P / N     (y and x derivative)      2S planes, one kernel
//     g   = C2R(G)                                       2S planes
//     u   = pml_sg (pml_sg u - dt / rho0 g)             one kernel
//     U   = R2C(u)                                       2S planes
//     U  *= kappa D- / N                                 one kernel, in place
//     du  = C2R(U)                                       2S planes
//     rho = pml (pml rho - dt rho0 du); Dirichlet source; p = c^2 (rho_y +
//           rho_x); sensors recorded                     one kernel
// with the constants of the vendored solver (kappa = sinc(c_ref dt |k| / 2),
// D+- = i k exp(+-i k d / 2) on k-Wave's wavenumber vectors, PML factors
// exp(-dt / 2 * 2 * c_ref / d * (distance / pml)^4)).  The step is captured
// once into a CUDA graph (the time index lives on the device) and replayed.
// Optional FIR decimation of the records (downsampleKWaveChannelData.m:
// MATLAB resample(x, 1, q, 24, 8.6)) runs on the device at the end.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace wust {

namespace {

constexpr int kSimThreads = 256;

#define WUST_CUFFT(call)                                                                      \
    do {                                                                                      \
        cufftResult r_ = (call);                                                              \
        if (r_ != CUFFT_SUCCESS) ::wust::fail(WUST_ERR_CUDA, "%s failed (cuFFT %d)", #call, (int)r_); \
    } while (0)

struct SimGeom {
    int Ny, Nx;          // expanded grid
    int Nyh;             // Ny / 2 + 1 (R2C along y)
    int S;               // transmitters in the batch
    size_t plane, cplane;
};

struct SimCoefs {
    const float *kappa;          // [Nx][Nyh]
    const float2 *dyp, *dyn;     // [Nyh] i k_y exp(+-i k_y dy / 2)
    const float2 *dxp, *dxn;     // [Nx]
    const float *pmly, *pmly_sg; // [Ny]
    const float *pmlx, *pmlx_sg; // [Nx]
    const float *c2;             // [Nx][Ny]
    float inv_n;                 // 1 / (Ny Nx): cuFFT's inverse is unnormalised
    float dt_rho0, dt_over_rho0;
};

// k-Wave's wavenumber of index i of an axis of n points (ifftshifted
// -n/2 .. n/2-1 for even n, -(n-1)/2 .. (n-1)/2 for odd n).
double kwave_k(int i, int n, double d) {
    const int m = i <= (n - 1) / 2 ? i : i - n;
    return 2.0 * M_PI * m / (n * d);
}

double pml_value(int i, int n, int pml, double d, double dt, double c_ref, bool staggered) {
    const double a = -0.5 * dt * 2.0 * c_ref / d, sh = staggered ? 0.5 : 0.0;
    if (i < pml) return std::exp(a * std::pow((i + sh - pml) / (double)(-pml), 4));
    if (i >= n - pml) return std::exp(a * std::pow((i - (n - pml) + sh + 1.0) / pml, 4));
    return 1.0;
}

// G[0..S) = kappa D+_y P / N,  G[S..2S) = kappa D+_x P / N
__global__ void sim_grad_kernel(SimGeom g, SimCoefs k, const float2 *__restrict__ P, float2 *__restrict__ G) {
    const size_t total = (size_t)g.S * g.cplane;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t e = i % g.cplane;
        const int iy = (int)(e % g.Nyh), ix = (int)(e / g.Nyh);
        const float kap = k.kappa[e] * k.inv_n;
        const float2 v = make_float2(P[i].x * kap, P[i].y * kap);
        G[i] = cmul(v, k.dyp[iy]);
        G[i + (size_t)g.S * g.cplane] = cmul(v, k.dxp[ix]);
    }
}

// u_y, u_x from the pressure gradient (two planes of g per transmitter)
__global__ void sim_velocity_kernel(SimGeom g, SimCoefs k, const float *__restrict__ grad, float *__restrict__ u) {
    const size_t half = (size_t)g.S * g.plane;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
        const size_t e = i % g.plane;
        const int iy = (int)(e % g.Ny), ix = (int)(e / g.Ny);
        const float py = k.pmly_sg[iy], px = k.pmlx_sg[ix];
        u[i] = py * (py * u[i] - k.dt_over_rho0 * grad[i]);
        u[i + half] = px * (px * u[i + half] - k.dt_over_rho0 * grad[i + half]);
    }
}

// U_y *= kappa D-_y / N, U_x *= kappa D-_x / N (in place)
__global__ void sim_div_kernel(SimGeom g, SimCoefs k, float2 *__restrict__ U) {
    const size_t half = (size_t)g.S * g.cplane;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
        const size_t e = i % g.cplane;
        const int iy = (int)(e % g.Nyh), ix = (int)(e / g.Nyh);
        const float kap = k.kappa[e] * k.inv_n;
        const float2 a = U[i], b = U[i + half];
        U[i] = cmul(make_float2(a.x * kap, a.y * kap), k.dyn[iy]);
        U[i + half] = cmul(make_float2(b.x * kap, b.y * kap), k.dxn[ix]);
    }
}

// split densities, Dirichlet source, pressure, sensors; the time index is
// read from *tstep (advanced by sim_tick_kernel after the step)
__global__ void sim_density_kernel(SimGeom g, SimCoefs k, const float *__restrict__ du, float *__restrict__ rho,
                                   float *__restrict__ p, const int *__restrict__ src_at, const float *__restrict__ src,
                                   const int *__restrict__ rx_slot, int n_rx, int nt, const int *__restrict__ tstep,
                                   float *__restrict__ record) {
    const int t = *tstep;
    const size_t half = (size_t)g.S * g.plane;
    const float sv = t < nt ? src[t] : 0.f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < half; i += (size_t)gridDim.x * blockDim.x) {
        const size_t e = i % g.plane;
        const int s = (int)(i / g.plane);
        const int iy = (int)(e % g.Ny), ix = (int)(e / g.Ny);
        const float py = k.pmly[iy], px = k.pmlx[ix];
        float ry = py * (py * rho[i] - k.dt_rho0 * du[i]);
        float rx = px * (px * rho[i + half] - k.dt_rho0 * du[i + half]);
        const float c2 = k.c2[e];
        if ((int)e == src_at[s]) ry = rx = sv / (2.f * c2);
        rho[i] = ry;
        rho[i + half] = rx;
        const float pv = c2 * (ry + rx);
        p[i] = pv;
        const int r = rx_slot[e];
        if (r >= 0 && t < nt) record[((size_t)s * n_rx + r) * nt + t] = pv;
    }
}

__global__ void sim_tick_kernel(int *tstep) { *tstep += 1; }

// y[m] = sum_j h[j] x[m q + M - j] over each record (x zero outside)
__global__ void sim_decimate_kernel(const float *__restrict__ in, int nt, int n_tr, const float *__restrict__ h, int L,
                                    int q, int ly, float *__restrict__ out) {
    const size_t total = (size_t)n_tr * ly;
    const int M = (L - 1) / 2;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(i % ly);
        const size_t tr = i / ly;
        const float *x = in + tr * nt;
        double acc = 0.0;
        const int c = m * q + M;
        const int j0 = std::max(0, c - (nt - 1)), j1 = std::min(L - 1, c);
        for (int j = j0; j <= j1; ++j) acc += (double)h[j] * (double)x[c - j];
        out[i] = (float)acc;
    }
}

int sim_grid(size_t n) { return (int)std::min<size_t>((n + kSimThreads - 1) / kSimThreads, 148 * 16); }

}  // namespace

// Taps of MATLAB resample(., 1, q, half_length, beta): the least-squares
// ideal low-pass (the truncated sinc, cut-off pi / q), Kaiser window, unit DC
// gain.
static std::vector<float> decimation_taps(int q, int half_length, double beta) {
    const int L = 2 * half_length * q + 1, M = half_length * q;
    auto bessel_i0 = [](double x) {
        double sum = 1.0, term = 1.0;
        for (int k = 1; k < 200; ++k) {
            term *= (x / (2.0 * k)) * (x / (2.0 * k));
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        return sum;
    };
    std::vector<double> h(L);
    double total = 0.0;
    for (int j = 0; j < L; ++j) {
        const double k = j - M, arg = M_PI * k / q;
        const double sinc = k == 0 ? 1.0 : std::sin(arg) / arg;
        const double r = 2.0 * j / (L - 1) - 1.0;
        const double w = bessel_i0(beta * std::sqrt(std::max(0.0, 1.0 - r * r))) / bessel_i0(beta);
        h[j] = sinc / q * w;
        total += h[j];
    }
    std::vector<float> hf(L);
    for (int j = 0; j < L; ++j) hf[j] = (float)(h[j] / total);
    return hf;
}

void simulate_rf(const SimulateArgs &a, float *rf, cudaStream_t caller) {
    // the work runs on a stream of its own, ordered after the caller's stream
    // (which may be the legacy default stream, where a graph cannot be
    // captured); the call returns when it is done
    struct StreamGuard {
        cudaStream_t s = nullptr;
        cudaEvent_t e = nullptr;
        ~StreamGuard() {
            if (s) {
                cudaStreamSynchronize(s);
                cudaStreamDestroy(s);
            }
            if (e) cudaEventDestroy(e);
        }
    } own;
    WUST_CUDA(cudaStreamCreateWithFlags(&own.s, cudaStreamNonBlocking));
    WUST_CUDA(cudaEventCreateWithFlags(&own.e, cudaEventDisableTiming));
    WUST_CUDA(cudaEventRecord(own.e, caller));
    WUST_CUDA(cudaStreamWaitEvent(own.s, own.e, 0));
    cudaStream_t st = own.s;
    const int ny = a.ny, nx = a.nx, P = a.pml;
    SimGeom g{};
    g.Ny = ny + 2 * P;
    g.Nx = nx + 2 * P;
    g.Nyh = g.Ny / 2 + 1;
    g.plane = (size_t)g.Ny * g.Nx;
    g.cplane = (size_t)g.Nyh * g.Nx;
    const int ntx = a.ntx, nrx = a.nrx, nt = a.nt;
    const int S = std::max(1, std::min(a.tx_batch > 0 ? a.tx_batch : ntx, ntx));
    g.S = S;
    const int q = std::max(1, a.decimation);
    const int ly = (nt + q - 1) / q;

    // ---- coefficients (host, FP64, stored in float) -------------------------
    std::vector<float> kappa(g.cplane), pmly(g.Ny), pmlys(g.Ny), pmlx(g.Nx), pmlxs(g.Nx), c2(g.plane);
    std::vector<float2> dyp(g.Nyh), dyn(g.Nyh), dxp(g.Nx), dxn(g.Nx);
    for (int ix = 0; ix < g.Nx; ++ix) {
        const double kx = kwave_k(ix, g.Nx, a.dx);
        for (int iy = 0; iy < g.Nyh; ++iy) {
            const double ky = kwave_k(iy, g.Ny, a.dy);
            const double arg = 0.5 * a.c_ref * a.dt * std::sqrt(kx * kx + ky * ky);
            kappa[(size_t)ix * g.Nyh + iy] = (float)(arg == 0.0 ? 1.0 : std::sin(arg) / arg);
        }
        dxp[ix] = make_float2((float)(-kx * std::sin(kx * a.dx / 2)), (float)(kx * std::cos(kx * a.dx / 2)));
        dxn[ix] = make_float2((float)(kx * std::sin(kx * a.dx / 2)), (float)(kx * std::cos(kx * a.dx / 2)));
        pmlx[ix] = (float)pml_value(ix, g.Nx, P, a.dx, a.dt, a.c_ref, false);
        pmlxs[ix] = (float)pml_value(ix, g.Nx, P, a.dx, a.dt, a.c_ref, true);
    }
    for (int iy = 0; iy < g.Nyh; ++iy) {
        const double ky = kwave_k(iy, g.Ny, a.dy);
        dyp[iy] = make_float2((float)(-ky * std::sin(ky * a.dy / 2)), (float)(ky * std::cos(ky * a.dy / 2)));
        dyn[iy] = make_float2((float)(ky * std::sin(ky * a.dy / 2)), (float)(ky * std::cos(ky * a.dy / 2)));
    }
    for (int iy = 0; iy < g.Ny; ++iy) {
        pmly[iy] = (float)pml_value(iy, g.Ny, P, a.dy, a.dt, a.c_ref, false);
        pmlys[iy] = (float)pml_value(iy, g.Ny, P, a.dy, a.dt, a.c_ref, true);
    }
    // the medium extended with its edge values
    for (int ix = 0; ix < g.Nx; ++ix)
        for (int iy = 0; iy < g.Ny; ++iy) {
            const int sy = std::min(std::max(iy - P, 0), ny - 1), sx = std::min(std::max(ix - P, 0), nx - 1);
            const double c = a.c[sy + (size_t)ny * sx];
            c2[(size_t)ix * g.Ny + iy] = (float)(c * c);
        }
    std::vector<int> rx_slot(g.plane, -1), src_at_all(ntx);
    auto padded = [&](int lin1) {
        const int iy = (lin1 - 1) % ny, ix = (lin1 - 1) / ny;
        return (ix + P) * g.Ny + (iy + P);
    };
    for (int r = 0; r < nrx; ++r) rx_slot[padded(a.rx_index[r])] = r;
    for (int s = 0; s < ntx; ++s) src_at_all[s] = padded(a.tx_index[s]);
    std::vector<float> srcf(nt);
    for (int t = 0; t < nt; ++t) srcf[t] = (float)a.source[t];

    // ---- device buffers (one allocation) ----------------------------------
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_coef = al(g.cplane * 4) + 4 * al(std::max<size_t>(g.Nyh, g.Nx) * 8) + 2 * al(g.Ny * 4) +
                          2 * al(g.Nx * 4) + al(g.plane * 4) + al(g.plane * 4) + al(ntx * 4) + al(nt * 4) + 256;
    const size_t b_fields = al((size_t)S * g.plane * 4) * 7;            // p, u (2), rho (2), g/du (2)
    const size_t b_spec = al((size_t)S * g.cplane * 8) * 3;             // P (1), G/U (2)
    const size_t b_rec = al((size_t)S * nrx * nt * 4);
    std::vector<float> taps;
    if (q > 1) taps = decimation_taps(q, 24, 8.6);
    const size_t b_taps = al(taps.size() * 4 + 4);
    uint8_t *base = nullptr;
    WUST_CUDA(cudaMallocAsync(&base, b_coef + b_fields + b_spec + b_rec + b_taps, st));
    uint8_t *q8 = base;
    auto take = [&](size_t b) { uint8_t *r = q8; q8 += al(b); return r; };
    SimCoefs k{};
    float *d_kappa = (float *)take(g.cplane * 4);
    float2 *d_dyp = (float2 *)take(std::max<size_t>(g.Nyh, g.Nx) * 8), *d_dyn = (float2 *)take(std::max<size_t>(g.Nyh, g.Nx) * 8);
    float2 *d_dxp = (float2 *)take(std::max<size_t>(g.Nyh, g.Nx) * 8), *d_dxn = (float2 *)take(std::max<size_t>(g.Nyh, g.Nx) * 8);
    float *d_pmly = (float *)take(g.Ny * 4), *d_pmlys = (float *)take(g.Ny * 4);
    float *d_pmlx = (float *)take(g.Nx * 4), *d_pmlxs = (float *)take(g.Nx * 4);
    float *d_c2 = (float *)take(g.plane * 4);
    int *d_rxslot = (int *)take(g.plane * 4);
    int *d_srcat = (int *)take(ntx * 4);
    float *d_src = (float *)take(nt * 4);
    int *d_t = (int *)take(4);
    q8 = base + b_coef;
    float *d_p = (float *)take((size_t)S * g.plane * 4);
    float *d_u = (float *)take((size_t)2 * S * g.plane * 4);
    q8 = base + b_coef + al((size_t)S * g.plane * 4) * 3;
    float *d_rho = (float *)take((size_t)2 * S * g.plane * 4);
    q8 = base + b_coef + al((size_t)S * g.plane * 4) * 5;
    float *d_g = (float *)take((size_t)2 * S * g.plane * 4);
    q8 = base + b_coef + b_fields;
    float2 *d_P = (float2 *)take((size_t)S * g.cplane * 8);
    float2 *d_G = (float2 *)take((size_t)2 * S * g.cplane * 8);
    q8 = base + b_coef + b_fields + b_spec;
    float *d_rec = (float *)take((size_t)S * nrx * nt * 4);
    q8 = base + b_coef + b_fields + b_spec + b_rec;
    float *d_taps = (float *)take(taps.size() * 4 + 4);

    WUST_CUDA(cudaMemcpyAsync(d_kappa, kappa.data(), g.cplane * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_dyp, dyp.data(), g.Nyh * 8, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_dyn, dyn.data(), g.Nyh * 8, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_dxp, dxp.data(), g.Nx * 8, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_dxn, dxn.data(), g.Nx * 8, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_pmly, pmly.data(), g.Ny * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_pmlys, pmlys.data(), g.Ny * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_pmlx, pmlx.data(), g.Nx * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_pmlxs, pmlxs.data(), g.Nx * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_c2, c2.data(), g.plane * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_rxslot, rx_slot.data(), g.plane * 4, cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(d_src, srcf.data(), nt * 4, cudaMemcpyHostToDevice, st));
    if (q > 1) WUST_CUDA(cudaMemcpyAsync(d_taps, taps.data(), taps.size() * 4, cudaMemcpyHostToDevice, st));
    k.kappa = d_kappa;
    k.dyp = d_dyp; k.dyn = d_dyn; k.dxp = d_dxp; k.dxn = d_dxn;
    k.pmly = d_pmly; k.pmly_sg = d_pmlys; k.pmlx = d_pmlx; k.pmlx_sg = d_pmlxs;
    k.c2 = d_c2;
    k.inv_n = (float)(1.0 / ((double)g.Ny * g.Nx));
    k.dt_rho0 = (float)(a.dt * a.rho0);
    k.dt_over_rho0 = (float)(a.dt / a.rho0);

    // ---- FFT plans: S planes (p) and 2S planes (g, u) ----------------------
    cufftHandle fwd1 = 0, fwd2 = 0, inv2 = 0;
    int n2[2] = {g.Nx, g.Ny};
    struct PlanGuard {
        cufftHandle *h[3];
        uint8_t *mem;
        cudaStream_t st;
        ~PlanGuard() {
            for (auto p : h)
                if (*p) cufftDestroy(*p);
            if (mem) cudaFreeAsync(mem, st);
        }
    } guard{{&fwd1, &fwd2, &inv2}, base, st};
    WUST_CUFFT(cufftPlanMany(&fwd1, 2, n2, nullptr, 1, (int)g.plane, nullptr, 1, (int)g.cplane, CUFFT_R2C, S));
    WUST_CUFFT(cufftPlanMany(&fwd2, 2, n2, nullptr, 1, (int)g.plane, nullptr, 1, (int)g.cplane, CUFFT_R2C, 2 * S));
    WUST_CUFFT(cufftPlanMany(&inv2, 2, n2, nullptr, 1, (int)g.cplane, nullptr, 1, (int)g.plane, CUFFT_C2R, 2 * S));
    for (cufftHandle h : {fwd1, fwd2, inv2}) WUST_CUFFT(cufftSetStream(h, st));

    const int gp = sim_grid((size_t)S * g.plane), gc = sim_grid((size_t)S * g.cplane);
    for (int s0 = 0; s0 < ntx; s0 += S) {
        const int sb = std::min(S, ntx - s0);
        std::vector<int> src_at(S, -1);
        for (int s = 0; s < sb; ++s) src_at[s] = src_at_all[s0 + s];
        WUST_CUDA(cudaMemcpyAsync(d_srcat, src_at.data(), S * 4, cudaMemcpyHostToDevice, st));
        WUST_CUDA(cudaMemsetAsync(d_p, 0, al((size_t)S * g.plane * 4) * 7, st));   // p, u, rho, g
        WUST_CUDA(cudaMemsetAsync(d_t, 0, 4, st));
        if (q == 1) WUST_CUDA(cudaMemsetAsync(d_rec, 0, (size_t)S * nrx * nt * 4, st));
        auto step = [&]() {
            WUST_CUFFT(cufftExecR2C(fwd1, d_p, (cufftComplex *)d_P));
            sim_grad_kernel<<<gc, kSimThreads, 0, st>>>(g, k, d_P, d_G);
            WUST_CUFFT(cufftExecC2R(inv2, (cufftComplex *)d_G, d_g));
            sim_velocity_kernel<<<gp, kSimThreads, 0, st>>>(g, k, d_g, d_u);
            WUST_CUFFT(cufftExecR2C(fwd2, d_u, (cufftComplex *)d_G));
            sim_div_kernel<<<gc, kSimThreads, 0, st>>>(g, k, d_G);
            WUST_CUFFT(cufftExecC2R(inv2, (cufftComplex *)d_G, d_g));
            sim_density_kernel<<<gp, kSimThreads, 0, st>>>(g, k, d_g, d_rho, d_p, d_srcat, d_src, d_rxslot, nrx, nt,
                                                           d_t, d_rec);
            sim_tick_kernel<<<1, 1, 0, st>>>(d_t);
        };
        // one step captured as a graph and replayed; launched directly if the
        // capture is refused
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool graphed = false;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
        } else {
            bool recorded = true;
            try {
                step();
            } catch (const WustError &) {
                recorded = false;
            }
            if (cudaStreamEndCapture(st, &graph) == cudaSuccess && graph && recorded &&
                cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess)
                graphed = true;
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
        }
        for (int t = 0; t < nt; ++t) {
            if (graphed) WUST_CUDA(cudaGraphLaunch(exec, st));
            else step();
        }
        if (exec) cudaGraphExecDestroy(exec);
        g_kernel_launches += 5LL * nt;
        WUST_LAUNCH_CHECK();
        // records [s][r][t] -> rf [t][r][tx] column-major, i.e. memory [tx][r][t]
        float *dst = rf + (size_t)s0 * nrx * ly;
        if (q == 1) {
            WUST_CUDA(cudaMemcpyAsync(dst, d_rec, (size_t)sb * nrx * nt * 4, cudaMemcpyDeviceToDevice, st));
        } else {
            const size_t n_out = (size_t)sb * nrx * ly;
            sim_decimate_kernel<<<sim_grid(n_out), kSimThreads, 0, st>>>(d_rec, nt, sb * nrx, d_taps, (int)taps.size(),
                                                                          q, ly, dst);
            ++g_kernel_launches;
            WUST_LAUNCH_CHECK();
        }
    }
    WUST_CUDA(cudaStreamSynchronize(st));
}

}  // namespace wust
