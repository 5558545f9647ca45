// C ABI of libwust_b200: the HelmholtzSolver object, the two legacy
// MEX-equivalent entry points and the oracle/curvature drivers.
#include <cmath>
#include <limits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <vector>

#include <cufft.h>

#include "common.cuh"
#include "kernels.cuh"

namespace wust {

thread_local long long g_kernel_launches = 0;
static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }

void fail(int status, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw WustError{status, std::string(buf)};
}

template <typename F>
static int guarded(F &&f) {
    try {
        f();
        return WUST_OK;
    } catch (const WustError &e) {
        set_last_error(e.message);
        return e.status;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return WUST_ERR_RUNTIME;
    } catch (...) {
        set_last_error("unknown error");
        return WUST_ERR_RUNTIME;
    }
}

static bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

template <typename T>
static T *dalloc(size_t n) {
    T *p = nullptr;
    if (n == 0) n = 1;
    WUST_CUDA(cudaMalloc(&p, n * sizeof(T)));
    return p;
}

static void dfree(void *p) {
    if (p) cudaFree(p);
}

// Stage an input array: device pointers are used in place, host arrays are
// copied into `staging` (grown on demand).
template <typename T>
static const T *stage_in(const T *src, size_t n, T *&staging, size_t &cap, cudaStream_t st) {
    if (is_device_ptr(src)) return src;
    if (cap < n) {
        dfree(staging);
        staging = dalloc<T>(n);
        cap = n;
    }
    WUST_CUDA(cudaMemcpyAsync(staging, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
    return staging;
}

static void check_finite_range(const double *v, size_t n, const char *what) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) fail(WUST_ERR_INVALID_INPUT, "%s must be finite", what);
}

}  // namespace wust

using namespace wust;

// ---------------------------------------------------------------------------
// Solver object
// ---------------------------------------------------------------------------
struct wust_solver {
    int ny = 0, nx = 0, smax = 0, precision = 0, refine_max = 8;
    double refine_tol = 1e-5;
    int factor_method = WUST_FACTOR_DEFAULT;
    int max_ctas = 0;      // > 0: cooperative grids capped (a solver confined to part of the GPU)
    int chunk_count = 0;   // > 0: column chunks of the chunked sweeps
    int sweep_method = WUST_SWEEP_DEFAULT;
    // NCG update on the device: real 2-D FFT plans of the grid, half spectrum,
    // block partials of the reductions (created on first use)
    bool fft_ready = false;
    cufftHandle fft_fwd = 0, fft_inv = 0;
    double2 *spec = nullptr;
    double *ncg_part = nullptr;
    double f = 0, sgn = -1, a0 = 0, L = 0, vmin = 0, vmax = 0;
    int ldr9 = 0;
    double dt = 0, cr = 0;
    std::vector<double> xs, ys;
    double h = 0, g = 0, b = 0, d = 0, e = 0;
    cudaStream_t st = nullptr;
    int device = 0;
    // medium + assembly
    double *vel = nullptr, *atten = nullptr, *exi = nullptr, *eyi = nullptr;
    double2 *c128[9] = {};
    float2 *c64[9] = {};
    double2 *mult = nullptr;
    int *status = nullptr;            // 64 ints
    // factor
    float2 *invT = nullptr;
    void *fscratch = nullptr;
    size_t fscratch_bytes = 0;
    // sweeps
    float2 *u = nullptr, *lam = nullptr, *tmp = nullptr, *work = nullptr;
    double2 *x64 = nullptr, *x64b = nullptr;   // FP64 refinement iterates (alternating)
    double2 *x64_last = nullptr;                // the one holding the last refined solution
    double2 *w9f = nullptr, *w9a = nullptr;     // interleaved FP64 weights of H and H^H for the residuals
    float2 *r32 = nullptr, *d32 = nullptr;
    double *rnorm2 = nullptr, *bnorm2 = nullptr, *dnorm2 = nullptr, *xnorm2 = nullptr;
    // objective
    int32_t *tx_lin = nullptr, *rx_lin = nullptr, *rx_at = nullptr;
    int tx_cap = 0, rx_cap = 0;
    float2 *Yd = nullptr;
    uint8_t *maskd = nullptr;
    size_t obs_cap = 0;
    float2 *resid = nullptr;
    double2 *scale = nullptr;     // all transmitters
    double *loss_src = nullptr;   // all transmitters
    double *grad = nullptr;
    double *dir = nullptr;
    // retained curvature state: forward fields of all transmitters
    float2 *ret_u = nullptr;
    size_t ret_cap = 0;
    int ret_ntx = 0, ret_nrx = 0, ret_valid = 0;
    // host staging for pageable inputs
    double *stage_d = nullptr; size_t stage_d_cap = 0;
    // tensor-core sweeps (TF32 profile): packed invT / invT^H operands, packed
    // B chunks, split-K partial tiles, barrier counters, wait-site flag
    uint8_t *tc_afwd = nullptr, *tc_aadj = nullptr, *tc_b = nullptr;
    float *tc_part = nullptr;
    unsigned *tc_sync = nullptr;
    int *tc_err = nullptr;
    TcSweepGeom tc_geom{};
    // column-chunked tensor-core sweeps (TF32 profile, default): packed
    // -Lambda_c pages, per-group B chunks, chunk and boundary states, counters
    bool use_chunks = false;
    TcChunkGeom ck_geom{};
    uint8_t *ck_lpack = nullptr, *ck_b = nullptr;
    float *ck_z = nullptr, *ck_sb = nullptr;
    float2 *ck_edges = nullptr;
    unsigned *ck_sync = nullptr;
    // BF16 operands of the correction sweeps (TF32 profile, chunked sweeps),
    // or of every sweep (BF16 profile)
    int correction_precision = WUST_CORRECTION_DEFAULT;
    bool bf16_corrections = false;
    bool bf16_all = false;
    uint8_t *tc_afwd16 = nullptr, *tc_aadj16 = nullptr, *ck_lpack16 = nullptr;
    TcChunkBuffers chunk_buffers() const {
        return TcChunkBuffers{ck_lpack, ck_b, ck_lpack16, ck_z, ck_sb, ck_edges, ck_sync, tc_err};
    }
    // Newton-Schulz factorization (TF32 profile)
    void *ns_scratch = nullptr;
    int ns_head = 3;                  // pages inverted directly before the Newton-Schulz run (learned)
    NsGeom ns_g{};
    long long ns_stats[4] = {};       // GEMMs, X updates, Newton-Schulz pages, Gauss-Jordan pages
    int ns_cluster = -1;              // last factorization: 1 cluster launches, 0 classic, -1 none
    float2 *stage_c = nullptr; size_t stage_c_cap = 0;
    double assembly_ms = 0, factor_ms = 0;
    int last_refine_iters = 0;
    double last_residual = 0;
    double last_error_est = 0;
    long long launches = 0;
    cudaEvent_t ev[4] = {};
    // device time of every block-LU sweep pair (forward + backward) since creation
    cudaEvent_t sw_ev[2] = {};
    double sweep_ms = 0;
    long long sweeps = 0;

    Coefs<float2> coefs64() const {
        Coefs<float2> c;
        c.Dd = c64[0]; c.Dl = c64[1]; c.Du = c64[2]; c.Ld = c64[3]; c.Ll = c64[4]; c.Lu = c64[5];
        c.Ud = c64[6]; c.Ul = c64[7]; c.Uu = c64[8];
        c.ny = ny; c.nx = nx;
        return c;
    }
    Coefs<double2> coefs128() const {
        Coefs<double2> c;
        c.Dd = c128[0]; c.Dl = c128[1]; c.Du = c128[2]; c.Ld = c128[3]; c.Ll = c128[4]; c.Lu = c128[5];
        c.Ud = c128[6]; c.Ul = c128[7]; c.Uu = c128[8];
        c.ny = ny; c.nx = nx;
        return c;
    }
    size_t plane() const { return (size_t)ny * nx; }
};

static size_t coef_elems(int which, int ny, int nx) {
    switch (which) {
        case 0: return (size_t)ny * nx;               // Dd
        case 1: case 2: return (size_t)(ny - 1) * nx; // Dl Du
        case 3: case 6: return (size_t)ny * (nx - 1); // Ld Ud
        default: return (size_t)(ny - 1) * (nx - 1); // Ll Lu Ul Uu
    }
}

static const char *kCoefNames[9] = {"Dd", "Dl", "Du", "Ld", "Ll", "Lu", "Ud", "Ul", "Uu"};

static void free_solver(wust_solver *s) {
    if (!s) return;
    void *ptrs[] = {s->vel, s->atten, s->exi, s->eyi, s->mult, s->status, s->invT, s->fscratch, s->u, s->lam,
                    s->tmp, s->work, s->x64, s->x64b, s->w9f, s->w9a, s->r32, s->d32, s->rnorm2, s->bnorm2, s->dnorm2, s->xnorm2, s->tx_lin, s->rx_lin,
                    s->rx_at, s->Yd, s->maskd, s->resid, s->scale, s->loss_src, s->grad, s->dir, s->ret_u,
                    s->stage_d, s->stage_c, s->tc_afwd, s->tc_aadj, s->tc_b, s->tc_part, s->tc_sync, s->tc_err, s->ns_scratch,
                    s->ck_lpack, s->ck_b, s->ck_z, s->ck_sb, s->ck_edges, s->ck_sync,
                    s->tc_afwd16, s->tc_aadj16, s->ck_lpack16};
    for (void *p : ptrs) dfree(p);
    if (s->fft_ready) {
        cufftDestroy(s->fft_fwd);
        cufftDestroy(s->fft_inv);
    }
    dfree(s->spec);
    dfree(s->ncg_part);
    for (int i = 0; i < 9; ++i) { dfree(s->c128[i]); dfree(s->c64[i]); }
    for (auto &e : s->ev) if (e) cudaEventDestroy(e);
    for (auto &e : s->sw_ev) if (e) cudaEventDestroy(e);
    delete s;
}

// numpy.linspace semantics: start + i * step, last sample = stop
static std::vector<double> linspace(double a, double b, int n) {
    std::vector<double> v(n);
    const double step = (b - a) / (n - 1);
    for (int i = 0; i < n; ++i) v[i] = a + i * step;
    v[n - 1] = b;
    return v;
}

// The tensor-core profiles: Newton-Schulz TF32 Schur inverses and tcgen05
// sweeps (TF32 operands, BF16 for corrections by default; the BF16 profile
// puts every sweep on BF16 operands).
static bool tensor_profile(const wust_solver *s) {
    return s->precision == WUST_PRECISION_TF32_REFINED || s->precision == WUST_PRECISION_BF16_REFINED;
}

static void assemble_and_factor(wust_solver *s, const double *vel_in, const double *atten_in) {
    cudaStream_t st = s->st;
    const size_t N = s->plane();
    // medium
    if (is_device_ptr(vel_in)) WUST_CUDA(cudaMemcpyAsync(s->vel, vel_in, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else {
        check_finite_range(vel_in, N, "vel");
        for (size_t i = 0; i < N; ++i)
            if (!(vel_in[i] > 0)) fail(WUST_ERR_INVALID_INPUT, "Expected a positive finite [ny,nx] medium");
        WUST_CUDA(cudaMemcpyAsync(s->vel, vel_in, N * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    const double *atten_dev = nullptr;
    if (atten_in) {
        if (!s->atten) s->atten = dalloc<double>(N);
        WUST_CUDA(cudaMemcpyAsync(s->atten, atten_in, N * sizeof(double), cudaMemcpyDefault, st));
        atten_dev = s->atten;
    }
    // PML profiles (HelmholtzSolver.m:74-84), imaginary parts of ex / ey
    const double pi = 3.14159265358979323846;
    const double xmin = s->xs.front(), xmax = s->xs.back(), ymin = s->ys.front(), ymax = s->ys.back();
    auto prof = [&](double lo, double hi, int n) {
        std::vector<double> e = linspace(lo, hi, 2 * (n - 1) + 1);
        const double ctr = (lo + hi) / 2, span = (hi - lo) / 2;
        for (double &v : e) {
            const double t = std::fmax(std::fabs(v - ctr) - span + s->L, 0.0) / s->L;
            const double sx = 2 * pi * s->a0 * s->f * (t * t);
            v = sx * s->sgn / (2 * pi * s->f);
        }
        return e;
    };
    std::vector<double> exi = prof(xmin, xmax, s->nx), eyi = prof(ymin, ymax, s->ny);
    WUST_CUDA(cudaMemcpyAsync(s->exi, exi.data(), exi.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    WUST_CUDA(cudaMemcpyAsync(s->eyi, eyi.data(), eyi.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    stencil_opt_params(s->vmin, s->vmax, s->f, s->h, s->g, &s->b, &s->d, &s->e);

    AssemblyInput in;
    in.ny = s->ny; in.nx = s->nx; in.f = s->f; in.sgn = s->sgn; in.a0 = s->a0; in.L = s->L;
    in.xmin = xmin; in.xmax = xmax; in.ymin = ymin; in.ymax = ymax; in.h = s->h; in.g = s->g;
    in.b = s->b; in.d = s->d; in.e = s->e; in.ldr9 = s->ldr9; in.dt = s->dt; in.cr = s->cr;
    WUST_CUDA(cudaMemsetAsync(s->status, 0, 64 * sizeof(int), st));
    WUST_CUDA(cudaEventRecord(s->ev[0], st));
    assemble_launch(in, s->vel, atten_dev, s->exi, s->eyi, s->c128, s->c64, s->mult, s->status, st);
    if (s->w9f) refine_weights_launch(s->coefs128(), s->w9f, s->w9a, st);
    WUST_CUDA(cudaEventRecord(s->ev[1], st));
    int hstat[3] = {0, 0, 0};
    auto check_assembly = [&](int astat) {
        if (astat == 1) fail(WUST_ERR_INVALID_INPUT, "Expected a positive finite [ny,nx] medium");
        if (astat == 2) fail(WUST_ERR_INVALID_INPUT, "k-Wave local dispersion target is evanescent");
        if (astat == 3) fail(WUST_ERR_NUMERICAL_FAILURE, "LDR-9 produced invalid wavenumber or derivative");
    };
    if (tensor_profile(s) && s->ns_scratch) {
        // the iteration needs a valid operator: check the assembly first
        int astat0 = 0;
        WUST_CUDA(cudaMemcpyAsync(&astat0, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        check_assembly(astat0);
        for (long long &v : s->ns_stats) v = 0;
        s->ns_cluster = -1;
        ns_factor(s->coefs64(), s->invT, s->ns_g, s->ns_scratch, s->fscratch, s->fscratch_bytes, st, s->ns_stats,
                  &s->ns_head, s->max_ctas, &s->ns_cluster);
    } else {
        factor_launch(s->coefs64(), s->invT, s->fscratch, s->fscratch_bytes, st, 10.0, hstat, 0, -1, s->max_ctas);
    }
    if (tensor_profile(s)) {
        if (s->bf16_corrections && s->use_chunks && s->ck_geom.kc == s->tc_geom.kc && s->ck_geom.mt == s->tc_geom.mt)
            tc_pack_invT_both(s->invT, s->ny, s->nx, s->ck_geom, s->tc_afwd, s->tc_aadj, s->tc_afwd16, s->tc_aadj16, st);
        else {
            tc_pack_invT(s->invT, s->ny, s->nx, s->tc_geom, s->tc_afwd, s->tc_aadj, st);
            if (s->bf16_corrections) tc_pack_invT16(s->invT, s->ny, s->nx, s->ck_geom, s->tc_afwd16, s->tc_aadj16, st);
        }
        if (s->use_chunks) tc_chunk_prepare(s->coefs64(), s->tc_afwd, s->tc_aadj, s->ck_geom, s->chunk_buffers(), st);
    }
    WUST_CUDA(cudaEventRecord(s->ev[2], st));
    int astat = 0;
    WUST_CUDA(cudaMemcpyAsync(&astat, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    WUST_CUDA(cudaStreamSynchronize(st));
    float ms0 = 0, ms1 = 0;
    WUST_CUDA(cudaEventElapsedTime(&ms0, s->ev[0], s->ev[1]));
    WUST_CUDA(cudaEventElapsedTime(&ms1, s->ev[1], s->ev[2]));
    s->assembly_ms = ms0;
    s->factor_ms = ms1;
    s->ret_valid = 0;
    check_assembly(astat);
    if (hstat[2]) fail(WUST_ERR_DEVICE_TIMEOUT, "factorization grid barrier %d timed out", hstat[2]);
    if (hstat[0]) fail(WUST_ERR_SINGULAR_SCHUR_BLOCK, "Schur block %d is singular at pivot %d", hstat[0], hstat[1] + 1);
}

static void ensure_obs(wust_solver *s, int n_tx, int n_rx) {
    if (n_tx > s->tx_cap) {
        dfree(s->tx_lin); dfree(s->scale); dfree(s->loss_src);
        s->tx_lin = dalloc<int32_t>(n_tx);
        s->scale = dalloc<double2>(n_tx);
        s->loss_src = dalloc<double>(n_tx);
        s->tx_cap = n_tx;
    }
    if (n_rx > s->rx_cap) {
        dfree(s->rx_lin); dfree(s->resid);
        s->rx_lin = dalloc<int32_t>(n_rx);
        s->resid = dalloc<float2>((size_t)n_rx * s->smax);
        s->rx_cap = n_rx;
    }
    const size_t nobs = (size_t)n_tx * n_rx;
    if (nobs > s->obs_cap) {
        dfree(s->Yd); dfree(s->maskd);
        s->Yd = dalloc<float2>(nobs);
        s->maskd = dalloc<uint8_t>(nobs);
        s->obs_cap = nobs;
    }
}

// One sweep pair (forward+backward) with the profile's arithmetic: CUDA-core
// complex single, or tcgen05 GEMMs on the packed invT operands (TF32, or BF16
// when bf16 is set and the solver holds BF16 operands).
static void run_sweep(wust_solver *s, const SrcView &src, int S, bool adjoint, float2 *out, bool bf16 = false) {
    WUST_CUDA(cudaEventRecord(s->sw_ev[0], s->st));
    if (tensor_profile(s)) {
        bf16 = bf16 && s->tc_afwd16 != nullptr;
        if (s->use_chunks)
            tc_chunk_solve(s->coefs64(), bf16 ? s->tc_afwd16 : s->tc_afwd, bf16 ? s->tc_aadj16 : s->tc_aadj, s->ck_geom,
                           s->chunk_buffers(), src, S, adjoint, out, bf16, s->st);
        else
            tc_sweep_solve(s->coefs64(), s->tc_afwd, s->tc_aadj, s->tc_geom, src, S, adjoint, out, s->tc_b,
                           s->tc_part, s->tc_sync, s->tc_err, s->st);
    } else {
        sweep_solve(s->coefs64(), s->invT, src, S, adjoint, out, s->tmp, s->st);
    }
    WUST_CUDA(cudaEventRecord(s->sw_ev[1], s->st));
    WUST_CUDA(cudaEventSynchronize(s->sw_ev[1]));
    float ms = 0;
    WUST_CUDA(cudaEventElapsedTime(&ms, s->sw_ev[0], s->sw_ev[1]));
    s->sweep_ms += ms;
    ++s->sweeps;
}

static void check_tc_err(wust_solver *s) {
    if (!s->tc_err) return;
    int e = 0;
    WUST_CUDA(cudaMemcpyAsync(&e, s->tc_err, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    WUST_CUDA(cudaStreamSynchronize(s->st));
    if (e) {
        WUST_CUDA(cudaMemsetAsync(s->tc_err, 0, sizeof(int), s->st));
        fail(WUST_ERR_DEVICE_TIMEOUT, "tensor-core pipeline wait expired (code %d)", e);
    }
}

// One block-LU solve with optional FP64 iterative refinement.  out must
// differ from the dense source buffer.
//
// Refinement: x_0 = solve(b); r_k = b - H x_k in FP64; d_{k+1} = solve(r_k);
// x_{k+1} = x_k + d_{k+1}, with x_0 the solve's c64 output, later x in FP64
// (two buffers, one step's input and output) and, from the second
// correction on, each step's c64 copy in out.  The stopping rule is on the forward error: the
// correction d_k measures the error of x_{k-1}, and the residual ratio
// rho_k = |r_k| / |r_{k-1}| is the contraction of one step, so
// |e_k| / |x_k| ~ rho_k |d_k| / |x_k|.  Refinement stops when that estimate is
// below refine_tol for every source (the residual alone is already small for
// the unrefined c64 solution while its error is not).  In the bf16-refined
// profile the estimate is taken with a margin of 1.5: residual and error
// contract at different rates there, and on the textured 552^2 medium the
// true error of an adjoint solve was 1.17 times the estimate.  With a TF32
// first sweep (tf32-refined) the estimate has stayed above the measured error
// at 552^2 (errors of 1.5-2.8e-6 where refinement stopped below 1e-5), and a
// margin there adds a correction sweep on the homogeneous medium (measured:
// 100 ms per gradient instead of 85).
static void solve_into(wust_solver *s, const SrcView &src, int S, bool adjoint, float2 *out) {
    cudaStream_t st = s->st;
    run_sweep(s, src, S, adjoint, out, s->bf16_all);
    s->last_refine_iters = 0;
    s->last_residual = -1;
    s->last_error_est = -1;
    if (s->precision == WUST_PRECISION_C64) return;
    std::vector<double> rn(S), rn_prev(S), bn(S), dn(S), xn(S);
    // BF16 corrections (half the operand bytes) as long as they contract the
    // residual at least kBf16Contraction-fold per correction; a weaker step
    // (poorly conditioned operators, long chunks whose BF16 propagators lose
    // accuracy) turns the rest of this solve's corrections to TF32 operands
    constexpr double kBf16Contraction = 0.2;
    bool bf16_corr = s->bf16_all || s->bf16_corrections;
    SrcView dense{};
    dense.mode = SRC_DENSE;
    dense.dense = s->r32;
    double2 *xa = nullptr, *xb = s->x64;         // the current FP64 iterate (none yet) and the next one
    const RefineWeights rw{s->w9f, s->w9a, s->ny, s->nx};
    refine_first_launch(rw, src, out, S, adjoint, s->r32, s->rnorm2, s->bnorm2, st);
    WUST_CUDA(cudaMemcpyAsync(rn.data(), s->rnorm2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
    WUST_CUDA(cudaMemcpyAsync(bn.data(), s->bnorm2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
    WUST_CUDA(cudaStreamSynchronize(st));
    check_tc_err(s);
    for (int k = 1;; ++k) {
        if (k > s->refine_max)
            fail(WUST_ERR_NOT_CONVERGED, "refinement did not reach %.1e after %d correction solves (estimate %.3e)",
                 s->refine_tol, s->refine_max, s->last_error_est);
        rn_prev = rn;
        run_sweep(s, dense, S, adjoint, s->d32, bf16_corr);
        if (!xa) {
            refine_step_launch(rw, src, s->d32, out, nullptr, S, adjoint, xb, nullptr, s->r32, s->rnorm2, s->dnorm2,
                               s->xnorm2, st);
            xa = xb;
            xb = s->x64b;
        } else {
            refine_step_launch(rw, src, s->d32, nullptr, xa, S, adjoint, xb, out, s->r32, s->rnorm2, s->dnorm2,
                               s->xnorm2, st);
            std::swap(xa, xb);
        }
        s->x64_last = xa;
        WUST_CUDA(cudaMemcpyAsync(rn.data(), s->rnorm2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaMemcpyAsync(dn.data(), s->dnorm2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaMemcpyAsync(xn.data(), s->xnorm2, S * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        check_tc_err(s);
        double worst_err = 0, worst_res = 0, worst_rho = 0;
        for (int q = 0; q < S; ++q) {
            if (!(std::isfinite(rn[q]) && std::isfinite(dn[q]) && std::isfinite(xn[q])))
                fail(WUST_ERR_NUMERICAL_FAILURE, "non-finite refinement residual");
            const double rho = rn_prev[q] > 0 ? std::sqrt(rn[q] / rn_prev[q]) : 0.0;
            const double rel_d = xn[q] > 0 ? std::sqrt(dn[q] / xn[q]) : 0.0;
            worst_err = std::fmax(worst_err, std::fmin(rho, 1.0) * rel_d);
            worst_rho = std::fmax(worst_rho, rho);
            worst_res = std::fmax(worst_res, bn[q] > 0 ? std::sqrt(rn[q] / bn[q]) : std::sqrt(rn[q]));
        }
        s->last_refine_iters = k;
        s->last_residual = worst_res;
        s->last_error_est = worst_err;
        const double margin = s->bf16_all ? 1.5 : 1.0;
        if (margin * worst_err <= s->refine_tol) break;
        if (worst_rho > kBf16Contraction) bf16_corr = false;
    }
    if (s->last_refine_iters == 1) refine_demote_launch(xa, out, s->plane() * S, st);   // out still holds x_0
}

extern "C" {

const char *wust_status_id(int status) {
    switch (status) {
        case WUST_OK: return "WUST:OK";
        case WUST_ERR_INVALID_INPUT: return "WUST:InvalidInput";
        case WUST_ERR_INVALID_OUTPUT: return "WUST:InvalidOutput";
        case WUST_ERR_CUDA: return "WUST:CUDAError";
        case WUST_ERR_CUBLAS: return "WUST:CUBLASError";
        case WUST_ERR_CUSOLVER: return "WUST:CUSOLVERError";
        case WUST_ERR_SINGULAR_SCHUR_BLOCK: return "WUST:SingularSchurBlock";
        case WUST_ERR_INVALID_SOLVER_ARGUMENT: return "WUST:InvalidSolverArgument";
        case WUST_ERR_RESOURCE_CLEANUP: return "WUST:ResourceCleanup";
        case WUST_ERR_RUNTIME: return "WUST:RuntimeError";
        case WUST_ERR_NUMERICAL_FAILURE: return "WUST:NumericalFailure";
        case WUST_ERR_DEVICE_TIMEOUT: return "WUST:DeviceTimeout";
        case WUST_ERR_NOT_CONVERGED: return "WUST:RefinementNotConverged";
        default: return "WUST:Unknown";
    }
}

const char *wust_last_error(void) { return g_last_error.c_str(); }

int wust_version(int *major, int *minor, int *patch) {
    if (major) *major = 0;
    if (minor) *minor = 1;
    if (patch) *patch = 0;
    return WUST_OK;
}

int wust_decomp_block_lu(const wust_c64 *Ld, const wust_c64 *Ll, const wust_c64 *Lu, const wust_c64 *Dd,
                         const wust_c64 *Dl, const wust_c64 *Du, const wust_c64 *Ud, const wust_c64 *Ul,
                         const wust_c64 *Uu, int Ny, int Nx, wust_c64 *invT, float *total_gpu_ms, void *stream) {
    return guarded([&] {
        const wust_c64 *in[9] = {Dd, Dl, Du, Ld, Ll, Lu, Ud, Ul, Uu};
        for (const wust_c64 *p : in)
            if (!p || !is_device_ptr(p)) fail(WUST_ERR_INVALID_INPUT, "decompBlockLU requires 9 gpuArray inputs.");
        if (Ny < 3 || Nx < 2 || (long long)Ny * Nx > 2147483647LL)
            fail(WUST_ERR_INVALID_INPUT, "Block-LU grid must have an interior and fit int indexing.");
        if (!invT || !is_device_ptr(invT)) fail(WUST_ERR_INVALID_OUTPUT, "decompBlockLU requires a device invT output.");
        cudaStream_t st = (cudaStream_t)stream;
        Coefs<float2> co;
        co.Dd = (const float2 *)Dd; co.Dl = (const float2 *)Dl; co.Du = (const float2 *)Du;
        co.Ld = (const float2 *)Ld; co.Ll = (const float2 *)Ll; co.Lu = (const float2 *)Lu;
        co.Ud = (const float2 *)Ud; co.Ul = (const float2 *)Ul; co.Uu = (const float2 *)Uu;
        co.ny = Ny; co.nx = Nx;
        const size_t bytes = factor_scratch_bytes(Ny);
        void *scratch = nullptr;
        WUST_CUDA(cudaMalloc(&scratch, bytes));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        int hstat[3] = {0, 0, 0};
        try {
            if (total_gpu_ms) {
                WUST_CUDA(cudaEventCreate(&e0));
                WUST_CUDA(cudaEventCreate(&e1));
                WUST_CUDA(cudaEventRecord(e0, st));
            }
            factor_launch(co, (float2 *)invT, scratch, bytes, st, 10.0, hstat);
            if (total_gpu_ms) {
                WUST_CUDA(cudaEventRecord(e1, st));
                WUST_CUDA(cudaEventSynchronize(e1));
                WUST_CUDA(cudaEventElapsedTime(total_gpu_ms, e0, e1));
            }
        } catch (...) {
            cudaFree(scratch);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            throw;
        }
        cudaFree(scratch);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (hstat[2]) fail(WUST_ERR_DEVICE_TIMEOUT, "factorization grid barrier %d timed out", hstat[2]);
        if (hstat[0]) fail(WUST_ERR_SINGULAR_SCHUR_BLOCK, "getrf block %d is singular at pivot %d", hstat[0], hstat[1] + 1);
    });
}

int wust_apply_block_lu(const wust_c64 *src, int Ny, int Nx, int n_src, const wust_c64 *Ld, const wust_c64 *Ll,
                        const wust_c64 *Lu, const wust_c64 *Ud, const wust_c64 *Ul, const wust_c64 *Uu,
                        const wust_c64 *invT, int adjoint, wust_c64 *u, void *stream) {
    return guarded([&] {
        const void *in[8] = {src, Ld, Ll, Lu, Ud, Ul, Uu, invT};
        for (const void *p : in)
            if (!p || !is_device_ptr(p))
                fail(WUST_ERR_INVALID_INPUT, "applyBlockLU inputs 1-8 must be gpuArray; input 9 must be a logical scalar.");
        if (Ny < 2 || Nx < 2 || n_src < 1 || (long long)Ny * Nx * n_src > 2147483647LL)
            fail(WUST_ERR_INVALID_INPUT, "Expected complex-single GPU arrays with 2D blocks and 3D inverse blocks/RHS pages.");
        if (!u || !is_device_ptr(u)) fail(WUST_ERR_INVALID_OUTPUT, "applyBlockLU requires exactly one output.");
        cudaStream_t st = (cudaStream_t)stream;
        Coefs<float2> co{};
        co.Ld = (const float2 *)Ld; co.Ll = (const float2 *)Ll; co.Lu = (const float2 *)Lu;
        co.Ud = (const float2 *)Ud; co.Ul = (const float2 *)Ul; co.Uu = (const float2 *)Uu;
        co.ny = Ny; co.nx = Nx;
        float2 *tmp = nullptr;
        WUST_CUDA(cudaMalloc(&tmp, sizeof(float2) * (size_t)Ny * n_src));
        SrcView sv{};
        sv.mode = SRC_DENSE;
        sv.dense = (const float2 *)src;
        try {
            sweep_solve(co, (const float2 *)invT, sv, n_src, adjoint != 0, (float2 *)u, tmp, st);
            WUST_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            cudaFree(tmp);
            throw;
        }
        cudaFree(tmp);
    });
}

int wust_solver_create(wust_solver **out, const wust_solver_options *o, const double *vel, const double *atten,
                       void *stream) {
    wust_solver *s = nullptr;
    int rc = guarded([&] {
        if (!out || !o || !vel) fail(WUST_ERR_INVALID_INPUT, "Explicit backend and fixed stencil_bounds are required");
        *out = nullptr;
        if (!(std::isfinite(o->stencil_vmin) && std::isfinite(o->stencil_vmax) && o->stencil_vmin > 0 &&
              o->stencil_vmax > o->stencil_vmin))
            fail(WUST_ERR_INVALID_INPUT, "stencil_bounds must be a positive ordered [min,max] pair");
        if (o->ny < 3 || o->nx < 3 || !o->x_m || !o->y_m)
            fail(WUST_ERR_INVALID_INPUT, "Expected a positive finite [ny,nx] medium");
        if ((long long)o->ny * o->nx > 2147483647LL) fail(WUST_ERR_INVALID_INPUT, "grid exceeds int indexing");
        if (!(o->frequency_hz > 0) || !(o->pml_m > 0) || !std::isfinite(o->pml_strength))
            fail(WUST_ERR_INVALID_INPUT, "frequency, pml_m and pml_strength must be positive and finite");
        if (o->precision < 0 || o->precision > 3) fail(WUST_ERR_INVALID_INPUT, "unknown precision profile");
        if (o->dispersion && !(o->time_step_s > 0 && o->reference_speed_mps > 0))
            fail(WUST_ERR_INVALID_INPUT, "LDR9 requires explicit simulation dispersion facts");
        s = new wust_solver();
        s->ny = o->ny; s->nx = o->nx;
        s->smax = o->max_sources > 0 ? o->max_sources : 256;
        if (o->factor_method < WUST_FACTOR_DEFAULT || o->factor_method > WUST_FACTOR_GAUSS_JORDAN)
            fail(WUST_ERR_INVALID_INPUT, "unknown factor_method %d", o->factor_method);
        s->factor_method = o->factor_method;
        if (o->sweep_method < WUST_SWEEP_DEFAULT || o->sweep_method > WUST_SWEEP_SEQUENTIAL)
            fail(WUST_ERR_INVALID_INPUT, "unknown sweep_method %d", o->sweep_method);
        s->sweep_method = o->sweep_method;
        if (o->correction_precision < WUST_CORRECTION_DEFAULT || o->correction_precision > WUST_CORRECTION_SAME)
            fail(WUST_ERR_INVALID_INPUT, "unknown correction_precision %d", o->correction_precision);
        s->correction_precision = o->correction_precision;
        if (o->max_ctas < 0 || o->chunk_count < 0) fail(WUST_ERR_INVALID_INPUT, "max_ctas and chunk_count must be >= 0");
        s->max_ctas = o->max_ctas;
        s->chunk_count = o->chunk_count;
        s->precision = o->precision;
        s->refine_max = o->refine_max_iters > 0 ? o->refine_max_iters : 8;
        s->refine_tol = o->refine_tol > 0 ? o->refine_tol : 1e-5;
        s->f = o->frequency_hz;
        s->sgn = o->sign_convention >= 0 ? (o->sign_convention > 0 ? 1.0 : 0.0) : -1.0;
        s->a0 = o->pml_strength; s->L = o->pml_m; s->vmin = o->stencil_vmin; s->vmax = o->stencil_vmax;
        s->ldr9 = o->dispersion; s->dt = o->time_step_s; s->cr = o->reference_speed_mps;
        s->xs.assign(o->x_m, o->x_m + o->nx);
        s->ys.assign(o->y_m, o->y_m + o->ny);
        // HelmholtzSolver.m:49-58: uniform increasing grids; h = mean(diff(x)), g = mean(diff(y)) / h
        auto mean_diff = [](const std::vector<double> &v, const char *what) {
            double sum = 0;
            for (size_t i = 1; i < v.size(); ++i) {
                if (!(v[i] > v[i - 1])) fail(WUST_ERR_INVALID_INPUT, "Uniform increasing grids required (%s)", what);
                sum += v[i] - v[i - 1];
            }
            const double m = sum / (v.size() - 1);
            for (size_t i = 1; i < v.size(); ++i)
                if (std::fabs((v[i] - v[i - 1]) - m) >= m * 1e-7) fail(WUST_ERR_INVALID_INPUT, "Uniform increasing grids required");
            return m;
        };
        s->h = mean_diff(s->xs, "x");
        s->g = mean_diff(s->ys, "y") / s->h;
        if (s->ldr9 && std::fabs(s->g - 1) >= 1e-10) fail(WUST_ERR_INVALID_INPUT, "LDR9 requires square grid cells");
        WUST_CUDA(cudaGetDevice(&s->device));
        s->st = (cudaStream_t)stream;
        for (auto &e : s->ev) WUST_CUDA(cudaEventCreate(&e));
        for (auto &e : s->sw_ev) WUST_CUDA(cudaEventCreate(&e));
        const size_t N = s->plane();
        const int ny = s->ny, nx = s->nx;
        s->vel = dalloc<double>(N);
        s->exi = dalloc<double>(2 * nx);
        s->eyi = dalloc<double>(2 * ny);
        for (int i = 0; i < 9; ++i) {
            s->c128[i] = dalloc<double2>(coef_elems(i, ny, nx));
            s->c64[i] = dalloc<float2>(coef_elems(i, ny, nx));
        }
        s->mult = dalloc<double2>(N);
        s->status = dalloc<int>(64);
        s->invT = dalloc<float2>((size_t)ny * ny * nx);
        s->fscratch_bytes = factor_scratch_bytes(ny);
        WUST_CUDA(cudaMalloc(&s->fscratch, s->fscratch_bytes));
        const size_t F = N * s->smax;
        s->u = dalloc<float2>(F);
        s->lam = dalloc<float2>(F);
        s->work = dalloc<float2>(F);
        s->tmp = dalloc<float2>((size_t)ny * s->smax);
        s->grad = dalloc<double>(N);
        s->dir = dalloc<double>(N);
        s->rx_at = dalloc<int32_t>(N);
        if (s->precision != WUST_PRECISION_C64) {
            s->x64 = dalloc<double2>(F);
            s->x64b = dalloc<double2>(F);
            s->w9f = dalloc<double2>(9 * N);
            s->w9a = dalloc<double2>(9 * N);
            s->r32 = dalloc<float2>(F);
            s->d32 = dalloc<float2>(F);
            s->rnorm2 = dalloc<double>(s->smax);
            s->bnorm2 = dalloc<double>(s->smax);
            s->dnorm2 = dalloc<double>(s->smax);
            s->xnorm2 = dalloc<double>(s->smax);
        }
        if (s->precision == WUST_PRECISION_BF16_REFINED && s->sweep_method != WUST_SWEEP_DEFAULT)
            fail(WUST_ERR_INVALID_INPUT, "the BF16 profile runs on the column-chunked sweeps (sweep_method default)");
        if (tensor_profile(s)) {
            auto capped = [&](int device_max) { return s->max_ctas > 0 ? std::min(device_max, s->max_ctas) : device_max; };
            s->tc_geom = tc_sweep_geom(ny, s->smax, capped(tc_sweep_max_ctas()));
            s->tc_afwd = dalloc<uint8_t>(s->tc_geom.page_bytes * nx);
            s->tc_aadj = dalloc<uint8_t>(s->tc_geom.page_bytes * nx);
            s->tc_b = dalloc<uint8_t>(s->tc_geom.b_bytes);
            s->tc_part = dalloc<float>(s->tc_geom.part_bytes / sizeof(float));
            s->tc_sync = dalloc<unsigned>(s->tc_geom.sync_words);
            if (s->factor_method == WUST_FACTOR_DEFAULT) {
                s->ns_g = ns_geom(ny, capped(ns_max_ctas()), s->max_ctas == 0);
                if (s->ns_g.ks > 0) WUST_CUDA(cudaMalloc(&s->ns_scratch, s->ns_g.scratch_bytes));
            }
            s->tc_err = dalloc<int>(4);
            WUST_CUDA(cudaMemset(s->tc_err, 0, 4 * sizeof(int)));
            if (s->sweep_method == WUST_SWEEP_DEFAULT) {
                s->ck_geom = tc_chunk_geom(ny, nx, capped(tc_chunk_max_ctas()), s->chunk_count);
                s->use_chunks = s->ck_geom.C >= 2;   // one chunk: the sequential kernel is faster
            }
            if (s->use_chunks) {
                if (s->ck_geom.lpack_bytes) s->ck_lpack = dalloc<uint8_t>(s->ck_geom.lpack_bytes);
                s->ck_b = dalloc<uint8_t>(s->ck_geom.b_bytes);
                s->ck_z = dalloc<float>(s->ck_geom.state_bytes / sizeof(float));
                s->ck_sb = dalloc<float>(s->ck_geom.state_bytes / sizeof(float));
                WUST_CUDA(cudaMemset(s->ck_z, 0, s->ck_geom.state_bytes));
                WUST_CUDA(cudaMemset(s->ck_sb, 0, s->ck_geom.state_bytes));
                s->ck_sync = dalloc<unsigned>(s->ck_geom.sync_words);
                s->ck_edges = dalloc<float2>(s->ck_geom.edge_bytes / sizeof(float2));
                // BF16 profile: every sweep on BF16 operands (correction_precision
                // SAME keeps the corrections on the profile's operands: BF16 too)
                s->bf16_all = s->precision == WUST_PRECISION_BF16_REFINED;
                s->bf16_corrections = s->bf16_all || s->correction_precision == WUST_CORRECTION_DEFAULT;
                if (s->bf16_corrections) {
                    s->tc_afwd16 = dalloc<uint8_t>(s->ck_geom.page_bytes16 * nx);
                    s->tc_aadj16 = dalloc<uint8_t>(s->ck_geom.page_bytes16 * nx);
                    if (s->ck_geom.lpack16_bytes) s->ck_lpack16 = dalloc<uint8_t>(s->ck_geom.lpack16_bytes);
                }
            }
            if (s->precision == WUST_PRECISION_BF16_REFINED && !s->use_chunks)
                fail(WUST_ERR_INVALID_INPUT, "the BF16 profile runs on the column-chunked sweeps; the grid has too "
                                             "few columns for two chunks (use tf32-refined)");
        }
        assemble_and_factor(s, vel, atten);
        *out = s;
    });
    if (rc != WUST_OK && s) free_solver(s);
    return rc;
}

int wust_solver_refactor(wust_solver *s, const double *vel, const double *atten, double frequency_hz) {
    return guarded([&] {
        if (!s || !vel) fail(WUST_ERR_INVALID_INPUT, "solver and medium required");
        if (!(frequency_hz > 0)) fail(WUST_ERR_INVALID_INPUT, "frequency must be positive");
        s->f = frequency_hz;
        assemble_and_factor(s, vel, atten);
    });
}

int wust_solver_destroy(wust_solver *s) {
    return guarded([&] { free_solver(s); });
}

int wust_solver_timings(const wust_solver *s, double *assembly_ms, double *factor_ms) {
    return guarded([&] {
        if (!s) fail(WUST_ERR_INVALID_INPUT, "null solver");
        if (assembly_ms) *assembly_ms = s->assembly_ms;
        if (factor_ms) *factor_ms = s->factor_ms;
    });
}

int wust_solver_stencil(const wust_solver *s, double *b, double *d, double *e) {
    return guarded([&] {
        if (!s) fail(WUST_ERR_INVALID_INPUT, "null solver");
        if (b) *b = s->b;
        if (d) *d = s->d;
        if (e) *e = s->e;
    });
}

int wust_solver_block(const wust_solver *s, const char *name, const void **ptr, int *rows, int *cols, int *pages) {
    return guarded([&] {
        if (!s || !name || !ptr) fail(WUST_ERR_INVALID_INPUT, "null argument");
        int r = 0, c = 0, p = 1;
        const void *q = nullptr;
        for (int i = 0; i < 9; ++i) {
            if (std::strcmp(name, kCoefNames[i]) == 0) {
                q = s->c64[i];
                r = (i == 0 || i == 3 || i == 6) ? s->ny : s->ny - 1;
                c = (i <= 2) ? s->nx : s->nx - 1;
            }
        }
        if (std::strcmp(name, "invT") == 0) { q = s->invT; r = s->ny; c = s->ny; p = s->nx; }
        if (std::strcmp(name, "mult") == 0) { q = s->mult; r = s->ny; c = s->nx; }
        if (!q) fail(WUST_ERR_INVALID_INPUT, "unknown block '%s'", name);
        *ptr = q;
        if (rows) *rows = r;
        if (cols) *cols = c;
        if (pages) *pages = p;
    });
}

int wust_solver_solve(wust_solver *s, const wust_c64 *src, int n_src, int adjoint, wust_c64 *out, wust_c64 *virt) {
    return guarded([&] {
        if (!s || !src || !out) fail(WUST_ERR_INVALID_INPUT, "solve requires src and out");
        if (n_src < 1 || n_src > s->smax) fail(WUST_ERR_INVALID_INPUT, "n_src must be in [1, max_sources]");
        const long long t0 = g_kernel_launches;
        cudaStream_t st = s->st;
        const size_t n = s->plane() * n_src;
        const float2 *dsrc = stage_in((const float2 *)src, n, s->stage_c, s->stage_c_cap, st);
        if (dsrc == (const float2 *)out) {   // in-place request: keep the source in a work buffer
            WUST_CUDA(cudaMemcpyAsync(s->work, dsrc, n * sizeof(float2), cudaMemcpyDeviceToDevice, st));
            dsrc = s->work;
        }
        SrcView sv{};
        sv.mode = SRC_DENSE;
        sv.dense = dsrc;
        const bool out_dev = is_device_ptr(out);
        float2 *dout = out_dev ? (float2 *)out : s->u;
        solve_into(s, sv, n_src, adjoint != 0, dout);
        if (virt) {
            const bool vdev = is_device_ptr(virt);
            float2 *dv = vdev ? (float2 *)virt : s->lam;
            virtual_source_launch(dout, s->mult, dv, s->ny, s->nx, n_src, st);
            if (!vdev) WUST_CUDA(cudaMemcpyAsync(virt, dv, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
        }
        if (!out_dev) WUST_CUDA(cudaMemcpyAsync(out, dout, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        s->launches = g_kernel_launches - t0;
    });
}

int wust_solver_mass_apply(wust_solver *s, const wust_c64 *v, int n, int adjoint, wust_c64 *out) {
    return guarded([&] {
        if (!s || !v || !out || n < 1) fail(WUST_ERR_INVALID_INPUT, "massApply requires v and out");
        cudaStream_t st = s->st;
        const size_t cnt = s->plane() * n;
        const bool in_dev = is_device_ptr(v), out_dev = is_device_ptr(out);
        if ((!in_dev || !out_dev) && n > s->smax) fail(WUST_ERR_INVALID_INPUT, "host massApply limited to max_sources");
        const float2 *dv = stage_in((const float2 *)v, cnt, s->stage_c, s->stage_c_cap, st);
        float2 *dout = out_dev ? (float2 *)out : s->work;
        if ((const void *)dv == (const void *)dout) fail(WUST_ERR_INVALID_INPUT, "massApply cannot run in place");
        mass_apply_launch(dv, dout, s->ny, s->nx, n, s->d, s->e, adjoint != 0, st);
        if (!out_dev) WUST_CUDA(cudaMemcpyAsync(out, dout, cnt * sizeof(float2), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
    });
}

int wust_solver_oracle(wust_solver *s, const int32_t *tx_index, int n_tx, const int32_t *rx_index, int n_rx,
                       const wust_c64 *Y, const uint8_t *mask, int source_batch_size, int flags, double *loss,
                       double *gradient) {
    return guarded([&] {
        if (!s || !tx_index || !rx_index || !Y || !mask || !loss) fail(WUST_ERR_INVALID_INPUT, "oracle arguments missing");
        const bool need_grad = (flags & WUST_NEED_GRADIENT) != 0;
        const bool retain = (flags & WUST_RETAIN_STATE) != 0;
        if (need_grad && !gradient) fail(WUST_ERR_INVALID_INPUT, "gradient output required");
        if (n_tx < 1 || n_rx < 1) fail(WUST_ERR_INVALID_INPUT, "empty transmitter or receiver set");
        const long long t0 = g_kernel_launches;
        cudaStream_t st = s->st;
        const int ny = s->ny, nx = s->nx;
        const size_t N = s->plane();
        ensure_obs(s, n_tx, n_rx);
        // indices: validate on the host (they are small), convert to 0-based
        std::vector<int32_t> tx(n_tx), rx(n_rx);
        WUST_CUDA(cudaMemcpy(tx.data(), tx_index, n_tx * sizeof(int32_t), cudaMemcpyDefault));
        WUST_CUDA(cudaMemcpy(rx.data(), rx_index, n_rx * sizeof(int32_t), cudaMemcpyDefault));
        std::vector<int32_t> at(N, -1);
        for (int i = 0; i < n_tx; ++i) {
            if (tx[i] < 1 || (size_t)tx[i] > N) fail(WUST_ERR_INVALID_INPUT, "tx_index out of range");
            tx[i] -= 1;
        }
        for (int i = 0; i < n_rx; ++i) {
            if (rx[i] < 1 || (size_t)rx[i] > N) fail(WUST_ERR_INVALID_INPUT, "rx_index out of range");
            rx[i] -= 1;
            if (at[rx[i]] >= 0) fail(WUST_ERR_INVALID_INPUT, "Distinct elements in one array collapse onto a grid sample");
            at[rx[i]] = i;
        }
        WUST_CUDA(cudaMemcpyAsync(s->tx_lin, tx.data(), n_tx * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        WUST_CUDA(cudaMemcpyAsync(s->rx_lin, rx.data(), n_rx * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        WUST_CUDA(cudaMemcpyAsync(s->rx_at, at.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice, st));
        const size_t nobs = (size_t)n_tx * n_rx;
        WUST_CUDA(cudaMemcpyAsync(s->Yd, Y, nobs * sizeof(float2), cudaMemcpyDefault, st));
        WUST_CUDA(cudaMemcpyAsync(s->maskd, mask, nobs, cudaMemcpyDefault, st));
        WUST_CUDA(cudaMemsetAsync(s->status, 0, 64 * sizeof(int), st));
        if (need_grad) WUST_CUDA(cudaMemsetAsync(s->grad, 0, N * sizeof(double), st));
        if (retain) {
            const size_t need = N * (size_t)n_tx;
            if (need > s->ret_cap) {
                dfree(s->ret_u);
                s->ret_u = dalloc<float2>(need);
                s->ret_cap = need;
            }
        }
        int bs = source_batch_size > 0 ? source_batch_size : n_tx;
        if (bs > s->smax) bs = s->smax;
        for (int first = 0; first < n_tx; first += bs) {
            const int nb = std::min(bs, n_tx - first);
            float2 *uf = retain ? s->ret_u + N * first : s->u;
            SrcView fwd{};
            fwd.mode = SRC_POINT;
            fwd.lin = s->tx_lin + first;
            solve_into(s, fwd, nb, false, uf);
            FitParams fp;
            fp.u = uf; fp.u64 = s->precision == WUST_PRECISION_C64 ? nullptr : s->x64_last; fp.rx_lin = s->rx_lin; fp.Y = s->Yd; fp.mask = s->maskd;
            fp.n_tx = n_tx; fp.n_rx = n_rx; fp.first_tx = first; fp.nb = nb; fp.ny = ny; fp.nx = nx;
            fp.residual = s->resid; fp.scale = s->scale + first; fp.loss_per_src = s->loss_src + first;
            fp.status = s->status;
            fit_launch(fp, st);
            if (need_grad) {
                SrcView adj{};
                adj.mode = SRC_SCATTER;
                adj.at = s->rx_at;
                adj.vals = s->resid;
                adj.n_slots = n_rx;
                solve_into(s, adj, nb, true, s->lam);
                gradient_launch(uf, s->lam, s->mult, s->scale + first, ny, nx, nb, s->d, s->e, s->grad, st);
            }
        }
        std::vector<double> ls(n_tx);
        int fstat = 0;
        WUST_CUDA(cudaMemcpyAsync(ls.data(), s->loss_src, n_tx * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaMemcpyAsync(&fstat, s->status, sizeof(int), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        if (fstat) fail(WUST_ERR_NUMERICAL_FAILURE, "Unusable source-scale denominator/numerator (transmitter %d)", fstat);
        double total = 0;
        for (double v : ls) total += v;
        if (!std::isfinite(total)) fail(WUST_ERR_NUMERICAL_FAILURE, "Nonfinite objective/gradient");
        *loss = total;
        if (need_grad) {
            if (is_device_ptr(gradient)) {
                WUST_CUDA(cudaMemcpyAsync(gradient, s->grad, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
                WUST_CUDA(cudaStreamSynchronize(st));
            } else {
                WUST_CUDA(cudaMemcpyAsync(gradient, s->grad, N * sizeof(double), cudaMemcpyDeviceToHost, st));
                WUST_CUDA(cudaStreamSynchronize(st));
                for (size_t i = 0; i < N; ++i)
                    if (!std::isfinite(gradient[i])) fail(WUST_ERR_NUMERICAL_FAILURE, "Nonfinite objective/gradient");
            }
        }
        s->ret_valid = retain ? 1 : 0;
        s->ret_ntx = n_tx;
        s->ret_nrx = n_rx;
        s->launches = g_kernel_launches - t0;
    });
}

int wust_solver_curvature(wust_solver *s, const double *direction, double *curvature) {
    return guarded([&] {
        if (!s || !direction || !curvature) fail(WUST_ERR_INVALID_INPUT, "curvature arguments missing");
        if (!s->ret_valid) fail(WUST_ERR_INVALID_INPUT, "no retained oracle state (call the oracle with WUST_RETAIN_STATE)");
        const long long t0 = g_kernel_launches;
        cudaStream_t st = s->st;
        const size_t N = s->plane();
        WUST_CUDA(cudaMemcpyAsync(s->dir, direction, N * sizeof(double), cudaMemcpyDefault, st));
        const int n_tx = s->ret_ntx, n_rx = s->ret_nrx;
        const int bs = s->smax;
        for (int first = 0; first < n_tx; first += bs) {
            const int nb = std::min(bs, n_tx - first);
            curvature_source_launch(s->ret_u + N * first, s->mult, s->dir, s->work, s->ny, s->nx, nb, s->d, s->e, st);
            SrcView sv{};
            sv.mode = SRC_DENSE;
            sv.dense = s->work;
            solve_into(s, sv, nb, false, s->u);
            curvature_reduce_launch(s->u, s->rx_lin, s->maskd, s->scale + first, n_tx, n_rx, first, nb, s->ny, s->nx,
                                    s->loss_src + first, st);
        }
        std::vector<double> part(n_tx);
        WUST_CUDA(cudaMemcpyAsync(part.data(), s->loss_src, n_tx * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        double k = 0;
        for (double v : part) k += v;
        if (!std::isfinite(k)) fail(WUST_ERR_NUMERICAL_FAILURE, "Nonfinite curvature");
        *curvature = k;
        s->launches = g_kernel_launches - t0;
    });
}

int wust_solver_gauss_newton_product(wust_solver *s, const double *direction, double *out, double *curvature) {
    return guarded([&] {
        if (!s || !direction || !out) fail(WUST_ERR_INVALID_INPUT, "Gauss-Newton product arguments missing");
        if (!s->ret_valid) fail(WUST_ERR_INVALID_INPUT, "no retained oracle state (call the oracle with WUST_RETAIN_STATE)");
        const long long t0 = g_kernel_launches;
        cudaStream_t st = s->st;
        const size_t N = s->plane();
        WUST_CUDA(cudaMemcpyAsync(s->dir, direction, N * sizeof(double), cudaMemcpyDefault, st));
        WUST_CUDA(cudaMemsetAsync(s->grad, 0, N * sizeof(double), st));
        const int n_tx = s->ret_ntx, n_rx = s->ret_nrx;
        const int bs = s->smax;
        for (int first = 0; first < n_tx; first += bs) {
            const int nb = std::min(bs, n_tx - first);
            const float2 *uf = s->ret_u + N * first;
            // J d: the linearized forward solve of directional_curvature.m
            curvature_source_launch(uf, s->mult, s->dir, s->work, s->ny, s->nx, nb, s->d, s->e, st);
            SrcView sv{};
            sv.mode = SRC_DENSE;
            sv.dense = s->work;
            solve_into(s, sv, nb, false, s->u);
            linearized_residual_launch(s->u, s->rx_lin, s->maskd, s->scale + first, n_tx, n_rx, first, nb, s->ny,
                                       s->nx, s->resid, s->loss_src + first, st);
            // Re(J^H q): the oracle's adjoint solve and gradient accumulation on q
            SrcView adj{};
            adj.mode = SRC_SCATTER;
            adj.at = s->rx_at;
            adj.vals = s->resid;
            adj.n_slots = n_rx;
            solve_into(s, adj, nb, true, s->lam);
            gradient_launch(uf, s->lam, s->mult, s->scale + first, s->ny, s->nx, nb, s->d, s->e, s->grad, st);
        }
        std::vector<double> part(n_tx);
        WUST_CUDA(cudaMemcpyAsync(part.data(), s->loss_src, n_tx * sizeof(double), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaMemcpyAsync(out, s->grad, N * sizeof(double), cudaMemcpyDefault, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        double k = 0;
        for (double v : part) k += v;
        if (!std::isfinite(k)) fail(WUST_ERR_NUMERICAL_FAILURE, "Nonfinite curvature");
        if (curvature) *curvature = k;
        s->launches = g_kernel_launches - t0;
    });
}

// ---------------------------------------------------------------------------
// NCG update on the device (wust_reconstruct.m:24-57)
// ---------------------------------------------------------------------------
static double *ncg_partials(wust_solver *s) {
    if (!s->ncg_part) s->ncg_part = dalloc<double>(3 * (size_t)kNcgMaxBlocks);
    return s->ncg_part;
}
// Sum `per` values over nb block partials, in block order.
static std::vector<double> ncg_sum(wust_solver *s, int nb, int per) {
    std::vector<double> h((size_t)nb * per), out(per, 0.0);
    WUST_CUDA(cudaMemcpyAsync(h.data(), s->ncg_part, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    WUST_CUDA(cudaStreamSynchronize(s->st));
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < per; ++k) out[k] += h[(size_t)b * per + k];
    return out;
}
static double mean_step(const std::vector<double> &v) {
    double t = 0;
    for (size_t i = 1; i < v.size(); ++i) t += v[i] - v[i - 1];
    return t / (double)(v.size() - 1);
}
static void check_cufft(cufftResult r, const char *what) {
    if (r != CUFFT_SUCCESS) fail(WUST_ERR_CUDA, "%s failed (cufft %d)", what, (int)r);
}

int wust_ncg_roi_gradient(wust_solver *s, const double *gradient, const uint8_t *update_mask, double c0,
                          double frequency_hz, double cutoff, double order, double *roi, double *z) {
    return guarded([&] {
        if (!s || !gradient || !update_mask || !roi || !z) fail(WUST_ERR_INVALID_INPUT, "roi_gradient arguments missing");
        if (!(std::isfinite(cutoff) && cutoff >= 0)) fail(WUST_ERR_INVALID_INPUT, "cutoff must be a finite nonnegative scalar");
        if (cutoff > 0 && !(std::isfinite(order) && order > 0 && std::isfinite(c0) && c0 > 0 && frequency_hz > 0))
            fail(WUST_ERR_INVALID_INPUT, "filter order, speed and frequency must be positive and finite");
        const long long t0 = g_kernel_launches;
        const size_t N = s->plane();
        cudaStream_t st = s->st;
        ncg_roi_launch(gradient, update_mask, roi, N, st);
        if (cutoff == 0) {
            WUST_CUDA(cudaMemcpyAsync(z, roi, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
        } else {
            if (!s->fft_ready) {
                // column-major ny x nx = row-major (nx, ny): half spectrum along y
                check_cufft(cufftPlan2d(&s->fft_fwd, s->nx, s->ny, CUFFT_D2Z), "cufftPlan2d");
                check_cufft(cufftPlan2d(&s->fft_inv, s->nx, s->ny, CUFFT_Z2D), "cufftPlan2d");
                s->spec = dalloc<double2>((size_t)s->nx * (s->ny / 2 + 1));
                s->fft_ready = true;
            }
            check_cufft(cufftSetStream(s->fft_fwd, st), "cufftSetStream");
            check_cufft(cufftSetStream(s->fft_inv, st), "cufftSetStream");
            check_cufft(cufftExecD2Z(s->fft_fwd, roi, reinterpret_cast<cufftDoubleComplex *>(s->spec)), "cufftExecD2Z");
            const double kc = (2.0 * frequency_hz / c0) * cutoff;
            ncg_butterworth_launch(s->spec, s->nx, s->ny, mean_step(s->xs), mean_step(s->ys), kc * kc, order, st);
            check_cufft(cufftExecZ2D(s->fft_inv, reinterpret_cast<cufftDoubleComplex *>(s->spec), z), "cufftExecZ2D");
            ncg_mask_scale_launch(z, update_mask, 1.0 / ((double)s->nx * s->ny), N, st);
        }
        s->launches = g_kernel_launches - t0;
    });
}

int wust_ncg_direction(wust_solver *s, const double *roi, const double *z, const double *prev_z, double prev_gz,
                       int same_frequency, double *direction, double *beta_out, double *gz_out) {
    return guarded([&] {
        if (!s || !roi || !z || !prev_z || !direction || !beta_out || !gz_out)
            fail(WUST_ERR_INVALID_INPUT, "ncg_direction arguments missing");
        const size_t N = s->plane();
        double *part = ncg_partials(s);
        const std::vector<double> d2 = ncg_sum(s, ncg_dot2_launch(roi, z, prev_z, N, part, s->st), 2);
        const double gz = d2[0];
        double beta = 0.0;
        if (same_frequency && prev_gz > 0) {
            const double beta_fr = gz / prev_gz, beta_pr = d2[1] / prev_gz;
            beta = std::min(std::max(beta_pr, 0.0), beta_fr);
        }
        std::vector<double> dd = ncg_sum(s, ncg_direction_launch(z, roi, beta, direction, N, part, s->st), 2);
        if (dd[0] >= 0) {                         // not a descent direction: restart with -z
            beta = 0.0;
            dd = ncg_sum(s, ncg_direction_launch(z, roi, 0.0, direction, N, part, s->st), 2);
        }
        if (dd[1] != 0 || !std::isfinite(gz) || gz < 0)
            fail(WUST_ERR_NUMERICAL_FAILURE, "Invalid preconditioned gradient");
        *beta_out = beta;
        *gz_out = gz;
    });
}

int wust_ncg_dot(wust_solver *s, const double *a, const double *b, double *out) {
    return guarded([&] {
        if (!s || !a || !b || !out) fail(WUST_ERR_INVALID_INPUT, "ncg_dot arguments missing");
        *out = ncg_sum(s, ncg_dot_launch(a, b, s->plane(), ncg_partials(s), s->st), 1)[0];
    });
}

int wust_ncg_project(wust_solver *s, double *c, const double *direction, double alpha, double step_damping,
                     double max_update_mps, double c_min, double c_max, const uint8_t *update_mask,
                     double *relative_update) {
    return guarded([&] {
        if (!s || !c || !direction || !update_mask) fail(WUST_ERR_INVALID_INPUT, "ncg_project arguments missing");
        if (!(c_min > 0 && c_max > c_min && max_update_mps > 0 && step_damping > 0 && std::isfinite(alpha)))
            fail(WUST_ERR_INVALID_INPUT, "Invalid speed bounds or step");
        const std::vector<double> r = ncg_sum(
            s, ncg_project_launch(c, direction, step_damping * alpha, max_update_mps, c_min, c_max, update_mask,
                                  s->plane(), ncg_partials(s), s->st), 3);
        if (r[0] != 0) fail(WUST_ERR_NUMERICAL_FAILURE, "Nonfinite slowness trial");
        if (relative_update)
            *relative_update = std::sqrt(r[1]) / std::max(std::sqrt(r[2]), std::numeric_limits<double>::min());
    });
}

int wust_dtft(const double *time_s, int n_time, const double *frequencies_hz, int n_f, const void *rf, int rf_is_double,
              int n_rx, int n_tx, const uint8_t *active, wust_c64 *Y, void *stream) {
    return guarded([&] {
        if (!time_s || !frequencies_hz || !rf || !active || !Y) fail(WUST_ERR_INVALID_INPUT, "dtft arguments missing");
        if (n_time < 2 || n_f < 1 || n_rx < 1 || n_tx < 1) fail(WUST_ERR_INVALID_INPUT, "Invalid sample times");
        for (int i = 0; i < n_time; ++i)
            if (!std::isfinite(time_s[i])) fail(WUST_ERR_INVALID_INPUT, "Invalid sample times");
        // wust_prepare.m:10-14: uniform sampling, frequencies below the saved Nyquist
        const double dt = time_s[1] - time_s[0];
        if (!(dt > 0)) fail(WUST_ERR_INVALID_INPUT, "Nonuniform time");
        for (int i = 1; i < n_time; ++i)
            if (std::fabs((time_s[i] - time_s[i - 1]) - dt) > dt * 1e-6) fail(WUST_ERR_INVALID_INPUT, "Nonuniform time");
        for (int k = 0; k < n_f; ++k)
            if (!(std::isfinite(frequencies_hz[k]) && frequencies_hz[k] > 0 && frequencies_hz[k] < 0.5 / dt))
                fail(WUST_ERR_INVALID_INPUT, "Frequency outside saved Nyquist");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        double *t_d = nullptr, *f_d = nullptr;
        double2 *K = nullptr;
        int *bad = nullptr;
        WUST_CUDA(cudaMallocAsync(&t_d, sizeof(double) * n_time, st));
        WUST_CUDA(cudaMallocAsync(&f_d, sizeof(double) * n_f, st));
        WUST_CUDA(cudaMallocAsync(&K, sizeof(double2) * (size_t)n_time * n_f, st));
        WUST_CUDA(cudaMallocAsync(&bad, sizeof(int), st));
        WUST_CUDA(cudaMemcpyAsync(t_d, time_s, sizeof(double) * n_time, cudaMemcpyHostToDevice, st));
        WUST_CUDA(cudaMemcpyAsync(f_d, frequencies_hz, sizeof(double) * n_f, cudaMemcpyHostToDevice, st));
        WUST_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
        dtft_launch(t_d, f_d, n_time, n_f, dt, rf, rf_is_double != 0, n_rx, n_tx, active, K,
                    reinterpret_cast<float2 *>(Y), bad, st);
        int h_bad = 0;
        WUST_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
        WUST_CUDA(cudaFreeAsync(t_d, st));
        WUST_CUDA(cudaFreeAsync(f_d, st));
        WUST_CUDA(cudaFreeAsync(K, st));
        WUST_CUDA(cudaFreeAsync(bad, st));
        WUST_CUDA(cudaStreamSynchronize(st));
        if (h_bad) fail(WUST_ERR_INVALID_INPUT, "Nonfinite RF on an active channel");
    });
}

int wust_simulate(const double *c_mps, int ny, int nx, double dy_m, double dx_m, double dt_s, int n_time,
                  const double *source, const int *tx_index, int n_tx, const int *rx_index, int n_rx, int pml_size,
                  double c_ref_mps, double rho0_kg_m3, int decimation, int tx_batch, float *rf, void *stream) {
    return guarded([&] {
        if (!c_mps || !source || !tx_index || !rx_index || !rf) fail(WUST_ERR_INVALID_INPUT, "simulate arguments missing");
        if (ny < 1 || nx < 1 || n_tx < 1 || n_rx < 1) fail(WUST_ERR_INVALID_INPUT, "Invalid medium");
        // wust_simulate.m:17-37
        double cmax = 0.0;
        for (size_t i = 0; i < (size_t)ny * nx; ++i) {
            if (!(std::isfinite(c_mps[i]) && c_mps[i] > 0)) fail(WUST_ERR_INVALID_INPUT, "Invalid medium");
            cmax = std::max(cmax, c_mps[i]);
        }
        if (!(dx_m > 0 && dy_m > 0 && std::isfinite(dx_m) && std::isfinite(dy_m)))
            fail(WUST_ERR_INVALID_INPUT, "Uniform grid required");
        if (!(dt_s > 0 && cmax * dt_s / std::min(dx_m, dy_m) <= 0.3)) fail(WUST_ERR_INVALID_INPUT, "CFL exceeds tested 0.3");
        if (!(rho0_kg_m3 > 0 && std::isfinite(rho0_kg_m3) && c_ref_mps >= cmax && std::isfinite(c_ref_mps)))
            fail(WUST_ERR_INVALID_INPUT, "Invalid density or reference speed");
        if (decimation < 1) fail(WUST_ERR_INVALID_INPUT, "Invalid decimation factor");
        if (pml_size < 1) fail(WUST_ERR_INVALID_INPUT, "Positive integer outside PML required");
        if (n_time < 2) fail(WUST_ERR_INVALID_INPUT, "Finite source waveform required");
        for (int t = 0; t < n_time; ++t)
            if (!std::isfinite(source[t])) fail(WUST_ERR_INVALID_INPUT, "Finite source waveform required");
        for (const int *ids : {tx_index, rx_index}) {
            const int n = ids == tx_index ? n_tx : n_rx;
            std::vector<int> v(ids, ids + n);
            std::sort(v.begin(), v.end());
            for (int i = 0; i < n; ++i)
                if (v[i] < 1 || (long long)v[i] > (long long)nx * ny || (i > 0 && v[i] == v[i - 1]))
                    fail(WUST_ERR_INVALID_INPUT, "Invalid/duplicate array indices");
        }
        SimulateArgs a{c_mps, ny, nx, dy_m, dx_m, dt_s, n_time, source, tx_index, n_tx, rx_index, n_rx, pml_size,
                       c_ref_mps, rho0_kg_m3, decimation, tx_batch};
        simulate_rf(a, rf, static_cast<cudaStream_t>(stream));
    });
}

int wust_solver_stats(const wust_solver *s, int *refine_iters, double *final_residual, double *error_estimate,
                      long long *kernel_launches) {
    return guarded([&] {
        if (!s) fail(WUST_ERR_INVALID_INPUT, "null solver");
        if (refine_iters) *refine_iters = s->last_refine_iters;
        if (final_residual) *final_residual = s->last_residual;
        if (error_estimate) *error_estimate = s->last_error_est;
        if (kernel_launches) *kernel_launches = s->launches;
    });
}

int wust_solver_sweep_times(const wust_solver *s, double *total_ms, long long *count) {
    return guarded([&] {
        if (!s) fail(WUST_ERR_INVALID_INPUT, "null solver");
        if (total_ms) *total_ms = s->sweep_ms;
        if (count) *count = s->sweeps;
    });
}

int wust_solver_factor_stats(const wust_solver *s, long long out[4]) {
    return guarded([&] {
        if (!s || !out) fail(WUST_ERR_INVALID_INPUT, "null solver or output");
        if (tensor_profile(s) && s->ns_scratch) {
            for (int i = 0; i < 4; ++i) out[i] = s->ns_stats[i];
        } else {
            out[0] = out[1] = out[2] = 0;
            out[3] = s->nx;
        }
    });
}

int wust_solver_factor_info(const wust_solver *s, int *k_slices, int *cluster) {
    return guarded([&] {
        if (!s) fail(WUST_ERR_INVALID_INPUT, "null solver");
        const bool ns = tensor_profile(s) && s->ns_scratch;
        if (k_slices) *k_slices = ns ? s->ns_g.ks : 0;
        if (cluster) *cluster = ns ? s->ns_cluster : -1;
    });
}

// Self-test hook: a device wait that nothing releases must give up after
// timeout_ms and report its site; returns WUST_ERR_DEVICE_TIMEOUT on success.
int wust_selftest_barrier_timeout(int timeout_ms, int *site) {
    return guarded([&] {
        int st = 0;
        int passed = barrier_selftest(timeout_ms * 1e-3, &st);
        if (site) *site = st;
        if (passed != 0) fail(WUST_ERR_RUNTIME, "barrier did not time out");
        fail(WUST_ERR_DEVICE_TIMEOUT, "bounded device wait expired at site %d", st);
    });
}

}  // extern "C"
