/*
 * wust_b200.h -- C ABI of the B200 (sm_100a) Helmholtz gradient library.
 *
 * The library replaces the GPU path of WaveformInversionUST's HelmholtzSolver
 * (Runtime/solver/HelmholtzSolver.m) and its two MEX kernels
 * (Runtime/solver/decompBlockLU.cu, Runtime/solver/applyBlockLU.cu), plus the
 * per-frequency misfit/gradient (Runtime/matlab/wust_oracle.m) and the
 * directional curvature (Runtime/matlab/directional_curvature.m).
 *
 * Conventions (identical to the reference):
 *   - 2-D grids are column-major [y, x] (y fastest), Ny rows by Nx columns;
 *     RHS stacks are [y, x, source].  Linear grid indices are 1-based
 *     (MATLAB sub2ind), as in obs.tx_index / obs.rx_index.
 *   - Complex numbers are interleaved (re, im).
 *   - Every call returns a wust_status; wust_status_id() maps it to the
 *     reference's error identifier and wust_last_error() gives the message
 *     of the last failing call on the calling thread.
 *   - Unless stated otherwise, array arguments may be host or device memory;
 *     the library detects which (cudaPointerGetAttributes) and stages host
 *     buffers through its own device copies.  The legacy MEX-equivalent
 *     entry points take device pointers only, like mxGPUArray data.
 *   - No entry point falls back to the CPU: without a usable CUDA device
 *     every compute call fails with WUST_ERR_CUDA.
 */
#ifndef WUST_B200_H
#define WUST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float re, im; } wust_c64;
typedef struct { double re, im; } wust_c128;

/* Status codes; names mirror the reference ids (block_lu_mex_utils.h:37-159,
 * wust_oracle.m:55-80). */
enum wust_status {
    WUST_OK = 0,
    WUST_ERR_INVALID_INPUT = 1,            /* WUST:InvalidInput */
    WUST_ERR_INVALID_OUTPUT = 2,           /* WUST:InvalidOutput */
    WUST_ERR_CUDA = 3,                     /* WUST:CUDAError */
    WUST_ERR_CUBLAS = 4,                   /* WUST:CUBLASError (id kept; no library GEMM is used) */
    WUST_ERR_CUSOLVER = 5,                 /* WUST:CUSOLVERError (id kept; no library solver is used) */
    WUST_ERR_SINGULAR_SCHUR_BLOCK = 6,     /* WUST:SingularSchurBlock */
    WUST_ERR_INVALID_SOLVER_ARGUMENT = 7,  /* WUST:InvalidSolverArgument */
    WUST_ERR_RESOURCE_CLEANUP = 8,         /* WUST:ResourceCleanup */
    WUST_ERR_RUNTIME = 9,                  /* WUST:RuntimeError */
    WUST_ERR_NUMERICAL_FAILURE = 10,       /* WUST:NumericalFailure */
    WUST_ERR_DEVICE_TIMEOUT = 11,          /* WUST:DeviceTimeout: a bounded device-side wait expired */
    WUST_ERR_NOT_CONVERGED = 12            /* WUST:RefinementNotConverged */
};

/* Precision profiles of the solver. */
enum wust_precision {
    WUST_PRECISION_C64 = 0,          /* plain complex-single block LU: the reference algorithm */
    WUST_PRECISION_C64_REFINED = 1,  /* c64 block LU + FP64-residual iterative refinement */
    WUST_PRECISION_BF16_REFINED = 2, /* BF16 tensor-core sweep GEMMs for every solve (TF32 Newton-Schulz
                                        Schur inverses) + FP64 refinement; needs the column-chunked sweeps */
    WUST_PRECISION_TF32_REFINED = 3  /* TF32 tensor-core Schur/solve GEMMs + FP64 refinement */
};

/* Oracle request flags (wust_oracle.m:5-6: nargout selects the work). */
enum wust_oracle_flags {
    WUST_NEED_GRADIENT = 1,   /* adjoint solve + slowness gradient */
    WUST_RETAIN_STATE = 2     /* keep forward fields and source scales for wust_solver_curvature */
};

const char *wust_status_id(int status);
const char *wust_last_error(void);
int wust_version(int *major, int *minor, int *patch);

/* ------------------------------------------------------------------------
 * Legacy MEX-equivalent entry points.  Device pointers, complex single.
 * ------------------------------------------------------------------------ */

/* Replaces `invT = decompBlockLU(Ld,Ll,Lu,Dd,Dl,Du,Ud,Ul,Uu)`
 * (Runtime/solver/decompBlockLU.cu:173-396; call site HelmholtzSolver.m:167-168).
 * Shapes (column-major): Ld, Ud: Ny x (Nx-1); Ll, Lu, Ul, Uu: (Ny-1) x (Nx-1);
 * Dd: Ny x Nx; Dl, Du: (Ny-1) x Nx.  Ny >= 3, Nx >= 2, Ny*Nx < 2^31.
 * invT: caller-allocated Ny x Ny x Nx; every page's border rows and columns
 * are written as zero and its interior holds inv(T_j interior).
 * total_gpu_ms (nullable) receives the device time like the optional timing
 * struct's total_gpu_ms field (decompBlockLU.cu:379-388).  stream may be NULL
 * (legacy default stream).  The call is synchronous, like the MEX. */
int wust_decomp_block_lu(const wust_c64 *Ld, const wust_c64 *Ll, const wust_c64 *Lu,
                         const wust_c64 *Dd, const wust_c64 *Dl, const wust_c64 *Du,
                         const wust_c64 *Ud, const wust_c64 *Ul, const wust_c64 *Uu,
                         int Ny, int Nx, wust_c64 *invT, float *total_gpu_ms, void *stream);

/* Largest Ny accepted by wust_decomp_block_lu_noalloc. */
#define WUST_NOALLOC_MAX_NY 1024

/* No counterpart in the reference (its MEX allocates through MATLAB).
 * The same factorization as wust_decomp_block_lu, for callers that must not
 * have the library allocate device memory: hosts whose own memory manager
 * owns the device heap, and latency-critical callers that cannot afford the
 * device synchronization of cudaMalloc/cudaFree.  It calls no cudaMalloc,
 * cudaFree or allocating library routine; its ~17.8 MB of scratch is a static
 * device array that every GPU loading the library holds until process exit.
 * Ny must not exceed WUST_NOALLOC_MAX_NY (larger grids: WUST_ERR_INVALID_INPUT).
 * All calls share that array, so calls that overlap on the GPU race; callers
 * must serialize them.  Every call looks up the array's address with the
 * caller's device current (so a device reset between calls is safe); the
 * first call on a device may load the module, so make it before any stream
 * capture.  No timing output. */
int wust_decomp_block_lu_noalloc(const wust_c64 *Ld, const wust_c64 *Ll, const wust_c64 *Lu,
                                 const wust_c64 *Dd, const wust_c64 *Dl, const wust_c64 *Du,
                                 const wust_c64 *Ud, const wust_c64 *Ul, const wust_c64 *Uu,
                                 int Ny, int Nx, wust_c64 *invT, void *stream);

/* Replaces `u = applyBlockLU(SRC,Ld,Ll,Lu,Ud,Ul,Uu,invT,adjoint)`
 * (Runtime/solver/applyBlockLU.cu:291-481; call site HelmholtzSolver.m:182-184).
 * src, u: Ny x Nx x n_src; u is caller-allocated and fully overwritten.
 * adjoint != 0 solves H^H u = src with the reference's sweep order. */
int wust_apply_block_lu(const wust_c64 *src, int Ny, int Nx, int n_src,
                        const wust_c64 *Ld, const wust_c64 *Ll, const wust_c64 *Lu,
                        const wust_c64 *Ud, const wust_c64 *Ul, const wust_c64 *Uu,
                        const wust_c64 *invT, int adjoint, wust_c64 *u, void *stream);

/* ------------------------------------------------------------------------
 * Solver object: one HelmholtzSolver instance (model + frequency).
 * ------------------------------------------------------------------------ */

typedef struct wust_solver wust_solver;

/* Constructor arguments of HelmholtzSolver(x, y, vel, atten, f,
 * signConvention, a0, L_PML, options) (HelmholtzSolver.m:32-52). */
typedef struct {
    int ny, nx;                    /* grid size including PML */
    const double *x_m;             /* host, nx increasing uniform samples */
    const double *y_m;             /* host, ny increasing uniform samples */
    double frequency_hz;
    double sign_convention;        /* wust_oracle passes -1 */
    double pml_strength;           /* a0 */
    double pml_m;                  /* L_PML */
    double stencil_vmin, stencil_vmax;   /* options.stencil_bounds */
    int dispersion;                /* 0: continuum; 1: kwave-ldr9 (needs the two below) */
    double time_step_s, reference_speed_mps;
    int precision;                 /* enum wust_precision */
    int refine_max_iters;          /* refined profiles: max refinement solves (0 -> 8) */
    double refine_tol;             /* refined profiles: relative FP64 residual target (0 -> 1e-5) */
    int max_sources;               /* largest RHS batch the object will see (0 -> 256) */
    int factor_method;             /* WUST_FACTOR_*: how the Schur pages are inverted */
    int sweep_method;              /* WUST_SWEEP_*: how the TF32 profile runs its sweeps */
    int correction_precision;      /* WUST_CORRECTION_*: operands of the refinement's correction sweeps */
    int max_ctas;                  /* > 0: cap on the CTAs (one per SM) of the solver's cooperative kernels, so that
                                      solvers on different streams can share the GPU; 0: the whole GPU */
    int chunk_count;               /* > 0: column chunks of the chunked sweeps (clamped to what fits); 0: about
                                      sqrt(2 (Nx - 1)) */
} wust_solver_options;

/* Schur-page inversion (no counterpart in the reference, which always uses
 * cuSOLVER LU).  DEFAULT: Newton-Schulz on the tensor cores for the TF32
 * profile, Gauss-Jordan otherwise; GAUSS_JORDAN: complex-single Gauss-Jordan
 * for every profile (the TF32 profile then keeps tensor-core sweeps only). */
enum wust_factor_method { WUST_FACTOR_DEFAULT = 0, WUST_FACTOR_GAUSS_JORDAN = 1 };

/* Sweeps of the TF32 profile (no counterpart in the reference, whose
 * applyBlockLU runs the columns one after the other).  DEFAULT: column
 * chunks solved concurrently and joined by their composed propagators
 * (formed once per factorization); SEQUENTIAL: one column step after the
 * other on all SMs.  Both apply the same block-LU operator. */
enum wust_sweep_method { WUST_SWEEP_DEFAULT = 0, WUST_SWEEP_SEQUENTIAL = 1 };

/* Operands of the correction sweeps of the refined TF32 profile (no
 * counterpart in the reference, which does not refine).  DEFAULT: BF16 pages
 * and propagators for the correction solves of the chunked sweeps (a
 * correction only has to be accurate to about 1e-2 for the refinement to
 * reach its target in the same number of steps; the BF16 operand stream is
 * half the bytes); SAME: the profile's TF32 operands for every solve. */
enum wust_correction_precision { WUST_CORRECTION_DEFAULT = 0, WUST_CORRECTION_SAME = 1 };

/* Assemble the nine-point PML operator on the GPU and factorize it.
 * vel, atten: ny x nx (atten may be NULL = zero).  stream may be NULL. */
int wust_solver_create(wust_solver **out, const wust_solver_options *options,
                       const double *vel, const double *atten, void *stream);
/* Re-assemble and re-factorize for a new medium and/or frequency on the
 * same grid, reusing all device buffers (one NCG step = one refactor). */
int wust_solver_refactor(wust_solver *s, const double *vel, const double *atten,
                         double frequency_hz);
int wust_solver_destroy(wust_solver *s);

/* Wall/device timings of the last construction (HelmholtzSolver.m:15-16). */
int wust_solver_timings(const wust_solver *s, double *assembly_ms, double *factor_ms);
/* Stencil mass weights b, d, e (obj.massD / obj.massE; stencilOptParams.m). */
int wust_solver_stencil(const wust_solver *s, double *b, double *d, double *e);

/* Device views of the factor blocks (HelmholtzSolver.m:18-24 properties).
 * names: "Dd","Dl","Du","Ld","Ll","Lu","Ud","Ul","Uu","invT","mult".
 * The pointer stays owned by the solver. */
int wust_solver_block(const wust_solver *s, const char *name, const void **device_ptr,
                      int *rows, int *cols, int *pages);

/* solve(src, adjoint) (HelmholtzSolver.m:174-203): out = H^{-1} src or
 * H^{-H} src for n_src right-hand sides; virt (nullable) receives the
 * virtual sources mult .* out. */
int wust_solver_solve(wust_solver *s, const wust_c64 *src, int n_src, int adjoint,
                      wust_c64 *out, wust_c64 *virt);

/* massApply(v, adjoint) (HelmholtzSolver.m:205-220). */
int wust_solver_mass_apply(wust_solver *s, const wust_c64 *v, int n, int adjoint, wust_c64 *out);

/* [loss, gradient, cache] = wust_oracle(c, obs, fi, cfg) for the solver's
 * model and frequency (wust_oracle.m:1-86).
 * tx_index, rx_index: 1-based linear grid indices (host or device, int32).
 * Y: n_tx x n_rx complex single observations of this frequency; mask: n_tx x
 * n_rx bytes (0/1).  source_batch_size <= 0 means all transmitters at once.
 * gradient (nullable unless WUST_NEED_GRADIENT): ny x nx double. */
int wust_solver_oracle(wust_solver *s, const int32_t *tx_index, int n_tx,
                       const int32_t *rx_index, int n_rx,
                       const wust_c64 *Y, const uint8_t *mask,
                       int source_batch_size, int flags,
                       double *loss, double *gradient);

/* directional_curvature(state, direction, rx_index, mask) on the state kept
 * by the last oracle call with WUST_RETAIN_STATE
 * (directional_curvature.m:1-26).  direction: ny x nx double. */
int wust_solver_curvature(wust_solver *s, const double *direction, double *curvature);

/* No counterpart in the reference (its NCG loop needs only the scalar
 * curvature of directional_curvature.m).  The Gauss-Newton Hessian-vector
 * product of the misfit along a direction, with the source scales frozen as
 * directional_curvature.m:1-26 freezes them, on the state kept by the last
 * oracle call with WUST_RETAIN_STATE:
 *     q = J d = -a (H^{-1} M (v .* d))(rx) .* mask,   out = Re(J^H q),
 * i.e. one more forward and one more adjoint solve, reusing the factors.
 * direction, out: ny x nx double (host or device); curvature (nullable)
 * receives d' out = ||q||^2, the value wust_solver_curvature returns. */
int wust_solver_gauss_newton_product(wust_solver *s, const double *direction, double *out, double *curvature);

/* The NCG update of wust_reconstruct (wust_reconstruct.m:24-57) on the GPU,
 * FP64, for hosts that keep the model, gradient and direction in device
 * memory between oracle calls (the reference runs these rules in MATLAB on
 * the host).  Every field is a device pointer to ny x nx column-major doubles
 * on the solver's grid; update masks are device bytes (0/1).  Calls are
 * ordered on the solver's stream; scalar outputs synchronize it. */

/* roi = M g; z = M F M g with F the ringing filter (wust_roi_gradient.m:1-10,
 * ringingRemovalFilt.m:1-45, FFT by cuFFT; cutoff 0: z = roi).  c0: the
 * reference speed the filter cutoff is scaled with (the mean initial speed). */
int wust_ncg_roi_gradient(wust_solver *s, const double *gradient, const uint8_t *update_mask, double c0,
                          double frequency_hz, double cutoff, double order, double *roi, double *z);
/* Clipped PR/FR direction with restart on non-descent (wust_ncg_direction.m:1-17).
 * direction: the previous direction on input, the new one on output. */
int wust_ncg_direction(wust_solver *s, const double *roi, const double *z, const double *prev_z, double prev_gz,
                       int same_frequency, double *direction, double *beta, double *gz);
/* sum a .* b over the grid (the directional slope roi' * direction). */
int wust_ncg_dot(wust_solver *s, const double *a, const double *b, double *out);
/* c <- projected update of the slowness 1/c + step_damping * alpha * direction
 * (wust_project_slowness_update.m:1-10); relative_update (nullable) receives
 * ||1/c_new - 1/c_old|| / ||1/c_old|| over the mask (wust_reconstruct.m:56). */
int wust_ncg_project(wust_solver *s, double *c, const double *direction, double alpha, double step_damping,
                     double max_update_mps, double c_min, double c_max, const uint8_t *update_mask,
                     double *relative_update);

/* The DTFT of the RF preparation (wust_prepare.m:30-37):
 *     Y(tx, rx, k) = single( sum_t exp(-2 pi i f_k t) dt * rf(t, rx, tx) ),
 * FP64 phases and sums over the record's sample times, the traces of channels
 * with active(tx, rx) == 0 taken as zero.  time_s (n_time), frequencies_hz
 * (n_f): host; rf: device [n_time, n_rx, n_tx] column-major, float
 * (rf_is_double == 0) or double; active: device bytes [n_tx, n_rx]; Y: device
 * complex single [n_tx, n_rx, n_f].  Rejects nonuniform sampling, frequencies
 * at or above the saved Nyquist and nonfinite samples on active channels with
 * the reference's messages.  Synchronizes the stream (NULL: legacy default). */
int wust_dtft(const double *time_s, int n_time, const double *frequencies_hz, int n_f, const void *rf, int rf_is_double,
              int n_rx, int n_tx, const uint8_t *active, wust_c64 *Y, void *stream);

/* RF simulation of wust_simulate.m:1-87 (its 'native-batch' and
 * 'matlab-serial' backends, which run k-Wave's 2-D first-order k-space solver
 * per transmitter): linear acoustics, scalar density rho0, no absorption, a
 * Dirichlet pressure source s(t) at each transmitter in turn, the pressure
 * recorded at every receiver, a PML of pml_size cells (alpha 2) outside the
 * grid, k-space correction at c_ref, then the FIR decimation of
 * downsampleKWaveChannelData.m when decimation > 1.  c_mps: host [ny, nx]
 * column-major (first axis y with spacing dy_m); source: host [n_time];
 * tx_index / rx_index: host 1-based column-major grid indices, distinct;
 * rf: device float [ceil(n_time / decimation), n_rx, n_tx] column-major (the
 * reference's pressure(time, receiver, transmitter)).  tx_batch transmitters
 * march together (0: all).  Checks the reference's preconditions (positive
 * finite medium, CFL c dt / min(dx, dy) <= 0.3, c_ref >= max c, rho0 > 0,
 * pml_size >= 1, decimation >= 1, at least two finite source samples, valid
 * distinct indices) and synchronizes the stream (NULL: legacy default). */
int wust_simulate(const double *c_mps, int ny, int nx, double dy_m, double dx_m, double dt_s, int n_time,
                  const double *source, const int *tx_index, int n_tx, const int *rx_index, int n_rx, int pml_size,
                  double c_ref_mps, double rho0_kg_m3, int decimation, int tx_batch, float *rf, void *stream);

/* Counters of the last solve/oracle call: correction solves of the last
 * refined solve, its final relative FP64 residual |b - Hx| / |b| and forward
 * error estimate (refined profiles; -1 otherwise), and the number of kernel
 * launches the call issued. */
int wust_solver_stats(const wust_solver *s, int *refine_iters, double *final_residual,
                      double *error_estimate, long long *kernel_launches);

/* Device time of the block-LU sweep pairs (one forward and one backward
 * sweep over a batch of right-hand sides; refined solves run one per
 * correction) since the solver was created, and their number (no counterpart
 * in the reference).  Each pair is bracketed by events on the solver stream,
 * so solves measure their sweeps at the cost of one stream synchronization
 * per pair. */
int wust_solver_sweep_times(const wust_solver *s, double *total_ms, long long *count);

/* Counters of the last factorization (no counterpart in the reference, which
 * always runs cuSOLVER LU per page): out[0] tensor-core GEMMs and out[1] X
 * updates of the Newton-Schulz pages, out[2] pages inverted by Newton-Schulz,
 * out[3] pages inverted directly: by Gauss-Jordan, or in closed form for the
 * Dirichlet columns (unit diagonal, no coupling: the identity page, after a
 * check of the coefficients).  Profiles other than
 * WUST_PRECISION_TF32_REFINED report {0, 0, 0, Nx}. */
int wust_solver_factor_stats(const wust_solver *s, long long out[4]);

/* How the last factorization ran its Newton-Schulz pages (no counterpart in
 * the reference): *k_slices the K split of each GEMM tile (0: no Newton-Schulz
 * pages for this profile or grid), *cluster 1 if the K slices of a tile ran as
 * one thread-block cluster (split-K partials summed through distributed
 * shared memory), 0 if as separate CTAs (partials through L2), -1 if no
 * Newton-Schulz launch ran.  Either pointer may be NULL. */
int wust_solver_factor_info(const wust_solver *s, int *k_slices, int *cluster);

/* Self-test of the bounded device-side wait used by the persistent kernels
 * (no counterpart in the reference, whose MEX calls are synchronous library
 * calls): one CTA waits at a grid barrier that can never fill; the wait must
 * give up after timeout_ms, leave the context usable and report its site.
 * Returns WUST_ERR_DEVICE_TIMEOUT when the timeout path works. */
int wust_selftest_barrier_timeout(int timeout_ms, int *site);

#ifdef __cplusplus
}
#endif

#endif /* WUST_B200_H */
