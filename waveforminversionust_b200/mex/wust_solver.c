/*
 * wust_solver MEX gateway over libwust_b200: the whole HelmholtzSolver object
 * on the GPU (assembly, factorization with a precision profile, refined
 * solves, massApply, the wust_oracle misfit/gradient and the directional
 * curvature), for MATLAB hosts.  It is what HelmholtzSolver.m's gpu backend
 * calls when options.precision is given (INTEGRATION.md shows that branch);
 * without precision the class keeps calling decompBlockLU / applyBlockLU.
 *
 *   h = wust_solver('create', x, y, vel, atten, f, signConvention, a0, L_PML, options)
 *       (HelmholtzSolver.m:32-172).  options: backend ('gpu'), stencil_bounds
 *       [min max] (both required, as the class requires them), dispersion
 *       ([] or a struct with time_step_s, reference_speed_mps), precision
 *       ('c64' | 'c64-refined' | 'tf32-refined', default 'c64'), refine_tol
 *       (default 1e-5), refine_max_iters (8), max_sources (256),
 *       factor_method ('default' | 'gauss-jordan'), sweep_method
 *       ('default' | 'sequential'), correction_precision ('default' | 'same'),
 *       max_ctas (0: the whole GPU), chunk_count (0: automatic).
 *       h is a uint64 scalar naming the live solver.
 *   wust_solver('refactor', h, vel, atten, f)       new medium / frequency, same grid
 *   [u, virt] = wust_solver('solve', h, src, adjoint)   (HelmholtzSolver.m:174-203)
 *       src: complex single [ny nx S] gpuArray (or host array); u, virt: gpuArrays.
 *   out = wust_solver('massApply', h, v, adjoint)       (HelmholtzSolver.m:205-220)
 *   [loss, gradient] = wust_solver('oracle', h, tx_index, rx_index, Y, mask, batch, retain)
 *       (wust_oracle.m:1-86 for the solver's medium and frequency): 1-based
 *       linear indices, Y complex single n_tx x n_rx, mask logical n_tx x n_rx,
 *       batch the source batch size (<= 0: all), retain true to keep the state
 *       for 'curvature'.  gradient: ny x nx double on the host.
 *   kappa = wust_solver('curvature', h, direction)      (directional_curvature.m:1-26)
 *   s = wust_solver('info', h)    assembly_seconds, factor_seconds, massB, massD,
 *       massE, refine_iters, final_residual, error_estimate (last refined solve)
 *   wust_solver('destroy', h)
 *
 * Errors carry the reference's identifiers (WUST:InvalidInput, WUST:CUDAError,
 * WUST:SingularSchurBlock, ...).  Solvers still alive when the MEX file is
 * cleared are destroyed.  Build (interleaved complex API):
 *   mexcuda -R2018a wust_solver.c -I<repo>/include -L<repo>/waveforminversionust_b200 -lwust_b200
 */
#include <stdint.h>
#include <string.h>

#include "mex.h"
#include "gpu/mxGPUArray.h"
#include "wust_b200.h"

#define MAX_SOLVERS 64

static wust_solver *live[MAX_SOLVERS];

static void destroy_all(void) {
    int i;
    for (i = 0; i < MAX_SOLVERS; ++i)
        if (live[i]) {
            wust_solver_destroy(live[i]);
            live[i] = NULL;
        }
}

static void check(int rc) {
    if (rc != WUST_OK) mexErrMsgIdAndTxt(wust_status_id(rc), "%s", wust_last_error());
}

static int slot_of(const mxArray *a) {
    uint64_t v;
    int i;
    if (!mxIsUint64(a) || mxGetNumberOfElements(a) != 1)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "solver handle must be a uint64 scalar");
    v = mxGetUint64s(a)[0];
    for (i = 0; i < MAX_SOLVERS; ++i)
        if (live[i] && (uint64_t)(uintptr_t)live[i] == v) return i;
    mexErrMsgIdAndTxt("WUST:InvalidInput", "invalid or destroyed solver handle");
    return -1;
}

static const double *host_doubles(const mxArray *a, size_t n, const char *what) {
    if (mxIsGPUArray(a) || !mxIsDouble(a) || mxIsComplex(a) || mxGetNumberOfElements(a) != n)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be a real double array with %zu elements", what, n);
    return mxGetDoubles(a);
}

static double scalar(const mxArray *a, const char *what) {
    if (mxIsGPUArray(a) || !mxIsNumeric(a) || mxIsComplex(a) || mxGetNumberOfElements(a) != 1)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be a real scalar", what);
    return mxGetScalar(a);
}

static int choice(const mxArray *opts, const char *field, const char *const *names, int n, int dflt) {
    const mxArray *f = mxGetField(opts, 0, field);
    char *s;
    int i;
    if (!f || mxIsEmpty(f)) return dflt;
    s = mxIsChar(f) ? mxArrayToString(f) : NULL;
    if (!s) mexErrMsgIdAndTxt("WUST:InvalidInput", "options.%s must be a character vector", field);
    for (i = 0; i < n; ++i)
        if (strcmp(s, names[i]) == 0) {
            mxFree(s);
            return i;
        }
    mxFree(s);
    mexErrMsgIdAndTxt("WUST:InvalidInput", "options.%s is not one of the accepted values", field);
    return -1;
}

static double option_scalar(const mxArray *opts, const char *field, double dflt) {
    const mxArray *f = mxGetField(opts, 0, field);
    return (!f || mxIsEmpty(f)) ? dflt : scalar(f, field);
}

/* Device or host pointer of a complex single array with the given element count. */
static const void *c64_data(const mxArray *a, const mxGPUArray **keep, size_t n, const char *what) {
    *keep = NULL;
    if (mxIsGPUArray(a)) {
        const mxGPUArray *g = mxGPUCreateFromMxArray(a);
        if (mxGPUGetClassID(g) != mxSINGLE_CLASS || mxGPUGetComplexity(g) != mxCOMPLEX ||
            mxGPUGetNumberOfElements(g) != n) {
            mxGPUDestroyGPUArray(g);
            mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be complex single with %zu elements", what, n);
        }
        *keep = g;
        return mxGPUGetDataReadOnly(g);
    }
    if (!mxIsSingle(a) || !mxIsComplex(a) || mxGetNumberOfElements(a) != n)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be complex single with %zu elements", what, n);
    return mxGetData(a);
}

static void cmd_create(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    static const char *const precisions[] = {"c64", "c64-refined", "bf16-refined", "tf32-refined"};
    static const char *const defaults2[] = {"default", "gauss-jordan"};
    static const char *const sweeps[] = {"default", "sequential"};
    static const char *const corrections[] = {"default", "same"};
    static const char *const backends[] = {"cpu", "gpu"};
    const mxArray *opts, *bounds, *disp;
    wust_solver_options o;
    const double *vel, *atten = NULL;
    wust_solver *s = NULL;
    size_t nx, ny;
    int slot, i;
    (void)nlhs;
    if (nrhs != 10) mexErrMsgIdAndTxt("WUST:InvalidInput", "create expects x, y, vel, atten, f, signConvention, a0, L_PML, options");
    opts = prhs[9];
    if (!mxIsStruct(opts) || !mxGetField(opts, 0, "backend") || !mxGetField(opts, 0, "stencil_bounds"))
        mexErrMsgIdAndTxt("WUST:InvalidInput", "Explicit backend and fixed stencil_bounds are required");
    bounds = mxGetField(opts, 0, "stencil_bounds");
    if (mxIsGPUArray(bounds) || !mxIsDouble(bounds) || mxIsComplex(bounds) || mxGetNumberOfElements(bounds) != 2 ||
        !(mxGetDoubles(bounds)[0] > 0) || !(mxGetDoubles(bounds)[1] > mxGetDoubles(bounds)[0]))
        mexErrMsgIdAndTxt("WUST:InvalidInput", "stencil_bounds must be a positive ordered [min,max] pair");
    if (choice(opts, "backend", backends, 2, -1) != 1)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "wust_solver runs the gpu backend only (backend must be 'gpu')");
    nx = mxGetNumberOfElements(prhs[1]);
    ny = mxGetNumberOfElements(prhs[2]);
    memset(&o, 0, sizeof(o));
    o.nx = (int)nx;
    o.ny = (int)ny;
    o.x_m = host_doubles(prhs[1], nx, "x");
    o.y_m = host_doubles(prhs[2], ny, "y");
    if (mxGetM(prhs[3]) != ny || mxGetN(prhs[3]) != nx)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "Expected a positive finite [ny,nx] medium");
    vel = host_doubles(prhs[3], nx * ny, "vel");
    if (!mxIsEmpty(prhs[4])) atten = host_doubles(prhs[4], nx * ny, "atten");
    o.frequency_hz = scalar(prhs[5], "f");
    o.sign_convention = scalar(prhs[6], "signConvention");
    o.pml_strength = scalar(prhs[7], "a0");
    o.pml_m = scalar(prhs[8], "L_PML");
    o.stencil_vmin = mxGetDoubles(bounds)[0];
    o.stencil_vmax = mxGetDoubles(bounds)[1];
    disp = mxGetField(opts, 0, "dispersion");
    if (disp && !mxIsEmpty(disp)) {
        if (!mxIsStruct(disp)) mexErrMsgIdAndTxt("WUST:InvalidInput", "options.dispersion must be [] or a struct");
        o.dispersion = 1;
        o.time_step_s = option_scalar(disp, "time_step_s", 0.0);
        o.reference_speed_mps = option_scalar(disp, "reference_speed_mps", 0.0);
    }
    o.precision = choice(opts, "precision", precisions, 4, WUST_PRECISION_C64);
    o.refine_tol = option_scalar(opts, "refine_tol", 1e-5);
    o.refine_max_iters = (int)option_scalar(opts, "refine_max_iters", 8);
    o.max_sources = (int)option_scalar(opts, "max_sources", 256);
    o.factor_method = choice(opts, "factor_method", defaults2, 2, WUST_FACTOR_DEFAULT);
    o.sweep_method = choice(opts, "sweep_method", sweeps, 2, WUST_SWEEP_DEFAULT);
    o.correction_precision = choice(opts, "correction_precision", corrections, 2, WUST_CORRECTION_DEFAULT);
    o.max_ctas = (int)option_scalar(opts, "max_ctas", 0);
    o.chunk_count = (int)option_scalar(opts, "chunk_count", 0);
    for (slot = -1, i = 0; i < MAX_SOLVERS; ++i)
        if (!live[i]) {
            slot = i;
            break;
        }
    if (slot < 0) mexErrMsgIdAndTxt("WUST:RuntimeError", "too many live solvers (%d); destroy some", MAX_SOLVERS);
    mexAtExit(destroy_all);
    mxInitGPU();
    check(wust_solver_create(&s, &o, vel, atten, NULL));
    live[slot] = s;
    plhs[0] = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
    mxGetUint64s(plhs[0])[0] = (uint64_t)(uintptr_t)s;
}

static void grid_of(wust_solver *s, int *ny, int *nx) {
    const void *p;
    int pages;
    check(wust_solver_block(s, "Dd", &p, ny, nx, &pages));
}

static void cmd_refactor(int nrhs, const mxArray *prhs[], int slot) {
    int ny, nx;
    const double *atten = NULL;
    if (nrhs != 5) mexErrMsgIdAndTxt("WUST:InvalidInput", "refactor expects h, vel, atten, f");
    grid_of(live[slot], &ny, &nx);
    if (!mxIsEmpty(prhs[3])) atten = host_doubles(prhs[3], (size_t)nx * ny, "atten");
    check(wust_solver_refactor(live[slot], host_doubles(prhs[2], (size_t)nx * ny, "vel"), atten,
                               scalar(prhs[4], "f")));
}

static void cmd_solve(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[], int slot, int mass) {
    const mxGPUArray *keep;
    const void *src;
    mxGPUArray *u, *virt = NULL;
    mwSize dims[3];
    size_t n;
    int ny, nx, rc, adjoint;
    if (nrhs != 4 || !mxIsLogicalScalar(prhs[3]))
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s expects h, an [ny nx n] array and a logical adjoint flag",
                          mass ? "massApply" : "solve");
    if (nlhs > (mass ? 1 : 2)) mexErrMsgIdAndTxt("WUST:InvalidOutput", "too many outputs");
    adjoint = mxIsLogicalScalarTrue(prhs[3]) ? 1 : 0;
    grid_of(live[slot], &ny, &nx);
    n = mxIsGPUArray(prhs[2]) ? 0 : mxGetNumberOfElements(prhs[2]);
    if (mxIsGPUArray(prhs[2])) {
        const mxGPUArray *g = mxGPUCreateFromMxArray(prhs[2]);
        n = mxGPUGetNumberOfElements(g);
        mxGPUDestroyGPUArray(g);
    }
    if (n == 0 || n % ((size_t)nx * ny) != 0)
        mexErrMsgIdAndTxt("WUST:InvalidInput", "source must be [ny, nx, n] on the solver's grid");
    src = c64_data(prhs[2], &keep, n, "source");
    dims[0] = (mwSize)ny;
    dims[1] = (mwSize)nx;
    dims[2] = (mwSize)(n / ((size_t)nx * ny));
    u = mxGPUCreateGPUArray(3, dims, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
    if (!mass && nlhs > 1) virt = mxGPUCreateGPUArray(3, dims, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
    if (mass)
        rc = wust_solver_mass_apply(live[slot], (const wust_c64 *)src, (int)dims[2], adjoint, (wust_c64 *)mxGPUGetData(u));
    else
        rc = wust_solver_solve(live[slot], (const wust_c64 *)src, (int)dims[2], adjoint, (wust_c64 *)mxGPUGetData(u),
                               virt ? (wust_c64 *)mxGPUGetData(virt) : NULL);
    if (keep) mxGPUDestroyGPUArray(keep);
    if (rc != WUST_OK) {
        mxGPUDestroyGPUArray(u);
        if (virt) mxGPUDestroyGPUArray(virt);
        check(rc);
    }
    plhs[0] = mxGPUCreateMxArrayOnGPU(u);
    mxGPUDestroyGPUArray(u);
    if (virt) {
        plhs[1] = mxGPUCreateMxArrayOnGPU(virt);
        mxGPUDestroyGPUArray(virt);
    }
}

/* 1-based linear indices as host int32. */
static int32_t *indices(const mxArray *a, size_t *n, const char *what) {
    size_t i, k = mxGetNumberOfElements(a);
    int32_t *out;
    if (mxIsGPUArray(a) || k == 0 || !(mxIsDouble(a) || mxIsInt32(a)) || mxIsComplex(a))
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be a non-empty real double or int32 index vector", what);
    out = (int32_t *)mxMalloc(k * sizeof(int32_t));
    for (i = 0; i < k; ++i) {
        const double v = mxIsInt32(a) ? (double)mxGetInt32s(a)[i] : mxGetDoubles(a)[i];
        if (!(v >= 1 && v <= 2147483647.0) || v != (double)(int32_t)v) {
            mxFree(out);
            mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must hold positive integer linear indices", what);
        }
        out[i] = (int32_t)v;
    }
    *n = k;
    return out;
}

static void cmd_oracle(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[], int slot) {
    const mxGPUArray *keep;
    const void *Y;
    int32_t *tx, *rx;
    size_t ntx, nrx;
    uint8_t *mask;
    size_t i;
    int ny, nx, flags, rc;
    double loss = 0.0;
    double *grad = NULL;
    if (nrhs != 8) mexErrMsgIdAndTxt("WUST:InvalidInput", "oracle expects h, tx_index, rx_index, Y, mask, batch, retain");
    if (nlhs > 2) mexErrMsgIdAndTxt("WUST:InvalidOutput", "oracle returns loss and gradient");
    grid_of(live[slot], &ny, &nx);
    tx = indices(prhs[2], &ntx, "tx_index");
    rx = indices(prhs[3], &nrx, "rx_index");
    if (mxIsGPUArray(prhs[5]) || !mxIsLogical(prhs[5]) || mxGetNumberOfElements(prhs[5]) != ntx * nrx) {
        mxFree(tx);
        mxFree(rx);
        mexErrMsgIdAndTxt("WUST:InvalidInput", "mask must be a logical n_tx x n_rx array");
    }
    mask = (uint8_t *)mxMalloc(ntx * nrx);
    for (i = 0; i < ntx * nrx; ++i) mask[i] = mxGetLogicals(prhs[5])[i] ? 1 : 0;
    Y = c64_data(prhs[4], &keep, ntx * nrx, "Y");
    flags = (nlhs > 1 ? WUST_NEED_GRADIENT : 0) | (mxIsLogicalScalarTrue(prhs[7]) ? WUST_RETAIN_STATE : 0);
    if (nlhs > 1) {
        plhs[1] = mxCreateDoubleMatrix((mwSize)ny, (mwSize)nx, mxREAL);
        grad = mxGetDoubles(plhs[1]);
    }
    rc = wust_solver_oracle(live[slot], tx, (int)ntx, rx, (int)nrx, (const wust_c64 *)Y, mask,
                            (int)scalar(prhs[6], "batch"), flags, &loss, grad);
    if (keep) mxGPUDestroyGPUArray(keep);
    mxFree(tx);
    mxFree(rx);
    mxFree(mask);
    check(rc);
    plhs[0] = mxCreateDoubleScalar(loss);
}

static void cmd_curvature(mxArray *plhs[], int nrhs, const mxArray *prhs[], int slot) {
    int ny, nx;
    double kappa = 0.0;
    if (nrhs != 3) mexErrMsgIdAndTxt("WUST:InvalidInput", "curvature expects h, direction");
    grid_of(live[slot], &ny, &nx);
    check(wust_solver_curvature(live[slot], host_doubles(prhs[2], (size_t)nx * ny, "direction"), &kappa));
    plhs[0] = mxCreateDoubleScalar(kappa);
}

static void cmd_info(mxArray *plhs[], int slot) {
    static const char *fields[8] = {"assembly_seconds", "factor_seconds", "massB", "massD", "massE",
                                    "refine_iters", "final_residual", "error_estimate"};
    double a, f, b, d, e, res, err;
    int it;
    long long launches;
    mxArray *s;
    check(wust_solver_timings(live[slot], &a, &f));
    check(wust_solver_stencil(live[slot], &b, &d, &e));
    check(wust_solver_stats(live[slot], &it, &res, &err, &launches));
    s = mxCreateStructMatrix(1, 1, 8, fields);
    mxSetField(s, 0, "assembly_seconds", mxCreateDoubleScalar(a * 1e-3));
    mxSetField(s, 0, "factor_seconds", mxCreateDoubleScalar(f * 1e-3));
    mxSetField(s, 0, "massB", mxCreateDoubleScalar(b));
    mxSetField(s, 0, "massD", mxCreateDoubleScalar(d));
    mxSetField(s, 0, "massE", mxCreateDoubleScalar(e));
    mxSetField(s, 0, "refine_iters", mxCreateDoubleScalar((double)it));
    mxSetField(s, 0, "final_residual", mxCreateDoubleScalar(res));
    mxSetField(s, 0, "error_estimate", mxCreateDoubleScalar(err));
    plhs[0] = s;
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    char *cmd;
    int slot;
    if (nrhs < 1 || !mxIsChar(prhs[0])) mexErrMsgIdAndTxt("WUST:InvalidInput", "first argument must be a command");
    cmd = mxArrayToString(prhs[0]);
    if (strcmp(cmd, "create") == 0) {
        mxFree(cmd);
        cmd_create(nlhs, plhs, nrhs, prhs);
        return;
    }
    if (nrhs < 2) {
        mxFree(cmd);
        mexErrMsgIdAndTxt("WUST:InvalidInput", "a solver handle is required");
    }
    slot = slot_of(prhs[1]);
    if (strcmp(cmd, "destroy") == 0) {
        mxFree(cmd);
        check(wust_solver_destroy(live[slot]));
        live[slot] = NULL;
    } else if (strcmp(cmd, "refactor") == 0) {
        mxFree(cmd);
        cmd_refactor(nrhs, prhs, slot);
    } else if (strcmp(cmd, "solve") == 0) {
        mxFree(cmd);
        cmd_solve(nlhs, plhs, nrhs, prhs, slot, 0);
    } else if (strcmp(cmd, "massApply") == 0) {
        mxFree(cmd);
        cmd_solve(nlhs, plhs, nrhs, prhs, slot, 1);
    } else if (strcmp(cmd, "oracle") == 0) {
        mxFree(cmd);
        cmd_oracle(nlhs, plhs, nrhs, prhs, slot);
    } else if (strcmp(cmd, "curvature") == 0) {
        mxFree(cmd);
        cmd_curvature(plhs, nrhs, prhs, slot);
    } else if (strcmp(cmd, "info") == 0) {
        mxFree(cmd);
        cmd_info(plhs, slot);
    } else {
        mxFree(cmd);
        mexErrMsgIdAndTxt("WUST:InvalidInput", "unknown command");
    }
}
