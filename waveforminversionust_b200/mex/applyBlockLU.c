/*
 * applyBlockLU MEX gateway over libwust_b200: drop-in for the reference's
 * Runtime/solver/applyBlockLU.cu (call site HelmholtzSolver.m:182-184).
 *
 *   u = applyBlockLU(SRC, Ld, Ll, Lu, Ud, Ul, Uu, invT, adjoint)
 *
 * SRC: Ny x Nx x S complex single gpuArray; the blocks as for decompBlockLU;
 * invT: Ny x Ny x Nx from decompBlockLU; adjoint: logical scalar.  Exactly
 * one output, like the reference (applyBlockLU.cu:327-388).  Build:
 *   mexcuda applyBlockLU.c -I<repo>/include -L<repo>/waveforminversionust_b200 -lwust_b200
 */
#include <stdint.h>

#include "mex.h"
#include "gpu/mxGPUArray.h"
#include "wust_b200.h"

static const mxGPUArray *in_gpu(const mxArray *a, const char *name) {
    if (!mxIsGPUArray(a)) mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be a gpuArray", name);
    const mxGPUArray *g = mxGPUCreateFromMxArray(a);
    if (mxGPUGetClassID(g) != mxSINGLE_CLASS || mxGPUGetComplexity(g) != mxCOMPLEX) {
        mxGPUDestroyGPUArray(g);
        mexErrMsgIdAndTxt("WUST:InvalidInput", "%s must be complex single", name);
    }
    return g;
}

static void release(const mxGPUArray **g, int n) {
    int i;
    for (i = 0; i < n; ++i) mxGPUDestroyGPUArray(g[i]);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    static const char *names[8] = {"SRC", "Ld", "Ll", "Lu", "Ud", "Ul", "Uu", "invT"};
    /* Block shapes relative to (Ny, Nx) (applyBlockLU.cu:377-388). */
    static const int drow[6] = {0, -1, -1, 0, -1, -1};
    const mxGPUArray *g[8];
    int i, rc, adjoint, ok;
    if (nlhs != 1) mexErrMsgIdAndTxt("WUST:InvalidOutput", "applyBlockLU requires exactly one output.");
    ok = nrhs == 9;
    for (i = 0; ok && i < 8; ++i) ok = mxIsGPUArray(prhs[i]);
    if (!ok || !mxIsLogicalScalar(prhs[8]))
        mexErrMsgIdAndTxt("WUST:InvalidInput",
                          "applyBlockLU inputs 1-8 must be gpuArray; input 9 must be a logical scalar.");
    adjoint = mxIsLogicalScalarTrue(prhs[8]) ? 1 : 0;
    mxInitGPU();
    for (i = 0; i < 8; ++i) g[i] = in_gpu(prhs[i], names[i]);
    {
        const mwSize nd = mxGPUGetNumberOfDimensions(g[0]);
        const mwSize *d = mxGPUGetDimensions(g[0]);
        const mwSize *t = mxGPUGetDimensions(g[7]);
        const mwSize ndt = mxGPUGetNumberOfDimensions(g[7]);
        const double numel = (double)mxGPUGetNumberOfElements(g[0]);
        const int Ny = (int)d[0], Nx = nd > 1 ? (int)d[1] : 1, S = nd > 2 ? (int)d[2] : 1;
        mxGPUArray *u;
        ok = nd >= 2 && nd <= 3 && d[0] >= 2 && d[1] >= 2 && numel > 0 && numel <= 2147483647.0 && ndt == 3 &&
             (int)t[0] == Ny && (int)t[1] == Ny && (int)t[2] == Nx;
        for (i = 1; ok && i < 7; ++i) {
            const mwSize *b = mxGPUGetDimensions(g[i]);
            ok = mxGPUGetNumberOfDimensions(g[i]) == 2 && (long)b[0] == Ny + drow[i - 1] && (long)b[1] == Nx - 1;
            mxFree((void *)b);
        }
        mxFree((void *)t);
        if (!ok) {
            mxFree((void *)d);
            release(g, 8);
            mexErrMsgIdAndTxt("WUST:InvalidInput", "Inconsistent Block-LU input shapes.");
        }
        u = mxGPUCreateGPUArray(nd, d, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
        mxFree((void *)d);
        rc = wust_apply_block_lu((const wust_c64 *)mxGPUGetDataReadOnly(g[0]), Ny, Nx, S,
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[1]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[2]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[3]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[4]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[5]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[6]),
                                 (const wust_c64 *)mxGPUGetDataReadOnly(g[7]), adjoint,
                                 (wust_c64 *)mxGPUGetData(u), NULL);
        release(g, 8);
        if (rc != WUST_OK) {
            mxGPUDestroyGPUArray(u);
            mexErrMsgIdAndTxt(wust_status_id(rc), "%s", wust_last_error());
        }
        plhs[0] = mxGPUCreateMxArrayOnGPU(u);
        mxGPUDestroyGPUArray(u);
    }
}
