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

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    static const char *names[8] = {"SRC", "Ld", "Ll", "Lu", "Ud", "Ul", "Uu", "invT"};
    const mxGPUArray *g[8];
    int i, rc, adjoint;
    if (nrhs != 9) mexErrMsgIdAndTxt("WUST:InvalidInput", "applyBlockLU expects 9 inputs");
    if (nlhs != 1) mexErrMsgIdAndTxt("WUST:InvalidOutput", "applyBlockLU returns exactly 1 output");
    if (!mxIsLogicalScalar(prhs[8])) mexErrMsgIdAndTxt("WUST:InvalidInput", "adjoint must be a logical scalar");
    adjoint = mxIsLogicalScalarTrue(prhs[8]) ? 1 : 0;
    mxInitGPU();
    for (i = 0; i < 8; ++i) g[i] = in_gpu(prhs[i], names[i]);
    {
        const mwSize nd = mxGPUGetNumberOfDimensions(g[0]);
        const mwSize *d = mxGPUGetDimensions(g[0]);
        const int Ny = (int)d[0], Nx = nd > 1 ? (int)d[1] : 1, S = nd > 2 ? (int)d[2] : 1;
        mxGPUArray *u = mxGPUCreateGPUArray(nd, d, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
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
        for (i = 0; i < 8; ++i) mxGPUDestroyGPUArray(g[i]);
        if (rc != WUST_OK) {
            mxGPUDestroyGPUArray(u);
            mexErrMsgIdAndTxt(wust_status_id(rc), "%s", wust_last_error());
        }
        plhs[0] = mxGPUCreateMxArrayOnGPU(u);
        mxGPUDestroyGPUArray(u);
    }
}
