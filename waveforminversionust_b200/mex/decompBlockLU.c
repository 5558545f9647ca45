/*
 * decompBlockLU MEX gateway over libwust_b200: drop-in for the reference's
 * Runtime/solver/decompBlockLU.cu (call site HelmholtzSolver.m:167-168).
 *
 *   invT = decompBlockLU(Ld, Ll, Lu, Dd, Dl, Du, Ud, Ul, Uu)
 *   [invT, info] = decompBlockLU(...)       info.total_gpu_ms, info.block_count
 *
 * Inputs are complex single gpuArrays with the reference's shapes
 * (Ld, Ud: Ny x (Nx-1); Ll, Lu, Ul, Uu: (Ny-1) x (Nx-1); Dd: Ny x Nx;
 * Dl, Du: (Ny-1) x Nx).  The library validates them and reports the
 * reference's error identifiers (WUST:InvalidInput, ...).  Build:
 *   mexcuda decompBlockLU.c -I<repo>/include -L<repo>/waveforminversionust_b200 -lwust_b200
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

/* Rows and columns of a 2-D gpuArray (0 x 0 when it has more dimensions). */
static void dims2(const mxGPUArray *g, mwSize *r, mwSize *c) {
    const mwSize *d = mxGPUGetDimensions(g);
    const mwSize nd = mxGPUGetNumberOfDimensions(g);
    *r = nd == 2 ? d[0] : 0;
    *c = nd == 2 ? d[1] : 0;
    mxFree((void *)d);
}

static void release(const mxGPUArray **g, int n) {
    int i;
    for (i = 0; i < n; ++i) mxGPUDestroyGPUArray(g[i]);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
    static const char *names[9] = {"Ld", "Ll", "Lu", "Dd", "Dl", "Du", "Ud", "Ul", "Uu"};
    /* Rows and columns of each block relative to (Ny, Nx): Ld, Ud are
     * Ny x (Nx-1); Ll, Lu, Ul, Uu (Ny-1) x (Nx-1); Dd Ny x Nx; Dl, Du
     * (Ny-1) x Nx (decompBlockLU.cu:247-258). */
    static const int drow[9] = {0, -1, -1, 0, -1, -1, 0, -1, -1};
    static const int dcol[9] = {-1, -1, -1, 0, 0, 0, -1, -1, -1};
    const mxGPUArray *g[9];
    const void *p[9];
    mwSize r, c;
    int i;
    if (nlhs > 2) mexErrMsgIdAndTxt("WUST:InvalidOutput", "decompBlockLU requires invT and optionally a timing struct.");
    if (nrhs != 9) mexErrMsgIdAndTxt("WUST:InvalidInput", "decompBlockLU requires 9 gpuArray inputs.");
    for (i = 0; i < 9; ++i)
        if (!mxIsGPUArray(prhs[i])) mexErrMsgIdAndTxt("WUST:InvalidInput", "decompBlockLU requires 9 gpuArray inputs.");
    mxInitGPU();
    for (i = 0; i < 9; ++i) {
        g[i] = in_gpu(prhs[i], names[i]);
        p[i] = mxGPUGetDataReadOnly(g[i]);
    }
    dims2(g[3], &r, &c);
    if (r < 3 || c < 2 || (double)r * (double)c > 2147483647.0) {
        release(g, 9);
        mexErrMsgIdAndTxt("WUST:InvalidInput", "Block-LU grid must have an interior and fit int indexing.");
    }
    {
        const int Ny = (int)r, Nx = (int)c;
        mwSize odims[3];
        mxGPUArray *invT;
        float ms = 0.f;
        int rc;
        for (i = 0; i < 9; ++i) {
            dims2(g[i], &r, &c);
            if ((long)r != Ny + drow[i] || (long)c != Nx + dcol[i]) {
                release(g, 9);
                mexErrMsgIdAndTxt("WUST:InvalidInput", "Block-LU diagonal/page dimensions disagree.");
            }
        }
        odims[0] = (mwSize)Ny;
        odims[1] = (mwSize)Ny;
        odims[2] = (mwSize)Nx;
        invT = mxGPUCreateGPUArray(3, odims, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
        rc = wust_decomp_block_lu((const wust_c64 *)p[0], (const wust_c64 *)p[1], (const wust_c64 *)p[2],
                                  (const wust_c64 *)p[3], (const wust_c64 *)p[4], (const wust_c64 *)p[5],
                                  (const wust_c64 *)p[6], (const wust_c64 *)p[7], (const wust_c64 *)p[8], Ny, Nx,
                                  (wust_c64 *)mxGPUGetData(invT), &ms, NULL);
        release(g, 9);
        if (rc != WUST_OK) {
            mxGPUDestroyGPUArray(invT);
            mexErrMsgIdAndTxt(wust_status_id(rc), "%s", wust_last_error());
        }
        plhs[0] = mxGPUCreateMxArrayOnGPU(invT);
        mxGPUDestroyGPUArray(invT);
        if (nlhs > 1) {
            static const char *fields[2] = {"total_gpu_ms", "block_count"};
            mxArray *info = mxCreateStructMatrix(1, 1, 2, fields);
            mxSetField(info, 0, "total_gpu_ms", mxCreateDoubleScalar((double)ms));
            mxSetField(info, 0, "block_count", mxCreateDoubleScalar((double)Nx));
            plhs[1] = info;
        }
    }
}
