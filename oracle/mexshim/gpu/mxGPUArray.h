/*
 * gpu/mxGPUArray.h of the MEX runtime stand-in (oracle/mexshim).  TEST
 * INFRASTRUCTURE ONLY; see matrix.h.  gpuArray data lives in device memory
 * of the current CUDA device, interleaved complex.  mxGPUGetDimensions
 * returns a copy that the caller releases with mxFree.
 */
#ifndef WUST_MEXSHIM_MXGPUARRAY_H
#define WUST_MEXSHIM_MXGPUARRAY_H

#include "../matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxGPUArray_tag mxGPUArray;

typedef enum { MX_GPU_DO_NOT_INITIALIZE = 0, MX_GPU_INITIALIZE_VALUES = 1 } mxGPUInitialize;

enum { MX_GPU_SUCCESS = 0, MX_GPU_FAILURE = 1 };

int mxInitGPU(void);
bool mxIsGPUArray(const mxArray *a);
const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a);
mxGPUArray *mxGPUCopyFromMxArray(const mxArray *a);
mxGPUArray *mxGPUCreateGPUArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity cplx,
                                mxGPUInitialize init);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g);
void mxGPUDestroyGPUArray(const mxGPUArray *g);
mxClassID mxGPUGetClassID(const mxGPUArray *g);
mxComplexity mxGPUGetComplexity(const mxGPUArray *g);
void *mxGPUGetData(mxGPUArray *g);
const void *mxGPUGetDataReadOnly(const mxGPUArray *g);
const mwSize *mxGPUGetDimensions(const mxGPUArray *g);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g);
mwSize mxGPUGetNumberOfElements(const mxGPUArray *g);

#ifdef __cplusplus
}
#endif

#endif
