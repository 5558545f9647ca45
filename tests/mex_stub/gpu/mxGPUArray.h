/* Minimal declarations of the MATLAB GPU MEX API (mxGPUArray) used by the
 * gateways in waveforminversionust_b200/mex/, written from MathWorks' public
 * API documentation for syntax checks without MATLAB. */
#ifndef WUST_TEST_MXGPUARRAY_STUB_H
#define WUST_TEST_MXGPUARRAY_STUB_H
#include "mex.h"
typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_INITIALIZE_VALUES = 0, MX_GPU_DO_NOT_INITIALIZE = 1 } mxGPUInitialize;
int mxInitGPU(void);
int mxIsGPUArray(const mxArray *a);
const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a);
mxClassID mxGPUGetClassID(const mxGPUArray *g);
mxComplexity mxGPUGetComplexity(const mxGPUArray *g);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g);
const mwSize *mxGPUGetDimensions(const mxGPUArray *g);
const void *mxGPUGetDataReadOnly(const mxGPUArray *g);
void *mxGPUGetData(mxGPUArray *g);
mxGPUArray *mxGPUCreateGPUArray(mwSize nd, const mwSize *dims, mxClassID c, mxComplexity x, mxGPUInitialize init);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g);
void mxGPUDestroyGPUArray(const mxGPUArray *g);
#endif
