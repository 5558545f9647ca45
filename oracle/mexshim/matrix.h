/*
 * matrix.h of the MEX runtime stand-in (oracle/mexshim).
 *
 * TEST INFRASTRUCTURE ONLY.  A functional stand-in, written from MathWorks'
 * public documentation of the MEX C API, for the parts of MATLAB's mxArray
 * API that the reference's two MEX kernels (Runtime/solver/decompBlockLU.cu,
 * Runtime/solver/applyBlockLU.cu) and this repository's MEX gateways
 * (the C files in waveforminversionust_b200/mex) use, so both can be compiled and run
 * without MATLAB: the reference's kernels to pin the oracle and time the
 * reference's GPU path, the gateways to test the drop-in boundary.  Complex
 * data is interleaved (re, im), as in MATLAB's interleaved complex API and
 * in gpuArray memory.  Not MATLAB's header.
 */
#ifndef WUST_MEXSHIM_MATRIX_H
#define WUST_MEXSHIM_MATRIX_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef bool mxLogical;
typedef char mxChar;

typedef enum {
    mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
    mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
    mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

void *mxMalloc(size_t n);
void *mxCalloc(size_t n, size_t size);
void mxFree(void *p);

mxArray *mxCreateDoubleScalar(double v);
mxArray *mxCreateLogicalScalar(bool v);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID cls, mxComplexity cplx);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity cplx);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity cplx);
mxArray *mxCreateString(const char *s);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names);
void mxDestroyArray(mxArray *a);

void mxSetField(mxArray *s, mwIndex index, const char *name, mxArray *value);
mxArray *mxGetField(const mxArray *s, mwIndex index, const char *name);

mxClassID mxGetClassID(const mxArray *a);
bool mxIsDouble(const mxArray *a);
bool mxIsSingle(const mxArray *a);
bool mxIsComplex(const mxArray *a);
bool mxIsChar(const mxArray *a);
bool mxIsStruct(const mxArray *a);
bool mxIsLogical(const mxArray *a);
bool mxIsNumeric(const mxArray *a);
bool mxIsInt32(const mxArray *a);
bool mxIsUint8(const mxArray *a);
bool mxIsUint64(const mxArray *a);
bool mxIsEmpty(const mxArray *a);
bool mxIsLogicalScalar(const mxArray *a);
bool mxIsLogicalScalarTrue(const mxArray *a);

mwSize mxGetNumberOfDimensions(const mxArray *a);
const mwSize *mxGetDimensions(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);

void *mxGetData(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
float *mxGetSingles(const mxArray *a);
int32_t *mxGetInt32s(const mxArray *a);
uint8_t *mxGetUint8s(const mxArray *a);
uint64_t *mxGetUint64s(const mxArray *a);
mxLogical *mxGetLogicals(const mxArray *a);
double mxGetScalar(const mxArray *a);
char *mxArrayToString(const mxArray *a);

#ifdef __cplusplus
}
#endif

#endif
