/* Minimal declarations of the MATLAB MEX C API used by the gateways in
 * waveforminversionust_b200/mex/, written from MathWorks' public API
 * documentation so the gateways can be syntax-checked where MATLAB is not
 * installed.  Not a replacement for MATLAB's own mex.h. */
#ifndef WUST_TEST_MEX_STUB_H
#define WUST_TEST_MEX_STUB_H
#include <stdbool.h>
#include <stddef.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mxFree(void *p);
bool mxIsLogicalScalar(const mxArray *a);
bool mxIsLogicalScalarTrue(const mxArray *a);
mxArray *mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char **names);
void mxSetField(mxArray *s, mwSize index, const char *name, mxArray *value);
mxArray *mxCreateDoubleScalar(double v);
#endif
