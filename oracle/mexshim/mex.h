/*
 * mex.h of the MEX runtime stand-in (oracle/mexshim).  TEST INFRASTRUCTURE
 * ONLY; see matrix.h.  mexErrMsgIdAndTxt does not return: the stand-in
 * raises a C++ exception that its call wrapper (mexshim_call) turns into the
 * error identifier and message, the way MATLAB turns it into an MException.
 * C gateways are therefore compiled with -fexceptions.
 */
#ifndef WUST_MEXSHIM_MEX_H
#define WUST_MEXSHIM_MEX_H

#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexErrMsgTxt(const char *msg);
void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...);
int mexAtExit(void (*fn)(void));
void mexLock(void);
void mexUnlock(void);

#ifdef __cplusplus
}
#endif

#endif
