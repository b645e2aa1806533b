/*
 * mex.h -- the mex* subset of the MATLAB External API used by WInDS's
 * BiotSavartMex (cuda/source/BiotSavartMex.cu:1-2,688) and by this library's
 * own mexFunction; declared from the public signatures. See matrix.h.
 *
 * mxshim_call() is not a MATLAB function: it is how a host without MATLAB
 * (Python/ctypes, C tests) invokes a mexFunction, turning mexErrMsg* into a
 * return code and message, and releasing mxCalloc'd memory afterwards.
 */
#ifndef WINDS_MEX_SHIM_H
#define WINDS_MEX_SHIM_H

#include "matrix.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void (*mex_function_t)(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#if defined(__GNUC__)
#define WINDS_MEX_NORETURN __attribute__((noreturn))
#else
#define WINDS_MEX_NORETURN
#endif

void mexErrMsgTxt(const char *msg) WINDS_MEX_NORETURN;
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) WINDS_MEX_NORETURN;
void mexWarnMsgTxt(const char *msg);
int mexPrintf(const char *fmt, ...);
int mexAtExit(void (*fn)(void));

/* Calls fn(nlhs, plhs, nrhs, prhs). Returns 0, or 1 when fn raised a MEX
 * error (id and message are copied into errid / errmsg, each of capacity
 * errcap). Output arrays stay owned by the caller (mxDestroyArray). */
int mxshim_call(mex_function_t fn, int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs,
                char *errid, char *errmsg, size_t errcap);

/* Runs and clears the functions registered with mexAtExit. */
void mxshim_run_atexit(void);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_MEX_SHIM_H */
