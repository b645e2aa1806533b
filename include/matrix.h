/*
 * matrix.h -- the mx* subset of the MATLAB External API that WInDS's MEX
 * layer uses, declared from the public API signatures so the engine and the
 * reference's MEX source can be built and called without MATLAB.
 *
 * The implementation (mx_shim.cpp) keeps MATLAB's semantics that matter here:
 * numeric arrays are zero-initialised column-major doubles, char arrays hold
 * 16-bit mxChar, mxCalloc'd memory is released when the MEX call returns, and
 * mexErrMsg* ends the call (here: a C++ exception caught by mxshim_call).
 * When the library is linked into a real MATLAB/Octave MEX file, MATLAB's own
 * headers and libmx replace these.
 */
#ifndef WINDS_MATRIX_SHIM_H
#define WINDS_MATRIX_SHIM_H

#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef unsigned short mxChar;
typedef struct mxArray_tag mxArray;

typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS,
  mxINT8_CLASS,
  mxUINT8_CLASS,
  mxINT16_CLASS,
  mxUINT16_CLASS,
  mxINT32_CLASS,
  mxUINT32_CLASS,
  mxINT64_CLASS,
  mxUINT64_CLASS,
  mxFUNCTION_CLASS
} mxClassID;

typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid,
                              mxComplexity flag);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray *mxCreateDoubleScalar(double value);
mxArray *mxCreateString(const char *str);
void mxDestroyArray(mxArray *pa);

double *mxGetPr(const mxArray *pa);
void *mxGetData(const mxArray *pa);
double mxGetScalar(const mxArray *pa);
const mwSize *mxGetDimensions(const mxArray *pa);
mwSize mxGetNumberOfDimensions(const mxArray *pa);
size_t mxGetNumberOfElements(const mxArray *pa);
size_t mxGetM(const mxArray *pa);
size_t mxGetN(const mxArray *pa);
mxClassID mxGetClassID(const mxArray *pa);
bool mxIsDouble(const mxArray *pa);
bool mxIsChar(const mxArray *pa);
bool mxIsComplex(const mxArray *pa);
int mxGetString(const mxArray *pa, char *buf, mwSize buflen);
char *mxArrayToString(const mxArray *pa);

void *mxCalloc(mwSize n, mwSize size);
void *mxMalloc(mwSize n);
void mxFree(void *ptr);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_MATRIX_SHIM_H */
