// mx_shim.cpp -- host implementation of the MATLAB External API subset declared
// in include/matrix.h and include/mex.h, so that a mexFunction (the engine's own
// or the reference's cuda/source/BiotSavartMex.cu:688) can run without MATLAB.
//
// Semantics kept from MATLAB: numeric arrays are zero-filled column-major;
// char arrays store mxChar; mxGetString returns 1 when the buffer is too
// short (it still writes a truncated, terminated string); mxCalloc'd memory
// is released when the MEX call returns; mexErrMsg* aborts the MEX call.
#include "mex.h"

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <vector>

struct mxArray_tag {
  mxClassID cls;
  std::vector<mwSize> dims;  // reported dimensions
  mwSize dimbuf[16];         // dims padded with 1s: callers may read 4 entries
  size_t nelem;
  size_t elsize;
  void *data;
};

namespace {

struct MexError : std::exception {
  std::string id, msg;
  MexError(std::string i, std::string m) : id(std::move(i)), msg(std::move(m)) {}
  const char *what() const noexcept override { return msg.c_str(); }
};

thread_local std::vector<void *> *g_call_allocs = nullptr;
std::mutex g_atexit_mu;
std::vector<void (*)(void)> g_atexit;

size_t class_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: case mxINT64_CLASS: case mxUINT64_CLASS: return 8;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    case mxCHAR_CLASS: case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
    case mxLOGICAL_CLASS: case mxINT8_CLASS: case mxUINT8_CLASS: return 1;
    default: return 0;
  }
}

mxArray *make(mxClassID cls, mwSize ndim, const mwSize *dims) {
  mxArray *a = new mxArray_tag;
  a->cls = cls;
  // MATLAB keeps at least 2 dims and drops trailing singleton dims beyond 2.
  size_t nd = ndim < 2 ? 2 : ndim;
  a->dims.assign(nd, 1);
  for (mwSize i = 0; i < ndim; ++i) a->dims[i] = dims[i];
  while (a->dims.size() > 2 && a->dims.back() == 1) a->dims.pop_back();
  for (int i = 0; i < 16; ++i) a->dimbuf[i] = i < (int)a->dims.size() ? a->dims[i] : 1;
  a->nelem = 1;
  for (mwSize d : a->dims) a->nelem *= d;
  a->elsize = class_size(cls);
  size_t bytes = a->nelem * a->elsize;
  a->data = std::calloc(bytes ? bytes : 1, 1);
  return a;
}

}  // namespace

extern "C" {

mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID classid,
                              mxComplexity flag) {
  if (flag != mxREAL || class_size(classid) == 0) return nullptr;
  return make(classid, ndim, dims);
}

mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag) {
  mwSize d[2] = {m, n};
  return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, flag);
}

mxArray *mxCreateDoubleScalar(double value) {
  mxArray *a = mxCreateDoubleMatrix(1, 1, mxREAL);
  *static_cast<double *>(a->data) = value;
  return a;
}

mxArray *mxCreateString(const char *str) {
  size_t n = std::strlen(str);
  mwSize d[2] = {static_cast<mwSize>(n ? 1 : 0), n};
  mxArray *a = make(mxCHAR_CLASS, 2, d);
  mxChar *c = static_cast<mxChar *>(a->data);
  for (size_t i = 0; i < n; ++i) c[i] = static_cast<unsigned char>(str[i]);
  return a;
}

void mxDestroyArray(mxArray *pa) {
  if (!pa) return;
  std::free(pa->data);
  delete pa;
}

double *mxGetPr(const mxArray *pa) {
  return pa && pa->cls == mxDOUBLE_CLASS ? static_cast<double *>(pa->data) : nullptr;
}
void *mxGetData(const mxArray *pa) { return pa ? pa->data : nullptr; }
double mxGetScalar(const mxArray *pa) {
  if (!pa || pa->nelem == 0) return 0.0;
  if (pa->cls == mxDOUBLE_CLASS) return static_cast<double *>(pa->data)[0];
  if (pa->cls == mxCHAR_CLASS) return static_cast<mxChar *>(pa->data)[0];
  return 0.0;
}
const mwSize *mxGetDimensions(const mxArray *pa) { return pa->dimbuf; }
mwSize mxGetNumberOfDimensions(const mxArray *pa) { return pa->dims.size(); }
size_t mxGetNumberOfElements(const mxArray *pa) { return pa->nelem; }
size_t mxGetM(const mxArray *pa) { return pa->dims[0]; }
size_t mxGetN(const mxArray *pa) { return pa->nelem / (pa->dims[0] ? pa->dims[0] : 1); }
mxClassID mxGetClassID(const mxArray *pa) { return pa->cls; }
bool mxIsDouble(const mxArray *pa) { return pa && pa->cls == mxDOUBLE_CLASS; }
bool mxIsChar(const mxArray *pa) { return pa && pa->cls == mxCHAR_CLASS; }
bool mxIsComplex(const mxArray *) { return false; }

int mxGetString(const mxArray *pa, char *buf, mwSize buflen) {
  if (!pa || pa->cls != mxCHAR_CLASS || buflen == 0) {
    if (buf && buflen) buf[0] = 0;
    return 1;
  }
  const mxChar *c = static_cast<const mxChar *>(pa->data);
  size_t n = pa->nelem;
  size_t k = n < buflen - 1 ? n : buflen - 1;
  for (size_t i = 0; i < k; ++i) buf[i] = static_cast<char>(c[i]);
  buf[k] = 0;
  return n < buflen ? 0 : 1;
}

char *mxArrayToString(const mxArray *pa) {
  if (!pa || pa->cls != mxCHAR_CLASS) return nullptr;
  char *s = static_cast<char *>(mxCalloc(pa->nelem + 1, 1));
  mxGetString(pa, s, pa->nelem + 1);
  return s;
}

void *mxCalloc(mwSize n, mwSize size) {
  void *p = std::calloc(n ? n : 1, size ? size : 1);
  if (g_call_allocs) g_call_allocs->push_back(p);
  return p;
}
void *mxMalloc(mwSize n) { return mxCalloc(n, 1); }
void mxFree(void *ptr) {
  if (!ptr) return;
  if (g_call_allocs) {
    for (auto &q : *g_call_allocs)
      if (q == ptr) q = nullptr;
  }
  std::free(ptr);
}

void mexErrMsgTxt(const char *msg) { throw MexError("", msg ? msg : ""); }

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt ? fmt : "", ap);
  va_end(ap);
  throw MexError(id ? id : "", buf);
}

void mexWarnMsgTxt(const char *) {}

int mexPrintf(const char *fmt, ...) {
  // MATLAB prints to its command window; outside MATLAB the text goes to
  // stderr only when WINDS_MEX_VERBOSE is set.
  if (!std::getenv("WINDS_MEX_VERBOSE")) return 0;
  va_list ap;
  va_start(ap, fmt);
  int n = std::vfprintf(stderr, fmt, ap);
  va_end(ap);
  return n;
}

int mexAtExit(void (*fn)(void)) {
  std::lock_guard<std::mutex> g(g_atexit_mu);
  for (auto f : g_atexit)
    if (f == fn) return 0;
  g_atexit.push_back(fn);
  return 0;
}

void mxshim_run_atexit(void) {
  std::vector<void (*)(void)> fns;
  {
    std::lock_guard<std::mutex> g(g_atexit_mu);
    fns.swap(g_atexit);
  }
  for (auto f : fns) f();
}

int mxshim_call(mex_function_t fn, int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs,
                char *errid, char *errmsg, size_t errcap) {
  std::vector<void *> allocs;
  std::vector<void *> *prev = g_call_allocs;
  g_call_allocs = &allocs;
  int rc = 0;
  if (errcap) {
    if (errid) errid[0] = 0;
    if (errmsg) errmsg[0] = 0;
  }
  try {
    fn(nlhs, plhs, nrhs, prhs);
  } catch (const MexError &e) {
    rc = 1;
    if (errcap && errid) std::snprintf(errid, errcap, "%s", e.id.c_str());
    if (errcap && errmsg) std::snprintf(errmsg, errcap, "%s", e.msg.c_str());
  } catch (const std::exception &e) {
    rc = 1;
    if (errcap && errid) std::snprintf(errid, errcap, "winds:mex:exception");
    if (errcap && errmsg) std::snprintf(errmsg, errcap, "%s", e.what());
  }
  for (void *p : allocs) std::free(p);
  g_call_allocs = prev;
  return rc;
}

}  // extern "C"
