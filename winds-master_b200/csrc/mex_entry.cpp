// mex_entry.cpp -- the [uind,L] = BiotSavartMex(F1,F2,P,gamma,rc,d,cmod,co,
// type,gpu,gpuhw) entry point of cuda/source/BiotSavartMex.cu:688-807, on top
// of the winds_bs C ABI. Linked into libwinds_bs.so (callable through the
// mx shim) and, for MATLAB/Octave, built as the BiotSavartMex MEX file.
//
// Kept from the reference: the 11-input / 2-output check (:720-723), the
// padding of a 2-D or 3-D P to 4-D (:729-764), uind shaped like the padded P
// and L shaped [P1, 1, P3, P4] (:776-783), zero-filled outputs, and the
// dispatch on the first four characters of `type` (:582,591,601).
// Changed on purpose:
//   * cmod and rc are honoured: cmod 'none' is the cut-off core with the
//     squared cut-off d, cmod 'visc' the Vatistas core of index n = d, as in
//     core/BiotSavart.m:102-109 (the reference MEX only had the cut-off and
//     ignored rc and co, :63-93);
//   * co is honoured (core/BiotSavart.m:111);
//   * type 'full' evaluates like 'fuln'/'fuls' (the reference's GPU branch
//     returned zeros for it, which silently dropped the pcc corrector's
//     induction, numerical/pcc.m:58,60);
//   * 'leng' returns |F2-F1| of filament i in L(i) for i < min(#P, #F)
//     (the reference kernel read past the filament arrays, :197-206);
//   * gpu is accepted but the engine always runs on the GPU; gpuhw(3) picks the
//     device and gpuhw(1) (threads per block) is superseded by the autotuner;
//   * errors are raised as winds:bs:* MEX errors instead of being printed.
// The arithmetic precision is FP32 + Kahan with FP64 near-singular terms
// unless the environment variable WINDS_BS_PRECISION is "f64".
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "mex.h"
#include "winds_bs.h"

namespace {

bool g_atexit_registered = false;

std::string get_string(const mxArray *a, const char *what) {
  if (!a || !mxIsChar(a)) mexErrMsgIdAndTxt("winds:bs:type", "%s must be a char array.", what);
  const size_t n = mxGetNumberOfElements(a) + 1;
  std::string s(n, '\0');
  if (mxGetString(a, &s[0], n)) mexErrMsgIdAndTxt("winds:bs:string", "Couldn't make %s string.", what);
  s.resize(std::strlen(s.c_str()));
  return s;
}

const double *get_doubles(const mxArray *a, const char *what) {
  if (!a || !mxIsDouble(a) || mxIsComplex(a))
    mexErrMsgIdAndTxt("winds:bs:type", "%s must be a real double array.", what);
  return mxGetPr(a);
}

double get_scalar(const mxArray *a, const char *what) {
  const double *p = get_doubles(a, what);
  if (mxGetNumberOfElements(a) < 1) mexErrMsgIdAndTxt("winds:bs:size", "%s is empty.", what);
  return p[0];
}

void dims4(const mxArray *a, long long out[4]) {
  const mwSize nd = mxGetNumberOfDimensions(a);
  const mwSize *d = mxGetDimensions(a);
  for (int i = 0; i < 4; ++i) out[i] = i < (int)nd ? (long long)d[i] : 1;
}

}  // namespace

extern "C" void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  if (nrhs != 11) mexErrMsgIdAndTxt("winds:bs:nrhs", "11 inputs expected.");
  if (nlhs != 2) mexErrMsgIdAndTxt("winds:bs:nlhs", "2 outputs expected.");
  if (!g_atexit_registered) {
    mexAtExit(winds_bs_shutdown);
    g_atexit_registered = true;
  }
  const mxArray *F1_in = prhs[0], *F2_in = prhs[1], *P_in = prhs[2], *G_in = prhs[3],
                *RC_in = prhs[4], *D_in = prhs[5], *CMOD_in = prhs[6], *CO_in = prhs[7],
                *TYPE_in = prhs[8], *GPU_in = prhs[9], *HW_in = prhs[10];
  const std::string cmod = get_string(CMOD_in, "Core Model");
  const std::string type = get_string(TYPE_in, "TYPE");
  (void)get_string(GPU_in, "GPU");

  const mwSize ndp = mxGetNumberOfDimensions(P_in);
  if (ndp < 2) mexErrMsgIdAndTxt("winds:bs:pdims", "Need more dimensions in P.");
  if (ndp > 4) mexErrMsgIdAndTxt("winds:bs:pdims", "Wrong dimensions in P.");
  long long pd[4], fd[4];
  dims4(P_in, pd);
  dims4(F1_in, fd);
  const double *P = get_doubles(P_in, "P");
  const double *F1 = get_doubles(F1_in, "F1");
  const double *F2 = get_doubles(F2_in, "F2");
  const double *gam = get_doubles(G_in, "gamma");
  const double *rc = get_doubles(RC_in, "rc");
  const double d = get_scalar(D_in, "d");
  const double co = get_scalar(CO_in, "co");
  const double *hw = get_doubles(HW_in, "gpuhw");

  mwSize od[4] = {(mwSize)pd[0], (mwSize)pd[1], (mwSize)pd[2], (mwSize)pd[3]};
  plhs[0] = mxCreateNumericArray(4, od, mxDOUBLE_CLASS, mxREAL);
  mwSize ld[4] = {(mwSize)pd[0], 1, (mwSize)pd[2], (mwSize)pd[3]};
  plhs[1] = mxCreateNumericArray(4, ld, mxDOUBLE_CLASS, mxREAL);
  double *uind = mxGetPr(plhs[0]);
  double *L = mxGetPr(plhs[1]);

  const long long nf = fd[0] * fd[2] * fd[3];
  const long long np = pd[0] * pd[2] * pd[3];
  if (fd[1] != 3 || mxGetNumberOfElements(F2_in) != (size_t)(3 * nf))
    mexErrMsgIdAndTxt("winds:bs:fdims", "F1 and F2 must both be [n,3,m,k].");
  if (pd[1] != 3) mexErrMsgIdAndTxt("winds:bs:pdims", "P must be [n,3,m,k].");
  if (mxGetNumberOfElements(G_in) != (size_t)nf || mxGetNumberOfElements(RC_in) != (size_t)nf)
    mexErrMsgIdAndTxt("winds:bs:gdims", "gamma and rc must hold one value per filament.");

  winds_bs_params prm;
  std::memset(&prm, 0, sizeof(prm));
  if (cmod.compare(0, 4, "visc") == 0)
    prm.core_model = WINDS_CORE_VATISTAS;
  else if (cmod == "none" || cmod.empty())
    prm.core_model = WINDS_CORE_CUTOFF;
  else
    mexErrMsgIdAndTxt("winds:bs:cmod", "Unknown core model '%s' (expected 'none' or 'visc').",
                      cmod.c_str());

  if (mxGetNumberOfElements(HW_in) >= 3) {
    const int dev = (int)hw[2];
    if (winds_bs_set_device(dev) != WINDS_BS_OK)
      mexErrMsgIdAndTxt("winds:bs:device", "%s", winds_bs_last_error());
  }

  const std::string t4 = type.substr(0, 4);
  if (t4 == "leng") {
    // L(i) = |F2(i)-F1(i)| for the first min(#P, #F) filaments (host arithmetic
    // of core/FilamentLength.m:27-44; no device round trip for O(n) work).
    const long long n = np < nf ? np : nf;
    for (long long f = 0; f < n; ++f) {
      const long long j = f / fd[0], i = f - j * fd[0];
      const long long b = i + fd[0] * 3 * j;
      const double dx = F2[b] - F1[b], dy = F2[b + fd[0]] - F1[b + fd[0]],
                   dz = F2[b + 2 * fd[0]] - F1[b + 2 * fd[0]];
      L[f] = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    return;
  }
  if (t4 != "fuln" && t4 != "fuls" && t4 != "full") return;  // zeros, as the reference
  if (np == 0) return;

  prm.d = d;
  prm.co = co;
  const char *pe = std::getenv("WINDS_BS_PRECISION");
  prm.precision = (pe && std::strcmp(pe, "f64") == 0) ? WINDS_PREC_F64 : WINDS_PREC_F32C;
  prm.flags = 0;

  winds_bs_family fam;
  fam.F1 = F1;
  fam.F2 = F2;
  fam.gamma = gam;
  fam.rc = rc;
  for (int i = 0; i < 4; ++i) fam.dims[i] = fd[i];
  const int rcode = winds_bs_eval_host(&fam, nf > 0 ? 1 : 0, P, pd, &prm, uind);
  if (rcode != WINDS_BS_OK)
    mexErrMsgIdAndTxt("winds:bs:eval", "BiotSavartMex failed (%d): %s", rcode, winds_bs_last_error());
}
