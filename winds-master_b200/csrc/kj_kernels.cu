// kj_kernels.cu -- device kernels of the Kutta-Joukowski fixed point
// (core/KuttaJoukowski.m:42-49 and kj(), :173-298) for every case of a batch.
//   kj_targets   lifting-line points of step s -> direct-sum targets (:216-219)
//   kj_update    blade-frame transform (:241-246), aoa (:258), interp1 of the
//                airfoil tables (:262-269), Γ = ½|V|c Cl (:277), relaxed update
//                (:281), relative residual in FP64 (:290), per station
//   kj_check     per case: converged when max |residual| <= tol (:45)
#include <cmath>

#include "bs_device.cuh"
#include "kj_launch.h"
#include "wake_types.h"

namespace winds {

__global__ void kj_targets(const WakeCase *cases, const KJCase *kc, const int *step,
                           const double *ll, double4 *tp, BBox *bb) {
  const WakeCase c = cases[blockIdx.y];
  const KJCase k = kc[blockIdx.y];
  const int ns = c.nst - 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (t < ns * c.nb) {
    const int i = t % ns, b = t / ns;
    const int s = *step;
    const double *p = ll + k.frame_off + i + (long long)ns * (3 * (s + (long long)c.nsteps * b));
    tp[k.t_off + t] = make_double4(p[0], p[ns], p[2 * ns], 0.0);
    for (int a = 0; a < 3; ++a) lo[a] = hi[a] = (float)p[a * ns];
  }
  bbox_accumulate(lo, hi, bb->tmin, bb->tmax);
}

// MATLAB interp1(x, y, xi): linear, NaN outside [x(1), x(end)].
__device__ double interp1(const double *x, const double *y, int n, double xi) {
  if (!(xi >= x[0] && xi <= x[n - 1])) return NAN;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (x[mid] <= xi) lo = mid; else hi = mid;
  }
  const double t = (xi - x[lo]) / (x[hi] - x[lo]);
  return y[lo] + t * (y[hi] - y[lo]);
}

__global__ void kj_update(const WakeCase *cases, const KJCase *kc, const int *step,
                          const double *uindb, const double *bxn, const double *byn,
                          const double *bzn, const double *vblade, const double *chord,
                          const int *foil, const int *foil_off, const double *aoa_t,
                          const double *cl_t, const double *cd_t, double relax, double *bound,
                          const int *converged, unsigned long long *res_max, int *diverged,
                          double *cl_out, double *cd_out, double *aoa_out) {
  const int ci = blockIdx.y;
  const WakeCase c = cases[ci];
  const KJCase k = kc[ci];
  const int ns = c.nst - 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * c.nb || converged[ci]) return;
  const int i = t % ns, b = t / ns;
  const int s = *step;
  const long long fo = k.frame_off + i + (long long)ns * (3 * (s + (long long)c.nsteps * b));
  const double *u = uindb + 3 * k.t_off + i + (long long)ns * 3 * b;  // [ns,3,nb] of this case
  double rot[3];
  const double *fr[3] = {bxn, byn, bzn};
  for (int a = 0; a < 3; ++a)
    rot[a] = fr[a][fo] * u[0] + fr[a][fo + ns] * u[ns] + fr[a][fo + 2 * ns] * u[2 * ns];
  const double vb0 = vblade[fo], vb1 = vblade[fo + ns], vb2 = vblade[fo + 2 * ns];
  const double tu = vb0 + rot[0], tv = vb1 + rot[1];
  const double Vinf = sqrt(vb0 * vb0 + vb1 * vb1 + vb2 * vb2);
  const double aoa = atan2(-tv, tu) * (180.0 / kPi);
  const int f = foil[k.station_off + i];
  const int o0 = foil_off[k.foil_base + f], o1 = foil_off[k.foil_base + f + 1];
  const double cl = interp1(aoa_t + o0, cl_t + o0, o1 - o0, aoa);
  const double cd = interp1(aoa_t + o0, cd_t + o0, o1 - o0, aoa);
  const long long q = c.bound_off + i + (long long)ns * b;  // station slot of the case
  cl_out[q] = cl;
  cd_out[q] = cd;
  aoa_out[q] = aoa;
  if (isnan(cl)) {
    atomicOr(&diverged[ci], 1);
    return;
  }
  const double gamma = 0.5 * Vinf * chord[k.station_off + i] * cl;
  const double dg = gamma - bound[q];
  bound[q] = bound[q] + relax * dg;
  const double r = fabs(dg / (fabs(gamma) + 1.0));
  atomicMax(&res_max[ci], (unsigned long long)__double_as_longlong(r));
}

// One thread per case: a case converged in this iteration stops updating.
__global__ void kj_check(int ncases, double tol, int *converged, int *iters,
                         unsigned long long *res_max, double *res_last, int *active) {
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci == 0) *active = 0;
  __syncthreads();
  if (ci >= ncases || converged[ci]) return;
  const double r = __longlong_as_double((long long)res_max[ci]);
  res_max[ci] = 0ull;
  res_last[ci] = r;
  iters[ci] += 1;
  if (r <= tol) converged[ci] = 1; else atomicOr(active, 1);
}

cudaError_t launch_kj_targets(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                              const int *step, const double *ll, double4 *tp, BBox *bb,
                              cudaStream_t s) {
  kj_targets<<<dim3((max_st + 127) / 128, ncases), 128, 0, s>>>(cases, kc, step, ll, tp, bb);
  return cudaGetLastError();
}

cudaError_t launch_kj_update(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                             const int *step, const double *uindb, const double *bxn,
                             const double *byn, const double *bzn, const double *vblade,
                             const double *chord, const int *foil, const int *foil_off,
                             const double *aoa_t, const double *cl_t, const double *cd_t,
                             double relax, double *bound, const int *converged,
                             unsigned long long *res_max, int *diverged, double *cl_out,
                             double *cd_out, double *aoa_out, cudaStream_t s) {
  kj_update<<<dim3((max_st + 127) / 128, ncases), 128, 0, s>>>(
      cases, kc, step, uindb, bxn, byn, bzn, vblade, chord, foil, foil_off, aoa_t, cl_t, cd_t,
      relax, bound, converged, res_max, diverged, cl_out, cd_out, aoa_out);
  return cudaGetLastError();
}

cudaError_t launch_kj_check(int ncases, double tol, int *converged, int *iters,
                            unsigned long long *res_max, double *res_last, int *active,
                            cudaStream_t s) {
  const int bs = ncases <= 1024 ? ((ncases + 31) / 32) * 32 : 1024;
  if (ncases > 1024) return cudaErrorInvalidValue;
  kj_check<<<1, bs, 0, s>>>(ncases, tol, converged, iters, res_max, res_last, active);
  return cudaGetLastError();
}

}  // namespace winds
