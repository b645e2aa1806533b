// kj_kernels.cu -- device kernels of the Kutta-Joukowski fixed point
// (core/KuttaJoukowski.m:42-49 and kj(), :173-298) for every case of a batch.
//   kj_targets   lifting-line points of step s -> direct-sum targets (:216-219)
//   kj_update    blade-frame transform (:241-246), aoa (:258), interp1 of the
//                airfoil tables (:262-269), Γ = ½|V|c Cl (:277), relaxed update
//                (:281), relative residual in FP64 (:290), per station
//   kj_check     per case: converged when max |residual| <= tol (:45)
//   kj_features, kj_apply_guess   inputs and result of the bound-circulation
//                MLP that replaces the previous-step start value (WInDS.m:131)
//   kj_loads     rotor thrust, torque and power (postproc/perform.m:18-62)
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

// The inflow features are the station's total inflow in the blade frame at
// this step with the induced velocity of the previous step's last iteration
// (uindb, zero before the first step): vblade + [bxn; byn; bzn] uindb, the
// velocity the first iteration of kj() would see (core/KuttaJoukowski.m:241-249).
// The history: bound (the last converged value), bound_last and bound_last2
// (the two before it; equal to bound before there were any).
__global__ void kj_features(const WakeCase *cases, const KJCase *kc, const int *step,
                            const double *bound, const double *bound_last,
                            const double *bound_last2,
                            const double *vblade, const double *bxn,
                            const double *byn, const double *bzn, const double *uindb,
                            const double *st_r, const double *st_c, const double *st_tw,
                            const double *azim, float *x) {
  const WakeCase c = cases[blockIdx.y];
  const KJCase k = kc[blockIdx.y];
  const int ns = c.nst - 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * c.nb) return;
  const int i = t % ns, b = t / ns;
  const int s = *step;
  const long long fo = k.frame_off + i + (long long)ns * (3 * (s + (long long)c.nsteps * b));
  const long long st = k.station_off + i;
  const double az = azim[k.az_off + s + (long long)c.nsteps * b];
  float *f = x + (k.t_off + t) * kKJFeatures;
  f[0] = (float)st_r[st];
  f[1] = (float)st_c[st];
  f[2] = (float)st_tw[st];
  f[3] = (float)sin(az);
  f[4] = (float)cos(az);
  const double *u = uindb + 3 * k.t_off + i + (long long)ns * 3 * b;
  const double *fr[3] = {bxn, byn, bzn};
  for (int a = 0; a < 3; ++a)
    f[5 + a] = (float)(vblade[fo + a * ns] +
                       (fr[a][fo] * u[0] + fr[a][fo + ns] * u[ns] + fr[a][fo + 2 * ns] * u[2 * ns]));
  const long long q = c.bound_off + i + (long long)ns * b;
  f[8] = (float)bound[q];
  f[9] = (float)(bound[q] - bound_last[q]);
  f[10] = (float)(bound_last[q] - bound_last2[q]);
}

// bound = base + out_scale * y, base Gamma_prev or, with *base != 0, its
// extrapolation Gamma_prev + dGamma_prev (feature 9 of the row). Two kinds of
// station keep Gamma_prev: those whose airfoil table has no lift (st_lift 0:
// Cl = 0 at every AoA, e.g. the cylinder root sections; their fixed point is
// Gamma = 0, the previous step already sits there, and the relaxed iteration
// damps any start error there by only 1 - relax per iteration), and those
// whose last converged AoA (aoa_prev) lies outside their table's stall bounds
// st_stall (the AoA of its lowest and highest Cl) less kStallMargin degrees:
// past stall a station can have more than one fixed point, and the previous
// step's value is the start that keeps the branch it is on.
// Nothing before the step the iteration starts at (WakeCase::kj_from).
constexpr double kStallMargin = 2.0;  // degrees
__global__ void kj_apply_guess(const WakeCase *cases, const KJCase *kc, const int *step,
                               const int *st_lift, const double2 *st_stall,
                               const double *aoa_prev, const float *y, const float *out_scale,
                               const float *feat, const float *base, double *bound) {
  const WakeCase c = cases[blockIdx.y];
  const KJCase k = kc[blockIdx.y];
  const int ns = c.nst - 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * c.nb || *step < c.kj_from) return;
  const int i = t % ns, b = t / ns;
  if (!st_lift[k.station_off + i]) return;
  const double2 sb = st_stall[k.station_off + i];
  const double ap = aoa_prev[c.bound_off + i + (long long)ns * b];
  if (!(ap > sb.x + kStallMargin && ap < sb.y - kStallMargin)) return;
  double g = bound[c.bound_off + i + (long long)ns * b];
  if (*base != 0.f) g += (double)feat[(k.t_off + t) * kKJFeatures + 9];
  bound[c.bound_off + i + (long long)ns * b] = g + (double)*out_scale * (double)y[k.t_off + t];
}

// Spanwise loads of one station (postproc/perform.m:20-55): the blade-frame
// velocity to the rotor frame, velX = -Rz(theta - 90 deg) vblade with theta =
// twist + pitch (DCMRot with the 'zzz' sequence [-90, twist, pitch]); inflow
// angle phi = aoa - theta; a/a' = TSR / tan(phi); a and a'; normal and
// tangential coefficients; dT, dQ, dP.
__global__ void kj_dloads(const WakeCase *cases, const KJCase *kc, const int *step,
                          const double *vblade, const double *cl, const double *cd,
                          const double *aoa, const double *st_tw, const double *chord,
                          const double *st_rr, const double *st_dr, const double *rpm,
                          const double *pitch, double *dl) {
  const WakeCase c = cases[blockIdx.y];
  const KJCase k = kc[blockIdx.y];
  const int ns = c.nst - 1;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ns * c.nb) return;
  const int i = t % ns, b = t / ns;
  const int s = *step;
  const long long fo = k.frame_off + i + (long long)ns * (3 * (s + (long long)c.nsteps * b));
  const long long st = k.station_off + i;
  const long long q = c.bound_off + i + (long long)ns * b;
  double th = st_tw[st] * (180.0 / kPi);  // deg
  if (k.has_pitch) th += pitch[k.az_off + s + (long long)c.nsteps * b];
  const double rot = (th - 90.0) * (kPi / 180.0);
  const double cr = cos(rot), sr = sin(rot);
  const double u0 = vblade[fo], u1 = vblade[fo + ns];
  const double v1 = -(cr * u0 - sr * u1);
  const double v2 = -(sr * u0 + cr * u1);
  const double tsr = v2 / v1;
  const double phi = aoa[q] - th;
  const double pr = phi * (kPi / 180.0);
  const double tp = tan(pr);
  const double aap = tsr / tp;
  const double a = aap * (v1 - tp * v2) / (aap * v1 + tp * v2);
  const double ap = a / aap;
  const double cz = cl[q] * cos(pr) + cd[q] * sin(pr);
  const double cx = cl[q] * sin(pr) - cd[q] * cos(pr);
  const double w1 = v1 * (1.0 - a), w2 = v2 * (1.0 + ap);
  const double w = w1 * w1 + w2 * w2;
  const double dT = 0.5 * k.rho * chord[st] * cz * w * st_dr[st];
  const double dQ = 0.5 * k.rho * chord[st] * cx * w * st_rr[st] * st_dr[st];
  double *o = dl + 3 * (k.t_off + t);
  o[0] = dT;
  o[1] = dQ;
  o[2] = (kPi / 30.0) * rpm[k.rpm_off + s] * dQ;
}

// Rotor totals, summed over stations and then blades as sum(sum(dT,1),4).
__global__ void kj_sum_loads(const WakeCase *cases, const KJCase *kc, int ncases,
                             const double *dl, double *out) {
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= ncases) return;
  const WakeCase c = cases[ci];
  const KJCase k = kc[ci];
  const int ns = c.nst - 1;
  double tot[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < c.nb; ++b) {
    double sb[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < ns; ++i)
      for (int a = 0; a < 3; ++a) sb[a] += dl[3 * (k.t_off + i + (long long)ns * b) + a];
    for (int a = 0; a < 3; ++a) tot[a] += sb[a];
  }
  for (int a = 0; a < 3; ++a) out[3 * ci + a] = tot[a];
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

// kj_check inside a graph's conditional WHILE node: the same per-case update,
// then one thread sets the loop condition -- continue while any case is active
// and fewer than maxiter iterations ran (the counter makes the loop finite).
__global__ void kj_check_cond(int ncases, double tol, int *converged, int *iters,
                              unsigned long long *res_max, double *res_last, int *active,
                              int *it_ctr, int maxiter, cudaGraphConditionalHandle h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int ci = threadIdx.x; ci < ncases; ci += blockDim.x) {
    if (converged[ci]) continue;
    const double r = __longlong_as_double((long long)res_max[ci]);
    res_max[ci] = 0ull;
    res_last[ci] = r;
    iters[ci] += 1;
    if (r <= tol) converged[ci] = 1; else atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *active = any;
    const int it = *it_ctr + 1;
    *it_ctr = it;
    cudaGraphSetConditional(h, (any && it < maxiter) ? 1u : 0u);
  }
}

// Upstream of a graph's WHILE node: no iteration at a step before the one the
// iteration starts at (WakeCase::kj_from, the same for every case; the
// reference's first step is core/initials.m's, which has none).
__global__ void kj_gate_cond(const WakeCase *cases, const int *step, cudaGraphConditionalHandle h) {
  if (threadIdx.x == 0 && *step < cases[0].kj_from) cudaGraphSetConditional(h, 0u);
}

cudaError_t launch_kj_gate_cond(const WakeCase *cases, const int *step,
                                cudaGraphConditionalHandle h, cudaStream_t s) {
  kj_gate_cond<<<1, 32, 0, s>>>(cases, step, h);
  return cudaGetLastError();
}

cudaError_t launch_kj_check_cond(int ncases, double tol, int *converged, int *iters,
                                 unsigned long long *res_max, double *res_last, int *active,
                                 int *it_ctr, int maxiter, cudaGraphConditionalHandle h,
                                 cudaStream_t s) {
  const int bs = ncases <= 1024 ? ((ncases + 31) / 32) * 32 : 1024;
  kj_check_cond<<<1, bs, 0, s>>>(ncases, tol, converged, iters, res_max, res_last, active, it_ctr,
                                 maxiter, h);
  return cudaGetLastError();
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

cudaError_t launch_kj_features(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                               const int *step, const double *bound, const double *bound_last,
                               const double *bound_last2, const double *vblade,
                               const double *bxn, const double *byn, const double *bzn,
                               const double *uindb, const double *st_r,
                               const double *st_c, const double *st_tw, const double *azim,
                               float *x, cudaStream_t s) {
  kj_features<<<dim3((max_st + 127) / 128, ncases), 128, 0, s>>>(
      cases, kc, step, bound, bound_last, bound_last2, vblade, bxn, byn, bzn, uindb, st_r, st_c,
      st_tw, azim, x);
  return cudaGetLastError();
}

cudaError_t launch_kj_apply_guess(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                                  const int *step, const int *st_lift, const double2 *st_stall,
                                  const double *aoa_prev, const float *y, const float *out_scale,
                                  const float *feat, const float *base, double *bound,
                                  cudaStream_t s) {
  kj_apply_guess<<<dim3((max_st + 127) / 128, ncases), 128, 0, s>>>(
      cases, kc, step, st_lift, st_stall, aoa_prev, y, out_scale, feat, base, bound);
  return cudaGetLastError();
}

cudaError_t launch_kj_loads(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                            const int *step, const double *vblade, const double *cl,
                            const double *cd, const double *aoa, const double *st_tw,
                            const double *chord, const double *st_rr, const double *st_dr,
                            const double *rpm, const double *pitch, double *dl, double *out,
                            cudaStream_t s) {
  kj_dloads<<<dim3((max_st + 127) / 128, ncases), 128, 0, s>>>(
      cases, kc, step, vblade, cl, cd, aoa, st_tw, chord, st_rr, st_dr, rpm, pitch, dl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  kj_sum_loads<<<(ncases + 127) / 128, 128, 0, s>>>(cases, kc, ncases, dl, out);
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
