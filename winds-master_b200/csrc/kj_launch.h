// kj_launch.h -- per-case table and launchers of the Kutta-Joukowski kernels.
#pragma once

#include <cuda_runtime.h>

#include "bs_types.h"
#include "wake_types.h"

namespace winds {

struct KJCase {
  long long frame_off;    // ns*3*nsteps*nb per case: ll, bxn, byn, bzn, vblade
  long long t_off;        // first lifting-line target (ns*nb per case)
  long long station_off;  // first station (ns per case): chord, foil
  long long az_off;       // nsteps*nb per case: blade azimuth (MLP features)
  long long rpm_off;      // nsteps per case: rotor speed (loads)
  double rho;             // air density (loads)
  int has_pitch;          // blade pitch per step at az_off (loads), else in the twist
  int foil_base;          // this case's first entry in the foil offset table
  int n_foils;
};

// Features of the bound-circulation MLP per lifting-line point (row t_off + t):
// r/R, chord/R, twist, sin and cos of the blade azimuth, the three
// blade-frame components of the local inflow (vblade at the step plus the
// previous step's induced velocity at the lifting line), the current bound
// circulation (the previous step's converged value), its change over the
// previous step and the change over the step before that.
constexpr int kKJFeatures = 11;

cudaError_t launch_kj_targets(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                              const int *step, const double *ll, double4 *tp, BBox *bb,
                              cudaStream_t s);
cudaError_t launch_kj_update(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                             const int *step, const double *uindb, const double *bxn,
                             const double *byn, const double *bzn, const double *vblade,
                             const double *chord, const int *foil, const int *foil_off,
                             const double *aoa_t, const double *cl_t, const double *cd_t,
                             double relax, double *bound, const int *converged,
                             unsigned long long *res_max, int *diverged, double *cl_out,
                             double *cd_out, double *aoa_out, cudaStream_t s);
cudaError_t launch_kj_features(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                               const int *step, const double *bound, const double *bound_last,
                               const double *bound_last2,
                               const double *vblade, const double *bxn, const double *byn,
                               const double *bzn, const double *uindb, const double *st_r,
                               const double *st_c, const double *st_tw, const double *azim,
                               float *x, cudaStream_t s);
// bound = base + out_scale * y (row order of the lifting-line targets); base
// Gamma_prev, or Gamma_prev + feature 9 (its change) when *base != 0;
// stations with st_lift 0 (no lift in their table), or whose last AoA
// (aoa_prev) is outside their table's stall bounds st_stall, keep Gamma_prev
cudaError_t launch_kj_apply_guess(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                                  const int *step, const int *st_lift, const double2 *st_stall,
                                  const double *aoa_prev, const float *y, const float *out_scale,
                                  const float *feat, const float *base, double *bound,
                                  cudaStream_t s);
// Rotor thrust, torque and power of every case at the step
// (postproc/perform.m:18-62): out[3*case + {0,1,2}] = T, Q, P; dl [rows][3]
// holds the spanwise terms.
cudaError_t launch_kj_loads(const WakeCase *cases, const KJCase *kc, int ncases, int max_st,
                            const int *step, const double *vblade, const double *cl,
                            const double *cd, const double *aoa, const double *st_tw,
                            const double *chord, const double *st_rr, const double *st_dr,
                            const double *rpm, const double *pitch, double *dl, double *out,
                            cudaStream_t s);
// Clears a graph WHILE condition at a step before WakeCase::kj_from.
cudaError_t launch_kj_gate_cond(const WakeCase *cases, const int *step,
                                cudaGraphConditionalHandle h, cudaStream_t s);
// kj_check that also sets a graph WHILE condition (see kj_kernels.cu).
cudaError_t launch_kj_check_cond(int ncases, double tol, int *converged, int *iters,
                                 unsigned long long *res_max, double *res_last, int *active,
                                 int *it_ctr, int maxiter, cudaGraphConditionalHandle h,
                                 cudaStream_t s);
cudaError_t launch_kj_check(int ncases, double tol, int *converged, int *iters,
                            unsigned long long *res_max, double *res_last, int *active,
                            cudaStream_t s);

}  // namespace winds
