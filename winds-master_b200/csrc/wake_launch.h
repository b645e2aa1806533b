// wake_launch.h -- host launchers of the batched wake-step kernels.
#pragma once

#include <cuda_runtime.h>

#include "bs_launch.h"
#include "wake_types.h"

namespace winds {

enum WakeConvectMode : int {
  kConvectFE = 0,         // numerical/fe.m:31 (also the pcc predictor, pcc.m:38)
  kConvectAB2 = 1,        // numerical/ab2.m:38-39
  kConvectAB4 = 2,        // numerical/ab4.m:77-81
  kConvectCorrector = 3,  // numerical/pcc.m:74-75
};

// Targets of a wake_live table.
enum WakeLiveMode : int {
  kLiveNodes = 0,      // the nodes of the step's live columns
  kLivePredicted = 1,  // the same, none before the pcc corrector starts
  kLiveAll = 2,        // every target of the group (lifting-line points)
};

// Kernels that depend on the wake's live columns read the step counter
// (*step, plus step_add for the pcc prediction of the next step).
// cols > 0: columns j < cols only (max_cols then nb * cols at most).
cudaError_t launch_wake_bookkeep(const WakeCase *cases, int ncases, long long max_cols,
                                 const int *step, int step_add, const double *bound,
                                 const double *trail_prev, double *shed, double *trail,
                                 cudaStream_t s, int cols = 0);
// The Kutta-Joukowski loop's repack: shed columns 0-1 and trailing column 0
// only; per_case is the largest nb * (2 (nst - 1) + nst) of the batch.
cudaError_t launch_wake_filaments_bound_cols(const WakeCase *cases, int ncases, long long per_case,
                                             const int *step, const double *dom,
                                             const double *shed, const double *trail,
                                             const double *rc_in_s, const double *rc_in_t,
                                             int model, double dcut, const PackedFilaments &pf,
                                             cudaStream_t s);
// ser: per-step time and initial core radius (WakeCase::ser_off).
cudaError_t launch_wake_filaments(const WakeCase *cases, int ncases, long long max_fil_pad,
                                  const int *step, int step_add, const double *ser,
                                  const double *dom, const double *shed, const double *trail,
                                  const double *len_old_s, const double *len_old_t, int have_old,
                                  int stretch, double *len_s, double *len_t, double *rc_s,
                                  double *rc_t, const double *rc_in_s, const double *rc_in_t,
                                  int model, double dcut, const PackedFilaments &pf, BBox *bb,
                                  cudaStream_t s);
cudaError_t launch_wake_targets(const WakeCase *cases, int ncases, long long max_nodes,
                                const int *step, int step_add, const double *dom, double4 *tp,
                                int *tgroup, BBox *bb, cudaStream_t s);
// live[case] for one evaluation of step *step + step_add (WakeLiveMode).
cudaError_t launch_wake_live(const WakeCase *cases, int ncases, const int *step, int step_add,
                             int mode, GroupLive *live, cudaStream_t s);
cudaError_t launch_wake_convect(const WakeCase *cases, int ncases, long long max_nodes,
                                const int *step, int mode, const double *dom, const double *uind,
                                const double *carry, const double *pred, const double *uind_pred,
                                double *vel, const double *h1, const double *h2, const double *h3,
                                const double *quarter, const double *trailing, const double *wind,
                                double *out, cudaStream_t s);
cudaError_t launch_wake_commit(const WakeCase *cases, int ncases, long long max_slots, int *step,
                               double *dom, const double *dom_new, double *vel, double *h1,
                               double *h2, double *h3, int keep_hist, double *trail_prev,
                               const double *trail_cur, double *len_old_s, const double *len_s,
                               double *len_old_t, const double *len_t, cudaStream_t s);

}  // namespace winds
