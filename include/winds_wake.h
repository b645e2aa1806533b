/*
 * winds_wake.h -- C ABI of the device-resident free-wake time step of
 * libwinds_bs: many rotor cases, each with its own span resolution and wake
 * length, stepped together; every step evaluates all cases' induced
 * velocities in one persistent direct-sum launch per evaluation and can be
 * replayed as one CUDA graph.
 *
 * What it replaces in the reference (ndevelder/WInDS-Master), per step:
 *   Γ bookkeeping          WInDS.m:131-140, numerical/pcc.m:43-49
 *   core growth + stretch  core/vcore.m:30-51, core/FilamentLength.m:27-44,
 *                          core/filamentmod.m:23-41
 *   induced velocity       WInDS.m:148-168 (two BiotSavart(Mex) calls),
 *                          numerical/pcc.m:55-71 (two more for the corrector)
 *   convection             numerical/fe.m:31, ab2.m:38-39, ab4.m:77-81, pcc.m:37-75
 *
 * Wake length. Each case holds `na` age columns of capacity. The wake starts
 * with `na_start` live columns and gains one per step, as the reference's
 * wake.domain{p} of p+1 columns does (core/initials.m:44-51,84-87, WInDS.m:127);
 * once it reaches `na` the oldest column is dropped every step (a truncated
 * wake). na_start = 2 starts from core/initials.m's wake.domain{1} (quarter
 * chord and trailing edge); na_start = na (or 0) keeps a truncated wake of na
 * columns from the first step. The live column count is kept on the device, so
 * one captured step graph stays valid while the wake grows.
 *
 * Start-up (winds_wake_params.startup). WINDS_STARTUP_REFERENCE follows the
 * reference's switches on the time index p = s + 1 of step s: step 0 is the
 * step of core/initials.m:138-152 (forward Euler, no Kutta-Joukowski
 * iteration); ab2 runs in full form from p = 2 (ab2.m:35), ab4 from p = 4
 * (ab4.m:35), the pcc corrector from p = 3 (pcc.m:40, `time>2`, before that
 * the predictor stands), filament stretching from time index 4
 * (filamentmod.m:26, `time>3`, for the corrector's evaluation of p+1 too),
 * and the corrector's induced velocity is added again at the next step
 * (pcc.m:71 then WInDS.m:168) only after a corrector step.
 * WINDS_STARTUP_FULL runs every part in its full form as soon as its history
 * exists (ab2 and ab4 as above, the corrector and stretching from step 0, the
 * iteration at every step): the form for a truncated wake that starts with a
 * history. Filament stretching compares new and previous lengths by column
 * index as filamentmod.m does.
 * Arrays use WInDS's MATLAB layout [span, xyz, age, blade], column-major.
 */
#ifndef WINDS_WAKE_H
#define WINDS_WAKE_H

#include "winds_bs.h"

#ifdef __cplusplus
extern "C" {
#endif

#define WINDS_INTEG_FE 0
#define WINDS_INTEG_AB2 1
#define WINDS_INTEG_AB4 2
#define WINDS_INTEG_PCC 3

#define WINDS_STARTUP_FULL 0
#define WINDS_STARTUP_REFERENCE 1

typedef struct winds_wake_batch winds_wake_batch;

/* One rotor case. Host arrays are copied at creation. */
typedef struct {
  int nst;            /* span nodes (trailing filaments per age column); ns = nst-1 stations */
  int nb;             /* blades */
  int na;             /* age columns of capacity (the most the wake keeps) */
  int nsteps;         /* time steps of kinematics and wind provided */
  double dt;          /* time step (1/user.t(3)) */
  double t0;          /* time of step 0 */
  const double *quarter;  /* [nst,3,nsteps,nb] quarter-chord nodes per step (pos.quarter) */
  const double *trailing; /* [nst,3,nsteps,nb] trailing-edge nodes per step (pos.trail)   */
  const double *wind;     /* [3,nsteps] freestream vector per step (wind.infty')         */
  double shear;           /* power-law exponent: wind * ((H+z)/H)^shear (0: uniform)     */
  double hub_height;      /* H                                                          */
  int core_mode;      /* 0: vcore.m, rc^2 = r0^2 + 4 alpha nu (1+a1 Re) t (absolute time)
                         1: age form rc^2 = rc0^2 + 4 alpha delta nu (1+a1 Re) age       */
  double r0, rc0, alpha, nu, a1, delta;
  const double *dom;         /* [nst,3,na,nb] initial node positions (wake.domain); only
                                the first na_start columns are read                    */
  const double *bound;       /* [nst-1,nb] bound circulation (shed column 1)            */
  const double *trail_gamma; /* [nst,na-1,nb] trailing circulation (wake.gamma.trail)   */
  int na_start;              /* live age columns at step 0: 2..na (0: na)                */
  const double *time;        /* [nsteps] absolute time of each step (fastout.Time), the
                                t of core_mode 0; NULL: t0 + step * dt                  */
  const double *r0_step;     /* [nsteps] initial core radius of each step (wake.r0(time),
                                core/initials.m:134-135, read by core/vcore.m:34);
                                NULL: the scalar r0                                     */
} winds_wake_case;

typedef struct {
  int integrator;      /* WINDS_INTEG_* */
  int core_model;      /* WINDS_CORE_* of the direct sum */
  double d;            /* cut-off d, or Vatistas index */
  double co;           /* reach cut-off */
  int precision;       /* WINDS_PREC_* */
  int pcc_double_add;  /* 1: the corrector's induced velocity is also added to the next
                          step's velocity (numerical/pcc.m:71 then WInDS.m:168) */
  int stretch;         /* 1: filament stretching (user.roll = 'true') */
  int startup;         /* WINDS_STARTUP_* (see the top of this file) */
} winds_wake_params;

/* Creates the batch on the current device and uploads every case. */
int winds_wake_create(const winds_wake_case *cases, int ncases, const winds_wake_params *prm,
                      winds_wake_batch **out);

/* Advances every case by `nsteps` steps. use_graph: capture one step into a
 * CUDA graph on the first call and replay it. Synchronous. */
int winds_wake_step(winds_wake_batch *b, int nsteps, int use_graph);

/* Copies one case's state to host arrays (any pointer may be NULL), in the
 * capacity's shapes: dom [nst,3,na,nb], bound [ns,nb], shed [ns,na,nb], trail
 * [nst,na-1,nb], rc_shed / rc_trail (effective squared cores of the last
 * evaluation, same shapes), uind [nst,3,na,nb] (induced velocity of the last
 * step's first evaluation). After k steps, dom holds the positions of step k
 * in its first live_cols(k) columns and the other arrays those of step k-1 in
 * their first live_cols(k-1) (shed, uind) or live_cols(k-1) - 1 (trail)
 * columns, live_cols(s) = min(na_start + s, na); winds_wake_get_live gives
 * the count. */
int winds_wake_get_state(winds_wake_batch *b, int icase, double *dom, double *bound,
                         double *shed, double *trail, double *rc_shed, double *rc_trail,
                         double *uind);

/* Live age columns of one case's wake at the current step (the columns of
 * the positions winds_wake_get_state returns) and the steps run so far. */
int winds_wake_get_live(winds_wake_batch *b, int icase, int *na_live, long long *steps_done);

/* Replaces one case's bound circulation [ns,nb] (e.g. after a Kutta-Joukowski
 * iteration); it enters at the next step's bookkeeping. */
int winds_wake_set_bound(winds_wake_batch *b, int icase, const double *bound);

/* Mean device time per step of the last winds_wake_step call (ms, CUDA
 * events around its steps), interactions per step over all cases and
 * evaluations (the mean over that call's steps while a wake grows), and the
 * number of kernels one step launches. */
int winds_wake_stats(winds_wake_batch *b, double *step_ms, long long *interactions,
                     int *launches_per_step);

/* ----------------------------------------------- Kutta-Joukowski (optional)
 * With a lifting line set, every step runs the fixed-point iteration of
 * core/KuttaJoukowski.m:42-49 after the convection (as WInDS.m:182 does after
 * pcc): each iteration evaluates every case's shed and trailing filaments at
 * its lifting-line points (kj(), :215-227) with the step's cores, transforms
 * to the blade frame, interpolates the airfoil tables and relaxes the bound
 * circulation; a case stops when max |dg/(|Γ|+1)| <= tol or after maxiter. */
typedef struct {
  const double *ll;        /* [ns,3,nsteps,nb] lifting-line points (pos.bound)          */
  const double *bxn;       /* [ns,3,nsteps,nb] blade-frame unit vectors (pos.nodes.bxn) */
  const double *byn;       /* [ns,3,nsteps,nb]                                         */
  const double *bzn;       /* [ns,3,nsteps,nb]                                         */
  const double *vblade;    /* [ns,3,nsteps,nb] blade-frame velocity (vel.blade)         */
  const double *chord;     /* [ns]                                                     */
  const int *foil;         /* [ns] airfoil table of each station (0-based, blade.NFoil) */
  int n_foils;
  const int *foil_points;  /* [n_foils] entries of each table                          */
  const double *aoa;       /* concatenated tables: AoA (deg, ascending), Cl, Cd        */
  const double *cl;
  const double *cd;
  /* Station inputs of the bound-circulation MLP (optional; all four needed by
   * winds_wake_set_mlp): */
  const double *r_over_R;     /* [ns] station radius / rotor radius               */
  const double *chord_over_R; /* [ns] chord / rotor radius                        */
  const double *twist;        /* [ns] local pitch (twist + blade pitch), rad      */
  const double *azimuth;      /* [nsteps,nb] blade azimuth per step, rad          */
  /* Rotor loads (optional; with twist, enables winds_wake_get_loads):
   * postproc/perform.m:18-62 per step. */
  const double *r_station;    /* [ns] station radius (blade.RNodes), m             */
  const double *dr_station;   /* [ns] station width (blade.DRNodes), m             */
  const double *rpm;          /* [nsteps] rotor speed (fastout.RotSpeed), rpm      */
  double rho;                 /* air density (const.rho), kg/m^3                  */
  /* Blade pitch per step and blade (fastout.BldPitch<b>), deg; optional. Given,
   * the loads rotate by and subtract twist + pitch(step, blade) as
   * perform.m:22-33 does and `twist` is the aerodynamic twist alone; NULL: a
   * constant pitch is part of `twist`. */
  const double *pitch;        /* [nsteps,nb]                                      */
} winds_kj_case;

typedef struct {
  double relax;  /* fixed-point relaxation (user.relax) */
  double tol;    /* convergence tolerance (user.tol)   */
  int maxiter;   /* iteration cap (user.maxiter)       */
  int ll_fp64;   /* 1: the iteration's induced velocity at the lifting lines in FP64 (the
                    plain FP64 direct sum) whatever the batch's precision; 0: the batch's */
} winds_kj_params;

/* Attaches one lifting line per case (host arrays copied) and enables the
 * iteration in every later winds_wake_step. */
int winds_wake_set_kj(winds_wake_batch *b, const winds_kj_case *kj, const winds_kj_params *prm);

/* Iterations and final residual of each case in the last step, and the number
 * of lifting-line induced-velocity evaluations that step ran. */
int winds_wake_kj_stats(winds_wake_batch *b, int *iterations, double *residual,
                        long long *ll_evaluations);

/* Cl, Cd and AoA [ns,nb] of one case from the last iteration of the last step. */
int winds_wake_get_perf(winds_wake_batch *b, int icase, double *cl, double *cd, double *aoa);

/* Starts every later step's iteration from the MLP's prediction instead of
 * the previous step's bound circulation (winds_mlp.h; NULL restores the
 * previous-step start). Features per station, in this order: r/R, chord/R,
 * twist, sin(azimuth), cos(azimuth), the local inflow in the blade frame
 * (3 components: vblade at the step plus the previous step's induced
 * velocity at the lifting line, transformed as kj() does), previous bound
 * circulation, its change over the previous step, the change over the step
 * before that; the start value is
 * Gamma_prev + out_scale * network(features) (on the extrapolated base:
 * Gamma_prev + its change + out_scale * network) at stations whose airfoil
 * table has lift, and Gamma_prev at the others (e.g. cylinder root sections:
 * Cl = 0 at every AoA, so their fixed point is Gamma = 0, and the relaxed
 * iteration damps a start error there by only 1 - relax per iteration).
 * The network must have 11 inputs and live on the batch's device; the
 * iteration and its tolerance are unchanged. No reference counterpart
 * (WInDS.m:131 always starts from the previous step). */
struct winds_mlp;
int winds_wake_set_mlp(winds_wake_batch *b, struct winds_mlp *m);

/* Rotor thrust (N), torque (N m) and power (W) of every case at the last step
 * (arrays of ncases; any may be NULL), from the converged Cl, Cd and AoA as
 * postproc/perform.m computes them. */
int winds_wake_get_loads(winds_wake_batch *b, double *thrust, double *torque, double *power);

/* The start value [ns,nb] of the last step's iteration for one case. */
int winds_wake_get_kj_guess(winds_wake_batch *b, int icase, double *guess);

/* The MLP features [ns*nb][11] (rows i + ns*b) of one case at the last step,
 * computed whenever the lifting lines carry the station inputs (training
 * pairs: these rows with the converged bound circulation). */
int winds_wake_get_kj_features(winds_wake_batch *b, int icase, float *x);

void winds_wake_destroy(winds_wake_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_WAKE_H */
