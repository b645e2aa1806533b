/*
 * winds_kin.h -- C ABI of the blade kinematics of libwinds_bs: the positions,
 * blade frames and blade-frame velocities that WInDS computes once per run
 * from the turbine time series, evaluated on the GPU for every node, step
 * and blade at once. The outputs are the wake engine's per-step inputs
 * (winds_wake_case.quarter/trailing, winds_kj_case.ll/bxn/byn/bzn/vblade).
 *
 * What it replaces in the reference (ndevelder/WInDS-Master):
 *   core/kinematics.m  hub position and blade points (rotor platform types;
 *                      the elliptical-wing sequence is not provided)
 *   core/velocity.m:36-88  bound-point velocity (numerical/ctdiff.m), blade
 *                      frames bxn/byn/bzn and bxt/byt/bzt, vel.blade
 *   core/DCMRot.m      the rotation sequences ('zyxz' hub, 'zzzyxxyzxyz' blade)
 * Angles in degrees; arrays column-major in WInDS's layout.
 */
#ifndef WINDS_KIN_H
#define WINDS_KIN_H

#include "winds_bs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nt;                    /* time steps (>= 5 for the velocity stencil)       */
  int nb;                    /* blades                                           */
  int nst;                   /* trailing nodes (blade.RTrail)                    */
  int ns;                    /* stations (blade.RNodes), >= 2                    */
  const double *time;        /* [nt] fastout.Time, s                             */
  const double *azimuth;     /* [nt] fastout.Azimuth                             */
  const double *pitch;       /* [nt,nb] fastout.BldPitch1..nb                    */
  const double *nac_yaw;     /* [nt] fastout.NacYaw                              */
  const double *ptfm;        /* [nt,6] PtfmSurge, PtfmSway, PtfmHeave (m),
                                PtfmRoll, PtfmPitch, PtfmYaw                     */
  const double *wind;        /* [nt,3] wind.infty, m/s                           */
  const double *r_trail;     /* [nst] blade.RTrail                               */
  const double *chord_trail; /* [nst] blade.ChordTrail                           */
  const double *twist_trail; /* [nst] blade.AeroTwstTrail                        */
  const double *r_nodes;     /* [ns] blade.RNodes                                */
  const double *chord;       /* [ns] blade.Chord                                 */
  const double *twist;       /* [ns] blade.AeroTwst                              */
  const double *precone;     /* [nb] turbine.PreCone                             */
  double overhang, shaft_tilt, tower_ht, twr2shft; /* turbine.OverHang, ShftTilt,
                                                      TowerHt, Twr2Shft          */
  double ptfm_ref;           /* platform.PtfmRef                                 */
} winds_kin_rotor;

/* Host output arrays; any pointer may be NULL. */
typedef struct {
  double *hub;                     /* [nt,3]          pos.hub                      */
  double *lead, *quarter, *trail;  /* [nst,3,nt,nb]   pos.lead, pos.quarter, pos.trail */
  double *bound, *colloc, *end;    /* [ns,3,nt,nb]    pos.bound, pos.colloc, pos.end */
  double *bxt, *byt, *bzt;         /* [nst,3,nt,nb]   pos.nodes.bxt, byt, bzt      */
  double *bxn, *byn, *bzn;         /* [ns,3,nt,nb]    pos.nodes.bxn, byn, bzn      */
  double *vbound, *vblade;         /* [ns,3,nt,nb]    vel.bound, vel.blade         */
} winds_kin_out;

/* Evaluates the kinematics on the current device (FP64). Synchronous. */
int winds_kinematics(const winds_kin_rotor *r, winds_kin_out *out);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_KIN_H */
