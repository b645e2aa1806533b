// wake_types.h -- per-case table of the batched wake step (device copy).
//
// All cases' arrays live in shared buffers; a case's slice starts at its
// offsets. Node arrays are [nst,3,na,nb], shed arrays [ns,na,nb], trailing
// arrays [nst,na-1,nb], bound [ns,nb], kinematics [nst,3,nsteps,nb], wind
// [3,nsteps] (MATLAB column-major within the slice).
#pragma once

namespace winds {

struct WakeCase {
  int nst, nb, na, nsteps;
  long long node_off;   // in nodes (x3 doubles for positions)
  long long shed_off;   // ns*na*nb per case
  long long trail_off;  // nst*(na-1)*nb per case
  long long bound_off;  // ns*nb per case
  long long fil_off;    // first packed filament (multiple of the filament pad)
  long long fil_count;  // ns*na*nb + nst*(na-1)*nb
  long long fil_pad;    // fil_count rounded up to the filament pad
  long long kin_off;    // nst*3*nsteps*nb per case
  long long wind_off;   // 3*nsteps per case
  double dt, t0, shear, hub, r0, rc0, alpha, nu, a1, delta;
  int core_mode, pad;
};

}  // namespace winds
