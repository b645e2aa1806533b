// wake_types.h -- per-case table of the batched wake step (device copy).
//
// All cases' arrays live in shared buffers; a case's slice starts at its
// offsets. Node arrays are [nst,3,na,nb], shed arrays [ns,na,nb], trailing
// arrays [nst,na-1,nb], bound [ns,nb], kinematics [nst,3,nsteps,nb], wind
// [3,nsteps] (MATLAB column-major within the slice). `na` is the capacity in
// age columns; at step s the first live_cols(c, s) columns of every blade
// hold the wake and the rest are unused.
#pragma once

namespace winds {

struct WakeCase {
  int nst, nb, na, nsteps;
  long long node_off;   // in nodes (x3 doubles for positions)
  long long shed_off;   // ns*na*nb per case
  long long trail_off;  // nst*(na-1)*nb per case
  long long bound_off;  // ns*nb per case
  long long fil_off;    // first packed filament (multiple of the filament pad)
  long long fil_count;  // ns*na*nb + nst*(na-1)*nb (at capacity)
  long long fil_pad;    // fil_count rounded up to the filament pad
  long long kin_off;    // nst*3*nsteps*nb per case
  long long wind_off;   // 3*nsteps per case
  long long ser_off;    // 2*nsteps per case: time, then r0 per step (has_time / has_r0)
  double dt, t0, shear, hub, r0, rc0, alpha, nu, a1, delta;
  int core_mode;
  int na0;              // live age columns at step 0 (na: a truncated wake from the start)
  int has_time, has_r0; // per-step time / initial core radius in the series buffer
  // first step index (or, for stretching, first time index s + step_add) at
  // which each part of the reference's start-up runs (0: from the start)
  int pcc_from;         // pcc corrector (numerical/pcc.m:40)
  int stretch_from;     // filament stretching (core/filamentmod.m:26)
  int kj_from;          // Kutta-Joukowski iteration (none in core/initials.m)
  int pad;
};

// Age columns of case c holding the wake at step s: na0 at step 0, one more
// per step, at most the capacity na (then the oldest column leaves).
__host__ __device__ __forceinline__ int live_cols(const WakeCase &c, long long s) {
  const long long m = (long long)c.na0 + s;
  return m < c.na ? (int)m : c.na;
}

// Filaments of case c with m live columns: ns*m*nb shed, then nst*(m-1)*nb trailing.
__host__ __device__ __forceinline__ long long live_filaments(const WakeCase &c, int m) {
  return (long long)(c.nst - 1) * m * c.nb + (long long)c.nst * (m - 1) * c.nb;
}

}  // namespace winds
