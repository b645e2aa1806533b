// wake_kernels.cu -- device kernels of the batched free-wake step (all cases in
// one launch each; blockIdx.y is the case). HBM-bound O(nodes) work around the
// direct sum:
//   wake_bookkeep    Γ bookkeeping, WInDS.m:131-140 / numerical/pcc.m:43-49
//   wake_filaments   FilamentLength + vcore + filamentmod + packing for the
//                    direct sum (core/FilamentLength.m:27-44, core/vcore.m:30-51,
//                    core/filamentmod.m:23-41)
//   wake_targets     node positions -> direct-sum targets
//   wake_convect     fe / ab2 / ab4 / pcc predictor and corrector
//                    (numerical/fe.m:31, ab2.m:38-39, ab4.m:77-81, pcc.m:37-75)
//   wake_commit      end of step: new positions, Γ and length history, counter
//   wake_live        live targets and filaments of every case for one
//                    evaluation (the direct sum's GroupLive table)
// A case keeps `na` age columns of capacity; at step s only its first
// live_cols(c, s) columns hold the wake (the reference's growing
// wake.domain{p} of core/initials.m:44-51 is live_cols = min(2 + s, na)).
// Memory is addressed with the capacity's strides; the packed filaments of
// the direct sum are numbered over the live columns only (shed, then
// trailing), so the live ones are the first of the case's range.
#include "bs_device.cuh"
#include "wake_launch.h"
#include "wake_types.h"

namespace winds {

namespace {

__device__ __forceinline__ double node_comp(const double *dom, const WakeCase &c, int i, int comp,
                                            int j, int b) {
  return dom[c.node_off * 3 + i + (long long)c.nst * (comp + 3 * (j + (long long)c.na * b))];
}
__device__ __forceinline__ long long node_idx(const WakeCase &c, int i, int comp, int j, int b) {
  return c.node_off * 3 + i + (long long)c.nst * (comp + 3 * (j + (long long)c.na * b));
}

// Freestream at (x,y,z) for step s: wind(:,s) * ((H + z)/H)^shear.
__device__ __forceinline__ void wind_at(const WakeCase &c, const double *wind, int s, double z,
                                        double &wx, double &wy, double &wz) {
  const double *w = wind + c.wind_off + 3 * (long long)s;
  double f = 1.0;
  if (c.shear != 0.0) f = pow(fmax(c.hub + z, 1e-3) / c.hub, c.shear);
  wx = w[0] * f;
  wy = w[1] * f;
  wz = w[2] * f;
}

// Squared core of vcore.m:30-37 (core_mode 0: r0(step)^2 + 4 alpha nu (1+a1 Re)
// Time(step)) or of the age form (core_mode 1, t = the filament's age).
__device__ __forceinline__ double core_sq(const WakeCase &c, double r0, double gamma, double t) {
  const double Re = fabs(gamma / c.nu);
  if (c.core_mode == 0) return r0 * r0 + 4.0 * c.alpha * c.nu * (1.0 + c.a1 * Re) * t;
  return c.rc0 * c.rc0 + 4.0 * c.alpha * c.delta * c.nu * (1.0 + c.a1 * Re) * t;
}

// Absolute time (fastout.Time) and initial core radius (wake.r0) of step s.
__device__ __forceinline__ double step_time(const WakeCase &c, const double *ser, int s) {
  return c.has_time ? ser[c.ser_off + s] : c.t0 + s * c.dt;
}
__device__ __forceinline__ double step_r0(const WakeCase &c, const double *ser, int s) {
  return c.has_r0 ? ser[c.ser_off + c.nsteps + s] : c.r0;
}

// trail(i, k, b) of the step being formed: column 0 from the bound circulation
// (diff([0; G; 0])), column k >= 1 from the previous step's column k-1.
__device__ __forceinline__ double trail_col(const WakeCase &c, const double *bound,
                                            const double *trail_prev, int i, int k, int b) {
  const int ns = c.nst - 1;
  if (k == 0) {
    const double *G = bound + c.bound_off + (long long)ns * b;
    const double hi = i < ns ? G[i] : 0.0;
    const double lo = i > 0 ? G[i - 1] : 0.0;
    return hi - lo;
  }
  return trail_prev[c.trail_off + i + (long long)c.nst * ((k - 1) + (long long)(c.na - 1) * b)];
}

}  // namespace

// One thread per (column j, blade b); the span loops are unrolled so a
// thread keeps several loads in flight (the data is small; latency bounds this).
// The step's live columns na_l = live_cols(c, *step + step_add): trailing
// columns 1..na_l-2 come from the previous step's columns 0..na_l-3 (all of
// them while the wake grows; at capacity the oldest is dropped).
// cols > 0: only columns j < cols (the Kutta-Joukowski loop's bound-dependent
// columns); the same arithmetic per column as the full pass.
__global__ void wake_bookkeep(const WakeCase *cases, const int *step, int step_add,
                              const double *bound, const double *trail_prev, double *shed,
                              double *trail, int cols) {
  const WakeCase c = cases[blockIdx.y];
  const int u = blockIdx.x * blockDim.x + threadIdx.x;  // (column j, blade b)
  const int na_l = live_cols(c, *step + step_add);
  const int nc = cols > 0 && cols < na_l ? cols : na_l;
  if (u >= nc * c.nb) return;
  const int j = u % nc, b = u / nc;
  const int ns = c.nst - 1, m = na_l - 1;  // m live trailing columns
  if (j < m) {
#pragma unroll 8
    for (int i = 0; i < c.nst; ++i)
      trail[c.trail_off + i + (long long)c.nst * (j + (long long)(c.na - 1) * b)] =
          trail_col(c, bound, trail_prev, i, j, b);
  }
  // shed(:, 0) = G; shed(:, j) = C_j - C_{j-1}, C_k = cumsum over span of trail(1:end-1, k),
  // C_m = 0 (WInDS.m:139-140)
  double *out = shed + c.shed_off + (long long)ns * (j + (long long)c.na * b);
  if (j == 0) {
#pragma unroll 8
    for (int i = 0; i < ns; ++i) out[i] = bound[c.bound_off + i + (long long)ns * b];
    return;
  }
  double cj = 0.0, cjm1 = 0.0;
#pragma unroll 8
  for (int i = 0; i < ns; ++i) {
    cjm1 += trail_col(c, bound, trail_prev, i, j - 1, b);
    if (j < m) cj += trail_col(c, bound, trail_prev, i, j, b);
    out[i] = cj - cjm1;
  }
}

// One thread per packed filament of the case's range. The live filaments of
// step s = *step + step_add (shed over the live columns, then trailing) get
// their length, core and stretching correction and are packed; the rest of
// the range is inert. Stretching (filamentmod.m:26-41) applies from the time
// index c.stretch_from on, to columns 1..m-2 against the previous lengths of
// the same column index.
__global__ void wake_filaments(const WakeCase *cases, const int *step, int step_add,
                               const double *ser, const double *dom, const double *shed,
                               const double *trail, const double *len_old_s,
                               const double *len_old_t, int have_old, int stretch, double *len_s,
                               double *len_t, double *rc_s, double *rc_t, const double *rc_in_s,
                               const double *rc_in_t, int model, double dcut, PackedFilaments pf,
                               BBox *bb) {
  const WakeCase c = cases[blockIdx.y];
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  float v[16];
  const int ns = c.nst - 1;
  const int s = *step + step_add;
  const int na_l = live_cols(c, s);
  const long long nsh = (long long)ns * na_l * c.nb;
  if (f < live_filaments(c, na_l)) {
    int i, j, b, m;
    double x1, y1, z1, x2, y2, z2, g, age;
    long long slot;
    const double *lold;
    double *lnew, *rcout;
    if (f < nsh) {  // shed: dom(i) -> dom(i+1) at column j
      const int fi = (int)f, q = fi / ns;  // per-case indices fit in 32 bits
      i = fi - q * ns;
      j = q % na_l;
      b = q / na_l;
      m = na_l;
      x1 = node_comp(dom, c, i, 0, j, b), y1 = node_comp(dom, c, i, 1, j, b);
      z1 = node_comp(dom, c, i, 2, j, b);
      x2 = node_comp(dom, c, i + 1, 0, j, b), y2 = node_comp(dom, c, i + 1, 1, j, b);
      z2 = node_comp(dom, c, i + 1, 2, j, b);
      slot = c.shed_off + i + (long long)ns * (j + (long long)c.na * b);
      g = shed[slot];
      age = j * c.dt;
      lold = len_old_s, lnew = len_s, rcout = rc_s;
      if (rc_in_s) rcout = nullptr;
    } else {  // trailing: dom(:, j+1) -> dom(:, j)
      const int ki = (int)(f - nsh), q = ki / c.nst;
      i = ki - q * c.nst;
      j = q % (na_l - 1);
      b = q / (na_l - 1);
      m = na_l - 1;
      x1 = node_comp(dom, c, i, 0, j + 1, b), y1 = node_comp(dom, c, i, 1, j + 1, b);
      z1 = node_comp(dom, c, i, 2, j + 1, b);
      x2 = node_comp(dom, c, i, 0, j, b), y2 = node_comp(dom, c, i, 1, j, b);
      z2 = node_comp(dom, c, i, 2, j, b);
      slot = c.trail_off + i + (long long)c.nst * (j + (long long)(c.na - 1) * b);
      g = trail[slot];
      age = (j + 0.5) * c.dt;
      lold = len_old_t, lnew = len_t, rcout = rc_t;
      if (rc_in_t) rcout = nullptr;
    }
    const double *rc_in = f < nsh ? rc_in_s : rc_in_t;
    double rc;
    if (rc_in) {  // cores held fixed (the Kutta-Joukowski loop keeps the step's vcore)
      rc = rc_in[slot];
    } else {
      const double dx = x2 - x1, dy = y2 - y1, dz = z2 - z1;
      const double L = sqrt(dx * dx + dy * dy + dz * dz);  // |L| (FilamentLength.m:43)
      rc = core_sq(c, step_r0(c, ser, s), g, c.core_mode == 0 ? step_time(c, ser, s) : age);
      if (stretch && have_old && s >= c.stretch_from && j >= 1 && j <= m - 2) {
        // filamentmod.m:29-41: lengths square-rooted again, same column index
        const double a = sqrt(L), o = sqrt(lold[slot]);
        const double strain = (a - o) / o;
        rc = rc * (1.0 / (1.0 + strain));
      }
      lnew[slot] = L;
      if (rcout) rcout[slot] = rc;
    }
    pf.ra[c.fil_off + f] = make_double4(x1, y1, z1, g);
    pf.rb[c.fil_off + f] = make_double4(x2, y2, z2, rc);
    filament_fields(x1, y1, z1, x2, y2, z2, g, rc, model, dcut, v);
    lo[0] = (float)fmin(x1, x2), lo[1] = (float)fmin(y1, y2), lo[2] = (float)fmin(z1, z2);
    hi[0] = (float)fmax(x1, x2), hi[1] = (float)fmax(y1, y2), hi[2] = (float)fmax(z1, z2);
  } else {
    inert_fields(v);
    if (f < c.fil_pad) {
      pf.ra[c.fil_off + f] = make_double4(kInertFar, kInertFar, kInertFar, 0.0);
      pf.rb[c.fil_off + f] = make_double4(kInertFar, kInertFar, kInertFar, 0.0);
    }
  }
  // fil_off and fil_pad are multiples of kFilamentPad, so both filaments of a
  // pair are in this warp and both are stored (real or inert) or neither is
  store_pair_fields(pf.pk, c.fil_off + f, v, f < c.fil_pad);
  bbox_accumulate(lo, hi, bb->fmin, bb->fmax);
}

// Repacks only the filaments whose circulation follows the bound iterate of
// the Kutta-Joukowski loop -- shed columns 0 and 1 and trailing column 0 (the
// bookkeeping's other columns come from the previous step) -- with the step's
// positions and held cores; the other records stay as the full pack before
// the loop wrote them. Same arithmetic and packed numbering (over the step's
// live columns) as wake_filaments, so the records are identical to a full
// repack. Needs at least two live columns (every step has them).
__global__ void wake_filaments_bound_cols(const WakeCase *cases, const int *step,
                                          const double *dom, const double *shed,
                                          const double *trail, const double *rc_in_s,
                                          const double *rc_in_t, int model, double dcut,
                                          PackedFilaments pf) {
  const WakeCase c = cases[blockIdx.y];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ns = c.nst - 1;
  const int n_shed = c.nb * 2 * ns;
  if (t >= n_shed + c.nb * c.nst) return;
  const int na_l = live_cols(c, *step);
  int i, j, b;
  double x1, y1, z1, x2, y2, z2, g, rc;
  long long f;
  if (t < n_shed) {  // shed column j in {0, 1}: dom(i) -> dom(i+1)
    b = t / (2 * ns);
    const int r = t - b * 2 * ns;
    j = r / ns;
    i = r - j * ns;
    f = i + (long long)ns * (j + (long long)na_l * b);
    const long long slot = c.shed_off + i + (long long)ns * (j + (long long)c.na * b);
    x1 = node_comp(dom, c, i, 0, j, b), y1 = node_comp(dom, c, i, 1, j, b);
    z1 = node_comp(dom, c, i, 2, j, b);
    x2 = node_comp(dom, c, i + 1, 0, j, b), y2 = node_comp(dom, c, i + 1, 1, j, b);
    z2 = node_comp(dom, c, i + 1, 2, j, b);
    g = shed[slot];
    rc = rc_in_s[slot];
  } else {  // trailing column 0: dom(:, 1) -> dom(:, 0)
    const int u = t - n_shed;
    b = u / c.nst;
    i = u - b * c.nst;
    const long long slot = c.trail_off + i + (long long)c.nst * ((long long)(c.na - 1) * b);
    f = (long long)ns * na_l * c.nb + i + (long long)c.nst * ((long long)(na_l - 1) * b);
    x1 = node_comp(dom, c, i, 0, 1, b), y1 = node_comp(dom, c, i, 1, 1, b);
    z1 = node_comp(dom, c, i, 2, 1, b);
    x2 = node_comp(dom, c, i, 0, 0, b), y2 = node_comp(dom, c, i, 1, 0, b);
    z2 = node_comp(dom, c, i, 2, 0, b);
    g = trail[slot];
    rc = rc_in_t[slot];
  }
  pack_filament(c.fil_off + f, x1, y1, z1, x2, y2, z2, g, rc, model, dcut, pf.pk, pf.ra, pf.rb);
}

// One thread per node slot of the case: nodes of the live columns of step
// *step + step_add become targets; the other slots are marked unused (w = 1),
// which sorts them after every live target of the case.
__global__ void wake_targets(const WakeCase *cases, const int *step, int step_add,
                             const double *dom, double4 *tp, int *tgroup, BBox *bb) {
  const WakeCase c = cases[blockIdx.y];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)c.nst * c.na * c.nb;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (t < n) {
    const int ti = (int)t, jk = ti / c.nst, i = ti - jk * c.nst;
    tgroup[c.node_off + t] = (int)blockIdx.y;
    if (jk % c.na < live_cols(c, *step + step_add)) {
      const long long base = c.node_off * 3 + i + c.nst * 3 * (long long)jk;
      const double x = dom[base], y = dom[base + c.nst], z = dom[base + 2 * c.nst];
      tp[c.node_off + t] = make_double4(x, y, z, 0.0);
      lo[0] = hi[0] = (float)x;
      lo[1] = hi[1] = (float)y;
      lo[2] = hi[2] = (float)z;
    } else {
      tp[c.node_off + t] = make_double4(0.0, 0.0, 0.0, 1.0);
    }
  }
  bbox_accumulate(lo, hi, bb->tmin, bb->tmax);
}

// One thread per node slot (i, j, b); nodes outside the step's live columns
// do nothing. Modes (WakeConvectMode): the node's velocity wind + uind
// (+ carry) is stored in `vel`, and the node's convected position is pushed
// to column j+1 of `out` (columns 0-1 of `out` come from the kinematics of
// step s+1; a column j+1 beyond the next step's live columns -- the oldest,
// once the wake is at capacity -- is dropped). The corrector reads the stored
// velocity and the predicted positions/induction of column j+1; before step
// c.pcc_from it keeps the predictor's positions (pcc.m:40: no corrector while
// time <= 2). The carry (the corrector's induced velocity, added again at the
// next step: pcc.m:71 then WInDS.m:168) is added only after a corrector step.
__global__ void wake_convect(const WakeCase *cases, const int *step, int mode, const double *dom,
                             const double *uind, const double *carry, const double *pred,
                             const double *uind_pred, double *vel, const double *h1,
                             const double *h2, const double *h3, const double *quarter,
                             const double *trailing, const double *wind, double *out) {
  const WakeCase c = cases[blockIdx.y];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)c.nst * c.na * c.nb;
  if (t >= n) return;
  const int s = *step;
  const int ti = (int)t, q = ti / c.nst;  // per-case indices fit in 32 bits
  const int i = ti - q * c.nst, j = q % c.na, b = q / c.na;
  if (j >= live_cols(c, s)) return;
  double v[3];
  if (mode != kConvectCorrector) {
    double w[3];
    wind_at(c, wind, s, node_comp(dom, c, i, 2, j, b), w[0], w[1], w[2]);
    const bool add_carry = carry && s - 1 >= c.pcc_from;
    for (int k = 0; k < 3; ++k) {
      const long long q = node_idx(c, i, k, j, b);
      v[k] = w[k] + uind[q] + (add_carry ? carry[q] : 0.0);
      vel[q] = v[k];
    }
  } else {
    for (int k = 0; k < 3; ++k) v[k] = vel[node_idx(c, i, k, j, b)];
  }
  if (j == 0) {  // columns 0-1 of the new domain: kinematics of step s+1
    for (int k = 0; k < 3; ++k) {
      const long long kq = c.kin_off + i + (long long)c.nst * (k + 3 * ((s + 1) + (long long)c.nsteps * b));
      out[node_idx(c, i, k, 0, b)] = quarter[kq];
      out[node_idx(c, i, k, 1, b)] = trailing[kq];
    }
    return;
  }
  if (j > live_cols(c, s + 1) - 2) return;  // the oldest column leaves a wake at capacity
  const double dt = c.dt;
  double x[3];
  for (int k = 0; k < 3; ++k) x[k] = node_comp(dom, c, i, k, j, b);
  if (mode == kConvectCorrector) {
    if (s < c.pcc_from) {
      for (int k = 0; k < 3; ++k) out[node_idx(c, i, k, j + 1, b)] = pred[node_idx(c, i, k, j + 1, b)];
      return;
    }
    double w[3];
    wind_at(c, wind, s + 1, node_comp(pred, c, i, 2, j + 1, b), w[0], w[1], w[2]);
    for (int k = 0; k < 3; ++k) {
      const double v1 = w[k] + uind_pred[node_idx(c, i, k, j + 1, b)];
      out[node_idx(c, i, k, j + 1, b)] = x[k] + dt / 2 * (v1 + v[k]);
    }
    return;
  }
  const int hist = s < 3 ? s : 3;  // velocities of earlier steps available
  for (int k = 0; k < 3; ++k) {
    double nx;
    if (mode == kConvectAB2 && hist >= 1) {  // ab2.m:35: full form from time index 2
      const double p1 = j >= 2 ? h1[node_idx(c, i, k, j - 1, b)] : 0.0;
      nx = x[k] + dt / 2 * (3.0 * v[k] - p1);
    } else if (mode == kConvectAB4 && hist >= 3) {  // ab4.m:35: from time index 4
      const double p1 = j >= 2 ? h1[node_idx(c, i, k, j - 1, b)] : 0.0;
      const double p2 = j >= 3 ? h2[node_idx(c, i, k, j - 2, b)] : 0.0;
      const double p3 = j >= 4 ? h3[node_idx(c, i, k, j - 3, b)] : 0.0;
      nx = x[k] + dt / 24 * (55.0 * v[k] - 59.0 * p1 + 37.0 * p2 - 9.0 * p3);
    } else {  // forward Euler (also the pcc predictor)
      nx = x[k] + dt * v[k];
    }
    out[node_idx(c, i, k, j + 1, b)] = nx;
  }
}

// End of step: positions, velocity history, previous trailing Γ and lengths
// (whole capacity slices; columns outside the live ones are never read).
__global__ void wake_commit(const WakeCase *cases, int *step, double *dom, const double *dom_new,
                            double *vel, double *h1, double *h2, double *h3, int keep_hist,
                            double *trail_prev, const double *trail_cur, double *len_old_s,
                            const double *len_s, double *len_old_t, const double *len_t) {
  const WakeCase c = cases[blockIdx.y];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nn = (long long)c.nst * c.na * c.nb;
  const long long nsh = (long long)(c.nst - 1) * c.na * c.nb;
  const long long ntr = (long long)c.nst * (c.na - 1) * c.nb;
  if (t < nn) {
    for (int k = 0; k < 3; ++k) {
      const long long q = c.node_off * 3 + k * nn + t;  // any bijection of the case's slice
      dom[q] = dom_new[q];
      if (keep_hist) {
        h3[q] = h2[q];
        h2[q] = h1[q];
        h1[q] = vel[q];
      }
    }
  }
  if (t < nsh) len_old_s[c.shed_off + t] = len_s[c.shed_off + t];
  if (t < ntr) {
    trail_prev[c.trail_off + t] = trail_cur[c.trail_off + t];
    len_old_t[c.trail_off + t] = len_t[c.trail_off + t];
  }
  // every kernel of this step that reads the counter ran before this one
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) step[0] += 1;
}

// The live part of every case for one direct-sum evaluation (one group per
// case, in case order): filaments of step s = *step + step_add up to the
// filament pad; as targets (mode kLiveNodes) the nodes of that step's live
// columns, (kLivePredicted) the same but none before the pcc corrector starts
// (pcc.m:40), (kLiveAll) every target of the group (lifting-line points).
__global__ void wake_live(const WakeCase *cases, int ncases, const int *step, int step_add,
                          int mode, GroupLive *live) {
  const int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= ncases) return;
  const WakeCase c = cases[ci];
  const int m = live_cols(c, *step + step_add);
  const long long nf = live_filaments(c, m);
  GroupLive g;
  g.f_end = (int)(c.fil_off + (nf + kFilamentPad - 1) / kFilamentPad * kFilamentPad);
  g.pad = 0;
  if (mode == kLiveAll)
    g.t_end = 0x7fffffffffffffffll;
  else if (mode == kLivePredicted && *step < c.pcc_from)
    g.t_end = c.node_off;
  else
    g.t_end = c.node_off + (long long)c.nst * m * c.nb;
  live[ci] = g;
}

// ------------------------------------------------------------ launchers
static dim3 case_grid(long long max_per_case, int ncases, int bs) {
  return dim3((unsigned)((max_per_case + bs - 1) / bs), (unsigned)ncases);
}

cudaError_t launch_wake_bookkeep(const WakeCase *cases, int ncases, long long max_cols,
                                 const int *step, int step_add, const double *bound,
                                 const double *trail_prev, double *shed, double *trail,
                                 cudaStream_t s, int cols) {
  wake_bookkeep<<<case_grid(max_cols, ncases, 128), 128, 0, s>>>(cases, step, step_add, bound,
                                                                  trail_prev, shed, trail, cols);
  return cudaGetLastError();
}

cudaError_t launch_wake_filaments_bound_cols(const WakeCase *cases, int ncases, long long per_case,
                                             const int *step, const double *dom,
                                             const double *shed, const double *trail,
                                             const double *rc_in_s, const double *rc_in_t,
                                             int model, double dcut, const PackedFilaments &pf,
                                             cudaStream_t s) {
  wake_filaments_bound_cols<<<case_grid(per_case, ncases, 128), 128, 0, s>>>(
      cases, step, dom, shed, trail, rc_in_s, rc_in_t, model, dcut, pf);
  return cudaGetLastError();
}

cudaError_t launch_wake_filaments(const WakeCase *cases, int ncases, long long max_fil_pad,
                                  const int *step, int step_add, const double *ser,
                                  const double *dom, const double *shed, const double *trail,
                                  const double *len_old_s, const double *len_old_t, int have_old,
                                  int stretch, double *len_s, double *len_t, double *rc_s,
                                  double *rc_t, const double *rc_in_s, const double *rc_in_t,
                                  int model, double dcut, const PackedFilaments &pf, BBox *bb,
                                  cudaStream_t s) {
  wake_filaments<<<case_grid(max_fil_pad, ncases, 256), 256, 0, s>>>(
      cases, step, step_add, ser, dom, shed, trail, len_old_s, len_old_t, have_old, stretch,
      len_s, len_t, rc_s, rc_t, rc_in_s, rc_in_t, model, dcut, pf, bb);
  return cudaGetLastError();
}

cudaError_t launch_wake_targets(const WakeCase *cases, int ncases, long long max_nodes,
                                const int *step, int step_add, const double *dom, double4 *tp,
                                int *tgroup, BBox *bb, cudaStream_t s) {
  wake_targets<<<case_grid(max_nodes, ncases, 256), 256, 0, s>>>(cases, step, step_add, dom, tp,
                                                                  tgroup, bb);
  return cudaGetLastError();
}

cudaError_t launch_wake_convect(const WakeCase *cases, int ncases, long long max_nodes,
                                const int *step, int mode, const double *dom, const double *uind,
                                const double *carry, const double *pred, const double *uind_pred,
                                double *vel, const double *h1, const double *h2, const double *h3,
                                const double *quarter, const double *trailing, const double *wind,
                                double *out, cudaStream_t s) {
  wake_convect<<<case_grid(max_nodes, ncases, 256), 256, 0, s>>>(
      cases, step, mode, dom, uind, carry, pred, uind_pred, vel, h1, h2, h3, quarter, trailing,
      wind, out);
  return cudaGetLastError();
}

cudaError_t launch_wake_commit(const WakeCase *cases, int ncases, long long max_slots, int *step,
                               double *dom, const double *dom_new, double *vel, double *h1,
                               double *h2, double *h3, int keep_hist, double *trail_prev,
                               const double *trail_cur, double *len_old_s, const double *len_s,
                               double *len_old_t, const double *len_t, cudaStream_t s) {
  wake_commit<<<case_grid(max_slots, ncases, 256), 256, 0, s>>>(
      cases, step, dom, dom_new, vel, h1, h2, h3, keep_hist, trail_prev, trail_cur, len_old_s,
      len_s, len_old_t, len_t);
  return cudaGetLastError();
}

cudaError_t launch_wake_live(const WakeCase *cases, int ncases, const int *step, int step_add,
                             int mode, GroupLive *live, cudaStream_t s) {
  wake_live<<<(ncases + 127) / 128, 128, 0, s>>>(cases, ncases, step, step_add, mode, live);
  return cudaGetLastError();
}

}  // namespace winds
