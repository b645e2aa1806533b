// kin_kernels.cu -- blade kinematics on the device (include/winds_kin.h):
// core/kinematics.m, core/velocity.m:36-88, core/DCMRot.m, numerical/ctdiff.m.
//
//   kin_hub     pos.hub: platform motion + DCMRot(hub_nominal, [PtfmYaw PtfmPitch
//               PtfmRoll NacYaw], 'zyxz') (kinematics.m, hub block)
//   kin_points  every node x step x blade: one DCM of the sequence
//               'zzzyxxyzxyz' = [twist 90 pitch precone Az_b Azimuth ShftTilt
//               NacYaw PtfmRoll PtfmPitch PtfmYaw], applied to the node's
//               local points (lead/quarter/trail or bound/colloc/end) + hub
//   kin_frames  blade frames (velocity.m:51-62), the bound-point velocity
//               -ctdiff(pos.bound) + wind (velocity.m:43-49) and vel.blade
//               (velocity.m:63-68)
// FP64 throughout with unfused products summed in the reference's order
// ((a0 b0 + a1 b1) + a2 b2); angles reduced by the nearest multiple of 90
// degrees before conversion, so multiples of 90 give exact 0 and +-1 as
// MATLAB's sind/cosd do.
#include <cmath>
#include <vector>

#include "bs_device.cuh"
#include "engine.h"
#include "winds_kin.h"

namespace winds {
namespace {

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dot3(const double *a, const double *b) {
  return add(add(mul(a[0], b[0]), mul(a[1], b[1])), mul(a[2], b[2]));
}

// (sind t, cosd t): nearest multiple of 90 degrees taken out exactly first.
__device__ __forceinline__ void sincosd(double t, double &s, double &c) {
  const double n = rint(t / 90.0);
  const double r = mul(sub(t, mul(90.0, n)), kPi / 180.0);
  const double s0 = sin(r), c0 = cos(r);
  int q = (int)fmod(n, 4.0);
  if (q < 0) q += 4;
  switch (q) {
    case 0: s = s0; c = c0; break;
    case 1: s = c0; c = -s0; break;
    case 2: s = -s0; c = -c0; break;
    default: s = -c0; c = s0; break;
  }
}

// A <- R A for a rotation of t degrees about axis 'x', 'y' or 'z' (DCMRot.m:27-45).
__device__ void rotate(double (&A)[9], char axis, double t) {
  double s, c;
  sincosd(t, s, c);
  double R[9];
  if (axis == 'x') {
    const double v[9] = {1.0, 0.0, 0.0, 0.0, c, -s, 0.0, s, c};
    for (int k = 0; k < 9; ++k) R[k] = v[k];
  } else if (axis == 'y') {
    const double v[9] = {c, 0.0, s, 0.0, 1.0, 0.0, -s, 0.0, c};
    for (int k = 0; k < 9; ++k) R[k] = v[k];
  } else {
    const double v[9] = {c, -s, 0.0, s, c, 0.0, 0.0, 0.0, 1.0};
    for (int k = 0; k < 9; ++k) R[k] = v[k];
  }
  double B[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      B[3 * i + j] = add(add(mul(R[3 * i], A[j]), mul(R[3 * i + 1], A[3 + j])), mul(R[3 * i + 2], A[6 + j]));
  for (int k = 0; k < 9; ++k) A[k] = B[k];
}

__device__ void apply3(const double (&A)[9], const double *x, double *y) {
  for (int i = 0; i < 3; ++i) y[i] = dot3(A + 3 * i, x);
}

struct KinDev {
  int nt, nb, nst, ns;
  const double *azimuth, *pitch, *nac_yaw, *ptfm, *wind;
  const double *r_trail, *chord_trail, *twist_trail, *r_nodes, *chord, *twist, *precone;
  double overhang, shaft_tilt, tower_ht, twr2shft, ptfm_ref, dx;
  double *hub;                       // [nt,3]
  double *lead, *quarter, *trail;    // [nst,3,nt,nb]
  double *bound, *colloc, *end;      // [ns,3,nt,nb]
  double *bxt, *byt, *bzt, *bxn, *byn, *bzn, *vbound, *vblade;
};

// element (i, c, t, b) of a [n,3,nt,nb] array
__device__ __forceinline__ long long at(const KinDev &k, int n, int i, int c, int t, int b) {
  return i + (long long)n * (c + 3 * (t + (long long)k.nt * b));
}

__global__ void kin_hub(const KinDev k) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k.nt) return;
  double s, c;
  sincosd(k.shaft_tilt, s, c);
  const double nom[3] = {mul(k.overhang, c), 0.0,
                         add(add(add(k.ptfm_ref, k.tower_ht), k.twr2shft), mul(k.overhang, s))};
  double A[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  rotate(A, 'z', k.ptfm[t + 5 * k.nt]);  // PtfmYaw
  rotate(A, 'y', k.ptfm[t + 4 * k.nt]);  // PtfmPitch
  rotate(A, 'x', k.ptfm[t + 3 * k.nt]);  // PtfmRoll
  rotate(A, 'z', k.nac_yaw[t]);          // NacYaw
  double y[3];
  apply3(A, nom, y);
  for (int i = 0; i < 3; ++i) k.hub[t + k.nt * i] = add(k.ptfm[t + i * k.nt], y[i]);
}

// One thread per (node, step, blade): trailing nodes first, then stations.
__global__ void kin_points(const KinDev k) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nodes = k.nst + k.ns;
  if (id >= nodes * k.nt * k.nb) return;
  const int node = (int)(id % nodes);
  const int t = (int)((id / nodes) % k.nt);
  const int b = (int)(id / (nodes * k.nt));
  const bool trailing = node < k.nst;
  const int i = trailing ? node : node - k.nst;
  const double tw = trailing ? k.twist_trail[i] : k.twist[i];
  double A[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  rotate(A, 'z', tw);
  rotate(A, 'z', 90.0);
  rotate(A, 'z', k.pitch[t + (long long)k.nt * b]);
  rotate(A, 'y', k.precone[b]);
  rotate(A, 'x', (360.0 / k.nb) * b);
  rotate(A, 'x', k.azimuth[t]);
  rotate(A, 'y', k.shaft_tilt);
  rotate(A, 'z', k.nac_yaw[t]);
  rotate(A, 'x', k.ptfm[t + 3 * k.nt]);
  rotate(A, 'y', k.ptfm[t + 4 * k.nt]);
  rotate(A, 'z', k.ptfm[t + 5 * k.nt]);
  const double h[3] = {k.hub[t], k.hub[t + k.nt], k.hub[t + 2 * k.nt]};
  const double r = trailing ? k.r_trail[i] : k.r_nodes[i];
  const double ch = trailing ? k.chord_trail[i] : k.chord[i];
  // local points: trailing (lead -c/4, quarter 0, trail 3c/4), stations (bound 0,
  // colloc c/4, end 3c/4), all at span r
  const double xs[3] = {trailing ? -0.25 * ch : 0.0, trailing ? 0.0 : 0.25 * ch, 0.75 * ch};
  double *dst[3] = {trailing ? k.lead : k.bound, trailing ? k.quarter : k.colloc,
                    trailing ? k.trail : k.end};
  const int n = trailing ? k.nst : k.ns;
  for (int p = 0; p < 3; ++p) {
    const double x[3] = {xs[p], 0.0, r};
    double y[3];
    apply3(A, x, y);
    for (int c = 0; c < 3; ++c) dst[p][at(k, n, i, c, t, b)] = add(y[c], h[c]);
  }
}

__device__ void unit3(const double *d, double *u) {
  const double n = __dsqrt_rn(add(add(mul(d[0], d[0]), mul(d[1], d[1])), mul(d[2], d[2])));
  for (int c = 0; c < 3; ++c) u[c] = __ddiv_rn(d[c], n);
}

__device__ void cross3(const double *a, const double *b, double *y) {
  y[0] = sub(mul(a[1], b[2]), mul(a[2], b[1]));
  y[1] = sub(mul(a[2], b[0]), mul(a[0], b[2]));
  y[2] = sub(mul(a[0], b[1]), mul(a[1], b[0]));
}

// numerical/ctdiff.m at step t of the series y(s) = p[at(.., s, ..)].
__device__ double ctdiff(const KinDev &k, const double *p, int n, int i, int c, int t, int b) {
  const int nt = k.nt;
  auto y = [&](int s) { return p[at(k, n, i, c, s, b)]; };
  const double h2 = mul(2.0, k.dx), h12 = mul(12.0, k.dx);
  if (t == 0) return __ddiv_rn(sub(add(-y(2), mul(4.0, y(1))), mul(3.0, y(0))), h2);
  if (t == 1) return __ddiv_rn(sub(y(2), y(0)), h2);
  if (t == nt - 1) return __ddiv_rn(add(sub(mul(3.0, y(nt - 1)), mul(4.0, y(nt - 2))), y(nt - 3)), h2);
  if (t == nt - 2) return __ddiv_rn(sub(y(nt - 1), y(nt - 3)), h2);
  return __ddiv_rn(add(sub(add(-y(t + 2), mul(8.0, y(t + 1))), mul(8.0, y(t - 1))), y(t - 2)), h12);
}

__global__ void kin_frames(const KinDev k) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nodes = k.nst + k.ns;
  if (id >= nodes * k.nt * k.nb) return;
  const int node = (int)(id % nodes);
  const int t = (int)((id / nodes) % k.nt);
  const int b = (int)(id / (nodes * k.nt));
  const bool trailing = node < k.nst;
  const int i = trailing ? node : node - k.nst;
  const int n = trailing ? k.nst : k.ns;
  const double *base = trailing ? k.quarter : k.bound;  // frame origin
  const double *tip = trailing ? k.trail : k.end;       // chordwise point
  double d[3], bx[3], bz[3], by[3];
  for (int c = 0; c < 3; ++c) d[c] = sub(tip[at(k, n, i, c, t, b)], base[at(k, n, i, c, t, b)]);
  unit3(d, bx);
  const int i1 = i == 0 ? 1 : i;  // diff along the span, first row repeated
  for (int c = 0; c < 3; ++c) d[c] = sub(base[at(k, n, i1, c, t, b)], base[at(k, n, i1 - 1, c, t, b)]);
  unit3(d, bz);
  cross3(bz, bx, by);
  double *fx = trailing ? k.bxt : k.bxn, *fy = trailing ? k.byt : k.byn, *fz = trailing ? k.bzt : k.bzn;
  for (int c = 0; c < 3; ++c) {
    fx[at(k, n, i, c, t, b)] = bx[c];
    fy[at(k, n, i, c, t, b)] = by[c];
    fz[at(k, n, i, c, t, b)] = bz[c];
  }
  if (trailing) return;
  double v[3];
  for (int c = 0; c < 3; ++c) {
    v[c] = add(-ctdiff(k, k.bound, n, i, c, t, b), k.wind[t + (long long)k.nt * c]);
    k.vbound[at(k, n, i, c, t, b)] = v[c];
  }
  k.vblade[at(k, n, i, 0, t, b)] = dot3(bx, v);
  k.vblade[at(k, n, i, 1, t, b)] = dot3(by, v);
  k.vblade[at(k, n, i, 2, t, b)] = dot3(bz, v);
}

}  // namespace
}  // namespace winds

using namespace winds;

extern "C" int winds_kinematics(const winds_kin_rotor *r, winds_kin_out *out) {
  if (!r || !out) return fail(WINDS_BS_ERR_ARG, "null argument");
  if (r->nt < 5 || r->nb < 1 || r->nst < 2 || r->ns < 2)
    return fail(WINDS_BS_ERR_ARG, "need nt >= 5, nb >= 1, nst >= 2, ns >= 2 (got %d, %d, %d, %d)",
                r->nt, r->nb, r->nst, r->ns);
  const double *req[] = {r->time, r->azimuth, r->pitch, r->nac_yaw, r->ptfm, r->wind, r->r_trail,
                         r->chord_trail, r->twist_trail, r->r_nodes, r->chord, r->twist, r->precone};
  for (const double *p : req)
    if (!p) return fail(WINDS_BS_ERR_ARG, "null input array");
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1)
    return fail(WINDS_BS_ERR_NODEV, "no CUDA device is visible");
  const long long nt = r->nt, nb = r->nb, nst = r->nst, ns = r->ns;
  // dx = |mean(diff(time))| (ctdiff.m), summed in order
  double acc = 0.0;
  for (long long s = 1; s < nt; ++s) acc += r->time[s] - r->time[s - 1];
  const double dx = std::fabs(acc / (double)(nt - 1));
  if (!(dx > 0.0)) return fail(WINDS_BS_ERR_ARG, "time must advance");
  // inputs and outputs in one device block
  const long long in_n = nt * (1 + nb + 1 + 6 + 3) + 3 * nst + 3 * ns + nb;
  const long long trail_n = nst * 3 * nt * nb, st_n = ns * 3 * nt * nb;
  const long long out_n = 3 * nt + 3 * trail_n + 3 * st_n + 3 * trail_n + 5 * st_n;
  double *blk = nullptr;
  cudaError_t e = cudaMalloc(&blk, (size_t)(in_n + out_n) * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "kinematics buffers");
  std::vector<double> h;
  h.reserve((size_t)in_n);
  auto put = [&](const double *p, long long n) {
    const long long off = (long long)h.size();
    h.insert(h.end(), p, p + n);
    return blk + off;
  };
  KinDev k;
  k.nt = r->nt, k.nb = r->nb, k.nst = r->nst, k.ns = r->ns;
  k.azimuth = put(r->azimuth, nt);
  k.pitch = put(r->pitch, nt * nb);
  k.nac_yaw = put(r->nac_yaw, nt);
  k.ptfm = put(r->ptfm, 6 * nt);
  k.wind = put(r->wind, 3 * nt);
  k.r_trail = put(r->r_trail, nst);
  k.chord_trail = put(r->chord_trail, nst);
  k.twist_trail = put(r->twist_trail, nst);
  k.r_nodes = put(r->r_nodes, ns);
  k.chord = put(r->chord, ns);
  k.twist = put(r->twist, ns);
  k.precone = put(r->precone, nb);
  k.overhang = r->overhang, k.shaft_tilt = r->shaft_tilt, k.tower_ht = r->tower_ht;
  k.twr2shft = r->twr2shft, k.ptfm_ref = r->ptfm_ref, k.dx = dx;
  double *o = blk + in_n;
  auto take = [&](long long n) {
    double *p = o;
    o += n;
    return p;
  };
  k.hub = take(3 * nt);
  k.lead = take(trail_n), k.quarter = take(trail_n), k.trail = take(trail_n);
  k.bound = take(st_n), k.colloc = take(st_n), k.end = take(st_n);
  k.bxt = take(trail_n), k.byt = take(trail_n), k.bzt = take(trail_n);
  k.bxn = take(st_n), k.byn = take(st_n), k.bzn = take(st_n), k.vbound = take(st_n),
  k.vblade = take(st_n);
  e = cudaMemcpy(blk, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  const long long threads = (nst + ns) * nt * nb;
  if (e == cudaSuccess) {
    kin_hub<<<(unsigned)((nt + 127) / 128), 128>>>(k);
    kin_points<<<(unsigned)((threads + 127) / 128), 128>>>(k);
    kin_frames<<<(unsigned)((threads + 127) / 128), 128>>>(k);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  struct Copy {
    double *dst;
    const double *src;
    long long n;
  };
  const Copy copies[] = {{out->hub, k.hub, 3 * nt},         {out->lead, k.lead, trail_n},
                         {out->quarter, k.quarter, trail_n}, {out->trail, k.trail, trail_n},
                         {out->bound, k.bound, st_n},        {out->colloc, k.colloc, st_n},
                         {out->end, k.end, st_n},            {out->bxt, k.bxt, trail_n},
                         {out->byt, k.byt, trail_n},         {out->bzt, k.bzt, trail_n},
                         {out->bxn, k.bxn, st_n},            {out->byn, k.byn, st_n},
                         {out->bzn, k.bzn, st_n},            {out->vbound, k.vbound, st_n},
                         {out->vblade, k.vblade, st_n}};
  for (const Copy &c : copies)
    if (e == cudaSuccess && c.dst)
      e = cudaMemcpy(c.dst, c.src, (size_t)c.n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(blk);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "kinematics");
}
