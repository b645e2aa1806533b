// bs_kernels.cu -- sm_100a kernels of the induced-velocity (Biot-Savart) direct
// sum that replaces core/BiotSavart.m:80-116 and the BiotSavart_naive /
// BiotSavart_sh kernels of cuda/source/BiotSavartMex.cu:131-193.
//
// Kernels
//   bs_pack_filaments  MATLAB-layout F1/F2/gamma/rc -> packed SoA float4 tiles
//                      (+ FP64 copies), the device-side replacement of the host
//                      crunch_f / crunch_rg packing (BiotSavartMex.cu:316-357)
//   bs_chain_count,    the same records laid out along the wake's lines of
//   bs_pack_chains     filaments (each lane of a record continuing the lane of
//                      the record before: x2 = previous x1), with a head bit per
//                      record where a line starts or the input has no link
//   bs_pack_targets    MATLAB-layout P -> double4 targets (crunch_p, :361-379)
//   bs_f32c            persistent FP32 direct sum on independent warp workers:
//                      each warp stages its filament tiles into its own shared
//                      memory by bulk copies (cp.async.bulk + mbarrier), keeps
//                      T register-resident targets per lane, Kahan-compensates
//                      the per-target sums, and recomputes the near-singular
//                      pairs in FP64 with all 32 lanes; on a chained stream
//                      (CHAIN) each interaction reuses the previous record's
//                      endpoint rsqrt
//   bs_f64             plain FP64 direct sum (the comparison GPU path)
//   bs_reduce          deterministic sum of the per-chunk partials, written in
//                      MATLAB layout (reassem_uind, :383-401)
//   bs_length          filament lengths (core/FilamentLength.m:27-44)
#include "bs_device.cuh"
#include "bs_launch.h"
#include "bs_types.h"

#include <cfloat>

#include <cub/device/device_radix_sort.cuh>

namespace winds {

// --------------------------------------------------------------- packing
__global__ void bs_bbox_init(BBox *bb) {
  if (threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      bb->tmin[c] = bb->fmin[c] = float_key(FLT_MAX);
      bb->tmax[c] = bb->fmax[c] = float_key(-FLT_MAX);
    }
  }
}

__global__ void bs_pack_filaments(const double *__restrict__ F1, const double *__restrict__ F2,
                                  const double *__restrict__ gam, const double *__restrict__ rc,
                                  long long d0, long long nf, long long off, int model, double dcut,
                                  float4 *pk, double4 *ra,
                                  double4 *rb, BBox *bb) {
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (f < nf) {
    const long long j = f / d0, i = f - j * d0;
    const long long b = i + d0 * 3 * j;
    const double x1 = F1[b], y1 = F1[b + d0], z1 = F1[b + 2 * d0];
    const double x2 = F2[b], y2 = F2[b + d0], z2 = F2[b + 2 * d0];
    const double g = gam[f], r = rc[f];
    pack_filament(off + f, x1, y1, z1, x2, y2, z2, g, r, model, dcut, pk, ra, rb);
    lo[0] = (float)fmin(x1, x2), lo[1] = (float)fmin(y1, y2), lo[2] = (float)fmin(z1, z2);
    hi[0] = (float)fmax(x1, x2), hi[1] = (float)fmax(y1, y2), hi[2] = (float)fmax(z1, z2);
  }
  bbox_accumulate(lo, hi, bb->fmin, bb->fmax);
}

// Inert filaments filling [from, to): far away, zero length, zero circulation.
__global__ void bs_pad_filaments(long long from, long long to, float4 *pk, double4 *ra,
                                 double4 *rb) {
  const long long f = from + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= to) return;
  pack_inert(f, pk, ra, rb);
}

// ------------------------------------------------------- chained packing
// WInDS's filaments meet at the wake's nodes: the shed call's F2(i) is its
// F1(i+1) (WInDS.m:150, along the first index) and the trailing call's
// F2(:,:,j) is its F1(:,:,j-1) (WInDS.m:153, along the third). Laid out so that
// each lane of a pair record follows one such line -- x2 of record r equal to
// x1 of record r - 1 -- the FP32 kernel reuses the previous record's endpoint
// term (interact_chain). bs_chain_count counts, per family, the filaments
// whose end is bitwise the start of their neighbour along each index;
// bs_pack_chains lays the family out along the index with more such links,
// lines paired in the two lanes of the records, and flags every record where
// either lane does not continue its predecessor (a head). Any layout of the
// input is evaluated correctly: a filament that does not continue a chain is
// a head, which the kernel evaluates from its own L.
__device__ __forceinline__ bool same_point(const double *__restrict__ F2, long long b2,
                                           const double *__restrict__ F1, long long b1,
                                           long long d0) {
  return F2[b2] == F1[b1] && F2[b2 + d0] == F1[b1 + d0] && F2[b2 + 2 * d0] == F1[b1 + 2 * d0];
}

__global__ void bs_chain_count(const double *__restrict__ F1, const double *__restrict__ F2,
                               long long d0, long long d2, long long nf,
                               unsigned long long *cnt) {
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool s = false, t = false;
  if (f < nf) {
    const long long jb = f / d0, i = f - jb * d0, j = jb % d2;
    const long long b = i + d0 * 3 * jb;
    if (i + 1 < d0) s = same_point(F2, b, F1, b + 1, d0);   // F2(i) == F1(i+1)
    if (j >= 1) t = same_point(F2, b, F1, b - 3 * d0, d0);  // F2(:,:,j) == F1(:,:,j-1)
  }
  const unsigned ns = __popc(__ballot_sync(0xffffffffu, s));
  const unsigned nt = __popc(__ballot_sync(0xffffffffu, t));
  if ((threadIdx.x & 31) == 0) {
    if (ns) atomicAdd(cnt, (unsigned long long)ns);
    if (nt) atomicAdd(cnt + 1, (unsigned long long)nt);
  }
}

// Records of nl lines of len filaments: pairs of lines side by side, and an
// odd last line split in two halves side by side.
__host__ __device__ __forceinline__ long long chain_layout_records(long long nl, long long len) {
  return nl / 2 * len + (nl & 1) * ((len + 1) / 2);
}

// One thread per lane slot of the family's nrec records from record rec_off:
// slot 2 r + h is lane h of record r. Order along the third index when cnt[1]
// > cnt[0] (lines (i, b), position k = j), else along the first (lines (j, b),
// position k = d0 - 1 - i). Line 2 m + h fills lane h of the m-th run of `len`
// records; an odd last line fills lane 0 with its first (len + 1) / 2
// positions and lane 1 with the rest. Slots past the lines are inert heads.
__global__ void bs_pack_chains(const double *__restrict__ F1, const double *__restrict__ F2,
                               const double *__restrict__ gam, const double *__restrict__ rc,
                               long long d0, long long d2, long long d3, long long rec_off,
                               long long nrec, const unsigned long long *__restrict__ cnt,
                               int model, double dcut, float4 *pk, double4 *ra, double4 *rb,
                               unsigned *heads, BBox *bb) {
  const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (slot < 2 * nrec) {
    const bool along3 = cnt[1] > cnt[0];
    const long long nl = along3 ? d0 * d3 : d2 * d3;
    const long long len = along3 ? d2 : d0;
    const long long r = slot >> 1;
    const long long h = slot & 1;
    const long long f = 2 * rec_off + slot;  // packed filament index
    long long k = 0, run = 0, line = -1;      // position in the line, in this lane's run
    const long long full = nl / 2 * len, half = (len + 1) / 2;
    if (r < full) {
      const long long m = r / len;
      run = k = r - m * len;
      line = 2 * m + h;
    } else if ((nl & 1) && r < full + half) {
      run = r - full;
      k = run + h * half;
      if (k < len) line = nl - 1;
    }
    bool head;
    if (line >= 0 && line < nl) {
      long long i, jb;
      if (along3) {
        const long long bl = line / d0;
        i = line - bl * d0;
        jb = k + d2 * bl;
      } else {
        i = d0 - 1 - k;
        jb = line;
      }
      const long long b = i + d0 * 3 * jb;
      const double x1 = F1[b], y1 = F1[b + d0], z1 = F1[b + 2 * d0];
      const double x2 = F2[b], y2 = F2[b + d0], z2 = F2[b + 2 * d0];
      const long long src = i + d0 * jb;
      pack_filament(f, x1, y1, z1, x2, y2, z2, gam[src], rc[src], model, dcut, pk, ra, rb);
      lo[0] = (float)fmin(x1, x2), lo[1] = (float)fmin(y1, y2), lo[2] = (float)fmin(z1, z2);
      hi[0] = (float)fmax(x1, x2), hi[1] = (float)fmax(y1, y2), hi[2] = (float)fmax(z1, z2);
      // the predecessor in the line is (i, j-1) along the third index, (i+1, j) along the first
      head = run == 0 || !(along3 ? same_point(F2, b, F1, b - 3 * d0, d0)
                                  : same_point(F2, b, F1, b + 1, d0));
    } else {
      pack_inert(f, pk, ra, rb);
      head = true;  // never continues a real lane (its x2 would not be its own)
    }
    if (head) atomicOr(heads + (f >> 6), 1u << ((f >> 1) & 31));
  }
  bbox_accumulate(lo, hi, bb->fmin, bb->fmax);
}

// Inert filaments filling [from, to) of a chained stream, their records heads.
__global__ void bs_pad_chains(long long from, long long to, float4 *pk, double4 *ra, double4 *rb,
                              unsigned *heads) {
  const long long f = from + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= to) return;
  pack_inert(f, pk, ra, rb);
  atomicOr(heads + (f >> 6), 1u << ((f >> 1) & 31));
}

__global__ void bs_pack_targets(const double *__restrict__ P, long long ns, long long np,
                                long long off, int group, double4 *tp, int *tgroup, BBox *bb) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (t < np) {
    const long long j = t / ns, i = t - j * ns;
    const long long b = i + ns * 3 * j;
    const double x = P[b], y = P[b + ns], z = P[b + 2 * ns];
    tp[off + t] = make_double4(x, y, z, 0.0);
    tgroup[off + t] = group;
    lo[0] = hi[0] = (float)x;
    lo[1] = hi[1] = (float)y;
    lo[2] = hi[2] = (float)z;
  }
  bbox_accumulate(lo, hi, bb->tmin, bb->tmax);
}

// Spreads the low 10 bits of v so that they occupy every third bit.
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
  unsigned long long x = v & 0x3ffu;
  x = (x | (x << 16)) & 0x30000ffull;
  x = (x | (x << 8)) & 0x300f00full;
  x = (x | (x << 4)) & 0x30c30c3ull;
  x = (x | (x << 2)) & 0x9249249ull;
  return x;
}

// Sort key of a target: group id above a 30-bit Morton code of its position
// in the targets' bounding box (bit 31: the target is unused).
__global__ void bs_target_keys(const double4 *__restrict__ tp, const int *__restrict__ tgroup,
                               long long n, const BBox *bb, unsigned long long *keys, int *vals) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const double4 p = tp[t];
  const double q[3] = {p.x, p.y, p.z};
  unsigned long long code = 0;
  for (int c = 0; c < 3; ++c) {
    const double lo = key_float(bb->tmin[c]), hi = key_float(bb->tmax[c]);
    const double w = hi > lo ? hi - lo : 1.0;
    double u = (q[c] - lo) / w * 1023.999;
    if (!(u >= 0.0)) u = 0.0;  // also catches NaN
    if (u > 1023.0) u = 1023.0;
    code |= spread3((unsigned)u) << c;
  }
  // a target marked unused (w != 0: past a growing wake's live columns) sorts
  // after every live target of its group
  if (p.w != 0.0) code |= 1ull << 31;
  keys[t] = ((unsigned long long)(unsigned)tgroup[t] << 32) | code;
  vals[t] = (int)t;
}

__global__ void bs_gather_targets(const double4 *__restrict__ src, const int *__restrict__ perm,
                                  long long n, double4 *dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = src[perm[t]];
}

// Largest possible squared target-endpoint distance from the bounds; the
// reach cut-off can only zero a term when co^2 is below it.
__device__ __forceinline__ bool co_can_trigger(const BBox *bb, double co) {
  double d2 = 0.0;
  for (int c = 0; c < 3; ++c) {
    const double a = (double)key_float(bb->tmax[c]) - (double)key_float(bb->fmin[c]);
    const double b = (double)key_float(bb->fmax[c]) - (double)key_float(bb->tmin[c]);
    const double m = fmax(fabs(a), fabs(b)) * (1.0 + 1e-6) + 1e-3;
    d2 += m * m;
  }
  return co * co < d2;  // false for NaN co: r > NaN is never true
}

// Cuts a work item to the live part of its group (GroupLive): the tile to its
// live targets, the filament range to the live filaments. False when nothing
// of the item is live; its partial sums are then neither written nor read.
__device__ __forceinline__ bool clip_live(const GroupLive *live, Item &it, Tile &tl) {
  const GroupLive gl = live[tl.group];
  const long long tn = gl.t_end - tl.t_begin;
  if (tn <= 0 || it.f_begin >= gl.f_end) return false;
  if (tn < tl.t_count) tl.t_count = (int)tn;
  if (it.f_end > gl.f_end) it.f_end = gl.f_end;
  return true;
}

// ------------------------------------------------------- FP32 direct sum
// Every warp is an independent worker: it takes work items (a tile of 32 x T
// targets against a filament range) from the persistent queue by itself and
// streams the range through its own ring of shared-memory stages, so warps
// never wait for one another (no CTA barrier in the kernel). A CTA holds kWarps
// workers that share nothing but the SM.
constexpr int kWarps = 4;
constexpr int kThreads = 32 * kWarps;
constexpr uint64_t kDefaultWaitNs = 2000000000ull;  // 2 s per tile: far above any real latency

template <int KF>
struct StageSmem {
  static constexpr int kBytes = KF * 64;  // KF/2 pair records of 128 B
  // stages in flight: a warp's tile takes ~10-50 us, a bulk copy ~2 us, so
  // one stage ahead suffices; three for the short 32-filament tiles
  static constexpr int kStages = KF >= 64 ? 2 : 3;
  // tiles per Kahan fold: the FP32 partial sums span 128 filaments
  static constexpr int kFold = KF >= 128 ? 1 : 128 / KF;
};

// Shared memory of one worker: its filament stages, the Kahan state of its
// targets (sum, compensation) x 3 components as floats, the near-singular bit
// words of the current tile (KF/4 words per lane), its full[s] barriers
// (bytes landed) and its target ball (centre, radius, threshold).
template <int T, int KF>
__host__ __device__ constexpr size_t warp_smem_bytes() {
  constexpr int S = StageSmem<KF>::kStages;
  return ((size_t)S * StageSmem<KF>::kBytes + (size_t)6 * 32 * T * sizeof(float) +
          (size_t)(KF / 4) * 32 * sizeof(unsigned) + S * sizeof(uint64_t) + 8 * sizeof(float) +
          127) / 128 * 128;
}

template <int T, int KF>
__host__ __device__ constexpr size_t f32c_smem_bytes_t() {
  return kWarps * warp_smem_bytes<T, KF>();
}

// Kahan step: (sum, comp) += v.
__device__ __forceinline__ void kahan_add(float &sum, float &comp, float v) {
  const float y = __fsub_rn(v, comp);
  const float s = __fadd_rn(sum, y);
  comp = __fsub_rn(__fsub_rn(s, sum), y);
  sum = s;
}

// Hands filaments f0 .. f0+KF to the copy engine into `stage`, completing on `bar`.
template <int KF>
__device__ __forceinline__ void issue_stage(const F32cArgs &a, unsigned char *stage, uint64_t *bar,
                                            int f0) {
  mbar_arrive_expect_tx(bar, StageSmem<KF>::kBytes);
  bulk_g2s(stage, a.pk + (size_t)(f0 / 2) * 8, KF * 64, bar);
}

// Orders this thread's earlier shared-memory accesses (generic proxy) before
// later bulk copies into the same bytes (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ----------------------------------------------------- packed FP32 arithmetic
// The direct sum runs on pairs of filaments: every FP32 operation is a packed
// f32x2 instruction (two independent IEEE operations, round to nearest) on the
// two filaments of a pair record, so one issue slot does two interactions'
// worth of arithmetic; the FMA pipe, not instruction issue, bounds the loop.
__device__ __forceinline__ float2 lo2(const float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4 v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 neg2(const float2 v) { return make_float2(-v.x, -v.y); }
__device__ __forceinline__ float2 rsqrt2(const float2 v) {
  return make_float2(rsqrt_approx(v.x), rsqrt_approx(v.y));
}
__device__ __forceinline__ float2 rcp2(const float2 v) {
  return make_float2(rcp_approx(v.x), rcp_approx(v.y));
}

// One filament pair of a stage, relative to this thread's centre c.
struct Fil2 {
  float2 qx, qy, qz;  // x1 - c (from the hi/lo split)
  float2 Lx, Ly, Lz, L2, D;
  float2 Mx, My, Mz;  // K L, K = gamma/4pi
  float2 Rn2;         // near-singular threshold (careful path)
};

// Pair record r (8 float4, layout in bs_types.h) into registers.
__device__ __forceinline__ void load_pair(const float4 *r, float2 ncx, float2 ncy, float2 ncz,
                                          Fil2 &f) {
  const float4 a0 = r[0], a1 = r[1], b0 = r[2], b1 = r[3];
  const float4 l0 = r[4], l1 = r[5], m0 = r[6], m1 = r[7];
  f.qx = __fadd2_rn(__fadd2_rn(lo2(a0), ncx), lo2(b0));
  f.qy = __fadd2_rn(__fadd2_rn(hi2(a0), ncy), hi2(b0));
  f.qz = __fadd2_rn(__fadd2_rn(lo2(a1), ncz), lo2(b1));
  f.L2 = hi2(a1);
  f.Rn2 = hi2(b1);
  f.Lx = lo2(l0);
  f.Ly = hi2(l0);
  f.Lz = lo2(l1);
  f.D = hi2(l1);
  f.Mx = lo2(m0);
  f.My = hi2(m0);
  f.Mz = lo2(m1);
}

// Internal form code of interact2: the pair term with its core left out,
// (i1 + i2) i1 i2 / e, for pairs where the core changes it by less than
// FP32's unit roundoff 2^-24. Vatistas: the warp screen places the targets
// at least kCoreFreeRatio core radii from the filament's line, where the
// factor 1/sqrt(1 + (rc/h)^4) is within (1/54)^4 / 2 = 5.9e-8 of 1.
// Cut-off: the targets are at least r from the segment with
// r^4 >= 2^24 d |L|^2, so the denominator's d |L|^2 gg^2 <= 2^-24 <= 2^-24 e
// (e >= 1 on the far path, where r1.r2 > 0).
constexpr int kCoreFree = 2;
constexpr float kCoreFreeRatio = 54.f;
constexpr float kCutoffFreeSq = 4096.f;  // r^2 >= 4096 sqrt(d |L|^2) is r^4 >= 2^24 d |L|^2

// One target against one filament pair, accumulated into the packed sums
// (ax, ay, az) (one lane per filament of the pair). (npx, npy, npz) = -(P - c)
// broadcast to both lanes. With NEAR it also tests r1.r2 < Rn^2 per lane: such
// terms are zeroed and recorded in `bits` (bit0 for the pair's first
// filament, bit1 for its second); they are redone in FP64 after the tile.
template <int MODEL, bool CO, bool NEAR>
__device__ __forceinline__ void interact2(float2 npx, float2 npy, float2 npz, const Fil2 &f,
                                          float2 Rn2, float co2, float2 &ax, float2 &ay,
                                          float2 &az, unsigned &bits, unsigned bit0,
                                          unsigned bit1) {
  const float2 nx = __fadd2_rn(f.qx, npx);  // x1 - P = -r1
  const float2 ny = __fadd2_rn(f.qy, npy);
  const float2 nz = __fadd2_rn(f.qz, npz);
  float2 r1s = __fmul2_rn(nx, nx);
  r1s = __ffma2_rn(ny, ny, r1s);
  r1s = __ffma2_rn(nz, nz, r1s);
  float2 ld = __fmul2_rn(f.Lx, nx);  // -L.r1
  ld = __ffma2_rn(f.Ly, ny, ld);
  ld = __ffma2_rn(f.Lz, nz, ld);
  const float2 dot = __fadd2_rn(r1s, ld);                   // r1 . r2
  const float2 r2s = __fadd2_rn(dot, __fadd2_rn(f.L2, ld));  // |r1 - L|^2
  const float2 i1 = rsqrt2(r1s), i2 = rsqrt2(r2s);
  const float2 gg = __fmul2_rn(i1, i2);
  const float2 e = __ffma2_rn(dot, gg, make_float2(1.f, 1.f));  // 1 + cos(theta)
  // K (r1 x r2) = K L x r1 = (x1 - P) x (K L): no cancellation for far or
  // collinear points
  const float2 cx = __ffma2_rn(ny, f.Mz, __fmul2_rn(nz, neg2(f.My)));
  const float2 cy = __ffma2_rn(nz, f.Mx, __fmul2_rn(nx, neg2(f.Mz)));
  const float2 cz = __ffma2_rn(nx, f.My, __fmul2_rn(ny, neg2(f.Mx)));
  float2 ub;
  if (MODEL == kCoreVatistas) {
    // Cnu / (r1 r2 (r1 r2 + r1.r2)) with h^2 = |L x r1|^2/|L|^2 and rc^4 folded:
    // Cnu = |c|^2 / sqrt(|c|^4 + D), c = K L x r1, D = (K^2 rc^2 |L|^2)^2
    float2 c2 = __fmul2_rn(cx, cx);
    c2 = __ffma2_rn(cy, cy, c2);
    c2 = __ffma2_rn(cz, cz, c2);
    const float2 q = __ffma2_rn(c2, c2, f.D);
    const float2 w = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg), c2);
    ub = __fmul2_rn(w, rsqrt2(__fmul2_rn(__fmul2_rn(e, e), q)));
  } else if (MODEL == kCoreFree) {
    // (r1+r2)/(r1r2(r1r2+r1.r2)) = (i1+i2) gg / e
    ub = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg), rcp2(e));
  } else {
    // (r1+r2)/(r1r2(r1r2+r1.r2) + d|L|^2) = (i1+i2) gg / (e + d|L|^2 gg^2)
    ub = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg),
                    rcp2(__ffma2_rn(f.D, __fmul2_rn(gg, gg), e)));
  }
  if (NEAR) {
    if (dot.x < Rn2.x) {
      bits |= bit0;
      ub.x = 0.f;
    }
    if (dot.y < Rn2.y) {
      bits |= bit1;
      ub.y = 0.f;
    }
  }
  if (CO) {
    if (fminf(r1s.x, r2s.x) > co2) ub.x = 0.f;
    if (fminf(r1s.y, r2s.y) > co2) ub.y = 0.f;
  }
  ax = __ffma2_rn(ub, cx, ax);
  ay = __ffma2_rn(ub, cy, ay);
  az = __ffma2_rn(ub, cz, az);
}

// interact2 on chained pair records. In a chained stream the second endpoint
// of each filament (per lane of the record) is the first endpoint of the same
// lane's filament in the previous record -- the wake's filaments meet at its
// nodes -- so 1/|x2 - P| is the previous record's 1/|x1 - P|, carried in `ti`:
// a chained record needs neither |r2|^2 nor its rsqrt (two FP32 operations and
// one MUFU result fewer per interaction). A record that starts a chain (HEAD)
// forms them from L as interact2 does. Either way 1/|x1 - P| is left in `ti`
// for the next record.
template <int MODEL, bool CO, bool NEAR, bool HEAD>
__device__ __forceinline__ void interact_chain(float2 npx, float2 npy, float2 npz, const Fil2 &f,
                                               float2 Rn2, float co2, float2 &ax, float2 &ay,
                                               float2 &az, unsigned &bits, unsigned bit0,
                                               unsigned bit1, float2 &ti) {
  const float2 nx = __fadd2_rn(f.qx, npx);  // x1 - P = -r1
  const float2 ny = __fadd2_rn(f.qy, npy);
  const float2 nz = __fadd2_rn(f.qz, npz);
  float2 r1s = __fmul2_rn(nx, nx);
  r1s = __ffma2_rn(ny, ny, r1s);
  r1s = __ffma2_rn(nz, nz, r1s);
  float2 ld = __fmul2_rn(f.Lx, nx);  // -L.r1
  ld = __ffma2_rn(f.Ly, ny, ld);
  ld = __ffma2_rn(f.Lz, nz, ld);
  const float2 dot = __fadd2_rn(r1s, ld);  // r1 . r2
  float2 r2s, i2;
  if (HEAD || CO) r2s = __fadd2_rn(dot, __fadd2_rn(f.L2, ld));  // |r1 - L|^2
  if (HEAD)
    i2 = rsqrt2(r2s);
  else
    i2 = ti;
  const float2 i1 = rsqrt2(r1s);
  const float2 gg = __fmul2_rn(i1, i2);
  const float2 e = __ffma2_rn(dot, gg, make_float2(1.f, 1.f));  // 1 + cos(theta)
  const float2 cx = __ffma2_rn(ny, f.Mz, __fmul2_rn(nz, neg2(f.My)));
  const float2 cy = __ffma2_rn(nz, f.Mx, __fmul2_rn(nx, neg2(f.Mz)));
  const float2 cz = __ffma2_rn(nx, f.My, __fmul2_rn(ny, neg2(f.Mx)));
  float2 ub;
  if (MODEL == kCoreVatistas) {
    float2 c2 = __fmul2_rn(cx, cx);
    c2 = __ffma2_rn(cy, cy, c2);
    c2 = __ffma2_rn(cz, cz, c2);
    const float2 q = __ffma2_rn(c2, c2, f.D);
    const float2 w = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg), c2);
    ub = __fmul2_rn(w, rsqrt2(__fmul2_rn(__fmul2_rn(e, e), q)));
  } else if (MODEL == kCoreFree) {
    ub = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg), rcp2(e));
  } else {
    ub = __fmul2_rn(__fmul2_rn(__fadd2_rn(i1, i2), gg),
                    rcp2(__ffma2_rn(f.D, __fmul2_rn(gg, gg), e)));
  }
  if (NEAR) {
    if (dot.x < Rn2.x) {
      bits |= bit0;
      ub.x = 0.f;
    }
    if (dot.y < Rn2.y) {
      bits |= bit1;
      ub.y = 0.f;
    }
  }
  if (CO) {
    if (fminf(r1s.x, r2s.x) > co2) ub.x = 0.f;
    if (fminf(r1s.y, r2s.y) > co2) ub.y = 0.f;
  }
  ax = __ffma2_rn(ub, cx, ax);
  ay = __ffma2_rn(ub, cy, ay);
  az = __ffma2_rn(ub, cz, az);
  ti = i1;
}

// One chained pair record against the lane's T targets, in form FORM
// (kCoreFree, or the kernel's model), the record starting a chain or not.
template <int T, int FORM, bool CO, bool NEAR>
__device__ __forceinline__ void chain_record(const float4 *rec, bool head, float2 ncx, float2 ncy,
                                             float2 ncz, const float2 (&npx)[T],
                                             const float2 (&npy)[T], const float2 (&npz)[T],
                                             float S2, float co2, float2 (&ax)[T],
                                             float2 (&ay)[T], float2 (&az)[T], float2 (&ti)[T],
                                             unsigned &nbits, int j) {
  Fil2 f;
  load_pair(rec, ncx, ncy, ncz, f);
  // near-singular threshold, raised for threads whose targets spread far
  // from their centre (as in the unchained careful path)
  const float2 Rn2 = NEAR ? make_float2(fmaxf(f.Rn2.x, S2), fmaxf(f.Rn2.y, S2)) : f.Rn2;
  if (head) {
#pragma unroll
    for (int t = 0; t < T; ++t)
      interact_chain<FORM, CO, NEAR, true>(npx[t], npy[t], npz[t], f, Rn2, co2, ax[t], ay[t],
                                           az[t], nbits, 1u << (8 * (2 * j) + t),
                                           1u << (8 * (2 * j + 1) + t), ti[t]);
  } else {
#pragma unroll
    for (int t = 0; t < T; ++t)
      interact_chain<FORM, CO, NEAR, false>(npx[t], npy[t], npz[t], f, Rn2, co2, ax[t], ay[t],
                                            az[t], nbits, 1u << (8 * (2 * j) + t),
                                            1u << (8 * (2 * j + 1) + t), ti[t]);
  }
}

// A near-singular pair of a tile, listed in the tile's consumed stage: the
// FP64 reference term `u` of filament `fidx` at the owner's target `slot`.
struct NearEntry {
  double u[3];
  int fidx, slot;
};

// One item: the lane's T targets against filaments [it.f_begin, it.f_end),
// streamed through the warp's S stages (tile g of the warp in stage g % S).
// Returns false, for the whole warp, when a bounded wait ran out (the item is
// abandoned after the copies in flight have landed).
template <int T, int KF, int MODEL, bool CO, bool CHAIN>
__device__ __forceinline__ bool f32c_item(const F32cArgs &a, const Item &it, unsigned char *stages,
                                          uint64_t *full, float *s_k, unsigned *s_nb,
                                          unsigned &gt, float2 (&npx)[T], float2 (&npy)[T],
                                          float2 (&npz)[T], float2 ncx, float2 ncy, float2 ncz,
                                          float S2, const float *ws, unsigned &near_cnt,
                                          unsigned long long &free_cnt,
                                          const Tile &tl) {
  constexpr int S = StageSmem<KF>::kStages;
  constexpr int kB = StageSmem<KF>::kBytes;
  const int lane = threadIdx.x & 31;
  const int ntiles = (it.f_end - it.f_begin) / KF;
  const float co2 = (float)(a.co * a.co);
  const int nslots = tl.t_count - lane * T;  // this lane's targets in the tile
  const unsigned live_slots = (unsigned)(nslots < 0 ? 0 : (nslots > T ? T : nslots));
  RefParams rp;
  rp.model = a.model;
  rp.d = a.d;
  rp.n = a.n;
  rp.co = a.co;
  // Between items every stage of the warp is free: each copy issued was
  // waited for and read before the previous item ended.
  int issued = ntiles < S ? ntiles : S;
  if (lane == 0)
    for (int j = 0; j < issued; ++j)
      issue_stage<KF>(a, stages + ((gt + j) % S) * kB, &full[(gt + j) % S], it.f_begin + j * KF);
  float2 ax[T], ay[T], az[T];
#pragma unroll
  for (int t = 0; t < T; ++t) ax[t] = ay[t] = az[t] = make_float2(0.f, 0.f);

  int i = 0;
  for (; i < ntiles; ++i) {
    const unsigned g = gt + i;
    const int st = g % S;
    const bool landed = mbar_wait_bounded(&full[st], (g / S) & 1u, a.err, a.wait_limit_ns);
    if (!__all_sync(0xffffffffu, landed)) break;
    const unsigned char *stage = stages + st * kB;
    const float4 *sP = reinterpret_cast<const float4 *>(stage);  // KF/2 pair records
    const float *sF = reinterpret_cast<const float *>(stage);
    // Hot loop: filaments in groups of 4 (two pair records). A warp-level
    // screen (one filament per lane, every 32 filaments) sends groups that are
    // far from all of the warp's targets down the plain path; the others test
    // every pair and put their near-singular bits (bit 8*j + t: filament
    // 4*kk+j, target t) in shared memory as one word. `careful` has bit g for
    // every such group g. A far group whose four filaments all leave every
    // target of the warp outside their core's reach (Vatistas: lines at least
    // kCoreFreeRatio core radii away; cut-off: segments far enough that the
    // d |L|^2 term is below FP32 resolution) takes the core-free form (`mf`
    // has a bit per such filament).
    unsigned careful = 0u;
#pragma unroll 1
    for (int w = 0; w < KF / 32; ++w) {
      unsigned m, mf = 0u;
      if (CO) {
        m = 0xffffffffu;
      } else {
        const int k = 32 * w + lane;
        const float *f = sF + (k >> 1) * 32 + (k & 1);  // field j of filament k at f[2 j]
        // the warp's target ball (centre, radius, largest S2), kept in shared
        // memory so it holds no registers across the hot loop
        const float wcx = ws[0], wcy = ws[1], wcz = ws[2], wr = ws[3], rn_floor = ws[4];
        const float big = fabsf(wcx) + fabsf(wcy) + fabsf(wcz);
        const float Ax = f[0], Ay = f[2], Az = f[4], L2 = f[6];
        const float mx = (Ax - wcx) + fmaf(0.5f, f[16], f[8]);
        const float my = (Ay - wcy) + fmaf(0.5f, f[18], f[10]);
        const float mz = (Az - wcz) + fmaf(0.5f, f[20], f[12]);
        const float d2 = mx * mx + my * my + mz * mz;
        const float reach = sqrtf(fmaf(0.25f, L2, fmaxf(f[14], rn_floor)));
        const float slack =
            1e-5f * (big + fabsf(Ax) + fabsf(Ay) + fabsf(Az)) + 1e-3f * (reach + wr);
        const float lim = wr + reach + slack;
        m = __ballot_sync(0xffffffffu, !(d2 > lim * lim));
        if (MODEL == kCoreVatistas) {
          // distance of the ball centre from the filament's line: |L x (x1 - c)| / |L|;
          // every target of the warp is at least that less wr from it
          const float Lx = f[16], Ly = f[18], Lz = f[20], rc = f[30];
          const float dx = Ax - wcx, dy = Ay - wcy, dz = Az - wcz;
          const float cx = Ly * dz - Lz * dy, cy = Lz * dx - Lx * dz, cz = Lx * dy - Ly * dx;
          const float R = fmaf(kCoreFreeRatio, rc, wr + slack);
          // zero length: the pair term is zero on either form; rc = 0 (no core,
          // or K = 0 and a zero term): the factor is 1
          const bool free_ =
              !(L2 > 0.f) || rc == 0.f || cx * cx + cy * cy + cz * cz >= R * R * L2;
          mf = __ballot_sync(0xffffffffu, free_);
        } else {
          // nearest approach of a warp target to the segment: its midpoint
          // distance less wr and |L|/2; D = d |L|^2 (record field 11)
          const float rmin = sqrtf(d2) - wr - 0.5f * sqrtf(L2) - slack;
          const bool free_ = rmin > 0.f && rmin * rmin >= kCutoffFreeSq * sqrtf(f[22]);
          mf = __ballot_sync(0xffffffffu, free_);
        }
      }
      if constexpr (CHAIN) {
        // Chained records: bit j of hm is set when record j of the word starts
        // a chain (the word's first record always does: no carry crosses a
        // word). The carry holds the previous record's x1 - P and 1/|x1 - P|.
        const unsigned r0 = (unsigned)((it.f_begin + i * KF + 32 * w) >> 1);
        const unsigned hm = ((__ldg(a.heads + (r0 >> 5)) >> (r0 & 31u)) & 0xffffu) | 1u;
        float2 ti[T];
        unsigned unused = 0;
        if (m == 0u && mf == 0xffffffffu) {
          free_cnt += 32u * live_slots;
#pragma unroll 2
          for (int j = 0; j < 16; ++j)
            chain_record<T, kCoreFree, false, false>(sP + (16 * w + j) * 8, (hm >> j) & 1u, ncx,
                                                     ncy, ncz, npx, npy, npz, S2, co2, ax, ay, az,
                                                     ti, unused, 0);
          continue;
        }
#pragma unroll 1
        for (int g = 0; g < 8; ++g) {
          const int kk = 32 * w + 4 * g;
          const unsigned hg = hm >> (2 * g);
          if (((m >> (4 * g)) & 0xfu) == 0u && ((mf >> (4 * g)) & 0xfu) == 0xfu) {
            free_cnt += 4u * live_slots;
#pragma unroll
            for (int j = 0; j < 2; ++j)
              chain_record<T, kCoreFree, false, false>(sP + (kk / 2 + j) * 8, (hg >> j) & 1u, ncx,
                                                       ncy, ncz, npx, npy, npz, S2, co2, ax, ay,
                                                       az, ti, unused, j);
          } else if (((m >> (4 * g)) & 0xfu) == 0u) {
#pragma unroll
            for (int j = 0; j < 2; ++j)
              chain_record<T, MODEL, false, false>(sP + (kk / 2 + j) * 8, (hg >> j) & 1u, ncx,
                                                   ncy, ncz, npx, npy, npz, S2, co2, ax, ay, az,
                                                   ti, unused, j);
          } else {
            careful |= 1u << (8 * w + g);
            unsigned nbits = 0;
#pragma unroll
            for (int j = 0; j < 2; ++j)
              chain_record<T, MODEL, CO, true>(sP + (kk / 2 + j) * 8, (hg >> j) & 1u, ncx, ncy,
                                               ncz, npx, npy, npz, S2, co2, ax, ay, az, ti,
                                               nbits, j);
            s_nb[(kk / 4) * 32 + lane] = nbits;
          }
        }
        continue;
      }
      if (m == 0u && mf == 0xffffffffu) {
        // the whole word far and core-free: one loop over its 16 pairs
        free_cnt += 32u * live_slots;
#pragma unroll 2
        for (int j = 0; j < 16; ++j) {
          Fil2 f;
          load_pair(sP + (16 * w + j) * 8, ncx, ncy, ncz, f);
          unsigned unused = 0;
#pragma unroll
          for (int t = 0; t < T; ++t)
            interact2<kCoreFree, false, false>(npx[t], npy[t], npz[t], f, f.Rn2, co2, ax[t],
                                               ay[t], az[t], unused, 0u, 0u);
        }
        continue;
      }
#pragma unroll 1
      for (int g = 0; g < 8; ++g) {
        const int kk = 32 * w + 4 * g;
        if (((m >> (4 * g)) & 0xfu) == 0u && ((mf >> (4 * g)) & 0xfu) == 0xfu) {
          free_cnt += 4u * live_slots;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            Fil2 f;
            load_pair(sP + (kk / 2 + j) * 8, ncx, ncy, ncz, f);
            unsigned unused = 0;
#pragma unroll
            for (int t = 0; t < T; ++t)
              interact2<kCoreFree, false, false>(npx[t], npy[t], npz[t], f, f.Rn2, co2, ax[t],
                                                 ay[t], az[t], unused, 0u, 0u);
          }
        } else if (((m >> (4 * g)) & 0xfu) == 0u) {
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            Fil2 f;
            load_pair(sP + (kk / 2 + j) * 8, ncx, ncy, ncz, f);
            unsigned unused = 0;
#pragma unroll
            for (int t = 0; t < T; ++t)
              interact2<MODEL, false, false>(npx[t], npy[t], npz[t], f, f.Rn2, co2, ax[t], ay[t],
                                             az[t], unused, 0u, 0u);
          }
        } else {
          careful |= 1u << (8 * w + g);
          unsigned nbits = 0;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            Fil2 f;
            load_pair(sP + (kk / 2 + j) * 8, ncx, ncy, ncz, f);
            // near-singular threshold, raised for threads whose targets spread
            // far from their centre (the FP32 differences lose ~eps * spread / |r1|)
            const float2 Rn2 = make_float2(fmaxf(f.Rn2.x, S2), fmaxf(f.Rn2.y, S2));
#pragma unroll
            for (int t = 0; t < T; ++t)
              interact2<MODEL, CO, true>(npx[t], npy[t], npz[t], f, Rn2, co2, ax[t], ay[t],
                                         az[t], nbits, 1u << (8 * (2 * j) + t),
                                         1u << (8 * (2 * j + 1) + t));
          }
          s_nb[(kk / 4) * 32 + lane] = nbits;
        }
      }
    }
    __syncwarp();
    // Kahan-fold the partial sums into the per-target totals every 128 filaments.
    if ((i + 1) % StageSmem<KF>::kFold == 0 || i + 1 == ntiles) {
#pragma unroll
      for (int t = 0; t < T; ++t) {
        const int sl = lane * T + t;
        kahan_add(s_k[0 * 32 * T + sl], s_k[1 * 32 * T + sl], ax[t].x + ax[t].y);
        kahan_add(s_k[2 * 32 * T + sl], s_k[3 * 32 * T + sl], ay[t].x + ay[t].y);
        kahan_add(s_k[4 * 32 * T + sl], s_k[5 * 32 * T + sl], az[t].x + az[t].y);
        ax[t] = ay[t] = az[t] = make_float2(0.f, 0.f);
      }
    }
    // Near-singular pairs of this tile: the reference formula in FP64, added to
    // the owner's Kahan state as an exact hi + lo pair. The pairs are listed in
    // the consumed stage (lane-major, in each lane's bit order), computed by all
    // lanes together, then added by their owners in list order, so every target
    // receives its terms in the same order as a lane-by-lane pass would.
    if (careful) {  // warp-uniform
      constexpr int kCap = kB / (int)sizeof(NearEntry);
      NearEntry *ne = reinterpret_cast<NearEntry *>(stages + st * kB);
      int cnt = 0;
      for (unsigned cg = careful; cg; cg &= cg - 1u) cnt += __popc(s_nb[(__ffs(cg) - 1) * 32 + lane]);
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int first = incl - cnt;
#pragma unroll 1
      for (int base = 0; base < total; base += kCap) {
        const int end = total < base + kCap ? total : base + kCap;
        if (first < end && first + cnt > base) {
          int k = first;
          for (unsigned cg = careful; cg && k < end; cg &= cg - 1u) {
            const int w = __ffs(cg) - 1;
            for (unsigned bits = s_nb[w * 32 + lane]; bits && k < end; bits &= bits - 1u, ++k) {
              if (k < base) continue;
              const int b = __ffs(bits) - 1;
              ne[k - base].fidx = it.f_begin + i * KF + 4 * w + (b >> 3);
              ne[k - base].slot = lane * T + (b & 7);
            }
          }
        }
        __syncwarp();
        for (int k = base + lane; k < end; k += 32) {
          NearEntry &e = ne[k - base];
          int local = e.slot;
          if (local >= tl.t_count) local = tl.t_count - 1;
          const double4 p = a.tp[tl.t_begin + local];
          double u0 = 0.0, u1 = 0.0, u2 = 0.0;
          ref_pair<false>(a.ra[e.fidx], a.rb[e.fidx], p.x, p.y, p.z, rp, u0, u1, u2);
          e.u[0] = u0;
          e.u[1] = u1;
          e.u[2] = u2;
        }
        __syncwarp();
        const int k0 = first > base ? first : base;
        const int k1 = first + cnt < end ? first + cnt : end;
        for (int k = k0; k < k1; ++k) {
          const NearEntry &e = ne[k - base];
          const int sl = e.slot;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float hi = (float)e.u[c];
            const float lo = (float)(e.u[c] - (double)hi);
            kahan_add(s_k[(2 * c) * 32 * T + sl], s_k[(2 * c + 1) * 32 * T + sl], hi);
            kahan_add(s_k[(2 * c) * 32 * T + sl], s_k[(2 * c + 1) * 32 * T + sl], lo);
          }
          ++near_cnt;
        }
        __syncwarp();
      }
    }
    // Every lane is done with the stage (tile and near list): refill it with
    // tile i + S.
    if (lane == 0 && issued < ntiles) {
      fence_proxy_async_smem();
      issue_stage<KF>(a, stages + st * kB, &full[st], it.f_begin + issued * KF);
      ++issued;
    }
    __syncwarp();
  }
  if (i < ntiles) {
    // A bounded wait ran out: let the copies already issued land (bounded)
    // before the warp leaves, so no bulk copy targets the shared memory of a
    // finished CTA.
    if (lane == 0)
      for (int j = i; j < issued; ++j) {
        const unsigned g = gt + j;
        mbar_wait_bounded(&full[g % S], (g / S) & 1u, a.err, a.wait_limit_ns);
      }
    __syncwarp();
    return false;
  }
  gt += ntiles;
  return true;
}

// Resident CTAs per SM the register allocation is capped for: 6 for T = 2
// (80 registers), 5 for T = 3 (96), 4 for T = 4 (128), 2 for T = 8 (255). The
// packed loop keeps each target as broadcast pairs and its sums as pairs (12
// registers a target). The chained kernel carries one more pair a target: 5
// for T = 2 (96), 4 for T = 3 and T = 4 (128; T = 4 then spills ~100 bytes,
// and measured faster so than at 3 CTAs with 168 registers on the cut-off
// core, slower on the Vatistas core, where T = 3 wins).
template <int T, bool CHAIN>
struct MinBlocks {
  static constexpr int value = CHAIN ? (T <= 2 ? 5 : (T <= 4 ? 4 : 2))
                                     : (T <= 2 ? 6 : (T == 3 ? 5 : (T <= 4 ? 4 : 2)));
};

template <int T, int KF, int MODEL, bool CHAIN>
__global__ void __launch_bounds__(kThreads, MinBlocks<T, CHAIN>::value) bs_f32c(const F32cArgs a) {
  static_assert(KF % 32 == 0 && KF / 4 <= 32, "one screen word per 32 filaments, one bit per group");
  constexpr int S = StageSmem<KF>::kStages;
  extern __shared__ __align__(128) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  unsigned char *stages = smem + (threadIdx.x >> 5) * warp_smem_bytes<T, KF>();
  float *s_k = reinterpret_cast<float *>(stages + S * StageSmem<KF>::kBytes);
  unsigned *s_nb = reinterpret_cast<unsigned *>(s_k + 6 * 32 * T);
  uint64_t *full = reinterpret_cast<uint64_t *>(s_nb + (KF / 4) * 32);
  float *ws = reinterpret_cast<float *>(full + S);
  if (lane == 0) {
    for (int st = 0; st < S; ++st) mbar_init(&full[st], 1);
    fence_mbar_init();
  }
  __syncwarp();
  const bool co_on = co_can_trigger(a.bbox, a.co);
  unsigned gt = 0;
  unsigned near_cnt = 0;
  unsigned long long free_cnt = 0;  // pairs of this lane that took the core-free form
  while (true) {
    int q = 0;
    if (lane == 0) q = (int)atomicAdd(a.work_ctr, 1u);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q >= a.n_items) break;
    const int item_id = a.order ? a.order[q] : q;
    Item it = a.items[item_id];
    Tile tl = a.tiles[it.tile];
    if (a.live && !clip_live(a.live, it, tl)) continue;
    if (tl.t_count <= 0 || ((it.f_end - it.f_begin) % KF) != 0) {
      if (lane == 0) atomicOr(a.err, kErrBadItem);
      continue;
    }
    // This lane's T consecutive targets, relative to the FP32 image of the first.
    float px[T], py[T], pz[T];
    float spread2 = 0.f;
    int l0 = lane * T;
    if (l0 >= tl.t_count) l0 = tl.t_count - 1;
    const double4 p0 = a.tp[tl.t_begin + l0];
    const float cx = (float)p0.x, cy = (float)p0.y, cz = (float)p0.z;
#pragma unroll
    for (int t = 0; t < T; ++t) {
      int l = lane * T + t;
      if (l >= tl.t_count) l = tl.t_count - 1;
      const double4 p = a.tp[tl.t_begin + l];
      px[t] = (float)(p.x - (double)cx);
      py[t] = (float)(p.y - (double)cy);
      pz[t] = (float)(p.z - (double)cz);
      spread2 = fmaxf(spread2, px[t] * px[t] + py[t] * py[t] + pz[t] * pz[t]);
#pragma unroll
      for (int c = 0; c < 6; ++c) s_k[c * 32 * T + lane * T + t] = 0.f;
    }
    const float S2 = 0.09f * spread2;  // pairs closer than 0.3 x spread go to FP64
    // -(P - c) in both lanes of a packed register, and -c likewise
    float2 npx[T], npy[T], npz[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
      npx[t] = make_float2(-px[t], -px[t]);
      npy[t] = make_float2(-py[t], -py[t]);
      npz[t] = make_float2(-pz[t], -pz[t]);
    }
    const float2 ncx = make_float2(-cx, -cx), ncy = make_float2(-cy, -cy),
                 ncz = make_float2(-cz, -cz);
    // The warp's targets lie in the ball (wc, wr) around the centre of their
    // bounding box. As r1.r2 = |P - m|^2 - |L|^2/4 (m the filament midpoint),
    // a filament whose midpoint is farther than wr + sqrt(|L|^2/4 + Rn^2)
    // from wc has r1.r2 >= Rn^2 for every target of the warp; rn_floor is
    // the warp's largest per-thread threshold S2.
    float blo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const float q[3] = {cx + px[t], cy + py[t], cz + pz[t]};
#pragma unroll
      for (int c = 0; c < 3; ++c) blo[c] = fminf(blo[c], q[c]), bhi[c] = fmaxf(bhi[c], q[c]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        blo[c] = fminf(blo[c], __shfl_xor_sync(0xffffffffu, blo[c], o));
        bhi[c] = fmaxf(bhi[c], __shfl_xor_sync(0xffffffffu, bhi[c], o));
      }
    const float wcx = 0.5f * (blo[0] + bhi[0]);
    const float wcy = 0.5f * (blo[1] + bhi[1]);
    const float wcz = 0.5f * (blo[2] + bhi[2]);
    float wr2 = 0.f;
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const float dx = (cx - wcx) + px[t], dy = (cy - wcy) + py[t], dz = (cz - wcz) + pz[t];
      wr2 = fmaxf(wr2, dx * dx + dy * dy + dz * dz);
    }
    float rn_floor = S2;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      wr2 = fmaxf(wr2, __shfl_xor_sync(0xffffffffu, wr2, o));
      rn_floor = fmaxf(rn_floor, __shfl_xor_sync(0xffffffffu, rn_floor, o));
    }
    if (lane == 0) {
      ws[0] = wcx;
      ws[1] = wcy;
      ws[2] = wcz;
      ws[3] = sqrtf(wr2);
      ws[4] = rn_floor;
    }
    __syncwarp();
    bool ok;
    if (co_on)
      ok = f32c_item<T, KF, MODEL, true, CHAIN>(a, it, stages, full, s_k, s_nb, gt, npx, npy, npz,
                                                ncx, ncy, ncz, S2, ws, near_cnt, free_cnt, tl);
    else
      ok = f32c_item<T, KF, MODEL, false, CHAIN>(a, it, stages, full, s_k, s_nb, gt, npx, npy,
                                                 npz, ncx, ncy, ncz, S2, ws, near_cnt, free_cnt,
                                                 tl);
    if (!ok) break;
    double *part = a.part + (size_t)item_id * 3 * a.tile_cap;
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const int l = lane * T + t;
      if (l < tl.t_count) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
          part[c * a.tile_cap + l] = (double)s_k[(2 * c) * 32 * T + l] -
                                     (double)s_k[(2 * c + 1) * 32 * T + l];
      }
    }
    __syncwarp();
  }
  if (a.near_ctr && near_cnt) atomicAdd(a.near_ctr, (unsigned long long)near_cnt);
  if (a.near_ctr && free_cnt) atomicAdd(a.near_ctr + 1, free_cnt);
}

// ------------------------------------------------------- FP64 direct sum
constexpr int kF64Threads = 128;
constexpr int kF64Tile = 128;  // filaments per shared-memory stage

__global__ void __launch_bounds__(kF64Threads) bs_f64(const F32cArgs a) {
  __shared__ double4 sA[2][kF64Tile], sB[2][kF64Tile];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  RefParams rp;
  rp.model = a.model;
  rp.d = a.d;
  rp.n = a.n;
  rp.co = a.co;
  while (true) {
    if (tid == 0) s_item = (int)atomicAdd(a.work_ctr, 1u);
    __syncthreads();
    const int q = s_item;
    __syncthreads();
    if (q >= a.n_items) break;
    const int item_id = a.order ? a.order[q] : q;
    Item it = a.items[item_id];
    Tile tl = a.tiles[it.tile];
    if (a.live && !clip_live(a.live, it, tl)) continue;  // uniform over the block
    int l = tid < tl.t_count ? tid : tl.t_count - 1;
    const double4 p = a.tp[tl.t_begin + l];
    double ux = 0.0, uy = 0.0, uz = 0.0;
    const int ntiles = (it.f_end - it.f_begin) / kF64Tile;
    // stage 0
    sA[0][tid] = a.ra[it.f_begin + tid];
    sB[0][tid] = a.rb[it.f_begin + tid];
    __syncthreads();
    for (int i = 0; i < ntiles; ++i) {
      const int b = i & 1;
      double4 nA, nB;
      const bool more = i + 1 < ntiles;
      if (more) {
        nA = a.ra[it.f_begin + (i + 1) * kF64Tile + tid];
        nB = a.rb[it.f_begin + (i + 1) * kF64Tile + tid];
      }
      for (int k = 0; k < kF64Tile; ++k) ref_pair(sA[b][k], sB[b][k], p.x, p.y, p.z, rp, ux, uy, uz);
      if (more) {
        sA[b ^ 1][tid] = nA;
        sB[b ^ 1][tid] = nB;
      }
      __syncthreads();
    }
    if (tid < tl.t_count) {
      double *part = a.part + (size_t)item_id * 3 * a.tile_cap;
      part[tid] = ux;
      part[a.tile_cap + tid] = uy;
      part[2 * a.tile_cap + tid] = uz;
    }
  }
}

// --------------------------------------------------------------- reduce
// With a live table, only the live targets of a tile are written, from the
// items before the group's live filament end (a tile's items cover increasing
// filament ranges, so those come first).
__global__ void bs_reduce(const Tile *__restrict__ tiles, const Group *__restrict__ groups,
                          const double *__restrict__ part, const int *__restrict__ perm,
                          int tile_cap, const Item *__restrict__ items,
                          const GroupLive *__restrict__ live) {
  Tile tl = tiles[blockIdx.x];
  const Group g = groups[tl.group];
  if (live) {
    const GroupLive gl = live[tl.group];
    const long long tn = gl.t_end - tl.t_begin;
    if (tn <= 0) return;
    if (tn < tl.t_count) tl.t_count = (int)tn;
    int k = 0;
    while (k < tl.n_items && items[tl.first_item + k].f_begin < gl.f_end) ++k;
    tl.n_items = k;
  }
  for (int l = threadIdx.x; l < tl.t_count; l += blockDim.x) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll 4
    for (int k = 0; k < tl.n_items; ++k) {
      const double *p = part + (size_t)(tl.first_item + k) * 3 * tile_cap;
      s0 += p[l];
      s1 += p[tile_cap + l];
      s2 += p[2 * tile_cap + l];
    }
    const long long local = (long long)perm[tl.t_begin + l] - g.t_begin;
    const long long j = local / g.ns_p, i = local - j * g.ns_p;
    double *o = g.out + i + 3 * g.ns_p * j;
    if (g.accumulate) {
      o[0] += s0;
      o[g.ns_p] += s1;
      o[2 * g.ns_p] += s2;
    } else {
      o[0] = s0;
      o[g.ns_p] = s1;
      o[2 * g.ns_p] = s2;
    }
  }
}

// --------------------------------------------------------------- lengths
__global__ void bs_length(const double *__restrict__ F1, const double *__restrict__ F2,
                          long long d0, long long nf, double *L) {
  const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const long long j = f / d0, i = f - j * d0;
  const long long b = i + d0 * 3 * j;
  const double dx = F2[b] - F1[b], dy = F2[b + d0] - F1[b + d0], dz = F2[b + 2 * d0] - F1[b + 2 * d0];
  L[f] = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
}

// ------------------------------------------------------- FP32 FMA peak probe
// Each thread runs 8 independent FMA chains; nothing but FFMA issues in the
// loop body, so the rate is the FP32 pipe's (the direct sum's roofline).
__global__ void __launch_bounds__(256) bs_ffma_peak(float *out, int iters, float a, float b) {
  float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-3f, x2 = x0 + 2e-3f, x3 = x0 + 3e-3f;
  float x4 = x0 + 4e-3f, x5 = x0 + 5e-3f, x6 = x0 + 6e-3f, x7 = x0 + 7e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fmaf(x0, a, b);
      x1 = fmaf(x1, a, b);
      x2 = fmaf(x2, a, b);
      x3 = fmaf(x3, a, b);
      x4 = fmaf(x4, a, b);
      x5 = fmaf(x5, a, b);
      x6 = fmaf(x6, a, b);
      x7 = fmaf(x7, a, b);
    }
  }
  const float r = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
  if (r == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = r;  // keeps the chains live
}

// ------------------------------------------------------- bounded-wait self-test
// Waits on an mbarrier that nothing arrives on, with the given limit; the
// bounded wait must give up, set the error word and let the kernel return.
__global__ void bs_wait_selftest(unsigned *err, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0u, err, limit_ns);
  __syncthreads();
}

// ============================================================ host launchers
namespace {
template <int T, int KF, int MODEL, bool CH>
cudaError_t launch_f32c_t(const F32cArgs &a, int grid, cudaStream_t s) {
  const size_t smem = f32c_smem_bytes_t<T, KF>();
  static unsigned attr_set = 0;  // one bit per device: the attribute is per context
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 32 || !(attr_set & (1u << dev))) {
    cudaError_t e = cudaFuncSetAttribute(bs_f32c<T, KF, MODEL, CH>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(bs_f32c<T, KF, MODEL, CH>,
                             cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    if (dev < 32) attr_set |= (1u << dev);
  }
  // `grid` counts workers (warps); kWarps of them per CTA
  bs_f32c<T, KF, MODEL, CH><<<(grid + kWarps - 1) / kWarps, kThreads, smem, s>>>(a);
  return cudaGetLastError();
}

template <int T, int KF, int MODEL, bool CH>
int occupancy_t() {
  const size_t smem = f32c_smem_bytes_t<T, KF>();
  cudaFuncSetAttribute(bs_f32c<T, KF, MODEL, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smem);
  cudaFuncSetAttribute(bs_f32c<T, KF, MODEL, CH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bs_f32c<T, KF, MODEL, CH>, kThreads, smem) !=
      cudaSuccess)
    return kWarps;
  return (n > 0 ? n : 1) * kWarps;  // resident workers per SM
}

#define WINDS_F32C_CASE(FN, M, TT, KK, ...) \
  case M * 1000 + TT * 100 + KK / 32: return FN<TT, KK, M, CH>(__VA_ARGS__);
#define WINDS_F32C_DISPATCH(FN, ...)                                                    \
  switch (model * 1000 + T * 100 + KF / 32) {                                          \
    WINDS_F32C_CASE(FN, 0, 2, 32, __VA_ARGS__) WINDS_F32C_CASE(FN, 0, 2, 64, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 2, 128, __VA_ARGS__) WINDS_F32C_CASE(FN, 0, 3, 32, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 3, 64, __VA_ARGS__) WINDS_F32C_CASE(FN, 0, 3, 128, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 4, 32, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 4, 64, __VA_ARGS__) WINDS_F32C_CASE(FN, 0, 4, 128, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 8, 32, __VA_ARGS__) WINDS_F32C_CASE(FN, 0, 8, 64, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 0, 8, 128, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 2, 32, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 2, 64, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 2, 128, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 3, 32, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 3, 64, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 3, 128, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 4, 32, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 4, 64, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 4, 128, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 8, 32, __VA_ARGS__) \
    WINDS_F32C_CASE(FN, 1, 8, 64, __VA_ARGS__) WINDS_F32C_CASE(FN, 1, 8, 128, __VA_ARGS__) \
    default: break;                                                                     \
  }
}  // namespace

bool f32c_config_supported(int T, int KF) {
  return (T == 2 || T == 3 || T == 4 || T == 8) && (KF == 32 || KF == 64 || KF == 128);
}

int f32c_threads() { return 32; }  // lanes of one worker: a tile holds 32 x T targets
int f64_threads() { return kF64Threads; }
int f64_tile() { return kF64Tile; }

namespace {
template <bool CH>
cudaError_t launch_f32c_ch(const F32cArgs &a, int model, int T, int KF, int grid, cudaStream_t s) {
  WINDS_F32C_DISPATCH(launch_f32c_t, a, grid, s)
  return cudaErrorInvalidValue;
}

template <bool CH>
int f32c_occupancy_ch(int model, int T, int KF) {
  WINDS_F32C_DISPATCH(occupancy_t)
  return 1;
}
}  // namespace

// a.heads set: the filament stream is chained (bs_pack_chains)
cudaError_t launch_f32c(const F32cArgs &a, int model, int T, int KF, int grid, cudaStream_t s) {
  return a.heads ? launch_f32c_ch<true>(a, model, T, KF, grid, s)
                 : launch_f32c_ch<false>(a, model, T, KF, grid, s);
}

int f32c_occupancy(int model, int T, int KF, bool chain) {
  return chain ? f32c_occupancy_ch<true>(model, T, KF) : f32c_occupancy_ch<false>(model, T, KF);
}

int f64_occupancy() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, bs_f64, kF64Threads, 0) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

cudaError_t launch_f64(const F32cArgs &a, int grid, cudaStream_t s) {
  bs_f64<<<grid, kF64Threads, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_bbox_init(BBox *bb, cudaStream_t s) {
  bs_bbox_init<<<1, 32, 0, s>>>(bb);
  return cudaGetLastError();
}

cudaError_t launch_pack_filaments(const double *F1, const double *F2, const double *gam,
                                  const double *rc, long long d0, long long nf, long long off,
                                  int model, double dcut, const PackedFilaments &pf, BBox *bb,
                                  cudaStream_t s) {
  if (nf <= 0) return cudaSuccess;
  const int bs = 256;
  const long long grid = (nf + bs - 1) / bs;
  bs_pack_filaments<<<(unsigned)grid, bs, 0, s>>>(F1, F2, gam, rc, d0, nf, off, model, dcut, pf.pk,
                                                 pf.ra, pf.rb, bb);
  return cudaGetLastError();
}

cudaError_t launch_pad_filaments(long long from, long long to, const PackedFilaments &pf,
                                 cudaStream_t s) {
  if (to <= from) return cudaSuccess;
  const int bs = 256;
  const long long grid = (to - from + bs - 1) / bs;
  bs_pad_filaments<<<(unsigned)grid, bs, 0, s>>>(from, to, pf.pk, pf.ra, pf.rb);
  return cudaGetLastError();
}

// Records of a [d0,3,d2,d3] family in a chained stream: room for the layout
// along either index (the device picks one; the rest of the room is inert).
long long chain_records(long long d0, long long d2, long long d3) {
  if (d0 <= 0 || d2 <= 0 || d3 <= 0) return 0;
  const long long a = chain_layout_records(d2 * d3, d0), b = chain_layout_records(d0 * d3, d2);
  return a > b ? a : b;
}

cudaError_t launch_pack_chains(const double *F1, const double *F2, const double *gam,
                               const double *rc, const long long d[4], long long rec_off,
                               unsigned long long *cnt, int model, double dcut,
                               const PackedFilaments &pf, unsigned *heads, BBox *bb,
                               cudaStream_t s) {
  const long long nf = d[0] * d[2] * d[3];
  const long long nrec = chain_records(d[0], d[2], d[3]);
  if (nf <= 0 || nrec <= 0) return cudaSuccess;
  const int bs = 256;
  cudaError_t e = cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  bs_chain_count<<<(unsigned)((nf + bs - 1) / bs), bs, 0, s>>>(F1, F2, d[0], d[2], nf, cnt);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  bs_pack_chains<<<(unsigned)((2 * nrec + bs - 1) / bs), bs, 0, s>>>(
      F1, F2, gam, rc, d[0], d[2], d[3], rec_off, nrec, cnt, model, dcut, pf.pk, pf.ra, pf.rb,
      heads, bb);
  return cudaGetLastError();
}

cudaError_t launch_pad_chains(long long from, long long to, const PackedFilaments &pf,
                              unsigned *heads, cudaStream_t s) {
  if (to <= from) return cudaSuccess;
  const int bs = 256;
  bs_pad_chains<<<(unsigned)((to - from + bs - 1) / bs), bs, 0, s>>>(from, to, pf.pk, pf.ra, pf.rb,
                                                                     heads);
  return cudaGetLastError();
}

cudaError_t launch_pack_targets(const double *P, long long ns, long long np, long long off,
                                int group, double4 *tp, int *tgroup, BBox *bb, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  const int bs = 256;
  const long long grid = (np + bs - 1) / bs;
  bs_pack_targets<<<(unsigned)grid, bs, 0, s>>>(P, ns, np, off, group, tp, tgroup, bb);
  return cudaGetLastError();
}

cudaError_t launch_target_keys(const double4 *tp, const int *tgroup, long long n, const BBox *bb,
                               unsigned long long *keys, int *vals, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  bs_target_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tp, tgroup, n, bb, keys, vals);
  return cudaGetLastError();
}

cudaError_t launch_gather_targets(const double4 *src, const int *perm, long long n, double4 *dst,
                                  cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  bs_gather_targets<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, perm, n, dst);
  return cudaGetLastError();
}

// Sorts (key, value) pairs with CUB's radix sort; temp == nullptr queries the
// scratch size into *temp_bytes.
cudaError_t sort_target_keys(void *temp, size_t *temp_bytes, const unsigned long long *kin,
                             unsigned long long *kout, const int *vin, int *vout, long long n,
                             cudaStream_t s) {
  return cub::DeviceRadixSort::SortPairs(temp, *temp_bytes, kin, kout, vin, vout, (int)n, 0, 64, s);
}

cudaError_t launch_reduce(const Tile *tiles, int n_tiles, const Group *groups, const double *part,
                          const int *perm, int tile_cap, cudaStream_t s, const Item *items,
                          const GroupLive *live) {
  if (n_tiles <= 0) return cudaSuccess;
  if (live && !items) return cudaErrorInvalidValue;
  const int bs = tile_cap >= 256 ? 256 : (tile_cap + 31) / 32 * 32;  // one thread per target
  bs_reduce<<<n_tiles, bs, 0, s>>>(tiles, groups, part, perm, tile_cap, items, live);
  return cudaGetLastError();
}

cudaError_t launch_length(const double *F1, const double *F2, long long d0, long long nf, double *L,
                          cudaStream_t s) {
  if (nf <= 0) return cudaSuccess;
  const int bs = 256;
  bs_length<<<(unsigned)((nf + bs - 1) / bs), bs, 0, s>>>(F1, F2, d0, nf, L);
  return cudaGetLastError();
}

unsigned long long default_wait_limit_ns() { return kDefaultWaitNs; }

cudaError_t launch_ffma_peak(float *out, int blocks, int iters, cudaStream_t s) {
  bs_ffma_peak<<<blocks, 256, 0, s>>>(out, iters, 0.999999f, 1e-7f);
  return cudaGetLastError();
}

cudaError_t launch_wait_selftest(unsigned *err, unsigned long long limit_ns, cudaStream_t s) {
  bs_wait_selftest<<<1, 32, 0, s>>>(err, limit_ns);
  return cudaGetLastError();
}

}  // namespace winds
