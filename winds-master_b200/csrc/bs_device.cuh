// bs_device.cuh -- device helpers shared by the induced-velocity kernels:
// mbarrier + bulk-copy (TMA) wrappers with bounded waits, fast FP32
// reciprocal square roots, ordered-float atomics, and the FP64 pair term that
// restates the reference formulas (used by the plain FP64 kernel and by the
// near-singular fix-up of the FP32 kernel).
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "bs_types.h"

namespace winds {

// ---------------------------------------------------------------- constants
constexpr double kPi = 3.14159265358979324;  // cuda/source/BiotSavartMex.cu:35
// (1.000/(4.000*pi)) as the reference's host loop folds it (BiotSavartMex.cu:260)
constexpr double kInv4PiMex = 1.000 / (4.000 * kPi);
// 4*pi as MATLAB evaluates it in core/BiotSavart.m:106,108
constexpr double k4Pi = 4.0 * 3.141592653589793;


// ------------------------------------------------------- PTX: barriers + bulk
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once on the barrier and add `bytes` to its expected transaction count.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Plain arrive (release) on the barrier.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// try_wait that lets the hardware suspend the thread for up to `hint_ns`
// while the phase is incomplete (no busy spinning).
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t *bar, uint32_t parity,
                                                    uint32_t hint_ns) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return ok != 0;
}

// Waits for the barrier phase with the given parity for at most `limit_ns`
// nanoseconds (the timer is read once per 32 suspended tries). On timeout it
// sets kErrWaitTimeout in *err and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, unsigned *err,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
#pragma unroll 1
    for (int k = 0; k < 32; ++k)
      if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
    if (global_timer_ns() - t0 > limit_ns) {
      atomicOr(err, kErrWaitTimeout);
      return false;
    }
  }
}

// One non-multicast bulk copy global -> this CTA's shared memory, completing
// `bytes` transactions on `bar`. Both addresses 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------ fast FP32 math
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Ordered mapping float <-> int so that atomicMin/atomicMax on ints order floats.
__device__ __forceinline__ int float_key(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__host__ __device__ inline float key_float(int k) {
  int i = k >= 0 ? k : k ^ 0x7fffffff;
  float f;
  memcpy(&f, &i, sizeof(f));
  return f;
}

// Block-level min/max of three floats, then one atomic per block and bound.
__device__ __forceinline__ void bbox_accumulate(const float lo[3], const float hi[3], int *gmin,
                                                int *gmax) {
  __shared__ float smin[3][32], smax[3][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    for (int o = 16; o > 0; o >>= 1) {
      l[c] = fminf(l[c], __shfl_xor_sync(0xffffffffu, l[c], o));
      h[c] = fmaxf(h[c], __shfl_xor_sync(0xffffffffu, h[c], o));
    }
    if (lane == 0) {
      smin[c][warp] = l[c];
      smax[c][warp] = h[c];
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int c = threadIdx.x;
    float a = FLT_MAX, b = -FLT_MAX;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = fminf(a, smin[c][w]);
      b = fmaxf(b, smax[c][w]);
    }
    // the box grows only at first: most blocks lie inside it already, so a
    // plain read spares the contended atomic (the bound only ever tightens
    // towards the block's value, so skipping a non-improving one is exact)
    const int ka = float_key(a), kb = float_key(b);
    if (a != FLT_MAX && ka < *(volatile const int *)&gmin[c]) atomicMin(&gmin[c], ka);
    if (b != -FLT_MAX && kb > *(volatile const int *)&gmax[c]) atomicMax(&gmax[c], kb);
  }
}

// ------------------------------------------------------- filament packing
// Field q of filament f in the pair-record layout (bs_types.h).
__device__ __forceinline__ float &pk_field(float4 *pk, long long f, int q) {
  return reinterpret_cast<float *>(pk)[(f >> 1) * 32 + 2 * q + (f & 1)];
}

// Writes filament f in the packed layout (see bs_types.h): FP32 hi/lo x1,
// |L|^2, near-singular radius Rn^2 = max(|L|^2, 9 rc^2), L, the core term and
// K L (K = gamma/4pi), plus the FP64 copy. A NaN/Inf ubar is zeroed by the
// reference (core/BiotSavart.m:111); with finite endpoints that happens
// exactly when gamma (or, Vatistas, rc; or, cut-off, d*|L|^2) is not finite,
// so such filaments get K = 0 and contribute nothing.
//
// Vatistas n=2 in FP32: with c = K L x r1, the core factor
// |L x r1|^2 / sqrt(|L x r1|^4 + (rc^2 |L|^2)^2) equals |c|^2 / sqrt(|c|^4 + D)
// for D = (K^2 rc^2 |L|^2)^2, so the kernel never multiplies by K.
//
// filament_fields computes the 16 FP32 fields; pack_filament writes them one
// float at a time, store_pair_fields lets the two lanes of a pair write the
// 128-byte record with four 16-byte stores each.
__device__ __forceinline__ void filament_fields(double x1, double y1, double z1, double x2,
                                                double y2, double z2, double g, double r,
                                                int model, double dcut, float v[16]) {
  const double Lx = x2 - x1, Ly = y2 - y1, Lz = z2 - z1;
  const double L2 = Lx * Lx + Ly * Ly + Lz * Lz;
  double K = g / k4Pi;
  if (!isfinite(g)) K = 0.0;
  double D;
  if (model == kCoreVatistas) {
    if (!isfinite(r)) K = 0.0;
    const double s = K * K * r * L2;
    D = s * s;
    if (!(D >= 1e-30)) D = 1e-30;  // also K = 0: the factor stays finite, K L = 0
    if (D > 1e30) D = 1e30;
  } else {
    D = dcut * L2;
    if (!isfinite(D)) K = 0.0, D = 0.0;
  }
  // Near-singular region: r1.r2 < Rn^2, a ball around the midpoint of radius
  // sqrt(|L|^2/4 + Rn^2) that contains every point within 3 core radii.
  double Rn2 = L2;
  if (isfinite(r) && 9.0 * r > Rn2) Rn2 = 9.0 * r;
  if (!(Rn2 > 1e-20)) Rn2 = 1e-20;
  const float hx = (float)x1, hy = (float)y1, hz = (float)z1;
  v[0] = hx, v[1] = hy, v[2] = hz, v[3] = (float)L2;
  v[4] = (float)(x1 - (double)hx), v[5] = (float)(y1 - (double)hy);
  v[6] = (float)(z1 - (double)hz), v[7] = (float)Rn2;
  v[8] = (float)Lx, v[9] = (float)Ly, v[10] = (float)Lz, v[11] = (float)D;
  v[12] = (float)(K * Lx), v[13] = (float)(K * Ly), v[14] = (float)(K * Lz);
  // the core radius, for the kernel's screen of pairs whose core factor is 1
  v[15] = model == kCoreVatistas && K != 0.0 ? (float)sqrt(fmax(r, 0.0)) : 0.f;
}

// Fields of an inert filament (far away, zero length, zero circulation) for padding.
__device__ __forceinline__ void inert_fields(float v[16]) {
  const float far = 1e18f;
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = 0.f;
  v[0] = v[1] = v[2] = far;
  v[11] = 1.f;
}
constexpr double kInertFar = 1e18;

__device__ __forceinline__ void pack_filament(long long f, double x1, double y1, double z1,
                                              double x2, double y2, double z2, double g, double r,
                                              int model, double dcut, float4 *pk, double4 *ra,
                                              double4 *rb) {
  ra[f] = make_double4(x1, y1, z1, g);
  rb[f] = make_double4(x2, y2, z2, r);
  float v[16];
  filament_fields(x1, y1, z1, x2, y2, z2, g, r, model, dcut, v);
#pragma unroll
  for (int q = 0; q < 16; ++q) pk_field(pk, f, q) = v[q];
}

__device__ __forceinline__ void pack_inert(long long f, float4 *pk, double4 *ra, double4 *rb) {
  float v[16];
  inert_fields(v);
#pragma unroll
  for (int q = 0; q < 16; ++q) pk_field(pk, f, q) = v[q];
  ra[f] = make_double4(kInertFar, kInertFar, kInertFar, 0.0);
  rb[f] = make_double4(kInertFar, kInertFar, kInertFar, 0.0);
}

// Pair record of filaments f and f ^ 1 from the two lanes holding them (f even
// on the even lane of the pair): every lane of the warp calls this; a lane
// with `active` false stores nothing (its pair partner must be inactive too).
// Float4 k of the record is {e[2k], o[2k], e[2k+1], o[2k+1]} (e, o the even
// and odd filament's fields); the even lane stores k = 0..3, the odd lane 4..7.
__device__ __forceinline__ void store_pair_fields(float4 *pk, long long f, const float v[16],
                                                  bool active) {
  const bool odd = (threadIdx.x & 1) != 0;
  // x: the partner's fields this lane stores -- the odd filament's 0..7 on
  // the even lane, the even filament's 8..15 on the odd lane
  float x[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) x[q] = __shfl_xor_sync(0xffffffffu, odd ? v[q] : v[q + 8], 1);
  if (!active) return;
  float4 *rec = pk + (f >> 1) * 8;
  if (!odd) {
#pragma unroll
    for (int k = 0; k < 4; ++k) rec[k] = make_float4(v[2 * k], x[2 * k], v[2 * k + 1], x[2 * k + 1]);
  } else {
#pragma unroll
    for (int k = 4; k < 8; ++k)
      rec[k] = make_float4(x[2 * k - 8], v[2 * k], x[2 * k - 7], v[2 * k + 1]);
  }
}

// ---------------------------------------------------- FP64 reference pair term
struct RefParams {
  int model;   // kCoreCutoff / kCoreVatistas
  double d;    // cut-off squared radius (cut-off model)
  double n;    // Vatistas index (Vatistas model)
  double co;   // reach cut-off
};

// Contribution of filament (A.xyz -> B.xyz, circulation A.w, squared core B.w)
// at point p, accumulated into u.
//
// Cut-off model: the operation sequence of the reference's host loop
// biot_p2p_nogpu (cuda/source/BiotSavartMex.cu:236-266), which is also the
// formula of core/BiotSavart.m:108, with no fused multiply-adds, so a
// sequential sum over filaments reproduces that loop bit for bit.
// Vatistas model: the sequence of core/BiotSavart.m:103-106.
// kGeneralN = false compiles only the n = 2 branch (the FP32 kernel's case).
// Both then apply core/BiotSavart.m:111: a NaN/Inf ubar, or r1>co and r2>co,
// gives ubar = 0 (the cross product still multiplies it, as in MATLAB).
template <bool kGeneralN = true>
__device__ __forceinline__ void ref_pair(const double4 A, const double4 B, double px, double py,
                                         double pz, const RefParams &rp, double &ux, double &uy,
                                         double &uz) {
  const double x1 = A.x, y1 = A.y, z1 = A.z, g = A.w;
  const double x2 = B.x, y2 = B.y, z2 = B.z, rc = B.w;
  const double pxx1 = __dsub_rn(px, x1), pxx2 = __dsub_rn(px, x2);
  const double pyy1 = __dsub_rn(py, y1), pyy2 = __dsub_rn(py, y2);
  const double pzz1 = __dsub_rn(pz, z1), pzz2 = __dsub_rn(pz, z2);
  const double r1 = sqrt(
      __dadd_rn(__dadd_rn(__dmul_rn(pxx1, pxx1), __dmul_rn(pyy1, pyy1)), __dmul_rn(pzz1, pzz1)));
  const double r2 = sqrt(
      __dadd_rn(__dadd_rn(__dmul_rn(pxx2, pxx2), __dmul_rn(pyy2, pyy2)), __dmul_rn(pzz2, pzz2)));
  const double r1dr2 =
      __dadd_rn(__dadd_rn(__dmul_rn(pxx1, pxx2), __dmul_rn(pyy1, pyy2)), __dmul_rn(pzz1, pzz2));
  const double r1tr2 = __dmul_rn(r1, r2);
  double ubar;
  if (rp.model == kCoreCutoff) {
    const double ldx = __dsub_rn(x1, x2), ldy = __dsub_rn(y1, y2), ldz = __dsub_rn(z1, z2);
    const double len =
        __dadd_rn(__dadd_rn(__dmul_rn(ldx, ldx), __dmul_rn(ldy, ldy)), __dmul_rn(ldz, ldz));
    const double den = __dadd_rn(__dmul_rn(r1tr2, __dadd_rn(r1tr2, r1dr2)), __dmul_rn(rp.d, len));
    ubar = __dmul_rn(__dmul_rn(g, __dadd_rn(r1, r2)), kInv4PiMex);
    ubar = __ddiv_rn(ubar, den);
  } else {
    const double x2x1 = __dsub_rn(x2, x1), y2y1 = __dsub_rn(y2, y1), z2z1 = __dsub_rn(z2, z1);
    const double L = __dadd_rn(__dadd_rn(__dmul_rn(x2x1, x2x1), __dmul_rn(y2y1, y2y1)),
                               __dmul_rn(z2z1, z2z1));
    const double ld = __dadd_rn(__dadd_rn(__dmul_rn(x2x1, pxx1), __dmul_rn(y2y1, pyy1)),
                                __dmul_rn(z2z1, pzz1));
    const double Ldr12 = __dmul_rn(ld, ld);
    double Cnu = __dsub_rn(__dmul_rn(r1, r1), __ddiv_rn(Ldr12, L));
    double base;
    if (!kGeneralN || rp.n == 2.0) {
      base = __dadd_rn(__dmul_rn(rc, rc), __dmul_rn(Cnu, Cnu));
      Cnu = __dmul_rn(Cnu, __ddiv_rn(1.0, sqrt(base)));
    } else {
      base = __dadd_rn(pow(rc, rp.n), pow(Cnu, rp.n));
      Cnu = __dmul_rn(Cnu, pow(base, -1.0 / rp.n));
    }
    ubar = __ddiv_rn(__dmul_rn(__ddiv_rn(__dmul_rn(Cnu, g), k4Pi), __dadd_rn(r1, r2)),
                     __dmul_rn(r1tr2, __dadd_rn(r1tr2, r1dr2)));
  }
  if (isnan(ubar) || isinf(ubar) || (r1 > rp.co && r2 > rp.co)) ubar = 0.0;
  ux = __dadd_rn(ux, __dmul_rn(ubar, __dsub_rn(__dmul_rn(pyy1, pzz2), __dmul_rn(pzz1, pyy2))));
  uy = __dadd_rn(uy, __dmul_rn(ubar, __dsub_rn(__dmul_rn(pzz1, pxx2), __dmul_rn(pxx1, pzz2))));
  uz = __dadd_rn(uz, __dmul_rn(ubar, __dsub_rn(__dmul_rn(pxx1, pyy2), __dmul_rn(pyy1, pxx2))));
}

}  // namespace winds
