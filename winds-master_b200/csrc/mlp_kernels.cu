// mlp_kernels.cu -- kernels of the MLP that predicts the converged bound
// circulation (the Kutta-Joukowski initial guess).
//
// GEMMs run on the 5th-generation tensor cores: operands are staged in shared
// memory in the no-swizzle core-matrix layout (8 rows x 16 bytes per core
// matrix), one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32,
// M = 128) into a tensor-memory accumulator and commits to an mbarrier, and
// the four warps read the accumulator back with tcgen05.ld (warp w owns
// lanes 32w..32w+31, one output row per thread) for a fused epilogue.
//
// One shared-memory tile serves both operand majors: the tile of a row-major
// [R][C] matrix is stored with element (r, c) at
//     (r / 8) * (C / 8) * 128 + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2   bytes,
// which is the K-major canonical layout when rows are M (or N) and columns K
// (LBO = 128 between K chunks, SBO = C/8*128 between row groups), and the
// MN-major canonical layout when rows are K and columns M (or N) (SBO = 128
// between M groups, LBO = C/8*128 between K groups). So activations stored
// [rows][features] and weights stored [out][in] feed the forward GEMM, the
// input-gradient GEMM and the weight-gradient GEMM without transposes.
#include <cuda_bf16.h>

#include "bs_device.cuh"
#include "mlp_launch.h"

namespace winds {
namespace {

constexpr int kGemmThreads = 128;
constexpr int kTileM = 128;
constexpr int kChunkK = 64;

// ------------------------------------------------------- tcgen05 wrappers
// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all >> 4), descriptor version 1 at bits 46-47.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;
  return d;
}

// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16
// (bits 7-9, 10-12 = 1), operand majors (bits 15, 16: 1 = MN-major),
// N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__device__ __forceinline__ uint32_t umma_idesc(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes made visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Arrives on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread i gets lane (base + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ----------------------------------------------------------- activation
// GELU, tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float kGeluA = 0.044715f;

__device__ __forceinline__ float gelu(float z) {
  const float u = kGeluC * fmaf(kGeluA * z, z * z, z);
  return 0.5f * z * (1.f + tanhf(u));
}

__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanhf(kGeluC * fmaf(kGeluA * z, z2, z));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * kGeluC * fmaf(3.f * kGeluA, z2, 1.f);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}

// Copies rows [r0, r0+R) x columns [c0, c0+C) of a row-major BF16 matrix
// (row stride ld) into the core-matrix tile; rows >= r_lim or columns >=
// c_lim read as zero (c_lim and c0 are multiples of 8).
template <int R, int C>
__device__ __forceinline__ void load_tile(unsigned char *dst, const __nv_bfloat16 *src,
                                          long long ld, long long r0, long long r_lim,
                                          long long c0, long long c_lim) {
  constexpr int V = R * (C / 8);
#pragma unroll 4
  for (int v = threadIdx.x; v < V; v += kGemmThreads) {
    const int r = v / (C / 8), c8 = v % (C / 8);
    const long long gr = r0 + r, gc = c0 + 8 * c8;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (gr < r_lim && gc < c_lim) val = *reinterpret_cast<const uint4 *>(src + gr * ld + gc);
    *reinterpret_cast<uint4 *>(dst + (r / 8) * (C / 8) * 128 + c8 * 128 + (r % 8) * 16) = val;
  }
}

struct __align__(1024) GemmSmem {
  unsigned char a[kTileM * kChunkK * 2];  // 16 KB
  unsigned char b[128 * kChunkK * 2];     // 16 KB
  float colsum[4][128];
  uint64_t mbar;
  uint32_t tmem_slot;
};

// Dynamic shared memory per CTA: the tiles plus padding so that at most four
// CTAs share an SM, whose 512 tensor-memory columns then always hold their
// 128-column accumulators (tcgen05.alloc never has to wait).
constexpr int kGemmSmemBytes = 56 * 1024;
static_assert(sizeof(GemmSmem) <= kGemmSmemBytes, "GEMM tile does not fit its shared memory");

template <int N, int EPI>
__global__ void __launch_bounds__(kGemmThreads) mlp_gemm(const MlpGemmArgs g) {
  extern __shared__ __align__(1024) unsigned char gemm_smem[];
  GemmSmem &sm = *reinterpret_cast<GemmSmem *>(gemm_smem);
  constexpr uint32_t kCols = N < 32 ? 32 : N;  // tensor-memory columns (power of 2, >= 32)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&sm.tmem_slot, kCols);
  if (tid == 0) {
    mbar_init(&sm.mbar, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem_slot;

  const long long m0 = (long long)blockIdx.x * kTileM;
  const long long kchunks = (g.K + kChunkK - 1) / kChunkK;
  const long long per = (kchunks + gridDim.z - 1) / gridDim.z;
  const long long kc0 = (long long)blockIdx.z * per;
  const long long kc1 = kc0 + per < kchunks ? kc0 + per : kchunks;

  const uint32_t idesc = umma_idesc(kTileM, N, g.a_mn, g.b_mn);
  const uint32_t sa = smem_u32(sm.a), sb = smem_u32(sm.b);
  const uint32_t a_lbo = g.a_mn ? (kTileM / 8) * 128 : 128;
  const uint32_t a_sbo = g.a_mn ? 128 : (kChunkK / 8) * 128;
  const uint32_t a_step = g.a_mn ? 2 * a_lbo : 256;  // 16 K per MMA: two K groups
  const uint32_t b_lbo = g.b_mn ? (N / 8) * 128 : 128;
  const uint32_t b_sbo = g.b_mn ? 128 : (kChunkK / 8) * 128;
  const uint32_t b_step = g.b_mn ? 2 * b_lbo : 256;

  uint32_t phase = 0;
  int issued = 0;
  bool ok = true;
  for (long long kc = kc0; kc < kc1; ++kc) {
    const long long k0 = kc * kChunkK;
    if (g.a_mn)
      load_tile<kChunkK, kTileM>(sm.a, g.A, g.lda, k0, g.K, m0, g.M);
    else
      load_tile<kTileM, kChunkK>(sm.a, g.A, g.lda, m0, g.M, k0, g.K);
    if (g.b_mn)
      load_tile<kChunkK, N>(sm.b, g.B, g.ldb, k0, g.K, 0, N);
    else
      load_tile<N, kChunkK>(sm.b, g.B, g.ldb, 0, N, k0, g.K);
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      long long rem = (g.K - k0 + 15) / 16;
      const int nk = rem < kChunkK / 16 ? (int)rem : kChunkK / 16;
      for (int j = 0; j < nk; ++j)
        tc_mma(tmem, umma_desc(sa + j * a_step, a_lbo, a_sbo),
               umma_desc(sb + j * b_step, b_lbo, b_sbo), idesc, (issued > 0 || j > 0) ? 1u : 0u);
      tc_commit(&sm.mbar);
    }
    ++issued;
    // the MMAs have read the tile (and written the accumulator) once the
    // barrier flips: the next chunk may overwrite shared memory
    ok = mbar_wait_bounded(&sm.mbar, phase, g.err, g.wait_limit_ns);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
  }
  if (!ok) {
    // a wait ran out: give the MMAs in flight one more bounded wait before
    // the accumulator is released
    if (tid == 0) mbar_wait_bounded(&sm.mbar, phase ^ 1u, g.err, g.wait_limit_ns);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kCols);
    return;
  }
  tc_fence_after();

  const long long row = m0 + warp * 32 + lane;
  const bool valid = row < g.M;
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
  for (int c = 0; c < N / 16; ++c) {
    float v[16];
    tmem_ld16(trow + 16 * c, v);  // every lane of the warp takes part
    if (issued == 0) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = 0.f;
    }
    const int n0 = 16 * c;
    if (EPI == kEpiPartial) {
      if (valid) {
        float4 *o = reinterpret_cast<float4 *>(g.out_f32 + (long long)blockIdx.z * g.M * g.ldo +
                                               row * g.ldo + n0);
#pragma unroll
        for (int q = 0; q < 4; ++q) o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
    } else if (EPI == kEpiBiasGelu) {
      if (valid) {
        float z[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) z[i] = v[i] + g.bias[n0 + i];
        if (g.z_out) {
          float4 *o = reinterpret_cast<float4 *>(g.z_out + row * g.ldo + n0);
#pragma unroll
          for (int q = 0; q < 4; ++q) o[q] = make_float4(z[4 * q], z[4 * q + 1], z[4 * q + 2], z[4 * q + 3]);
        }
        uint32_t p[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) p[i] = pack_bf16(gelu(z[2 * i]), gelu(z[2 * i + 1]));
        uint4 *o = reinterpret_cast<uint4 *>(g.a_out + row * g.ldo + n0);
        o[0] = make_uint4(p[0], p[1], p[2], p[3]);
        o[1] = make_uint4(p[4], p[5], p[6], p[7]);
      }
    } else {  // kEpiGeluBwd
      float dz[16];
      if (valid) {
        const float4 *zi = reinterpret_cast<const float4 *>(g.z_in + row * g.ldo + n0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 z = zi[q];
          dz[4 * q] = v[4 * q] * gelu_grad(z.x);
          dz[4 * q + 1] = v[4 * q + 1] * gelu_grad(z.y);
          dz[4 * q + 2] = v[4 * q + 2] * gelu_grad(z.z);
          dz[4 * q + 3] = v[4 * q + 3] * gelu_grad(z.w);
        }
        uint32_t p[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) p[i] = pack_bf16(dz[2 * i], dz[2 * i + 1]);
        uint4 *o = reinterpret_cast<uint4 *>(g.dz_out + row * g.ldo + n0);
        o[0] = make_uint4(p[0], p[1], p[2], p[3]);
        o[1] = make_uint4(p[4], p[5], p[6], p[7]);
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) dz[i] = 0.f;
      }
      // column sums of this warp's 32 rows, fixed shuffle order
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        float s = dz[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sm.colsum[warp][n0 + i] = s;
      }
    }
  }
  if (EPI == kEpiGeluBwd) {
    __syncthreads();
    if (tid < N)
      g.colsum_part[(long long)blockIdx.x * N + tid] =
          ((sm.colsum[0][tid] + sm.colsum[1][tid]) + sm.colsum[2][tid]) + sm.colsum[3][tid];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kCols);
}

// ------------------------------------------------------------- CUDA cores
__global__ void mlp_prep(const float *__restrict__ x, long long n, int n_in,
                         const float *__restrict__ shift, const float *__restrict__ scale,
                         __nv_bfloat16 *__restrict__ X) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * kMlpInPad) return;
  const long long r = i / kMlpInPad;
  const int c = (int)(i % kMlpInPad);
  const float v = c < n_in ? (x[r * n_in + c] - shift[c]) * scale[c] : 0.f;
  X[i] = __float2bfloat16_rn(v);
}

__global__ void mlp_gather(const __nv_bfloat16 *__restrict__ X, const float *__restrict__ t,
                           const int *__restrict__ idx, long long nb, __nv_bfloat16 *__restrict__ Xb,
                           float *__restrict__ tb) {
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nb) return;
  const long long s = idx[r];
  const uint4 *src = reinterpret_cast<const uint4 *>(X + s * kMlpInPad);
  uint4 *dst = reinterpret_cast<uint4 *>(Xb + r * kMlpInPad);
  dst[0] = src[0];
  dst[1] = src[1];
  tb[r] = t[s];
}

// One warp per row: lane l holds columns 4l .. 4l+3.
__global__ void mlp_head_fwd(const __nv_bfloat16 *__restrict__ a4, long long n,
                             const float *__restrict__ w5, const float *__restrict__ b5,
                             float *__restrict__ y) {
  const long long r = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(a4 + r * kMlpWidth + 4 * lane);
  const float2 u = __bfloat1622float2(p[0]), w = __bfloat1622float2(p[1]);
  float s = u.x * w5[4 * lane] + u.y * w5[4 * lane + 1] + w.x * w5[4 * lane + 2] +
            w.y * w5[4 * lane + 3];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[r] = s + b5[0];
}

// Thread j owns column j of a block of rows.
__global__ void mlp_head_bwd(const float *__restrict__ y, const float *__restrict__ t,
                             const float *__restrict__ z4, const __nv_bfloat16 *__restrict__ a4,
                             const float *__restrict__ w5, long long n, float inv_n,
                             __nv_bfloat16 *__restrict__ dz4, float *__restrict__ dw5_part,
                             float *__restrict__ db4_part, float *__restrict__ db5_part,
                             float *__restrict__ loss_part, int rows_per_block) {
  const int j = threadIdx.x;
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  long long r1 = r0 + rows_per_block;
  if (r1 > n) r1 = n;
  const float w = w5[j];
  float adw = 0.f, adb = 0.f, ady = 0.f, al = 0.f;
  for (long long r = r0; r < r1; ++r) {
    const float e = y[r] - t[r];
    const float dy = e * inv_n;
    const float dz = dy * w * gelu_grad(z4[r * kMlpWidth + j]);
    dz4[r * kMlpWidth + j] = __float2bfloat16_rn(dz);
    adw = fmaf(dy, __bfloat162float(a4[r * kMlpWidth + j]), adw);
    adb += dz;
    ady += dy;
    al = fmaf(e, e, al);
  }
  dw5_part[(long long)blockIdx.x * kMlpWidth + j] = adw;
  db4_part[(long long)blockIdx.x * kMlpWidth + j] = adb;
  if (j == 0) {
    db5_part[blockIdx.x] = ady;
    loss_part[blockIdx.x] = al;
  }
}

__global__ void mlp_reduce(const MlpReduceJob *__restrict__ jobs) {
  const MlpReduceJob jb = jobs[blockIdx.y];
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= jb.n) return;
  float s = 0.f;
  for (int k = 0; k < jb.count; ++k) s += jb.part[(long long)k * jb.n + e];
  jb.dst[e] = s * jb.scale;
}

// Adam with bias corrections c1 = 1 - b1^t, c2 = 1 - b2^t (and decoupled
// weight decay wd).
__global__ void mlp_adam(float *__restrict__ theta, __nv_bfloat16 *__restrict__ theta_bf,
                         const float *__restrict__ grad, float *__restrict__ m,
                         float *__restrict__ v, long long n, float lr, float b1, float b2,
                         float eps, float wd, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grad[i];
  const float mi = fmaf(b1, m[i], (1.f - b1) * g);
  const float vi = fmaf(b2, v[i], (1.f - b2) * g * g);
  m[i] = mi;
  v[i] = vi;
  float th = theta[i];
  th -= lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * th);
  theta[i] = th;
  theta_bf[i] = __float2bfloat16_rn(th);
}

__global__ void mlp_to_bf16(const float *__restrict__ theta, __nv_bfloat16 *__restrict__ theta_bf,
                            long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) theta_bf[i] = __float2bfloat16_rn(theta[i]);
}

unsigned blocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

cudaError_t launch_mlp_gemm(const MlpGemmArgs &g, int N, int epi, int ksplit, cudaStream_t s) {
  if (g.M <= 0) return cudaSuccess;
  if (ksplit < 1 || (epi != kEpiPartial && ksplit != 1)) return cudaErrorInvalidValue;
  const dim3 grid((unsigned)((g.M + kTileM - 1) / kTileM), 1, (unsigned)ksplit);
  void (*k)(const MlpGemmArgs);
  if (N == 128 && epi == kEpiPartial)
    k = mlp_gemm<128, kEpiPartial>;
  else if (N == 16 && epi == kEpiPartial)
    k = mlp_gemm<16, kEpiPartial>;
  else if (N == 128 && epi == kEpiBiasGelu)
    k = mlp_gemm<128, kEpiBiasGelu>;
  else if (N == 128 && epi == kEpiGeluBwd)
    k = mlp_gemm<128, kEpiGeluBwd>;
  else
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmemBytes);
  if (e != cudaSuccess) return e;
  k<<<grid, kGemmThreads, kGemmSmemBytes, s>>>(g);
  return cudaGetLastError();
}

cudaError_t launch_mlp_prep(const float *x, long long n, int n_in, const float *shift,
                            const float *scale, __nv_bfloat16 *X, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  mlp_prep<<<blocks(n * kMlpInPad, 256), 256, 0, s>>>(x, n, n_in, shift, scale, X);
  return cudaGetLastError();
}

cudaError_t launch_mlp_gather(const __nv_bfloat16 *X, const float *t, const int *idx, long long nb,
                              __nv_bfloat16 *Xb, float *tb, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  mlp_gather<<<blocks(nb, 256), 256, 0, s>>>(X, t, idx, nb, Xb, tb);
  return cudaGetLastError();
}

cudaError_t launch_mlp_head_fwd(const __nv_bfloat16 *a4, long long n, const float *w5,
                                const float *b5, float *y, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  mlp_head_fwd<<<blocks(n, 8), 256, 0, s>>>(a4, n, w5, b5, y);
  return cudaGetLastError();
}

cudaError_t launch_mlp_head_bwd(const float *y, const float *t, const float *z4,
                                const __nv_bfloat16 *a4, const float *w5, long long n, float inv_n,
                                __nv_bfloat16 *dz4, float *dw5_part, float *db4_part,
                                float *db5_part, float *loss_part, int rows_per_block,
                                cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  mlp_head_bwd<<<blocks(n, rows_per_block), kMlpWidth, 0, s>>>(
      y, t, z4, a4, w5, n, inv_n, dz4, dw5_part, db4_part, db5_part, loss_part, rows_per_block);
  return cudaGetLastError();
}

cudaError_t launch_mlp_reduce(const MlpReduceJob *jobs_dev, int njobs, int max_n, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  mlp_reduce<<<dim3(blocks(max_n, 256), (unsigned)njobs), 256, 0, s>>>(jobs_dev);
  return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float *theta, __nv_bfloat16 *theta_bf, const float *grad, float *m,
                            float *v, long long n, float lr, float b1, float b2, float eps,
                            float wd, float c1, float c2, cudaStream_t s) {
  mlp_adam<<<blocks(n, 256), 256, 0, s>>>(theta, theta_bf, grad, m, v, n, lr, b1, b2, eps, wd, c1,
                                          c2);
  return cudaGetLastError();
}

cudaError_t launch_mlp_to_bf16(const float *theta, __nv_bfloat16 *theta_bf, long long n,
                               cudaStream_t s) {
  mlp_to_bf16<<<blocks(n, 256), 256, 0, s>>>(theta, theta_bf, n);
  return cudaGetLastError();
}

}  // namespace winds
