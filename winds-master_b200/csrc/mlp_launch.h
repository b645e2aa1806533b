// mlp_launch.h -- kernels of the bound-circulation MLP (BF16 tcgen05 GEMMs
// with FP32 accumulation in tensor memory, CUDA-core head, reductions, Adam).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace winds {

constexpr int kMlpWidth = 128;  // hidden width (the GEMM tile's N and M)
constexpr int kMlpInPad = 16;   // input features padded to one K step of the MMA

// Epilogue of one GEMM tile (D = A B accumulated in tensor memory):
enum MlpEpi : int {
  kEpiPartial = 0,   // out_f32[blockIdx.z][m][n] = D (split-K partial sums)
  kEpiBiasGelu = 1,  // z = D + bias; z_out = z (FP32, optional); a_out = bf16(gelu(z))
  kEpiGeluBwd = 2,   // dz = D * gelu'(z_in); dz_out = bf16(dz); colsum_part[blockIdx.x][n] = sum_m dz
};

// D[M x N] = A[M x K] B[K x N], BF16 operands, FP32 accumulation.
// A stored row-major either as [M][K] (a_mn = 0) or as [K][M] (a_mn = 1),
// B as [N][K] (b_mn = 0) or [K][N] (b_mn = 1); leading dimensions in
// elements, multiples of 8, base pointers 16-byte aligned. K is a multiple
// of 16; M of 8 when A is stored [K][M].
struct MlpGemmArgs {
  const __nv_bfloat16 *A;
  long long lda;
  int a_mn;
  const __nv_bfloat16 *B;
  long long ldb;
  int b_mn;
  long long M, K;
  const float *bias;
  float *out_f32;
  long long ldo;
  float *z_out;
  __nv_bfloat16 *a_out;
  const float *z_in;
  __nv_bfloat16 *dz_out;
  float *colsum_part;
  unsigned *err;
  unsigned long long wait_limit_ns;
};

// N = 16 or 128; ksplit CTAs share the K range (kEpiPartial only).
cudaError_t launch_mlp_gemm(const MlpGemmArgs &g, int N, int epi, int ksplit, cudaStream_t s);

// Raw FP32 features [n][n_in] -> standardised, zero-padded BF16 [n][16].
cudaError_t launch_mlp_prep(const float *x, long long n, int n_in, const float *shift,
                            const float *scale, __nv_bfloat16 *X, cudaStream_t s);
// Rows idx[i] of X [.][16] and t [.] -> Xb [nb][16], tb [nb].
cudaError_t launch_mlp_gather(const __nv_bfloat16 *X, const float *t, const int *idx, long long nb,
                              __nv_bfloat16 *Xb, float *tb, cudaStream_t s);
// y[r] = a4[r] . w5 + b5 (a4 BF16 [n][128]).
cudaError_t launch_mlp_head_fwd(const __nv_bfloat16 *a4, long long n, const float *w5,
                                const float *b5, float *y, cudaStream_t s);
// Squared-error head gradient: dy = (y - t) * inv_n; dz4 = bf16(dy w5 gelu'(z4));
// per block of rows: partial sums of dw5 = sum dy a4, db4 = sum dz4, db5 = sum dy,
// loss = sum (y - t)^2. Returns the number of blocks through *nblocks.
cudaError_t launch_mlp_head_bwd(const float *y, const float *t, const float *z4,
                                const __nv_bfloat16 *a4, const float *w5, long long n, float inv_n,
                                __nv_bfloat16 *dz4, float *dw5_part, float *db4_part,
                                float *db5_part, float *loss_part, int rows_per_block,
                                cudaStream_t s);

struct MlpReduceJob {
  const float *part;  // [count][n]
  int count;
  int n;
  float *dst;         // [n]: dst[e] = sum_k part[k][e], summed in k order
  float scale;
};
cudaError_t launch_mlp_reduce(const MlpReduceJob *jobs_dev, int njobs, int max_n, cudaStream_t s);

// One Adam step over the flat parameter vector; writes the BF16 copy.
cudaError_t launch_mlp_adam(float *theta, __nv_bfloat16 *theta_bf, const float *grad, float *m,
                            float *v, long long n, float lr, float b1, float b2, float eps,
                            float wd, float c1, float c2, cudaStream_t s);
cudaError_t launch_mlp_to_bf16(const float *theta, __nv_bfloat16 *theta_bf, long long n,
                               cudaStream_t s);

}  // namespace winds
