// mlp_engine.h -- internal host side of the bound-circulation MLP (the C ABI
// is include/winds_mlp.h); shared with the wake engine, which runs the
// network's forward pass on its own stream for the Kutta-Joukowski guess.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "engine.h"
#include "winds_mlp.h"

namespace winds {

// Activations and partial sums for up to `cap` rows.
struct MlpWork {
  long long cap = 0;
  bool train = false;
  DevBuf X, t, y, Z[4], A[4], dZa, dZb, part_w[4], part_b[4], dw5p, db5p, lossp, xraw;
  int ensure(long long n, bool train, cudaStream_t s);
  void release();
};

// Runs the forward pass on rows X (BF16 [n][16], standardised) into y [n];
// with w.train the pre-activations are kept for a backward pass.
int mlp_forward(const winds_mlp *m, const __nv_bfloat16 *X, long long n, MlpWork &w, float *y,
                cudaStream_t s);

// Device copies of the input standardisation and the output scale.
const float *mlp_shift_dev(const winds_mlp *m);
const float *mlp_scale_dev(const winds_mlp *m);
float mlp_out_scale(const winds_mlp *m);
const float *mlp_out_scale_dev(const winds_mlp *m);
const float *mlp_base_dev(const winds_mlp *m);
int mlp_n_in(const winds_mlp *m);
int mlp_device(const winds_mlp *m);
unsigned *mlp_err_word(const winds_mlp *m);

}  // namespace winds
