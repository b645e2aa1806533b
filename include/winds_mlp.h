/*
 * winds_mlp.h -- C ABI of the bound-circulation MLP of libwinds_bs: a small
 * network that predicts the converged Kutta-Joukowski bound circulation of a
 * blade station from its local state, used as the fixed point's initial
 * guess in place of the previous step's value (WInDS.m:131; the iteration of
 * core/KuttaJoukowski.m:42-49 then runs to the same tolerance, so converged
 * results are unchanged and only iterations are saved).
 *
 * No reference counterpart: the reference always starts the iteration from
 * the previous step's bound circulation.
 *
 * Network: n_in inputs (<= 16, zero-padded to 16), four hidden layers of
 * width 128 with GELU (tanh form), one linear output. Weights are FP32 master
 * copies with BF16 copies for the GEMMs; GEMMs run on the tensor cores with
 * FP32 accumulation; the output layer, loss and Adam run on the CUDA cores.
 *
 * Parameter vector (FP32, this order): W1 [128][16] (row = output unit,
 * column = input; columns >= n_in stay zero), b1 [128], W2 [128][128], b2,
 * W3 [128][128], b3, W4 [128][128], b4, w5 [128], b5 [1].
 *
 * Inputs are standardised inside the library: x_std = (x - shift) * scale.
 * The model output is the raw network value; a caller maps it to its target
 * (the wake engine uses Gamma = Gamma_prev + out_scale * y).
 */
#ifndef WINDS_MLP_H
#define WINDS_MLP_H

#include "winds_bs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct winds_mlp winds_mlp;

typedef struct {
  int n_in;                 /* input features, 1..16 */
  unsigned long long seed;  /* initial weights: normal(0, 1/fan_in), biases zero */
} winds_mlp_config;

typedef struct {
  int epochs;
  int batch;                /* rows per Adam step */
  float lr;
  float beta1, beta2, eps;
  float weight_decay;       /* decoupled (AdamW); 0 for plain Adam */
  unsigned long long seed;  /* row shuffling */
} winds_mlp_train_params;

/* Creates the network on the current device. */
int winds_mlp_create(const winds_mlp_config *cfg, winds_mlp **out);

/* Number of parameters (the length of the vectors below). */
long long winds_mlp_param_count(const winds_mlp *m);

/* FP32 master parameters to / from a host vector. */
int winds_mlp_get_params(winds_mlp *m, float *theta);
int winds_mlp_set_params(winds_mlp *m, const float *theta);

/* Input standardisation (n_in entries each) and the output scale. */
int winds_mlp_set_scaling(winds_mlp *m, const float *shift, const float *scale, float out_scale);
int winds_mlp_get_scaling(winds_mlp *m, float *shift, float *scale, float *out_scale);

/* What the wake engine adds the scaled output to when the network is its
 * lifting-line start value: the previous step's converged bound circulation
 * (the reference's start, WInDS.m:131; the default) or its linear
 * extrapolation over the last two steps, Gamma_prev + (Gamma_prev - Gamma_prev2),
 * so that the network learns the residual of the extrapolation. */
#define WINDS_MLP_BASE_PREVIOUS 0
#define WINDS_MLP_BASE_EXTRAPOLATED 1
int winds_mlp_set_base(winds_mlp *m, int base);
int winds_mlp_get_base(const winds_mlp *m);

/* y[i] = network(x[i]) for host rows x [n][n_in]. Synchronous. */
int winds_mlp_forward_host(winds_mlp *m, const float *x, long long n, float *y);

/* Loss 0.5 * mean((y - t)^2) over host rows and its gradient with respect to
 * the parameter vector (as the training step computes it). Synchronous. */
int winds_mlp_loss_grad_host(winds_mlp *m, const float *x, const float *t, long long n,
                             double *loss, float *grad);

/* Adam training on host rows (copied to the device once); epoch_loss
 * (optional, `epochs` entries) receives each epoch's mean loss. */
int winds_mlp_train_host(winds_mlp *m, const float *x, const float *t, long long n,
                         const winds_mlp_train_params *prm, float *epoch_loss);

/* Device time of the last winds_mlp_train_host call (ms) and its Adam steps. */
int winds_mlp_train_stats(winds_mlp *m, double *ms, long long *steps);

void winds_mlp_destroy(winds_mlp *m);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_MLP_H */
