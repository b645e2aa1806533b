// mlp_engine.cu -- host side of the bound-circulation MLP: parameters,
// forward / backward launch sequences, Adam training, C ABI (winds_mlp.h).
//
// One training step on a batch of n rows (15 launches):
//   forward   4 x GEMM (bias + GELU epilogue, pre-activations kept), head
//   backward  head (loss, dz4 and the output-layer partial sums), then for
//             layers 4, 3, 2: weight-gradient GEMM (split over rows) and
//             input-gradient GEMM (GELU' epilogue with bias-gradient column
//             sums); layer 1: weight-gradient GEMM; one reduction of every
//             partial sum in a fixed order (deterministic)
//   update    Adam on the FP32 master vector, BF16 copy for the GEMMs
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "bs_launch.h"
#include "mlp_engine.h"
#include "mlp_launch.h"

struct winds_mlp {
  int dev = 0;
  int n_in = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  winds::DevBuf theta, theta_bf, grad, mom, vel, shift, scale, err, jobs, loss, lossbuf, idx;
  winds::DevBuf Xall, Tall, xall_raw;
  float out_scale = 1.f;
  int base = 0;  // start value the output is added to (winds_mlp_set_base)
  float h_shift[16], h_scale[16];
  long long adam_t = 0;
  winds::MlpWork w;
  double train_ms = 0.0;
  long long train_steps = 0;
};

namespace winds {
namespace {

constexpr int W = kMlpWidth;
constexpr int kHeadRows = 64;  // rows per block of the head's backward kernel

// Offsets in the parameter vector.
constexpr long long kOffW[4] = {0, 2176, 18688, 35200};
constexpr long long kOffB[4] = {2048, 18560, 35072, 51584};
constexpr long long kOffW5 = 51712;
constexpr long long kOffB5 = 51840;
constexpr long long kNParam = 51841;
constexpr int kInK[4] = {kMlpInPad, W, W, W};  // input width of each GEMM layer

template <class T>
T *P(DevBuf &b) {
  return static_cast<T *>(b.p);
}
template <class T>
const T *P(const DevBuf &b) {
  return static_cast<const T *>(b.p);
}

long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

int ksplit_for(long long n) {
  const long long chunks = cdiv(n, 64);
  long long ks = chunks / 4;
  if (ks < 1) ks = 1;
  if (ks > 256) ks = 256;
  return (int)ks;
}

MlpGemmArgs gemm_args(const winds_mlp *m) {
  MlpGemmArgs g;
  std::memset(&g, 0, sizeof(g));
  g.err = static_cast<unsigned *>(m->err.p);
  g.wait_limit_ns = default_wait_limit_ns();
  return g;
}

int check_err(winds_mlp *m) {
  unsigned word = 0;
  cudaError_t e = cudaMemcpy(&word, m->err.p, sizeof(word), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "mlp error word");
  if (word) {
    cudaMemset(m->err.p, 0, sizeof(unsigned));
    return fail(word & kErrWaitTimeout ? WINDS_BS_ERR_TIMEOUT : WINDS_BS_ERR_CUDA,
                "mlp kernels reported error word 0x%x", word);
  }
  return WINDS_BS_OK;
}

// Backward pass of the rows the last forward (with train) ran on, targets t:
// gradient into m->grad, 0.5 * mean squared error into m->loss.
int mlp_backward(winds_mlp *m, const __nv_bfloat16 *X, const float *t, long long n, MlpWork &w,
                 cudaStream_t s) {
  const float *theta = P<float>(m->theta);
  const __nv_bfloat16 *wbf = P<__nv_bfloat16>(m->theta_bf);
  const int nb_head = (int)cdiv(n, kHeadRows);
  const int nb_rows = (int)cdiv(n, 128);
  const int ks = ksplit_for(n);
  cudaError_t e = launch_mlp_head_bwd(P<float>(w.y), t, P<float>(w.Z[3]), P<__nv_bfloat16>(w.A[3]),
                                      theta + kOffW5, n, (float)(1.0 / (double)n),
                                      P<__nv_bfloat16>(w.dZa), P<float>(w.dw5p),
                                      P<float>(w.part_b[3]), P<float>(w.db5p), P<float>(w.lossp),
                                      kHeadRows, s);
  __nv_bfloat16 *dz = P<__nv_bfloat16>(w.dZa), *dz_next = P<__nv_bfloat16>(w.dZb);
  for (int L = 3; L >= 0 && e == cudaSuccess; --L) {
    // weight gradient: dW_L[out][in] = sum_rows dz[row][out] * a_{L-1}[row][in]
    MlpGemmArgs g = gemm_args(m);
    g.A = dz;
    g.lda = W;
    g.a_mn = 1;
    g.B = L > 0 ? P<__nv_bfloat16>(w.A[L - 1]) : X;
    g.ldb = kInK[L];
    g.b_mn = 1;
    g.M = W;
    g.K = n;
    g.out_f32 = P<float>(w.part_w[L]);
    g.ldo = kInK[L];
    e = launch_mlp_gemm(g, kInK[L], kEpiPartial, ks, s);
    if (L == 0 || e != cudaSuccess) break;
    // input gradient through GELU: dz_{L-1} = (dz W_L) * gelu'(z_{L-1})
    MlpGemmArgs h = gemm_args(m);
    h.A = dz;
    h.lda = W;
    h.a_mn = 0;
    h.B = wbf + kOffW[L];
    h.ldb = W;
    h.b_mn = 1;
    h.M = n;
    h.K = W;
    h.z_in = P<float>(w.Z[L - 1]);
    h.dz_out = dz_next;
    h.colsum_part = P<float>(w.part_b[L - 1]);
    h.ldo = W;
    e = launch_mlp_gemm(h, W, kEpiGeluBwd, 1, s);
    std::swap(dz, dz_next);
  }
  if (e != cudaSuccess) return cuda_fail(e, "mlp backward");
  float *grad = P<float>(m->grad);
  std::vector<MlpReduceJob> jobs;
  for (int L = 0; L < 4; ++L) {
    jobs.push_back({P<float>(w.part_w[L]), ks, W * kInK[L], grad + kOffW[L], 1.f});
    jobs.push_back({P<float>(w.part_b[L]), L == 3 ? nb_head : nb_rows, W, grad + kOffB[L], 1.f});
  }
  jobs.push_back({P<float>(w.dw5p), nb_head, W, grad + kOffW5, 1.f});
  jobs.push_back({P<float>(w.db5p), nb_head, 1, grad + kOffB5, 1.f});
  jobs.push_back({P<float>(w.lossp), nb_head, 1, P<float>(m->loss), (float)(0.5 / (double)n)});
  e = cudaMemcpyAsync(m->jobs.p, jobs.data(), jobs.size() * sizeof(MlpReduceJob),
                      cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_mlp_reduce(P<MlpReduceJob>(m->jobs), (int)jobs.size(), W * W, s);
  // the host vector must outlive the (pageable, staged) copy
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp gradient reduction");
}

int adam_step(winds_mlp *m, const winds_mlp_train_params &p, cudaStream_t s) {
  ++m->adam_t;
  const double c1 = 1.0 - std::pow((double)p.beta1, (double)m->adam_t);
  const double c2 = 1.0 - std::pow((double)p.beta2, (double)m->adam_t);
  cudaError_t e = launch_mlp_adam(P<float>(m->theta), P<__nv_bfloat16>(m->theta_bf),
                                  P<float>(m->grad), P<float>(m->mom), P<float>(m->vel), kNParam,
                                  p.lr, p.beta1, p.beta2, p.eps, p.weight_decay, (float)c1,
                                  (float)c2, s);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp adam");
}

int upload_inputs(winds_mlp *m, const float *x, long long n, MlpWork &w, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(w.xraw.p, x, (size_t)n * m->n_in * sizeof(float),
                                  cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_mlp_prep(P<float>(w.xraw), n, m->n_in, P<float>(m->shift), P<float>(m->scale),
                        P<__nv_bfloat16>(w.X), s);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp input upload");
}

}  // namespace

int MlpWork::ensure(long long n, bool tr, cudaStream_t s) {
  if (n <= cap && (train || !tr)) return WINDS_BS_OK;
  const long long c = n > cap ? n : cap;
  const bool t2 = tr || train;
  int rc;
  if ((rc = X.ensure(c * kMlpInPad * 2, s)) || (rc = t.ensure(c * 4, s)) ||
      (rc = y.ensure(c * 4, s)) || (rc = xraw.ensure(c * 16 * 4, s)))
    return rc;
  for (int L = 0; L < 4; ++L) {
    if ((rc = A[L].ensure(c * W * 2, s))) return rc;
    if (t2 && (rc = Z[L].ensure(c * W * 4, s))) return rc;
  }
  if (t2) {
    const int ks = ksplit_for(c);
    const long long nbh = cdiv(c, kHeadRows), nbr = cdiv(c, 128);
    if ((rc = dZa.ensure(c * W * 2, s)) || (rc = dZb.ensure(c * W * 2, s)) ||
        (rc = dw5p.ensure(nbh * W * 4, s)) || (rc = db5p.ensure(nbh * 4, s)) ||
        (rc = lossp.ensure(nbh * 4, s)))
      return rc;
    for (int L = 0; L < 4; ++L) {
      if ((rc = part_w[L].ensure((size_t)ks * W * kInK[L] * 4, s))) return rc;
      if ((rc = part_b[L].ensure((size_t)(L == 3 ? nbh : nbr) * W * 4, s))) return rc;
    }
  }
  cap = c;
  train = t2;
  return WINDS_BS_OK;
}

void MlpWork::release() {
  for (DevBuf *b : {&X, &t, &y, &dZa, &dZb, &dw5p, &db5p, &lossp, &xraw}) b->release();
  for (int L = 0; L < 4; ++L) {
    Z[L].release();
    A[L].release();
    part_w[L].release();
    part_b[L].release();
  }
  cap = 0;
  train = false;
}

int mlp_forward(const winds_mlp *m, const __nv_bfloat16 *X, long long n, MlpWork &w, float *y,
                cudaStream_t s) {
  if (n <= 0) return WINDS_BS_OK;
  const float *theta = static_cast<const float *>(m->theta.p);
  const __nv_bfloat16 *wbf = static_cast<const __nv_bfloat16 *>(m->theta_bf.p);
  cudaError_t e = cudaSuccess;
  for (int L = 0; L < 4 && e == cudaSuccess; ++L) {
    MlpGemmArgs g = gemm_args(m);
    g.A = L == 0 ? X : P<__nv_bfloat16>(w.A[L - 1]);
    g.lda = kInK[L];
    g.a_mn = 0;
    g.B = wbf + kOffW[L];
    g.ldb = kInK[L];
    g.b_mn = 0;
    g.M = n;
    g.K = kInK[L];
    g.bias = theta + kOffB[L];
    g.z_out = w.train ? P<float>(w.Z[L]) : nullptr;
    g.a_out = P<__nv_bfloat16>(w.A[L]);
    g.ldo = W;
    e = launch_mlp_gemm(g, W, kEpiBiasGelu, 1, s);
  }
  if (e == cudaSuccess)
    e = launch_mlp_head_fwd(P<__nv_bfloat16>(w.A[3]), n, theta + kOffW5, theta + kOffB5, y, s);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp forward");
}

const float *mlp_shift_dev(const winds_mlp *m) { return static_cast<const float *>(m->shift.p); }
const float *mlp_scale_dev(const winds_mlp *m) { return static_cast<const float *>(m->scale.p); }
float mlp_out_scale(const winds_mlp *m) { return m->out_scale; }
// out_scale and the base flag on the device (after the 16 input scales), read
// when a captured step replays
const float *mlp_out_scale_dev(const winds_mlp *m) { return static_cast<const float *>(m->scale.p) + 16; }
const float *mlp_base_dev(const winds_mlp *m) { return static_cast<const float *>(m->scale.p) + 17; }
int mlp_n_in(const winds_mlp *m) { return m->n_in; }
int mlp_device(const winds_mlp *m) { return m->dev; }
unsigned *mlp_err_word(const winds_mlp *m) { return static_cast<unsigned *>(m->err.p); }

}  // namespace winds

using namespace winds;

extern "C" {

int winds_mlp_create(const winds_mlp_config *cfg, winds_mlp **out) {
  if (!cfg || !out || cfg->n_in < 1 || cfg->n_in > kMlpInPad)
    return fail(WINDS_BS_ERR_ARG, "n_in must be 1..16");
  *out = nullptr;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1) return fail(WINDS_BS_ERR_NODEV, "no CUDA device");
  winds_mlp *m = new winds_mlp();
  cudaGetDevice(&m->dev);
  m->n_in = cfg->n_in;
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&m->e0);
  if (e == cudaSuccess) e = cudaEventCreate(&m->e1);
  if (e != cudaSuccess) {
    delete m;
    return cuda_fail(e, "mlp stream");
  }
  cudaStream_t s = m->stream;
  int rc;
  if ((rc = m->theta.ensure(kNParam * 4, s)) || (rc = m->theta_bf.ensure(kNParam * 2, s)) ||
      (rc = m->grad.ensure(kNParam * 4, s)) || (rc = m->mom.ensure(kNParam * 4, s)) ||
      (rc = m->vel.ensure(kNParam * 4, s)) || (rc = m->shift.ensure(64, s)) ||
      (rc = m->scale.ensure(128, s)) || (rc = m->err.ensure(16, s)) ||
      (rc = m->jobs.ensure(32 * sizeof(MlpReduceJob), s)) || (rc = m->loss.ensure(16, s))) {
    winds_mlp_destroy(m);
    return rc;
  }
  // initial weights normal(0, 1/fan_in), biases zero, padded inputs zero
  std::vector<float> th(kNParam, 0.f);
  std::mt19937_64 gen(cfg->seed);
  for (int L = 0; L < 4; ++L) {
    const int fan = L == 0 ? cfg->n_in : W;
    std::normal_distribution<double> nd01(0.0, 1.0 / std::sqrt((double)fan));
    for (int o = 0; o < W; ++o)
      for (int i = 0; i < fan; ++i) th[kOffW[L] + (long long)o * kInK[L] + i] = (float)nd01(gen);
  }
  std::normal_distribution<double> nd5(0.0, 1.0 / std::sqrt((double)W));
  for (int j = 0; j < W; ++j) th[kOffW5 + j] = (float)nd5(gen);
  for (int i = 0; i < 16; ++i) m->h_shift[i] = 0.f, m->h_scale[i] = 1.f;
  e = cudaMemcpy(m->theta.p, th.data(), kNParam * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m->shift.p, m->h_shift, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m->scale.p, m->h_scale, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(P<float>(m->scale) + 16, &m->out_scale, 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(P<float>(m->scale) + 17, 0, 4);  // base 0
  if (e == cudaSuccess) e = cudaMemset(m->mom.p, 0, kNParam * 4);
  if (e == cudaSuccess) e = cudaMemset(m->vel.p, 0, kNParam * 4);
  if (e == cudaSuccess) e = cudaMemset(m->err.p, 0, 16);
  if (e == cudaSuccess) e = launch_mlp_to_bf16(P<float>(m->theta), P<__nv_bfloat16>(m->theta_bf), kNParam, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    winds_mlp_destroy(m);
    return cuda_fail(e, "mlp init");
  }
  *out = m;
  return WINDS_BS_OK;
}

long long winds_mlp_param_count(const winds_mlp *m) { return m ? kNParam : 0; }

int winds_mlp_get_params(winds_mlp *m, float *theta) {
  if (!m || !theta) return fail(WINDS_BS_ERR_ARG, "null argument");
  cudaSetDevice(m->dev);
  cudaStreamSynchronize(m->stream);
  cudaError_t e = cudaMemcpy(theta, m->theta.p, kNParam * 4, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp params");
}

int winds_mlp_set_params(winds_mlp *m, const float *theta) {
  if (!m || !theta) return fail(WINDS_BS_ERR_ARG, "null argument");
  cudaSetDevice(m->dev);
  cudaStreamSynchronize(m->stream);
  std::vector<float> th(theta, theta + kNParam);
  for (int o = 0; o < W; ++o)  // padded inputs of layer 1 stay zero
    for (int i = m->n_in; i < kMlpInPad; ++i) th[kOffW[0] + (long long)o * kMlpInPad + i] = 0.f;
  cudaError_t e = cudaMemcpy(m->theta.p, th.data(), kNParam * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = launch_mlp_to_bf16(P<float>(m->theta), P<__nv_bfloat16>(m->theta_bf), kNParam, m->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->mom.p, 0, kNParam * 4, m->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->vel.p, 0, kNParam * 4, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  m->adam_t = 0;
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp params");
}

int winds_mlp_set_scaling(winds_mlp *m, const float *shift, const float *scale, float out_scale) {
  if (!m || !shift || !scale || !std::isfinite(out_scale))
    return fail(WINDS_BS_ERR_ARG, "bad scaling");
  cudaSetDevice(m->dev);
  for (int i = 0; i < 16; ++i) {
    m->h_shift[i] = i < m->n_in ? shift[i] : 0.f;
    m->h_scale[i] = i < m->n_in ? scale[i] : 1.f;
  }
  m->out_scale = out_scale;
  cudaStreamSynchronize(m->stream);
  cudaError_t e = cudaMemcpy(m->shift.p, m->h_shift, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(m->scale.p, m->h_scale, 64, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(P<float>(m->scale) + 16, &out_scale, 4, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "mlp scaling");
}

int winds_mlp_set_base(winds_mlp *m, int base) {
  if (!m || (base != WINDS_MLP_BASE_PREVIOUS && base != WINDS_MLP_BASE_EXTRAPOLATED))
    return fail(WINDS_BS_ERR_ARG, "bad start-value base %d", base);
  cudaSetDevice(m->dev);
  cudaStreamSynchronize(m->stream);
  const float f = (float)base;
  cudaError_t e = cudaMemcpy(P<float>(m->scale) + 17, &f, 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "mlp base");
  m->base = base;
  return WINDS_BS_OK;
}

int winds_mlp_get_base(const winds_mlp *m) { return m ? m->base : -1; }

int winds_mlp_get_scaling(winds_mlp *m, float *shift, float *scale, float *out_scale) {
  if (!m) return fail(WINDS_BS_ERR_ARG, "null model");
  for (int i = 0; i < m->n_in; ++i) {
    if (shift) shift[i] = m->h_shift[i];
    if (scale) scale[i] = m->h_scale[i];
  }
  if (out_scale) *out_scale = m->out_scale;
  return WINDS_BS_OK;
}

int winds_mlp_forward_host(winds_mlp *m, const float *x, long long n, float *y) {
  if (!m || n < 0 || (n > 0 && (!x || !y))) return fail(WINDS_BS_ERR_ARG, "bad arguments");
  if (n == 0) return WINDS_BS_OK;
  cudaSetDevice(m->dev);
  cudaStream_t s = m->stream;
  const long long chunk = 1 << 16;
  for (long long r0 = 0; r0 < n; r0 += chunk) {
    const long long k = n - r0 < chunk ? n - r0 : chunk;
    int rc = m->w.ensure(k, false, s);
    if (!rc) rc = upload_inputs(m, x + r0 * m->n_in, k, m->w, s);
    if (!rc) rc = mlp_forward(m, P<__nv_bfloat16>(m->w.X), k, m->w, P<float>(m->w.y), s);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(y + r0, m->w.y.p, k * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "mlp forward");
  }
  return check_err(m);
}

int winds_mlp_loss_grad_host(winds_mlp *m, const float *x, const float *t, long long n,
                             double *loss, float *grad) {
  if (!m || n < 1 || !x || !t) return fail(WINDS_BS_ERR_ARG, "bad arguments");
  cudaSetDevice(m->dev);
  cudaStream_t s = m->stream;
  int rc = m->w.ensure(n, true, s);
  if (!rc) rc = upload_inputs(m, x, n, m->w, s);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(m->w.t.p, t, n * 4, cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "mlp targets");
  if ((rc = mlp_forward(m, P<__nv_bfloat16>(m->w.X), n, m->w, P<float>(m->w.y), s))) return rc;
  if ((rc = mlp_backward(m, P<__nv_bfloat16>(m->w.X), P<float>(m->w.t), n, m->w, s))) return rc;
  float l = 0.f;
  e = cudaMemcpy(&l, m->loss.p, 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && grad) e = cudaMemcpy(grad, m->grad.p, kNParam * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "mlp gradient read");
  if (loss) *loss = l;
  return check_err(m);
}

int winds_mlp_train_host(winds_mlp *m, const float *x, const float *t, long long n,
                         const winds_mlp_train_params *p, float *epoch_loss) {
  if (!m || !p || n < 1 || !x || !t || p->epochs < 0 || p->batch < 1 || !(p->lr > 0))
    return fail(WINDS_BS_ERR_ARG, "bad training arguments");
  cudaSetDevice(m->dev);
  cudaStream_t s = m->stream;
  const long long B = p->batch < n ? p->batch : n;
  const long long nbatch = cdiv(n, B);
  int rc;
  if ((rc = m->xall_raw.ensure(n * m->n_in * 4, s)) || (rc = m->Xall.ensure(n * kMlpInPad * 2, s)) ||
      (rc = m->Tall.ensure(n * 4, s)) || (rc = m->idx.ensure(n * 4, s)) ||
      (rc = m->lossbuf.ensure(nbatch * 4, s)) || (rc = m->w.ensure(B, true, s)))
    return rc;
  cudaError_t e = cudaMemcpyAsync(m->xall_raw.p, x, n * m->n_in * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(m->Tall.p, t, n * 4, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_mlp_prep(P<float>(m->xall_raw), n, m->n_in, P<float>(m->shift), P<float>(m->scale),
                        P<__nv_bfloat16>(m->Xall), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "mlp training upload");
  std::vector<int> perm(n);
  for (long long i = 0; i < n; ++i) perm[i] = (int)i;
  std::mt19937_64 gen(p->seed);
  std::vector<float> bl(nbatch);
  m->train_steps = 0;
  float total_ms = 0.f;
  for (int ep = 0; ep < p->epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), gen);
    e = cudaMemcpy(m->idx.p, perm.data(), n * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "mlp shuffle upload");
    cudaEventRecord(m->e0, s);
    for (long long b = 0; b < nbatch; ++b) {
      const long long r0 = b * B, nb = n - r0 < B ? n - r0 : B;
      e = launch_mlp_gather(P<__nv_bfloat16>(m->Xall), P<float>(m->Tall), P<int>(m->idx) + r0, nb,
                            P<__nv_bfloat16>(m->w.X), P<float>(m->w.t), s);
      if (e != cudaSuccess) return cuda_fail(e, "mlp gather");
      if ((rc = mlp_forward(m, P<__nv_bfloat16>(m->w.X), nb, m->w, P<float>(m->w.y), s))) return rc;
      if ((rc = mlp_backward(m, P<__nv_bfloat16>(m->w.X), P<float>(m->w.t), nb, m->w, s))) return rc;
      e = cudaMemcpyAsync(P<float>(m->lossbuf) + b, m->loss.p, 4, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_fail(e, "mlp loss copy");
      if ((rc = adam_step(m, *p, s))) return rc;
      ++m->train_steps;
    }
    cudaEventRecord(m->e1, s);
    e = cudaMemcpyAsync(bl.data(), m->lossbuf.p, nbatch * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "mlp epoch");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, m->e0, m->e1);
    total_ms += ms;
    if (epoch_loss) {
      double acc = 0.0;
      for (long long b = 0; b < nbatch; ++b) {
        const long long nb = n - b * B < B ? n - b * B : B;
        acc += (double)bl[b] * (double)nb;
      }
      epoch_loss[ep] = (float)(acc / (double)n);
    }
    if ((rc = check_err(m))) return rc;
  }
  m->train_ms = total_ms;
  return WINDS_BS_OK;
}

int winds_mlp_train_stats(winds_mlp *m, double *ms, long long *steps) {
  if (!m) return fail(WINDS_BS_ERR_ARG, "null model");
  if (ms) *ms = m->train_ms;
  if (steps) *steps = m->train_steps;
  return WINDS_BS_OK;
}

void winds_mlp_destroy(winds_mlp *m) {
  if (!m) return;
  cudaSetDevice(m->dev);
  if (m->stream) cudaStreamSynchronize(m->stream);
  m->w.release();
  for (DevBuf *b : {&m->theta, &m->theta_bf, &m->grad, &m->mom, &m->vel, &m->shift, &m->scale,
                    &m->err, &m->jobs, &m->loss, &m->lossbuf, &m->idx, &m->Xall, &m->Tall,
                    &m->xall_raw})
    b->release();
  if (m->e0) cudaEventDestroy(m->e0);
  if (m->e1) cudaEventDestroy(m->e1);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}

}  // extern "C"
