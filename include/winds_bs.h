/*
 * winds_bs.h -- C ABI of libwinds_bs, the sm_100a induced-velocity engine that
 * replaces WInDS's Biot-Savart hot path.
 *
 * Every entry point takes plain pointers and sizes. Arrays keep WInDS's MATLAB
 * layout: column-major doubles shaped [span, component, age, blade].
 *
 * What each entry point replaces in the reference (ndevelder/WInDS-Master):
 *   winds_bs_eval_host    core/BiotSavart.m:1-119 (the [uind,L]=BiotSavart(...)
 *                         'full' call) and cuda/source/BiotSavartMex.cu:452-685
 *                         (biot_calc: pack, copy in, kernel, copy out).
 *   winds_bs_eval_device  the same evaluation on device-resident arrays
 *                         (cuda/source/BiotSavartMex.cu:131-193, the
 *                         BiotSavart_naive / BiotSavart_sh kernels).
 *   winds_bs_length_*     core/FilamentLength.m:27-44 and the 'leng' branch of
 *                         cuda/source/BiotSavartMex.cu:197-206,582-587.
 *   mexFunction           cuda/source/BiotSavartMex.cu:688-807, the 11-argument
 *                         [uind,L]=BiotSavartMex(F1,F2,P,gamma,rc,d,cmod,co,
 *                         type,gpu,gpuhw) contract.
 *
 * All functions return WINDS_BS_OK (0) or a positive WINDS_BS_ERR_* code; the
 * message of the last failure on the calling thread is available from
 * winds_bs_last_error(). Nothing prints.
 */
#ifndef WINDS_BS_H
#define WINDS_BS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WINDS_BS_OK 0
#define WINDS_BS_ERR_ARG 1      /* bad shape, pointer or option */
#define WINDS_BS_ERR_CUDA 2     /* a CUDA runtime call failed */
#define WINDS_BS_ERR_TIMEOUT 3  /* a bounded device wait ran out; context stays usable */
#define WINDS_BS_ERR_NOMEM 4    /* device or pinned allocation failed */
#define WINDS_BS_ERR_NODEV 5    /* no CUDA device, or the library was built without one */
#define WINDS_BS_ERR_DIVERGED 6 /* Kutta-Joukowski: Cl is NaN (KuttaJoukowski.m:272-274) */

/* Core models of core/BiotSavart.m:102-109. */
#define WINDS_CORE_CUTOFF 0   /* ubar = G/4pi (r1+r2)/(r1r2(r1r2+r1.r2) + d|L|^2)      (:108) */
#define WINDS_CORE_VATISTAS 1 /* ubar scaled by Cnu = h^2 (rc^n + h^2n)^(-1/n), n = d  (:103-106) */

/* Arithmetic of the direct sum. */
#define WINDS_PREC_F32C 0 /* FP32 tiles + per-target Kahan, FP64 near-singular terms (default) */
#define WINDS_PREC_F64 1  /* plain FP64 direct sum (the comparison GPU path) */

/* One filament family, e.g. the shed call F1=dom(1:end-1,:,:,:),
 * F2=dom(2:end,:,:,:) of WInDS.m:150 or the trailing call of WInDS.m:153. */
typedef struct {
  const double *F1;    /* [dims0, 3, dims2, dims3] first endpoints            */
  const double *F2;    /* [dims0, 3, dims2, dims3] second endpoints           */
  const double *gamma; /* [dims0, 1, dims2, dims3] circulation                */
  const double *rc;    /* [dims0, 1, dims2, dims3] squared core radius (rc^2) */
  long long dims[4];   /* dims[1] must be 3 */
} winds_bs_family;

/* Flags of winds_bs_params.flags. */
#define WINDS_BS_FLAG_SEQUENTIAL 1 /* FP64: one pass per target over all filaments in order
                                      (reproduces the reference's serial host loop,
                                      BiotSavartMex.cu:268-282, bit for bit, cut-off model) */

typedef struct {
  int core_model; /* WINDS_CORE_* */
  double d;       /* cut-off: squared cut-off (user.d); Vatistas: index n */
  double co;      /* reach cut-off: a term is zero when r1>co and r2>co (BiotSavart.m:111) */
  int precision;  /* WINDS_PREC_* ; Vatistas n != 2 and non-finite or negative d use FP64 */
  int flags;      /* WINDS_BS_FLAG_* */
} winds_bs_params;

/* Library version string. */
const char *winds_bs_version(void);

/* Message of the last failure on this thread ("" if none). */
const char *winds_bs_last_error(void);

/* Number of visible CUDA devices (0 on a machine without a GPU). */
int winds_bs_device_count(int *n);

/* Select the device later calls on this thread use (gpuhw(3) of the MEX). */
int winds_bs_set_device(int device);

/* Induced velocity at every point of P from every filament of fams[0..nfam).
 * Device pointers. P is [pdims0, 3, pdims2, pdims3] (a 2-D or 3-D P is passed
 * with trailing dims 1); uind has P's layout and is overwritten. stream is a
 * cudaStream_t (NULL: the library's own stream); the call is asynchronous on
 * it except that it waits for completion when it must report a device error.
 * Replaces core/BiotSavart.m:80-116 / cuda/source/BiotSavartMex.cu:131-193. */
int winds_bs_eval_device(const winds_bs_family *fams, int nfam, const double *P,
                         const long long pdims[4], const winds_bs_params *prm,
                         double *uind, void *stream);

/* Same evaluation from host arrays: copies in, evaluates, copies uind out and
 * synchronises. Replaces cuda/source/BiotSavartMex.cu:452-685 (biot_calc). */
int winds_bs_eval_host(const winds_bs_family *fams, int nfam, const double *P,
                       const long long pdims[4], const winds_bs_params *prm,
                       double *uind);

/* The same evaluation as winds_bs_eval_device for callers that must not
 * allocate device memory. No counterpart in the reference: it exists because
 * winds_bs_eval_device grows its buffers with cudaMalloc, which a host that
 * owns all device memory through its own pool cannot allow and which, by
 * synchronising the device, stalls a solver that calls the engine every step.
 * All scratch lives in one static __device__ array of
 * WINDS_BS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds
 * until exit. Inputs and outputs are those of winds_bs_eval_device (device
 * pointers), with two differences: the work runs on the calling thread's
 * current CUDA device (winds_bs_eval_device uses the device chosen by
 * winds_bs_set_device, which also makes it current on that thread), and a
 * NULL stream is the legacy default stream (winds_bs_eval_device: the
 * library's own stream). Limits: at most WINDS_BS_NOALLOC_MAX_FILAMENTS
 * filaments and WINDS_BS_NOALLOC_MAX_TARGETS targets per call
 * (WINDS_BS_ERR_ARG beyond). The call waits for its stream and reports
 * device-side errors. Every call looks up the array's device address (a
 * host-side lookup); the first call on a device also loads the library's
 * device code, which commits the array's memory: make that first call before
 * any stream capture. Calls share the array: calls that overlap on the GPU
 * race. */
#define WINDS_BS_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define WINDS_BS_NOALLOC_MAX_FILAMENTS 131072
#define WINDS_BS_NOALLOC_MAX_TARGETS 65536
int winds_bs_eval_device_noalloc(const winds_bs_family *fams, int nfam, const double *P,
                                 const long long pdims[4], const winds_bs_params *prm,
                                 double *uind, void *stream);

/* Filament lengths sqrt(|F2-F1|^2), MATLAB layout [dims0,1,dims2,dims3].
 * Replaces core/FilamentLength.m:27-44. Device pointers. */
int winds_bs_length_device(const double *F1, const double *F2, const long long dims[4],
                           double *L, void *stream);

/* Wall-free timing hook for benchmarks: device time in ms of the last
 * winds_bs_eval_* call's main direct-sum kernel(s), measured with CUDA events
 * on the launch stream; also reports how many kernels that call launched and
 * how many near-singular pairs its FP32c direct sum recomputed in FP64 (0 for
 * the FP64 path). */
int winds_bs_last_stats(double *main_ms, int *launches, long long *near_pairs);

/* How many pairs of the last winds_bs_eval_host / winds_bs_eval_device call's
 * FP32c direct sum took the core-free form, where leaving the core out
 * changes the pair term by less than FP32's unit roundoff 2^-24 (one-sided):
 * Vatistas, targets at least 54 core radii from the filament's line (the
 * factor 1/sqrt(1 + (rc/h)^4) is within 5.9e-8 of 1); cut-off, targets at
 * least r from the segment with r^4 >= 2^24 d |L|^2. A screen of 32
 * filaments against a warp's targets decides. 0 for the FP64 path. */
int winds_bs_last_core_free(long long *pairs);

/* 1 when the last winds_bs_eval_host / winds_bs_eval_device call's FP32c
 * direct sum ran on the chained filament stream, else 0. The chained stream
 * lays each line of connected filaments (the shed call's along the span, the
 * trailing call's along the wake age: BiotSavart calls of WInDS.m:150,153)
 * along one lane of consecutive pair records, so that each interaction takes
 * its second endpoint's inverse distance from the previous filament's first
 * one (one rsqrt fewer); the autotuner picks it or the input order per size
 * bucket together with the tiling (no reference counterpart: the reference's
 * kernel evaluates every filament on its own, BiotSavartMex.cu:131-193). */
int winds_bs_last_chained(int *chained);

/* Synchronises `stream` (NULL: the library's stream) and reports a device-side
 * error (WINDS_BS_ERR_TIMEOUT for a bounded wait that ran out) recorded by an
 * earlier asynchronous call; the error word is cleared. */
int winds_bs_sync(void *stream);

/* Autotuner control. The first FP32 evaluation of a (core model, log2 targets,
 * log2 filaments) bucket on the library's own stream times the candidate
 * tilings (targets per thread T in {2,3,4}, filaments per tile KF in {32,64,128},
 * work-queue depth: items per resident warp) on both filament stream layouts
 * (input order and chained) and caches the fastest tiling and layout (T = 8
 * is settable). Evaluations on another stream, or with the autotuner off, use
 * the cached choice or the untuned default (T = 4, or 2 below 2048 targets;
 * KF = 64; input order).
 * set_tuning / get_tuning read and write that cache directly (e.g. to restore
 * a saved choice). */
int winds_bs_set_autotune(int on);
int winds_bs_set_tuning(int core_model, long long n_targets, long long n_filaments, int T, int KF,
                        double waves);
int winds_bs_get_tuning(int core_model, long long n_targets, long long n_filaments, int *T,
                        int *KF, double *waves);
/* Sets the FP32c evaluations' stream layout of a bucket (1: chained, 0: input
 * order; see winds_bs_last_chained), keeping its tiling (the untuned default
 * when the bucket has none); set_tuning resets the bucket to input order. */
int winds_bs_set_layout(int core_model, long long n_targets, long long n_filaments, int chained);

/* Measured FP32 FMA throughput of this GPU in TFLOP/s (a ~0.1 s probe of
 * independent FFMA chains): the roofline denominator of the direct sum. */
int winds_bs_fp32_peak(double *tflops);

/* Failure-detection self-test: launches a kernel whose bounded mbarrier wait
 * (limit_ns) has no producer, so it must run out. Returns WINDS_BS_ERR_TIMEOUT
 * when the timeout was detected and reported; the context stays usable. */
int winds_bs_selftest_wait_timeout(unsigned long long limit_ns);

/* Frees every device buffer, stream and event of every device context
 * (the mexAtExit hook of the MEX layer). */
void winds_bs_shutdown(void);

#ifdef __cplusplus
}
#endif

#endif /* WINDS_BS_H */
