// engine.h -- internal host-side types of libwinds_bs (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "bs_types.h"
#include "winds_bs.h"

namespace winds {

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes, cudaStream_t s);  // grows (after a stream sync); keeps no contents
  void release();
};

struct HostBuf {  // pinned
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes);
  void release();
};

struct TargetSpec {
  const double *P;  // device, MATLAB layout [ns, 3, ...]
  long long ns;
  long long count;
  double *out;      // device, P's layout
  int accumulate;
};

struct GroupSpec {
  double *out;
  long long t_begin, t_count, ns_p;
  int f_begin, f_end;
  int accumulate;
};

struct Plan {
  int tile_cap = 0;
  std::vector<Group> groups;
  std::vector<Tile> tiles;
  std::vector<Item> items;
  std::vector<int> order;  // work queue: queue position -> item
};

struct TuneChoice {
  int T = 4;
  int KF = 64;
  double waves = 8.0;
  bool chain = false;  // FP32c on the chained filament stream (evaluation entry points)
};

struct Context {
  int dev = 0;
  int num_sms = 0;
  int cc_major = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_main0 = nullptr, ev_main1 = nullptr, ev_upload = nullptr;
  // packed inputs; targets sorted (tp) from their packed order (tp_raw)
  DevBuf pk, ra, rb, tp, tp_raw, tgroup, keys, vals, perm, sort_tmp;
  // plan tables and partial sums
  DevBuf groups, tiles, items, order, part;
  // small words
  DevBuf bbox, ctr, err, nearctr;
  // chained filament stream (FP32c path): head bit per pair record, and the
  // per-family link counts that choose each family's layout
  DevBuf heads, chaincnt;
  bool chained = false;  // the packed filaments are a chained stream
  // device copies of host inputs/outputs (host API)
  DevBuf in_P, in_F, out_u;
  HostBuf htab, hstat;
  Plan plan;
  // what the uploaded plan was built from: a call with the same groups and
  // tiling reuses it (no host rebuild, no upload)
  std::vector<GroupSpec> plan_gs;
  int plan_tile_cap = -1, plan_resident = -1, plan_quantum = -1;
  double plan_waves = -1.0;
  int launches = 0;
  bool timed = false;
  bool autotune = true;
};

int fail(int code, const char *fmt, ...);
void build_plan(Plan &pl, const std::vector<GroupSpec> &gs, int tile_cap, int resident,
                double waves, int chunk_quantum);
int resolve_model(const winds_bs_params *prm, int *model, double *dcut, double *n, int *prec);
int validate_family(const winds_bs_family &f);
TuneChoice default_choice(long long nt);
// Tuned tilings per (model, log2 targets, log2 filaments) bucket, apart for
// the evaluation entry points (eval = true: their choice includes the stream
// layout) and the callers that pack their own unchained stream.
bool lookup_tune(int model, long long nt, long long nf, TuneChoice *out, bool eval = false);
void store_tune(int model, long long nt, long long nf, const TuneChoice &ch, bool eval = false);
int cuda_fail(cudaError_t e, const char *what);
Context *get_context(int *rc);
int eval_device(Context *c, const winds_bs_family *fams, int nfam,
                const std::vector<TargetSpec> &tsets, const winds_bs_params *prm, cudaStream_t s,
                bool sequential);
int autotune(Context *c, const std::vector<GroupSpec> &gs, int model, double dcut, double n,
             double co, TuneChoice *best, float *best_ms);
int check_device_error(Context *c, cudaStream_t s);

}  // namespace winds
