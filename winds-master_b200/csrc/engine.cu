// engine.cu -- host side of libwinds_bs: per-device contexts (stream, events,
// grow-only HBM buffers that persist across calls), work planning for the
// persistent direct-sum kernels, the autotuner, and the C ABI of winds_bs.h.
//
// The reference allocates, copies and frees every device buffer on every call
// (cuda/source/BiotSavartMex.cu:538-575,655-665) and packs on the host
// (:523-526). Here inputs are copied once in MATLAB layout and packed on the
// device; buffers are reused by the next call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "bs_launch.h"
#include "engine.h"
#include "winds_bs.h"

namespace winds {

// ------------------------------------------------------------- error state
static thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? WINDS_BS_ERR_NOMEM : WINDS_BS_ERR_CUDA,
              "%s: %s", what, cudaGetErrorString(e));
}

const char *last_error() { return g_last_error.c_str(); }

// ------------------------------------------------------------- buffers
int DevBuf::ensure(size_t bytes, cudaStream_t s) {
  if (bytes <= cap) return WINDS_BS_OK;
  if (p) {
    // the old buffer may still be read on any stream of this device
    (void)s;
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "sync before buffer growth");
    cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  size_t want = bytes + bytes / 4 + 256;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    return cuda_fail(e, "cudaMalloc");
  }
  cap = want;
  return WINDS_BS_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

int HostBuf::ensure(size_t bytes) {
  if (bytes <= cap) return WINDS_BS_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  size_t want = bytes + bytes / 4 + 256;
  cudaError_t e = cudaMallocHost(&p, want);
  if (e != cudaSuccess) {
    p = nullptr;
    return cuda_fail(e, "cudaMallocHost");
  }
  cap = want;
  return WINDS_BS_OK;
}

void HostBuf::release() {
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
}

// ------------------------------------------------------------- contexts
static std::mutex g_ctx_mu;
static std::map<int, Context *> g_ctx;
static thread_local int g_device = -1;

Context *get_context(int *rc) {
  int dev = g_device;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  }
  std::lock_guard<std::mutex> g(g_ctx_mu);
  auto it = g_ctx.find(dev);
  if (it != g_ctx.end()) {
    cudaSetDevice(dev);
    *rc = WINDS_BS_OK;
    return it->second;
  }
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    *rc = fail(WINDS_BS_ERR_NODEV, "no CUDA device is visible");
    return nullptr;
  }
  if (dev >= n) {
    *rc = fail(WINDS_BS_ERR_ARG, "device %d requested, %d visible", dev, n);
    return nullptr;
  }
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    *rc = cuda_fail(e, "cudaSetDevice");
    return nullptr;
  }
  Context *c = new Context();
  c->dev = dev;
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  c->num_sms = prop.multiProcessorCount;
  c->cc_major = prop.major;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&c->ev_main0)) != cudaSuccess ||
      (e = cudaEventCreate(&c->ev_main1)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&c->ev_upload, cudaEventDisableTiming)) != cudaSuccess) {
    *rc = cuda_fail(e, "stream/event creation");
    delete c;
    return nullptr;
  }
  // small fixed buffers: bbox, counters, error word, near-pair counter
  if ((*rc = c->bbox.ensure(sizeof(BBox), c->stream)) ||
      (*rc = c->ctr.ensure(64 * sizeof(unsigned), c->stream)) ||
      (*rc = c->err.ensure(sizeof(unsigned), c->stream)) ||
      (*rc = c->nearctr.ensure(2 * sizeof(unsigned long long), c->stream)) ||
      (*rc = c->hstat.ensure(64))) {
    delete c;
    return nullptr;
  }
  cudaMemsetAsync(c->err.p, 0, sizeof(unsigned), c->stream);
  cudaMemsetAsync(c->nearctr.p, 0, 2 * sizeof(unsigned long long), c->stream);
  g_ctx[dev] = c;
  *rc = WINDS_BS_OK;
  return c;
}

void shutdown_all() {
  std::lock_guard<std::mutex> g(g_ctx_mu);
  for (auto &kv : g_ctx) {
    Context *c = kv.second;
    cudaSetDevice(c->dev);
    cudaStreamSynchronize(c->stream);
    for (DevBuf *b : {&c->pk, &c->ra, &c->rb, &c->tp, &c->tp_raw,
                      &c->tgroup, &c->keys, &c->vals, &c->perm, &c->sort_tmp, &c->groups,
                      &c->tiles, &c->items, &c->order, &c->part, &c->bbox, &c->ctr, &c->err,
                      &c->nearctr,
                      &c->in_P, &c->in_F, &c->out_u})
      b->release();
    c->htab.release();
    c->hstat.release();
    cudaEventDestroy(c->ev_main0);
    cudaEventDestroy(c->ev_main1);
    cudaEventDestroy(c->ev_upload);
    cudaStreamDestroy(c->stream);
    delete c;
  }
  g_ctx.clear();
}

// ------------------------------------------------------------- planning
static long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

// Splits each group into tiles of tile_cap targets and each tile's filament
// range into chunks, aiming at `waves` rounds of the resident workers so the
// persistent kernel's work queue stays balanced. The last part of every
// tile's range (a fraction min(1/4, 2/waves) of the work) is cut into
// quarter-size chunks that the queue hands out after all full-size ones, so
// the workers finish together (guided scheduling). Items stay tile-major in
// `items` (the reduce sums a tile's partials in filament order); `order`
// is the queue: queue position -> item.
void build_plan(Plan &pl, const std::vector<GroupSpec> &gs, int tile_cap, int resident,
                double waves, int chunk_quantum) {
  pl.tile_cap = tile_cap;
  pl.groups.clear();
  pl.tiles.clear();
  pl.items.clear();
  pl.order.clear();
  std::vector<int> tail_items;
  double total_work = 0.0;
  long long total_tiles = 0;
  for (const GroupSpec &g : gs) {
    long long nt = (g.t_count + tile_cap - 1) / tile_cap;
    total_tiles += nt;
    total_work += (double)nt * (double)(g.f_end - g.f_begin);
  }
  const double want_items = std::max((double)resident * waves, (double)total_tiles);
  long long chunk = (long long)std::ceil(total_work / want_items);
  chunk = std::max<long long>(round_up(std::max<long long>(chunk, 1), chunk_quantum),
                              chunk_quantum);
  const long long tail_chunk = round_up(std::max<long long>(chunk / 4, 1), chunk_quantum);
  const double tail_frac = waves > 0.0 && tail_chunk < chunk ? std::min(0.25, 2.0 / waves) : 0.0;
  for (size_t gi = 0; gi < gs.size(); ++gi) {
    const GroupSpec &g = gs[gi];
    Group G;
    G.out = g.out;
    G.t_begin = g.t_begin;
    G.t_count = g.t_count;
    G.ns_p = g.ns_p;
    G.f_begin = g.f_begin;
    G.f_end = g.f_end;
    G.accumulate = g.accumulate;
    G.pad = 0;
    pl.groups.push_back(G);
    if (g.t_count <= 0) continue;
    for (long long t0 = 0; t0 < g.t_count; t0 += tile_cap) {
      Tile T;
      T.t_begin = g.t_begin + t0;
      T.t_count = (int)std::min<long long>(tile_cap, g.t_count - t0);
      T.group = (int)gi;
      T.first_item = (int)pl.items.size();
      T.n_items = 0;
      const long long range = (long long)g.f_end - g.f_begin;
      const long long tail = (long long)(tail_frac * (double)range) / tail_chunk * tail_chunk;
      const long long f_mid = g.f_end - tail;
      for (long long f0 = g.f_begin; f0 < g.f_end;) {
        const bool in_tail = f0 >= f_mid;
        const long long f1 = std::min<long long>(f0 + (in_tail ? tail_chunk : chunk),
                                                 in_tail ? g.f_end : f_mid);
        Item I;
        I.tile = (int)pl.tiles.size();
        I.f_begin = (int)f0;
        I.f_end = (int)f1;
        I.pad = 0;
        (in_tail ? tail_items : pl.order).push_back((int)pl.items.size());
        pl.items.push_back(I);
        ++T.n_items;
        f0 = f1;
      }
      if (T.n_items == 0) {  // empty filament range: one empty item writes zeros
        Item I;
        I.tile = (int)pl.tiles.size();
        I.f_begin = I.f_end = g.f_begin;
        I.pad = 0;
        pl.order.push_back((int)pl.items.size());
        pl.items.push_back(I);
        T.n_items = 1;
      }
      pl.tiles.push_back(T);
    }
  }
  pl.order.insert(pl.order.end(), tail_items.begin(), tail_items.end());
}

int upload_plan(Context *c, const Plan &pl, cudaStream_t s) {
  const size_t gb = pl.groups.size() * sizeof(Group);
  const size_t tb = pl.tiles.size() * sizeof(Tile);
  const size_t ib = pl.items.size() * sizeof(Item);
  const size_t ob = pl.order.size() * sizeof(int);
  int rc;
  if ((rc = c->groups.ensure(gb + 16, s)) || (rc = c->tiles.ensure(tb + 16, s)) ||
      (rc = c->items.ensure(ib + 16, s)) || (rc = c->order.ensure(ob + 16, s)))
    return rc;
  // the pinned staging may still feed the previous upload
  cudaEventSynchronize(c->ev_upload);
  if ((rc = c->htab.ensure(gb + tb + ib + ob + 64))) return rc;
  char *h = static_cast<char *>(c->htab.p);
  std::memcpy(h, pl.groups.data(), gb);
  std::memcpy(h + gb, pl.tiles.data(), tb);
  std::memcpy(h + gb + tb, pl.items.data(), ib);
  std::memcpy(h + gb + tb + ib, pl.order.data(), ob);
  cudaError_t e;
  if ((e = cudaMemcpyAsync(c->groups.p, h, gb, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(c->tiles.p, h + gb, tb, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(c->items.p, h + gb + tb, ib, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(c->order.p, h + gb + tb + ib, ob, cudaMemcpyHostToDevice, s)) !=
          cudaSuccess)
    return cuda_fail(e, "plan upload");
  cudaEventRecord(c->ev_upload, s);
  return WINDS_BS_OK;
}

// ------------------------------------------------------------- packing
// chain: lay the filaments out as a chained stream (the FP32c kernel's
// faster form; bs_pack_chains), else in input order.
int pack_inputs(Context *c, const winds_bs_family *fams, int nfam,
                const std::vector<TargetSpec> &tsets, int model, double dcut, cudaStream_t s,
                long long *nf_real, long long *nf_pad, long long *nt_total, bool chain) {
  long long nf = 0, nrec = 0;
  for (int k = 0; k < nfam; ++k) {
    const long long *d = fams[k].dims;
    nf += d[0] * d[2] * d[3];
    nrec += chain_records(d[0], d[2], d[3]);
  }
  const long long nfp =
      std::max<long long>(round_up(chain ? 2 * nrec : nf, kFilamentPad), kFilamentPad);
  long long nt = 0;
  for (const TargetSpec &t : tsets) nt += t.count;
  int rc;
  if ((rc = c->pk.ensure(nfp * 4 * sizeof(float4), s)) ||
      (rc = c->ra.ensure(nfp * sizeof(double4), s)) ||
      (rc = c->rb.ensure(nfp * sizeof(double4), s)) ||
      (rc = c->tp.ensure(std::max<long long>(nt, 1) * sizeof(double4), s)) ||
      (rc = c->tp_raw.ensure(std::max<long long>(nt, 1) * sizeof(double4), s)) ||
      (rc = c->tgroup.ensure(std::max<long long>(nt, 1) * sizeof(int), s)) ||
      (rc = c->keys.ensure(std::max<long long>(nt, 1) * 2 * sizeof(unsigned long long), s)) ||
      (rc = c->vals.ensure(std::max<long long>(nt, 1) * sizeof(int), s)) ||
      (rc = c->perm.ensure(std::max<long long>(nt, 1) * sizeof(int), s)))
    return rc;
  if (chain && ((rc = c->heads.ensure((nfp / 64 + 1) * sizeof(unsigned), s)) ||
                (rc = c->chaincnt.ensure(std::max(nfam, 1) * 2 * sizeof(unsigned long long), s))))
    return rc;
  size_t sort_bytes = 0;
  if (sort_target_keys(nullptr, &sort_bytes, nullptr, nullptr, nullptr, nullptr, nt, s) !=
      cudaSuccess)
    return fail(WINDS_BS_ERR_CUDA, "target sort size query failed");
  if ((rc = c->sort_tmp.ensure(sort_bytes + 256, s))) return rc;
  PackedFilaments pf{(float4 *)c->pk.p, (double4 *)c->ra.p, (double4 *)c->rb.p};
  cudaError_t e = launch_bbox_init((BBox *)c->bbox.p, s);
  c->launches += 1;
  c->chained = chain;
  if (chain) {
    unsigned *heads = (unsigned *)c->heads.p;
    if (e == cudaSuccess) e = cudaMemsetAsync(heads, 0, (nfp / 64 + 1) * sizeof(unsigned), s);
    long long roff = 0;
    for (int k = 0; k < nfam && e == cudaSuccess; ++k) {
      const long long *d = fams[k].dims;
      e = launch_pack_chains(fams[k].F1, fams[k].F2, fams[k].gamma, fams[k].rc, d,
                             roff, (unsigned long long *)c->chaincnt.p + 2 * k, model, dcut, pf,
                             heads, (BBox *)c->bbox.p, s);
      c->launches += d[0] * d[2] * d[3] > 0 ? 2 : 0;
      roff += chain_records(d[0], d[2], d[3]);
    }
    if (e == cudaSuccess) {
      e = launch_pad_chains(2 * nrec, nfp, pf, heads, s);
      c->launches += nfp > 2 * nrec;
    }
  } else {
    long long off = 0;
    for (int k = 0; k < nfam && e == cudaSuccess; ++k) {
      const long long *d = fams[k].dims;
      const long long n = d[0] * d[2] * d[3];
      e = launch_pack_filaments(fams[k].F1, fams[k].F2, fams[k].gamma, fams[k].rc, d[0], n, off,
                                model, dcut, pf, (BBox *)c->bbox.p, s);
      c->launches += n > 0;
      off += n;
    }
    if (e == cudaSuccess) {
      e = launch_pad_filaments(nf, nfp, pf, s);
      c->launches += nfp > nf;
    }
  }
  long long toff = 0;
  int gid = 0;
  for (const TargetSpec &t : tsets) {
    if (e != cudaSuccess) break;
    e = launch_pack_targets(t.P, t.ns, t.count, toff, gid++, (double4 *)c->tp_raw.p,
                            (int *)c->tgroup.p, (BBox *)c->bbox.p, s);
    c->launches += t.count > 0;
    toff += t.count;
  }
  // Sort targets by (set, Morton code) so each thread's targets lie close together.
  unsigned long long *k0 = (unsigned long long *)c->keys.p, *k1 = k0 + std::max<long long>(nt, 1);
  if (e == cudaSuccess)
    e = launch_target_keys((const double4 *)c->tp_raw.p, (const int *)c->tgroup.p, nt,
                           (const BBox *)c->bbox.p, k0, (int *)c->vals.p, s);
  if (e == cudaSuccess && nt > 0)
    e = sort_target_keys(c->sort_tmp.p, &sort_bytes, k0, k1, (const int *)c->vals.p,
                         (int *)c->perm.p, nt, s);
  if (e == cudaSuccess)
    e = launch_gather_targets((const double4 *)c->tp_raw.p, (const int *)c->perm.p, nt,
                              (double4 *)c->tp.p, s);
  c->launches += nt > 0 ? 5 : 0;  // keys, 3 radix-sort passes (library), gather (approx.)
  if (e != cudaSuccess) return cuda_fail(e, "pack kernels");
  *nf_real = nf;
  *nf_pad = nfp;
  *nt_total = nt;
  return WINDS_BS_OK;
}

// ------------------------------------------------------------- autotuner
struct TuneKey {
  int model;
  int tb, fb;  // log2 buckets of targets and filaments
  bool eval;   // the evaluation entry points (layout included in the choice)
  bool operator<(const TuneKey &o) const {
    return std::tie(model, tb, fb, eval) < std::tie(o.model, o.tb, o.fb, o.eval);
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneChoice> g_tune;

static int log2_bucket(long long n) {
  int b = 0;
  while (n > 1) {
    n >>= 1;
    ++b;
  }
  return b;
}

// Untuned tiling: 4 targets per thread (2 for small sets). T = 8 unrolls
// twice as much code per path; where warps alternate between the screened
// far path and the careful path it runs ~35% slower (64-case wake batch).
TuneChoice default_choice(long long nt) {
  TuneChoice ch;
  ch.T = nt >= 2048 ? 4 : 2;
  ch.KF = 64;
  ch.waves = 32.0;
  return ch;
}

bool lookup_tune(int model, long long nt, long long nf, TuneChoice *out, bool eval) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tune.find(TuneKey{model, log2_bucket(nt), log2_bucket(nf), eval});
  if (it == g_tune.end()) return false;
  *out = it->second;
  return true;
}

void store_tune(int model, long long nt, long long nf, const TuneChoice &ch, bool eval) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[TuneKey{model, log2_bucket(nt), log2_bucket(nf), eval}] = ch;
}

// ------------------------------------------------------------- evaluation
int run_direct_sum(Context *c, const std::vector<GroupSpec> &gs, int model, double d, double n,
                   double co, int precision, bool sequential, const TuneChoice &ch,
                   cudaStream_t s, bool time_main) {
  Plan &pl = c->plan;
  int tile_cap, resident, quantum;
  if (precision == WINDS_PREC_F64) {
    tile_cap = f64_threads();
    resident = f64_occupancy() * c->num_sms;
    quantum = f64_tile();
  } else {
    if (!f32c_config_supported(ch.T, ch.KF)) return fail(WINDS_BS_ERR_ARG, "bad tile choice");
    tile_cap = f32c_threads() * ch.T;
    resident = f32c_occupancy(model, ch.T, ch.KF, c->chained) * c->num_sms;
    quantum = kFilamentPad;
  }
  // sequential: one chunk per tile, so every target sums its filaments in order
  const double waves = sequential ? 0.0 : ch.waves;
  if (sequential) quantum = 1 << 30;
  bool same = c->plan_tile_cap == tile_cap && c->plan_resident == resident &&
              c->plan_quantum == quantum && c->plan_waves == waves &&
              c->plan_gs.size() == gs.size();
  for (size_t k = 0; same && k < gs.size(); ++k) {
    const GroupSpec &x = gs[k], &y = c->plan_gs[k];
    same = x.out == y.out && x.t_begin == y.t_begin && x.t_count == y.t_count &&
           x.ns_p == y.ns_p && x.f_begin == y.f_begin && x.f_end == y.f_end &&
           x.accumulate == y.accumulate;
  }
  int rc;
  if (same) {
    // the tables on the device are this plan's; order after their upload
    cudaError_t e = cudaStreamWaitEvent(s, c->ev_upload, 0);
    if (e != cudaSuccess) return cuda_fail(e, "plan reuse");
  } else {
    c->plan_tile_cap = -1;
    build_plan(pl, gs, tile_cap, resident, waves, quantum);
    if ((rc = upload_plan(c, pl, s))) return rc;
    c->plan_gs = gs;
    c->plan_tile_cap = tile_cap;
    c->plan_resident = resident;
    c->plan_quantum = quantum;
    c->plan_waves = waves;
  }
  const size_t part_bytes = pl.items.size() * 3 * (size_t)tile_cap * sizeof(double);
  if ((rc = c->part.ensure(part_bytes + 16, s))) return rc;
  F32cArgs a;
  a.pk = (const float4 *)c->pk.p;
  a.ra = (const double4 *)c->ra.p;
  a.rb = (const double4 *)c->rb.p;
  a.tp = (const double4 *)c->tp.p;
  a.groups = (const Group *)c->groups.p;
  a.tiles = (const Tile *)c->tiles.p;
  a.items = (const Item *)c->items.p;
  a.order = (const int *)c->order.p;
  a.n_items = (int)pl.items.size();
  a.tile_cap = tile_cap;
  a.part = (double *)c->part.p;
  a.work_ctr = (unsigned *)c->ctr.p;
  a.err = (unsigned *)c->err.p;
  a.near_ctr = (unsigned long long *)c->nearctr.p;
  a.bbox = (const BBox *)c->bbox.p;
  a.model = model;
  a.d = d;
  a.n = n;
  a.co = co;
  a.wait_limit_ns = default_wait_limit_ns();
  a.heads = precision == WINDS_PREC_F32C && c->chained ? (const unsigned *)c->heads.p : nullptr;
  cudaError_t e = cudaMemsetAsync(c->ctr.p, 0, sizeof(unsigned), s);
  // near-singular pairs are counted per evaluation
  if (e == cudaSuccess) e = cudaMemsetAsync(c->nearctr.p, 0, 2 * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "work counter reset");
  const int grid = (int)std::max<long long>(1, std::min<long long>(a.n_items, resident));
  if (time_main) cudaEventRecord(c->ev_main0, s);
  if (precision == WINDS_PREC_F64)
    e = launch_f64(a, grid, s);
  else
    e = launch_f32c(a, model, ch.T, ch.KF, grid, s);
  if (time_main) cudaEventRecord(c->ev_main1, s);
  c->launches += 1;
  c->timed = time_main;
  if (e != cudaSuccess) return cuda_fail(e, "direct-sum launch");
  e = launch_reduce((const Tile *)c->tiles.p, (int)pl.tiles.size(), (const Group *)c->groups.p,
                    (const double *)c->part.p, (const int *)c->perm.p, tile_cap, s);
  c->launches += 1;
  if (e != cudaSuccess) return cuda_fail(e, "reduce launch");
  return WINDS_BS_OK;
}

int validate_family(const winds_bs_family &f) {
  const long long *d = f.dims;
  if (d[1] != 3 || d[0] < 0 || d[2] < 0 || d[3] < 0)
    return fail(WINDS_BS_ERR_ARG, "filament arrays must be [n,3,m,k] (got [%lld,%lld,%lld,%lld])",
                d[0], d[1], d[2], d[3]);
  const long long n = d[0] * d[2] * d[3];
  if (n > 0 && (!f.F1 || !f.F2 || !f.gamma || !f.rc))
    return fail(WINDS_BS_ERR_ARG, "null filament pointer");
  if (n > (1ll << 30)) return fail(WINDS_BS_ERR_ARG, "too many filaments (%lld)", n);
  return WINDS_BS_OK;
}

int resolve_model(const winds_bs_params *prm, int *model, double *dcut, double *n, int *prec) {
  if (!prm) return fail(WINDS_BS_ERR_ARG, "null params");
  *prec = prm->precision;
  if (*prec != WINDS_PREC_F32C && *prec != WINDS_PREC_F64)
    return fail(WINDS_BS_ERR_ARG, "unknown precision %d", *prec);
  if (prm->core_model == WINDS_CORE_CUTOFF) {
    *model = kCoreCutoff;
    *dcut = prm->d;
    *n = 0.0;
    // A negative or non-finite squared cut-off can make the denominator vanish;
    // only the FP64 path reproduces the reference there.
    if (!(prm->d >= 0.0) || !std::isfinite(prm->d)) *prec = WINDS_PREC_F64;
  } else if (prm->core_model == WINDS_CORE_VATISTAS) {
    *model = kCoreVatistas;
    *dcut = 0.0;
    *n = prm->d;
    // The FP32 kernel folds the n = 2 core; other indices run in FP64.
    if (prm->d != 2.0) *prec = WINDS_PREC_F64;
    if (prm->d == 0.0) {  // n = 0 is the cut-off branch with d = 0 (BiotSavart.m:102)
      *model = kCoreCutoff;
      *dcut = 0.0;
    }
  } else {
    return fail(WINDS_BS_ERR_ARG, "unknown core model %d", prm->core_model);
  }
  return WINDS_BS_OK;
}

// Packs the inputs in one layout and describes one group per target set.
static int pack_groups(Context *c, const winds_bs_family *fams, int nfam,
                       const std::vector<TargetSpec> &tsets, int model, double dcut,
                       cudaStream_t s, bool chain, std::vector<GroupSpec> *gs, long long *nf,
                       long long *nt) {
  long long nfp;
  int rc;
  if ((rc = pack_inputs(c, fams, nfam, tsets, model, dcut, s, nf, &nfp, nt, chain))) return rc;
  gs->clear();
  long long toff = 0;
  for (const TargetSpec &t : tsets) {
    GroupSpec g;
    g.out = t.out;
    g.t_begin = toff;
    g.t_count = t.count;
    g.ns_p = t.ns;
    g.f_begin = 0;
    g.f_end = (int)nfp;
    g.accumulate = t.accumulate;
    gs->push_back(g);
    toff += t.count;
  }
  return WINDS_BS_OK;
}

int eval_device(Context *c, const winds_bs_family *fams, int nfam,
                const std::vector<TargetSpec> &tsets, const winds_bs_params *prm,
                cudaStream_t s, bool sequential) {
  int model, prec, rc;
  double dcut, n;
  if ((rc = resolve_model(prm, &model, &dcut, &n, &prec))) return rc;
  for (int k = 0; k < nfam; ++k)
    if ((rc = validate_family(fams[k]))) return rc;
  c->launches = 0;
  long long nf = 0, nt = 0;
  for (int k = 0; k < nfam; ++k) nf += fams[k].dims[0] * fams[k].dims[2] * fams[k].dims[3];
  for (const TargetSpec &t : tsets) nt += t.count;
  // The FP64 path (and the sequential mode that reproduces the reference's
  // order) runs on the input order. FP32c runs on the layout its tuned choice
  // names; the autotuner times both layouts, each with every tiling.
  const bool fast = prec == WINDS_PREC_F32C && !sequential;
  TuneChoice ch = default_choice(nt);
  std::vector<GroupSpec> gs;
  if (fast && nt > 0 && !lookup_tune(model, nt, nf, &ch, true) && c->autotune && s == c->stream) {
    float best_ms = 1e30f;
    for (int layout = 0; layout < 2; ++layout) {
      TuneChoice tc;
      float ms = 1e30f;
      if ((rc = pack_groups(c, fams, nfam, tsets, model, dcut, s, layout == 1, &gs, &nf, &nt)) ||
          (rc = autotune(c, gs, model, dcut, n, prm->co, &tc, &ms)))
        return rc;
      tc.chain = layout == 1;
      if (ms < best_ms) best_ms = ms, ch = tc;
    }
    store_tune(model, nt, nf, ch, true);
  }
  if ((rc = pack_groups(c, fams, nfam, tsets, model, dcut, s, fast && ch.chain, &gs, &nf, &nt)))
    return rc;
  if (nt == 0) return WINDS_BS_OK;
  return run_direct_sum(c, gs, model, dcut, n, prm->co, prec, sequential, ch, s, true);
}

// Times each candidate (T, KF, waves) twice after a warm-up on the inputs as
// packed and returns the fastest with its time.
int autotune(Context *c, const std::vector<GroupSpec> &gs, int model, double dcut, double n,
             double co, TuneChoice *best, float *best_ms_out) {
  // T = 8 (supported, settable) is left out: its unrolled paths run slower
  const int Ts[3] = {2, 3, 4};
  const int KFs[3] = {32, 64, 128};
  const double Ws[3] = {16.0, 32.0, 64.0};
  float best_ms = 1e30f;
  TuneChoice bc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int T : Ts) {
    for (int KF : KFs)
      for (double w : Ws) {
        TuneChoice ch;
        ch.T = T;
        ch.KF = KF;
        ch.waves = w;
        int rc = run_direct_sum(c, gs, model, dcut, n, co, WINDS_PREC_F32C, false, ch, c->stream,
                                false);
        if (rc) return rc;
        float ms = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {  // the faster of two timed runs
          cudaEventRecord(e0, c->stream);
          rc = run_direct_sum(c, gs, model, dcut, n, co, WINDS_PREC_F32C, false, ch, c->stream,
                              false);
          if (rc) return rc;
          cudaEventRecord(e1, c->stream);
          cudaError_t e = cudaEventSynchronize(e1);
          if (e != cudaSuccess) return cuda_fail(e, "autotune");
          float t = 0.f;
          cudaEventElapsedTime(&t, e0, e1);
          ms = std::min(ms, t);
        }
        if (ms < best_ms) {
          best_ms = ms;
          bc = ch;
        }
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *best = bc;
  *best_ms_out = best_ms;
  return WINDS_BS_OK;
}

int check_device_error(Context *c, cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
  unsigned *h = static_cast<unsigned *>(c->hstat.p);
  e = cudaMemcpy(h, c->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "error word read");
  if (*h) {
    const unsigned v = *h;
    cudaMemset(c->err.p, 0, sizeof(unsigned));
    if (v & kErrWaitTimeout)
      return fail(WINDS_BS_ERR_TIMEOUT, "a bounded device wait ran out (error word 0x%x)", v);
    return fail(WINDS_BS_ERR_CUDA, "device reported error word 0x%x", v);
  }
  return WINDS_BS_OK;
}

}  // namespace winds

// =================================================================== C ABI
using namespace winds;

extern "C" {

const char *winds_bs_version(void) { return "winds_bs 0.1 (sm_100a)"; }

const char *winds_bs_last_error(void) { return last_error(); }

int winds_bs_device_count(int *n) {
  if (!n) return fail(WINDS_BS_ERR_ARG, "null pointer");
  int k = 0;
  if (cudaGetDeviceCount(&k) != cudaSuccess) k = 0;
  *n = k;
  return WINDS_BS_OK;
}

int winds_bs_set_device(int device) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0)
    return fail(WINDS_BS_ERR_NODEV, "no CUDA device is visible");
  if (device < 0 || device >= n) return fail(WINDS_BS_ERR_ARG, "device %d of %d", device, n);
  g_device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return WINDS_BS_OK;
}

static int targets_from(const double *P, const long long pdims[4], double *uind,
                        std::vector<TargetSpec> *ts) {
  if (!pdims) return fail(WINDS_BS_ERR_ARG, "null P dims");
  if (pdims[1] != 3 || pdims[0] < 0 || pdims[2] < 0 || pdims[3] < 0)
    return fail(WINDS_BS_ERR_ARG, "P must be [n,3,m,k] (got [%lld,%lld,%lld,%lld])", pdims[0],
                pdims[1], pdims[2], pdims[3]);
  TargetSpec t;
  t.P = P;
  t.ns = pdims[0];
  t.count = pdims[0] * pdims[2] * pdims[3];
  t.out = uind;
  t.accumulate = 0;
  if (t.count > 0 && (!P || !uind)) return fail(WINDS_BS_ERR_ARG, "null P or uind");
  ts->push_back(t);
  return WINDS_BS_OK;
}

int winds_bs_eval_device(const winds_bs_family *fams, int nfam, const double *P,
                         const long long pdims[4], const winds_bs_params *prm, double *uind,
                         void *stream) {
  if (nfam < 0 || (nfam > 0 && !fams)) return fail(WINDS_BS_ERR_ARG, "bad family list");
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  std::vector<TargetSpec> ts;
  if ((rc = targets_from(P, pdims, uind, &ts))) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  const bool seq = prm && (prm->flags & WINDS_BS_FLAG_SEQUENTIAL);
  if (nfam == 0 || ts[0].count == 0) {
    if (ts[0].count > 0) {
      cudaError_t e = cudaMemsetAsync(uind, 0, ts[0].count * 3 * sizeof(double), s);
      if (e != cudaSuccess) return cuda_fail(e, "zero output");
    }
    return WINDS_BS_OK;
  }
  return eval_device(c, fams, nfam, ts, prm, s, seq);
}

int winds_bs_eval_host(const winds_bs_family *fams, int nfam, const double *P,
                       const long long pdims[4], const winds_bs_params *prm, double *uind) {
  if (nfam < 0 || (nfam > 0 && !fams)) return fail(WINDS_BS_ERR_ARG, "bad family list");
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  std::vector<TargetSpec> ts;
  if ((rc = targets_from(P, pdims, uind, &ts))) return rc;
  const long long np = ts[0].count;
  cudaStream_t s = c->stream;
  if (np == 0) return WINDS_BS_OK;
  for (int k = 0; k < nfam; ++k)
    if ((rc = validate_family(fams[k]))) return rc;
  // device copies of the MATLAB arrays: P, then per family F1, F2, gamma, rc
  size_t fbytes = 0;
  for (int k = 0; k < nfam; ++k) {
    const long long n = fams[k].dims[0] * fams[k].dims[2] * fams[k].dims[3];
    fbytes += (size_t)n * 8 * sizeof(double);
  }
  if ((rc = c->in_P.ensure(np * 3 * sizeof(double), s)) || (rc = c->in_F.ensure(fbytes + 64, s)) ||
      (rc = c->out_u.ensure(np * 3 * sizeof(double), s)))
    return rc;
  cudaError_t e = cudaMemcpyAsync(c->in_P.p, P, np * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
  std::vector<winds_bs_family> dev(nfam);
  double *base = (double *)c->in_F.p;
  for (int k = 0; k < nfam && e == cudaSuccess; ++k) {
    const long long n = fams[k].dims[0] * fams[k].dims[2] * fams[k].dims[3];
    dev[k] = fams[k];
    dev[k].F1 = base;
    dev[k].F2 = base + 3 * n;
    dev[k].gamma = base + 6 * n;
    dev[k].rc = base + 7 * n;
    if (n > 0) {
      e = cudaMemcpyAsync((void *)dev[k].F1, fams[k].F1, 3 * n * sizeof(double),
                          cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync((void *)dev[k].F2, fams[k].F2, 3 * n * sizeof(double),
                            cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync((void *)dev[k].gamma, fams[k].gamma, n * sizeof(double),
                            cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync((void *)dev[k].rc, fams[k].rc, n * sizeof(double),
                            cudaMemcpyHostToDevice, s);
    }
    base += 8 * n;
  }
  if (e != cudaSuccess) return cuda_fail(e, "host to device copy");
  std::vector<TargetSpec> dts = ts;
  dts[0].P = (const double *)c->in_P.p;
  dts[0].out = (double *)c->out_u.p;
  const bool seq = prm && (prm->flags & WINDS_BS_FLAG_SEQUENTIAL);
  if (nfam == 0) {
    e = cudaMemsetAsync(c->out_u.p, 0, np * 3 * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "zero output");
  } else if ((rc = eval_device(c, dev.data(), nfam, dts, prm, s, seq))) {
    return rc;
  }
  e = cudaMemcpyAsync(uind, c->out_u.p, np * 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_fail(e, "device to host copy");
  return check_device_error(c, s);
}

int winds_bs_length_device(const double *F1, const double *F2, const long long dims[4], double *L,
                           void *stream) {
  if (!dims || dims[1] != 3) return fail(WINDS_BS_ERR_ARG, "filament arrays must be [n,3,m,k]");
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  const long long n = dims[0] * dims[2] * dims[3];
  if (n > 0 && (!F1 || !F2 || !L)) return fail(WINDS_BS_ERR_ARG, "null pointer");
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  cudaError_t e = launch_length(F1, F2, dims[0], n, L, s);
  if (e != cudaSuccess) return cuda_fail(e, "length kernel");
  return WINDS_BS_OK;
}

int winds_bs_sync(void *stream) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  return check_device_error(c, stream ? (cudaStream_t)stream : c->stream);
}

int winds_bs_last_stats(double *main_ms, int *launches, long long *near_pairs) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "stats sync");
  if (main_ms) {
    float ms = 0.f;
    if (c->timed) cudaEventElapsedTime(&ms, c->ev_main0, c->ev_main1);
    *main_ms = ms;
  }
  if (launches) *launches = c->launches;
  if (near_pairs) {
    unsigned long long v = 0;
    cudaMemcpy(&v, c->nearctr.p, sizeof(v), cudaMemcpyDeviceToHost);
    cudaMemset(c->nearctr.p, 0, sizeof(v));
    *near_pairs = (long long)v;
  }
  return WINDS_BS_OK;
}

int winds_bs_last_chained(int *chained) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  if (!chained) return WINDS_BS_ERR_ARG;
  *chained = c->chained ? 1 : 0;
  return WINDS_BS_OK;
}

int winds_bs_last_core_free(long long *pairs) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  if (!pairs) return WINDS_BS_ERR_ARG;
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "stats sync");
  unsigned long long v = 0;
  e = cudaMemcpy(&v, (const unsigned long long *)c->nearctr.p + 1, sizeof(v),
                 cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "stats read");
  *pairs = (long long)v;
  return WINDS_BS_OK;
}

int winds_bs_set_autotune(int on) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  c->autotune = on != 0;
  return WINDS_BS_OK;
}

int winds_bs_set_tuning(int core_model, long long n_targets, long long n_filaments, int T, int KF,
                        double waves) {
  if (!f32c_config_supported(T, KF) || !(waves > 0))
    return fail(WINDS_BS_ERR_ARG, "unsupported tile choice T=%d KF=%d", T, KF);
  TuneChoice ch;
  ch.T = T;
  ch.KF = KF;
  ch.waves = waves;
  // for every FP32c path of the bucket: the evaluations' chained stream and
  // the unchained ones
  const int model = core_model == WINDS_CORE_CUTOFF ? kCoreCutoff : kCoreVatistas;
  store_tune(model, n_targets, n_filaments, ch, true);
  store_tune(model, n_targets, n_filaments, ch, false);
  return WINDS_BS_OK;
}

int winds_bs_set_layout(int core_model, long long n_targets, long long n_filaments, int chained) {
  const int model = core_model == WINDS_CORE_CUTOFF ? kCoreCutoff : kCoreVatistas;
  TuneChoice ch;
  if (!lookup_tune(model, n_targets, n_filaments, &ch, true)) ch = default_choice(n_targets);
  ch.chain = chained != 0;
  store_tune(model, n_targets, n_filaments, ch, true);
  return WINDS_BS_OK;
}

int winds_bs_get_tuning(int core_model, long long n_targets, long long n_filaments, int *T, int *KF,
                        double *waves) {
  TuneChoice ch;
  const int model = core_model == WINDS_CORE_CUTOFF ? kCoreCutoff : kCoreVatistas;
  if (!lookup_tune(model, n_targets, n_filaments, &ch, true) &&
      !lookup_tune(model, n_targets, n_filaments, &ch, false))
    ch = default_choice(n_targets);
  if (T) *T = ch.T;
  if (KF) *KF = ch.KF;
  if (waves) *waves = ch.waves;
  return WINDS_BS_OK;
}

int winds_bs_fp32_peak(double *tflops) {
  if (!tflops) return fail(WINDS_BS_ERR_ARG, "null pointer");
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  const int blocks = c->num_sms * 8, iters = 4096;
  if ((rc = c->part.ensure((size_t)blocks * 256 * sizeof(float), c->stream))) return rc;
  cudaError_t e = launch_ffma_peak((float *)c->part.p, blocks, 64, c->stream);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, c->stream);
  if (e == cudaSuccess) e = launch_ffma_peak((float *)c->part.p, blocks, iters, c->stream);
  cudaEventRecord(e1, c->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "FP32 peak probe");
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return WINDS_BS_OK;
}

int winds_bs_selftest_wait_timeout(unsigned long long limit_ns) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  cudaError_t e = launch_wait_selftest((unsigned *)c->err.p, limit_ns, c->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wait self-test launch");
  return check_device_error(c, c->stream);
}

void winds_bs_shutdown(void) { shutdown_all(); }

}  // extern "C"
