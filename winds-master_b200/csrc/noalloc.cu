// noalloc.cu -- winds_bs_eval_device_noalloc: the induced-velocity evaluation
// for callers that must not allocate device memory.
//
// Who cannot allocate: a host that owns every byte of device memory through
// its own pool or caching allocator (and must not have a library call
// cudaMalloc behind its back), and a time-stepping loop that must not stall:
// cudaMalloc and cudaFree synchronise the device, so a solver calling the
// engine every step cannot afford them. winds_bs_eval_device grows buffers
// with cudaMalloc the first time it sees a larger problem; this entry point
// never does. All of its scratch lives in one file-scope __device__ array of
// WINDS_BS_NOALLOC_SCRATCH_BYTES (64 MiB) that every GPU loading the library
// holds until the process exits.
//
// Rules of use (also in include/winds_bs.h):
//   * every call looks up the array's device address on the current device
//     (cudaGetSymbolAddress, a host-side lookup, so the address is never stale
//     after a device reset); the first call on a device also loads the
//     module, which commits the array: make that first call before any
//     stream capture;
//   * the work runs on the calling thread's current device and on `stream`
//     (NULL: the legacy default stream), not on the library's own device
//     choice and stream as winds_bs_eval_device does;
//   * every call shares the one array and overwrites it: calls that overlap on
//     the GPU (two streams, or two host threads) race and corrupt each other;
//   * sizes are limited to WINDS_BS_NOALLOC_MAX_FILAMENTS filaments and
//     WINDS_BS_NOALLOC_MAX_TARGETS targets; larger calls are rejected.
#include <cuda_runtime.h>

#include <algorithm>

#include "bs_launch.h"
#include "engine.h"
#include "winds_bs.h"

namespace winds {
namespace {

constexpr size_t kNoallocBytes = (size_t)WINDS_BS_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxItems = 2048;
constexpr size_t kPartBudget = (size_t)24 << 20;  // partial sums: 3 doubles per target per item

// The scratch array. In host code this name is only a stand-in for the
// symbol: the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// Device address of the scratch array on the current device, looked up on
// every call: nothing is cached that a device reset could invalidate.
int scratch_address(unsigned char **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
  *out = static_cast<unsigned char *>(p);
  return WINDS_BS_OK;
}

// One target set: tile j holds targets [j*tile_cap, ...), item i is tile
// i / n_chunks against filament chunk i % n_chunks.
__global__ void bs_noalloc_plan(Group *groups, Tile *tiles, Item *items, double *out,
                                long long nt, long long ns_p, int nf_pad, int tile_cap,
                                int chunk, int n_chunks, int n_tiles) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    Group g;
    g.out = out;
    g.t_begin = 0;
    g.t_count = nt;
    g.ns_p = ns_p;
    g.f_begin = 0;
    g.f_end = nf_pad;
    g.accumulate = 0;
    g.pad = 0;
    groups[0] = g;
  }
  if (i < n_tiles) {
    Tile t;
    t.t_begin = (long long)i * tile_cap;
    const long long left = nt - t.t_begin;
    t.t_count = (int)(left < tile_cap ? left : tile_cap);
    t.group = 0;
    t.first_item = i * n_chunks;
    t.n_items = n_chunks;
    tiles[i] = t;
  }
  if (i < n_tiles * n_chunks) {
    Item it;
    it.tile = i / n_chunks;
    it.f_begin = (i % n_chunks) * chunk;
    it.f_end = it.f_begin + chunk < nf_pad ? it.f_begin + chunk : nf_pad;
    it.pad = 0;
    items[i] = it;
  }
}

struct Carve {
  unsigned char *base;
  size_t off = 0;
  template <class U>
  U *take(size_t n) {
    off = (off + 255) & ~(size_t)255;
    U *p = reinterpret_cast<U *>(base + off);
    off += n * sizeof(U);
    return p;
  }
};

}  // namespace
}  // namespace winds

using namespace winds;

extern "C" int winds_bs_eval_device_noalloc(const winds_bs_family *fams, int nfam, const double *P,
                                            const long long pdims[4], const winds_bs_params *prm,
                                            double *uind, void *stream) {
  if (nfam < 0 || (nfam > 0 && !fams)) return fail(WINDS_BS_ERR_ARG, "bad family list");
  if (!pdims || pdims[1] != 3 || pdims[0] < 0 || pdims[2] < 0 || pdims[3] < 0)
    return fail(WINDS_BS_ERR_ARG, "P must be [n,3,m,k]");
  int model, prec, rc;
  double dcut, n;
  if ((rc = resolve_model(prm, &model, &dcut, &n, &prec))) return rc;
  long long nf = 0;
  for (int k = 0; k < nfam; ++k) {
    if ((rc = validate_family(fams[k]))) return rc;
    nf += fams[k].dims[0] * fams[k].dims[2] * fams[k].dims[3];
  }
  const long long nt = pdims[0] * pdims[2] * pdims[3];
  if (nt > 0 && (!P || !uind)) return fail(WINDS_BS_ERR_ARG, "null P or uind");
  if (nf > WINDS_BS_NOALLOC_MAX_FILAMENTS || nt > WINDS_BS_NOALLOC_MAX_TARGETS)
    return fail(WINDS_BS_ERR_ARG,
                "noalloc evaluation limited to %d filaments and %d targets (got %lld and %lld); "
                "use winds_bs_eval_device",
                WINDS_BS_NOALLOC_MAX_FILAMENTS, WINDS_BS_NOALLOC_MAX_TARGETS, nf, nt);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if (nt == 0) return WINDS_BS_OK;
  if (nf == 0) {
    e = cudaMemsetAsync(uind, 0, nt * 3 * sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail(e, "zero output");
    e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "stream synchronize");
  }
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  unsigned char *base = nullptr;
  if ((rc = scratch_address(&base))) return rc;
  int sms = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
      sms <= 0)
    return e != cudaSuccess ? cuda_fail(e, "multiprocessor count")
                            : fail(WINDS_BS_ERR_CUDA, "device %d reports no multiprocessors", dev);

  // ---- plan (sizes only; the tables are written by a kernel)
  const long long nfp = std::max<long long>((nf + kFilamentPad - 1) / kFilamentPad * kFilamentPad,
                                            kFilamentPad);
  TuneChoice ch = default_choice(nt);
  if (prec == WINDS_PREC_F32C) lookup_tune(model, nt, nf, &ch);
  int tile_cap, resident, quantum;
  if (prec == WINDS_PREC_F64) {
    tile_cap = f64_threads();
    resident = f64_occupancy() * sms;
    quantum = f64_tile();
  } else {
    tile_cap = f32c_threads() * ch.T;
    resident = f32c_occupancy(model, ch.T, ch.KF) * sms;
    quantum = kFilamentPad;
  }
  const int n_tiles = (int)((nt + tile_cap - 1) / tile_cap);
  const long long max_items =
      std::min<long long>(kMaxItems, (long long)(kPartBudget / (3 * sizeof(double) * tile_cap)));
  long long want = std::max<long long>((long long)(resident * ch.waves), n_tiles);
  want = std::min<long long>(want, max_items);
  long long chunk = (n_tiles * nfp + want - 1) / want;
  chunk = std::max<long long>((chunk + quantum - 1) / quantum * quantum, quantum);
  int n_chunks = (int)((nfp + chunk - 1) / chunk);
  while ((long long)n_tiles * n_chunks > max_items) {  // bounded partial-sum slots
    chunk += quantum;
    n_chunks = (int)((nfp + chunk - 1) / chunk);
  }
  const int n_items = n_tiles * n_chunks;

  // ---- carve the scratch array
  size_t sort_bytes = 0;
  if (sort_target_keys(nullptr, &sort_bytes, nullptr, nullptr, nullptr, nullptr, nt, s) !=
      cudaSuccess)
    return fail(WINDS_BS_ERR_CUDA, "target sort size query failed");
  Carve cv{base};
  BBox *bbox = cv.take<BBox>(1);
  unsigned *ctr = cv.take<unsigned>(4);
  unsigned *err = cv.take<unsigned>(4);
  unsigned long long *nearc = cv.take<unsigned long long>(2);  // near, core-free pairs
  PackedFilaments pf{cv.take<float4>(nfp * 4), cv.take<double4>(nfp), cv.take<double4>(nfp)};
  double4 *tp = cv.take<double4>(nt);
  double4 *tp_raw = cv.take<double4>(nt);
  int *tgroup = cv.take<int>(nt);
  int *vals = cv.take<int>(nt);
  int *perm = cv.take<int>(nt);
  unsigned long long *k0 = cv.take<unsigned long long>(nt);
  unsigned long long *k1 = cv.take<unsigned long long>(nt);
  void *sort_tmp = cv.take<unsigned char>(sort_bytes);
  Group *groups = cv.take<Group>(1);
  Tile *tiles = cv.take<Tile>(n_tiles);
  Item *items = cv.take<Item>(n_items);
  double *part = cv.take<double>((size_t)n_items * 3 * tile_cap);
  if (cv.off > kNoallocBytes)
    return fail(WINDS_BS_ERR_ARG, "noalloc scratch too small: need %zu of %zu bytes", cv.off,
                kNoallocBytes);

  // ---- state carried over from the previous call: clear what starts at zero
  if ((e = cudaMemsetAsync(ctr, 0, 4 * sizeof(unsigned), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(err, 0, 4 * sizeof(unsigned), s)) != cudaSuccess ||
      (e = cudaMemsetAsync(nearc, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess)
    return cuda_fail(e, "scratch reset");

  // ---- pack (the same kernels as winds_bs_eval_device)
  e = launch_bbox_init(bbox, s);
  long long off = 0;
  for (int k = 0; k < nfam && e == cudaSuccess; ++k) {
    const long long *d = fams[k].dims;
    const long long m = d[0] * d[2] * d[3];
    e = launch_pack_filaments(fams[k].F1, fams[k].F2, fams[k].gamma, fams[k].rc, d[0], m, off,
                              model, dcut, pf, bbox, s);
    off += m;
  }
  if (e == cudaSuccess) e = launch_pad_filaments(nf, nfp, pf, s);
  if (e == cudaSuccess) e = launch_pack_targets(P, pdims[0], nt, 0, 0, tp_raw, tgroup, bbox, s);
  if (e == cudaSuccess) e = launch_target_keys(tp_raw, tgroup, nt, bbox, k0, vals, s);
  if (e == cudaSuccess) e = sort_target_keys(sort_tmp, &sort_bytes, k0, k1, vals, perm, nt, s);
  if (e == cudaSuccess) e = launch_gather_targets(tp_raw, perm, nt, tp, s);
  if (e == cudaSuccess) {
    const int grid = (n_items + 255) / 256;
    bs_noalloc_plan<<<grid, 256, 0, s>>>(groups, tiles, items, uind, nt, pdims[0], (int)nfp,
                                         tile_cap, (int)chunk, n_chunks, n_tiles);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return cuda_fail(e, "noalloc pack/plan kernels");

  // ---- direct sum and reduction
  F32cArgs a;
  a.pk = pf.pk;
  a.ra = pf.ra;
  a.rb = pf.rb;
  a.tp = tp;
  a.groups = groups;
  a.tiles = tiles;
  a.items = items;
  a.order = nullptr;  // items are generated in queue order
  a.n_items = n_items;
  a.tile_cap = tile_cap;
  a.part = part;
  a.work_ctr = ctr;
  a.err = err;
  a.near_ctr = nearc;
  a.bbox = bbox;
  a.model = model;
  a.d = dcut;
  a.n = n;
  a.co = prm->co;
  a.wait_limit_ns = default_wait_limit_ns();
  const int grid = std::max(1, std::min(n_items, resident));
  e = prec == WINDS_PREC_F64 ? launch_f64(a, grid, s) : launch_f32c(a, model, ch.T, ch.KF, grid, s);
  if (e == cudaSuccess) e = launch_reduce(tiles, n_tiles, groups, part, perm, tile_cap, s);
  if (e != cudaSuccess) return cuda_fail(e, "noalloc direct-sum launch");

  // ---- synchronous: report a device-side timeout recorded in the error word,
  // read on the call's own stream (no wait on the device's other streams)
  unsigned word = 0;
  if ((e = cudaMemcpyAsync(&word, err, sizeof(word), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
    return cuda_fail(e, "error word read");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cuda_fail(e, "stream synchronize");
  if (word & kErrWaitTimeout)
    return fail(WINDS_BS_ERR_TIMEOUT, "a bounded device wait ran out (error word 0x%x)", word);
  if (word) return fail(WINDS_BS_ERR_CUDA, "device reported error word 0x%x", word);
  return WINDS_BS_OK;
}
