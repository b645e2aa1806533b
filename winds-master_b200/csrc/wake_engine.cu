// wake_engine.cu -- host side of the batched free-wake step (include/winds_wake.h).
//
// One batch holds every case's state in shared device buffers. A step is a
// fixed sequence of kernel launches on the batch's stream:
//   bookkeeping -> [pack filaments + targets -> sort -> direct sum -> reduce]
//   -> convect (fe/ab2/ab4, or pcc predictor) -> (pcc: bookkeeping for p+1
//   -> [direct sum at the predicted nodes] -> corrector) -> commit.
// All sizes are fixed at creation (each wake has a capacity of na columns),
// so the plan tables of the persistent direct-sum kernel are built once and
// the whole step can be captured once as a CUDA graph and replayed. The step
// counter lives on the device, so a replayed graph reads the right kinematics
// row and the right live column count of a growing wake: every evaluation
// first writes a live table (wake_live) that limits the direct sum and its
// reduction to the live targets and filaments of each case.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "bs_launch.h"
#include "engine.h"
#include "kj_launch.h"
#include "mlp_engine.h"
#include "mlp_launch.h"
#include "wake_launch.h"
#include "winds_wake.h"

using namespace winds;

struct winds_wake_batch {
  int dev = 0;
  int ncases = 0;
  winds_wake_params prm{};
  int model = kCoreVatistas, prec = WINDS_PREC_F32C;
  double dcut = 0.0, nidx = 2.0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<WakeCase> cases;
  long long nodes = 0, shed_n = 0, trail_n = 0, bound_n = 0, fil_pad = 0, kin_n = 0, wind_n = 0;
  long long ser_n = 0;
  long long max_nodes = 0, max_cols = 0, max_fil = 0, max_slots = 0;
  int max_nb = 0;  // most blades of a case
  long long interactions = 0;  // per step of the last winds_wake_step call
  int launches = 0;
  int pcc_from = 0, kj_from = 0;  // first step of the corrector / the iteration (startup)
  // state and work buffers
  DevBuf cases_d, step_d;
  DevBuf dom, dom_pred, dom_new, vel, h1, h2, h3, uind, uind_pred;
  DevBuf bound, trail_prev, shed_cur, trail_cur, shed_next, trail_next;
  DevBuf rc_s, rc_t, len_old_s, len_old_t, len_s, len_t, len_ps, len_pt;
  DevBuf quarter, trailing, wind, ser;
  DevBuf live_main, live_pred, live_kj;  // GroupLive per case, per evaluation kind
  // direct-sum buffers
  DevBuf pk, ra, rb, tp, tp_raw, tgroup, keys, vals, perm, sort_tmp;
  DevBuf groups_main, groups_pred, tiles, items, order, part, bbox, ctr, err, nearctr;
  size_t sort_bytes = 0;
  int n_tiles = 0, n_items = 0, tile_cap = 0, grid = 0;
  TuneChoice ch;
  long long steps_done = 0;
  bool tuned = true;         // tiling from the autotuner's cache (or not FP32c)
  long long min_nsteps = 0;  // kinematics rows available in every case
  int timed_steps = 0;       // steps between ev0 and ev1
  // Kutta-Joukowski lifting lines
  bool kj = false;
  winds_kj_params kjp{};
  std::vector<KJCase> kjc;
  long long n_ll = 0, frames_n = 0, stations_n = 0;
  int max_st = 0;
  long long max_bound_cols = 0;  // largest nb (2 ns + nst): the loop's repack
  DevBuf kjc_d, ll, bxn, byn, bzn, vblade, chord, foil, foil_off, aoa_t, cl_t, cd_t;
  DevBuf tp_ll, perm_ll, uindb, kj_groups, kj_tiles, kj_items, kj_order, kj_part;
  DevBuf conv, iters, res_max, res_last, active, diverged, cl_o, cd_o, aoa_o;
  int kj_ntiles = 0, kj_nitems = 0, kj_grid = 0, kj_tile_cap = 0, kj_T = 2, kj_KF = 64;
  long long kj_evals = 0;
  // bound-circulation MLP start value
  bool mlp_inputs = false;      // every case gave the station arrays
  bool loads = false;           // every case gave the loads inputs
  DevBuf st_rr, st_dr, rpm, pitch, dl, loads_out;
  DevBuf st_r, st_c, st_tw, azim, guess, feat, bound_last, bound_last2;
  DevBuf st_lift;   // per station: 1 when its airfoil table has lift (start value applies)
  DevBuf st_stall;  // per station: AoA (deg) of its table's lowest and highest Cl
  winds_mlp *mlp = nullptr;
  MlpWork mw;
  cudaGraphExec_t exec_pre = nullptr, exec_kj = nullptr, exec_post = nullptr;
  cudaGraph_t g_pre = nullptr, g_kj = nullptr, g_post = nullptr;
  // whole step with the iteration as a conditional WHILE node (no host round trip)
  cudaGraphExec_t exec_step = nullptr;
  cudaGraph_t g_step = nullptr;
  cudaStream_t body_stream = nullptr;
  bool cond_ok = true;  // false after a failed build: host loop instead
  int step_launches = 0;
  DevBuf kj_it;         // iterations run in the current step
};

namespace {

template <class T>
T *P(DevBuf &b) {
  return static_cast<T *>(b.p);
}

int alloc_all(winds_wake_batch *b) {
  cudaStream_t s = b->stream;
  const size_t n3 = (size_t)b->nodes * 3 * sizeof(double);
  int rc;
  for (DevBuf *x : {&b->dom, &b->dom_pred, &b->dom_new, &b->vel, &b->h1, &b->h2, &b->h3, &b->uind,
                    &b->uind_pred})
    if ((rc = x->ensure(n3, s))) return rc;
  const size_t sb = std::max<long long>(b->shed_n, 1) * sizeof(double);
  const size_t tb = std::max<long long>(b->trail_n, 1) * sizeof(double);
  for (DevBuf *x : {&b->shed_cur, &b->shed_next, &b->rc_s, &b->len_old_s, &b->len_s, &b->len_ps})
    if ((rc = x->ensure(sb, s))) return rc;
  for (DevBuf *x : {&b->trail_prev, &b->trail_cur, &b->trail_next, &b->rc_t, &b->len_old_t,
                    &b->len_t, &b->len_pt})
    if ((rc = x->ensure(tb, s))) return rc;
  if ((rc = b->bound.ensure(b->bound_n * sizeof(double), s)) ||
      (rc = b->quarter.ensure(b->kin_n * sizeof(double), s)) ||
      (rc = b->trailing.ensure(b->kin_n * sizeof(double), s)) ||
      (rc = b->wind.ensure(b->wind_n * sizeof(double), s)) ||
      (rc = b->ser.ensure(std::max<long long>(b->ser_n, 1) * sizeof(double), s)) ||
      (rc = b->live_main.ensure(b->ncases * sizeof(GroupLive), s)) ||
      (rc = b->live_pred.ensure(b->ncases * sizeof(GroupLive), s)) ||
      (rc = b->live_kj.ensure(b->ncases * sizeof(GroupLive), s)) ||
      (rc = b->cases_d.ensure(b->ncases * sizeof(WakeCase), s)) ||
      (rc = b->step_d.ensure(4 * sizeof(int), s)))
    return rc;
  const long long nf = b->fil_pad, nt = std::max<long long>(b->nodes, 1);
  if ((rc = b->pk.ensure(nf * 4 * sizeof(float4), s)) ||
      (rc = b->ra.ensure(nf * sizeof(double4), s)) || (rc = b->rb.ensure(nf * sizeof(double4), s)) ||
      (rc = b->tp.ensure(nt * sizeof(double4), s)) ||
      (rc = b->tp_raw.ensure(nt * sizeof(double4), s)) ||
      (rc = b->tgroup.ensure(nt * sizeof(int), s)) ||
      (rc = b->keys.ensure(nt * 2 * sizeof(unsigned long long), s)) ||
      (rc = b->vals.ensure(nt * sizeof(int), s)) || (rc = b->perm.ensure(nt * sizeof(int), s)) ||
      (rc = b->bbox.ensure(sizeof(BBox), s)) || (rc = b->ctr.ensure(64, s)) ||
      (rc = b->err.ensure(64, s)) || (rc = b->nearctr.ensure(64, s)))
    return rc;
  if (sort_target_keys(nullptr, &b->sort_bytes, nullptr, nullptr, nullptr, nullptr, b->nodes, s) !=
      cudaSuccess)
    return fail(WINDS_BS_ERR_CUDA, "target sort size query failed");
  return b->sort_tmp.ensure(b->sort_bytes + 256, s);
}

// Direct-sum plan: case c's nodes (one group) against case c's filaments.
int build_plans(winds_wake_batch *b) {
  std::vector<GroupSpec> gs;
  for (const WakeCase &c : b->cases) {
    GroupSpec g;
    g.out = P<double>(b->uind) + c.node_off * 3;
    g.t_begin = c.node_off;
    g.t_count = (long long)c.nst * c.na * c.nb;
    g.ns_p = c.nst;
    g.f_begin = (int)c.fil_off;
    g.f_end = (int)(c.fil_off + c.fil_pad);
    g.accumulate = 0;
    gs.push_back(g);
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
  int resident, quantum;
  if (b->prec == WINDS_PREC_F64) {
    b->tile_cap = f64_threads();
    resident = f64_occupancy() * sms;
    quantum = f64_tile();
  } else {
    b->tile_cap = f32c_threads() * b->ch.T;
    resident = f32c_occupancy(b->model, b->ch.T, b->ch.KF) * sms;
    quantum = kFilamentPad;
  }
  Plan pl;
  build_plan(pl, gs, b->tile_cap, resident, b->ch.waves, quantum);
  b->n_tiles = (int)pl.tiles.size();
  b->n_items = (int)pl.items.size();
  b->grid = std::max(1, std::min(b->n_items, resident));
  std::vector<Group> gp = pl.groups;
  for (size_t k = 0; k < gp.size(); ++k) gp[k].out = P<double>(b->uind_pred) + b->cases[k].node_off * 3;
  int rc;
  cudaStream_t s = b->stream;
  if ((rc = b->groups_main.ensure(pl.groups.size() * sizeof(Group), s)) ||
      (rc = b->groups_pred.ensure(gp.size() * sizeof(Group), s)) ||
      (rc = b->tiles.ensure(pl.tiles.size() * sizeof(Tile), s)) ||
      (rc = b->items.ensure(pl.items.size() * sizeof(Item), s)) ||
      (rc = b->order.ensure(pl.order.size() * sizeof(int), s)) ||
      (rc = b->part.ensure((size_t)b->n_items * 3 * b->tile_cap * sizeof(double), s)))
    return rc;
  cudaError_t e;
  if ((e = cudaMemcpy(b->groups_main.p, pl.groups.data(), pl.groups.size() * sizeof(Group),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->groups_pred.p, gp.data(), gp.size() * sizeof(Group),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->tiles.p, pl.tiles.data(), pl.tiles.size() * sizeof(Tile),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->items.p, pl.items.data(), pl.items.size() * sizeof(Item),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->order.p, pl.order.data(), pl.order.size() * sizeof(int),
                      cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(e, "wake plan upload");
  return WINDS_BS_OK;
}

// One induced-velocity evaluation of every case (nodes of `dom`, Γ, cores) at
// step *step + step_add; live_mode kLiveNodes or kLivePredicted (wake_live).
cudaError_t enqueue_eval(winds_wake_batch *b, const double *dom, const double *shed,
                         const double *trail, int step_add, const double *lold_s,
                         const double *lold_t, int have_old, double *lnew_s, double *lnew_t,
                         double *rc_s, double *rc_t, DevBuf &groups, int &launches,
                         int live_mode = kLiveNodes) {
  cudaStream_t s = b->stream;
  const WakeCase *cd = P<const WakeCase>(b->cases_d);
  const int *step = P<const int>(b->step_d);
  PackedFilaments pf{P<float4>(b->pk),
                     P<double4>(b->ra), P<double4>(b->rb)};
  BBox *bb = P<BBox>(b->bbox);
  GroupLive *live = P<GroupLive>(live_mode == kLivePredicted ? b->live_pred : b->live_main);
  cudaError_t e = launch_bbox_init(bb, s);
  if (e == cudaSuccess) e = launch_wake_live(cd, b->ncases, step, step_add, live_mode, live, s);
  if (e == cudaSuccess)
    e = launch_wake_filaments(cd, b->ncases, b->max_fil, step, step_add, P<const double>(b->ser),
                              dom, shed, trail, lold_s, lold_t, have_old, b->prm.stretch, lnew_s,
                              lnew_t, rc_s, rc_t, nullptr, nullptr, b->model, b->dcut, pf, bb, s);
  if (e == cudaSuccess)
    e = launch_wake_targets(cd, b->ncases, b->max_nodes, step, step_add, dom,
                            P<double4>(b->tp_raw), P<int>(b->tgroup), bb, s);
  unsigned long long *k0 = P<unsigned long long>(b->keys), *k1 = k0 + std::max<long long>(b->nodes, 1);
  if (e == cudaSuccess)
    e = launch_target_keys(P<const double4>(b->tp_raw), P<const int>(b->tgroup), b->nodes, bb, k0,
                           P<int>(b->vals), s);
  if (e == cudaSuccess)
    e = sort_target_keys(b->sort_tmp.p, &b->sort_bytes, k0, k1, P<const int>(b->vals),
                         P<int>(b->perm), b->nodes, s);
  if (e == cudaSuccess)
    e = launch_gather_targets(P<const double4>(b->tp_raw), P<const int>(b->perm), b->nodes,
                              P<double4>(b->tp), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->ctr.p, 0, sizeof(unsigned), s);
  F32cArgs a;
  a.pk = pf.pk;
  a.ra = pf.ra;
  a.rb = pf.rb;
  a.tp = P<const double4>(b->tp);
  a.groups = P<const Group>(groups);
  a.tiles = P<const Tile>(b->tiles);
  a.items = P<const Item>(b->items);
  a.order = P<const int>(b->order);
  a.n_items = b->n_items;
  a.tile_cap = b->tile_cap;
  a.part = P<double>(b->part);
  a.work_ctr = P<unsigned>(b->ctr);
  a.err = P<unsigned>(b->err);
  a.near_ctr = P<unsigned long long>(b->nearctr);
  a.bbox = bb;
  a.model = b->model;
  a.d = b->dcut;
  a.n = b->nidx;
  a.co = b->prm.co;
  a.wait_limit_ns = default_wait_limit_ns();
  a.live = live;
  if (e == cudaSuccess)
    e = b->prec == WINDS_PREC_F64 ? launch_f64(a, b->grid, s)
                                  : launch_f32c(a, b->model, b->ch.T, b->ch.KF, b->grid, s);
  if (e == cudaSuccess)
    e = launch_reduce(P<const Tile>(b->tiles), b->n_tiles, P<const Group>(groups),
                      P<const double>(b->part), P<const int>(b->perm), b->tile_cap, s,
                      P<const Item>(b->items), live);
  launches += 13;  // bbox, live, filaments, targets, keys, sort (4), gather, memset, sum, reduce
  return e;
}

cudaError_t enqueue_pre(winds_wake_batch *b, int &launches) {
  cudaStream_t s = b->stream;
  const WakeCase *cd = P<const WakeCase>(b->cases_d);
  const int *step = P<const int>(b->step_d);
  launches = 0;
  const bool pcc = b->prm.integrator == WINDS_INTEG_PCC;
  cudaError_t e = launch_wake_bookkeep(cd, b->ncases, b->max_cols, step, 0,
                                       P<const double>(b->bound), P<const double>(b->trail_prev),
                                       P<double>(b->shed_cur), P<double>(b->trail_cur), s);
  ++launches;
  // previous lengths exist from creation on (the initial lengths: zero strain
  // at step 0); the start-up's first stretching step is checked on the device
  if (e == cudaSuccess)
    e = enqueue_eval(b, P<const double>(b->dom), P<const double>(b->shed_cur),
                     P<const double>(b->trail_cur), 0, P<const double>(b->len_old_s),
                     P<const double>(b->len_old_t), 1, P<double>(b->len_s), P<double>(b->len_t),
                     P<double>(b->rc_s), P<double>(b->rc_t), b->groups_main, launches);
  int mode = kConvectFE;
  if (b->prm.integrator == WINDS_INTEG_AB2) mode = kConvectAB2;
  if (b->prm.integrator == WINDS_INTEG_AB4) mode = kConvectAB4;
  const double *carry = pcc && b->prm.pcc_double_add ? P<const double>(b->uind_pred) : nullptr;
  if (e == cudaSuccess)
    e = launch_wake_convect(cd, b->ncases, b->max_nodes, step, mode, P<const double>(b->dom),
                            P<const double>(b->uind), carry, nullptr, nullptr, P<double>(b->vel),
                            P<const double>(b->h1), P<const double>(b->h2), P<const double>(b->h3),
                            P<const double>(b->quarter), P<const double>(b->trailing),
                            P<const double>(b->wind), pcc ? P<double>(b->dom_pred) : P<double>(b->dom_new), s);
  ++launches;
  if (pcc) {
    if (e == cudaSuccess)
      e = launch_wake_bookkeep(cd, b->ncases, b->max_cols, step, 1, P<const double>(b->bound),
                               P<const double>(b->trail_cur), P<double>(b->shed_next),
                               P<double>(b->trail_next), s);
    ++launches;
    if (e == cudaSuccess)
      e = enqueue_eval(b, P<const double>(b->dom_pred), P<const double>(b->shed_next),
                       P<const double>(b->trail_next), 1, P<const double>(b->len_s),
                       P<const double>(b->len_t), 1, P<double>(b->len_ps), P<double>(b->len_pt),
                       nullptr, nullptr, b->groups_pred, launches, kLivePredicted);
    if (e == cudaSuccess)
      e = launch_wake_convect(cd, b->ncases, b->max_nodes, step, kConvectCorrector,
                              P<const double>(b->dom), nullptr, nullptr, P<const double>(b->dom_pred),
                              P<const double>(b->uind_pred), P<double>(b->vel), nullptr, nullptr,
                              nullptr, P<const double>(b->quarter), P<const double>(b->trailing),
                              P<const double>(b->wind), P<double>(b->dom_new), s);
    ++launches;
  }
  return e;
}

// End of step: (with lifting lines) Γ of the converged bound circulation,
// then the new positions and histories.
cudaError_t enqueue_post(winds_wake_batch *b, int &launches) {
  cudaStream_t s = b->stream;
  const WakeCase *cd = P<const WakeCase>(b->cases_d);
  cudaError_t e = cudaSuccess;
  if (b->kj) {
    e = launch_wake_bookkeep(cd, b->ncases, b->max_cols, P<const int>(b->step_d), 0,
                             P<const double>(b->bound), P<const double>(b->trail_prev),
                             P<double>(b->shed_cur), P<double>(b->trail_cur), s);
    ++launches;
    if (e == cudaSuccess && b->loads) {
      e = launch_kj_loads(cd, P<const KJCase>(b->kjc_d), b->ncases, b->max_st,
                          P<const int>(b->step_d), P<const double>(b->vblade),
                          P<const double>(b->cl_o), P<const double>(b->cd_o),
                          P<const double>(b->aoa_o), P<const double>(b->st_tw),
                          P<const double>(b->chord), P<const double>(b->st_rr),
                          P<const double>(b->st_dr), P<const double>(b->rpm),
                          P<const double>(b->pitch), P<double>(b->dl), P<double>(b->loads_out), s);
      launches += 2;
    }
  }
  const int keep_hist = b->prm.integrator == WINDS_INTEG_AB2 || b->prm.integrator == WINDS_INTEG_AB4;
  if (e == cudaSuccess)
    e = launch_wake_commit(cd, b->ncases, b->max_slots, P<int>(b->step_d), P<double>(b->dom),
                           P<const double>(b->dom_new), P<double>(b->vel), P<double>(b->h1),
                           P<double>(b->h2), P<double>(b->h3), keep_hist, P<double>(b->trail_prev),
                           P<const double>(b->trail_cur), P<double>(b->len_old_s),
                           P<const double>(b->len_s), P<double>(b->len_old_t),
                           P<const double>(b->len_t), s);
  ++launches;
  return e;
}

cudaError_t enqueue_step(winds_wake_batch *b, int &launches) {
  launches = 0;
  cudaError_t e = enqueue_pre(b, launches);
  int l2 = 0;
  if (e == cudaSuccess) e = enqueue_post(b, l2);
  launches += l2;
  return e;
}

// One Kutta-Joukowski iteration of every active case: Γ from the bound
// iterate, filaments with the step's cores, induced velocity at the lifting
// lines, station update and per-case convergence.
cudaError_t enqueue_kj_iter(winds_wake_batch *b, int &launches, cudaStream_t s,
                            const cudaGraphConditionalHandle *cond = nullptr) {
  const WakeCase *cd = P<const WakeCase>(b->cases_d);
  const KJCase *kd = P<const KJCase>(b->kjc_d);
  PackedFilaments pf{P<float4>(b->pk),
                     P<double4>(b->ra), P<double4>(b->rb)};
  BBox *bb = P<BBox>(b->bbox);
  // Γ of the bound iterate: columns 0-1 follow it (the others come from the
  // previous step); only those are recomputed and repacked (enqueue_kj_begin
  // did every column and every filament with the step's positions and cores)
  const int *step = P<const int>(b->step_d);
  cudaError_t e = launch_wake_bookkeep(cd, b->ncases, 2LL * b->max_nb, step, 0,
                                       P<const double>(b->bound), P<const double>(b->trail_prev),
                                       P<double>(b->shed_cur), P<double>(b->trail_cur), s, 2);
  if (e == cudaSuccess)
    e = launch_wake_filaments_bound_cols(cd, b->ncases, b->max_bound_cols, step,
                                         P<const double>(b->dom), P<const double>(b->shed_cur),
                                         P<const double>(b->trail_cur), P<const double>(b->rc_s),
                                         P<const double>(b->rc_t), b->model, b->dcut, pf, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->ctr.p, 0, sizeof(unsigned), s);
  F32cArgs a;
  a.pk = pf.pk;
  a.ra = pf.ra;
  a.rb = pf.rb;
  a.tp = P<const double4>(b->tp_ll);
  a.live = P<const GroupLive>(b->live_kj);
  a.groups = P<const Group>(b->kj_groups);
  a.tiles = P<const Tile>(b->kj_tiles);
  a.items = P<const Item>(b->kj_items);
  a.order = P<const int>(b->kj_order);
  a.n_items = b->kj_nitems;
  a.tile_cap = b->kj_tile_cap;
  a.part = P<double>(b->kj_part);
  a.work_ctr = P<unsigned>(b->ctr);
  a.err = P<unsigned>(b->err);
  a.near_ctr = P<unsigned long long>(b->nearctr);
  a.bbox = bb;
  a.model = b->model;
  a.d = b->dcut;
  a.n = b->nidx;
  a.co = b->prm.co;
  a.wait_limit_ns = default_wait_limit_ns();
  if (e == cudaSuccess)
    e = b->prec == WINDS_PREC_F64 || b->kjp.ll_fp64 ? launch_f64(a, b->kj_grid, s)
                                  : launch_f32c(a, b->model, b->kj_T, b->kj_KF, b->kj_grid, s);
  if (e == cudaSuccess)
    e = launch_reduce(P<const Tile>(b->kj_tiles), b->kj_ntiles, P<const Group>(b->kj_groups),
                      P<const double>(b->kj_part), P<const int>(b->perm_ll), b->kj_tile_cap, s,
                      P<const Item>(b->kj_items), P<const GroupLive>(b->live_kj));
  if (e == cudaSuccess)
    e = launch_kj_update(cd, kd, b->ncases, b->max_st, P<const int>(b->step_d),
                         P<const double>(b->uindb), P<const double>(b->bxn), P<const double>(b->byn),
                         P<const double>(b->bzn), P<const double>(b->vblade),
                         P<const double>(b->chord), P<const int>(b->foil), P<const int>(b->foil_off),
                         P<const double>(b->aoa_t), P<const double>(b->cl_t), P<const double>(b->cd_t),
                         b->kjp.relax, P<double>(b->bound), P<const int>(b->conv),
                         P<unsigned long long>(b->res_max), P<int>(b->diverged), P<double>(b->cl_o),
                         P<double>(b->cd_o), P<double>(b->aoa_o), s);
  if (e == cudaSuccess)
    e = cond ? launch_kj_check_cond(b->ncases, b->kjp.tol, P<int>(b->conv), P<int>(b->iters),
                                    P<unsigned long long>(b->res_max), P<double>(b->res_last),
                                    P<int>(b->active), P<int>(b->kj_it), b->kjp.maxiter, *cond, s)
             : launch_kj_check(b->ncases, b->kjp.tol, P<int>(b->conv), P<int>(b->iters),
                               P<unsigned long long>(b->res_max), P<double>(b->res_last),
                               P<int>(b->active), s);
  launches = 8;
  return e;
}

// Lifting-line targets and the per-step reset of the iteration state.
cudaError_t enqueue_kj_begin(winds_wake_batch *b) {
  cudaStream_t s = b->stream;
  cudaError_t e = launch_bbox_init(P<BBox>(b->bbox), s);
  // the step's live filaments; every lifting-line point is a target
  if (e == cudaSuccess)
    e = launch_wake_live(P<const WakeCase>(b->cases_d), b->ncases, P<const int>(b->step_d), 0,
                         kLiveAll, P<GroupLive>(b->live_kj), s);
  if (e == cudaSuccess)
    e = launch_kj_targets(P<const WakeCase>(b->cases_d), P<const KJCase>(b->kjc_d), b->ncases,
                          b->max_st, P<const int>(b->step_d), P<const double>(b->ll),
                          P<double4>(b->tp_ll), P<BBox>(b->bbox), s);
  for (DevBuf *x : {&b->conv, &b->iters, &b->diverged, &b->res_max})
    if (e == cudaSuccess) e = cudaMemsetAsync(x->p, 0, b->ncases * 8, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->kj_it.p, 0, sizeof(int), s);
  const WakeCase *cd = P<const WakeCase>(b->cases_d);
  const KJCase *kd = P<const KJCase>(b->kjc_d);
  if (e == cudaSuccess && b->mlp_inputs)
    e = launch_kj_features(cd, kd, b->ncases, b->max_st, P<const int>(b->step_d),
                           P<const double>(b->bound), P<const double>(b->bound_last),
                           P<const double>(b->bound_last2), P<const double>(b->vblade),
                           P<const double>(b->bxn), P<const double>(b->byn),
                           P<const double>(b->bzn), P<const double>(b->uindb),
                           P<const double>(b->st_r), P<const double>(b->st_c),
                           P<const double>(b->st_tw), P<const double>(b->azim), P<float>(b->feat),
                           s);
  // the history one step on, for the next step's change features
  if (e == cudaSuccess && b->mlp_inputs)
    e = cudaMemcpyAsync(b->bound_last2.p, b->bound_last.p, b->bound_n * sizeof(double),
                        cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && b->mlp_inputs)
    e = cudaMemcpyAsync(b->bound_last.p, b->bound.p, b->bound_n * sizeof(double),
                        cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess && b->mlp) {
    // start value Gamma_prev + out_scale * network(features)
    e = launch_mlp_prep(P<float>(b->feat), b->n_ll, kKJFeatures, mlp_shift_dev(b->mlp),
                        mlp_scale_dev(b->mlp), P<__nv_bfloat16>(b->mw.X), s);
    if (e == cudaSuccess &&
        mlp_forward(b->mlp, P<__nv_bfloat16>(b->mw.X), b->n_ll, b->mw, P<float>(b->mw.y), s))
      e = cudaErrorLaunchFailure;
    if (e == cudaSuccess)
      e = launch_kj_apply_guess(cd, kd, b->ncases, b->max_st, P<const int>(b->step_d),
                                P<const int>(b->st_lift), P<const double2>(b->st_stall),
                                P<const double>(b->aoa_o), P<const float>(b->mw.y),
                                mlp_out_scale_dev(b->mlp),
                                P<const float>(b->feat), mlp_base_dev(b->mlp), P<double>(b->bound),
                                s);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->guess.p, b->bound.p, b->bound_n * sizeof(double),
                        cudaMemcpyDeviceToDevice, s);
  // every filament at the step's positions with the step's cores held fixed
  // (as kj() does), Γ from the start value; the iterations repack only the
  // columns that follow the bound iterate
  if (e == cudaSuccess)
    e = launch_wake_bookkeep(cd, b->ncases, b->max_cols, P<const int>(b->step_d), 0,
                             P<const double>(b->bound), P<const double>(b->trail_prev),
                             P<double>(b->shed_cur), P<double>(b->trail_cur), s);
  if (e == cudaSuccess) {
    PackedFilaments pf{P<float4>(b->pk), P<double4>(b->ra), P<double4>(b->rb)};
    e = launch_wake_filaments(cd, b->ncases, b->max_fil, P<const int>(b->step_d), 0,
                              P<const double>(b->ser), P<const double>(b->dom),
                              P<const double>(b->shed_cur),
                              P<const double>(b->trail_cur), nullptr, nullptr, 0, 0, nullptr,
                              nullptr, nullptr, nullptr, P<const double>(b->rc_s),
                              P<const double>(b->rc_t), b->model, b->dcut, pf, P<BBox>(b->bbox), s);
  }
  return e;
}

int kj_step_errors(winds_wake_batch *b);

// One step as one graph: the part before the iteration, the lifting-line set-up,
// a conditional WHILE node whose body is one iteration (kj_check_cond ends it),
// then the commit. Built once, replayed every step.
int build_step_graph(winds_wake_batch *b) {
  cudaStream_t s = b->stream;
  cudaError_t e = cudaSuccess;
  if (!b->body_stream) e = cudaStreamCreateWithFlags(&b->body_stream, cudaStreamNonBlocking);
  int l1 = 0, l2 = 0, l3 = 0;
  cudaGraph_t g = nullptr;
  bool capturing = false;
  if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  capturing = e == cudaSuccess;
  if (e == cudaSuccess) e = enqueue_pre(b, l1);
  if (e == cudaSuccess) e = enqueue_kj_begin(b);
  cudaGraphConditionalHandle h = 0;
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) {
    cudaStreamCaptureStatus st;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    // no iteration at a step before the start-up's first (the condition is
    // reset to 1 at every launch of the graph)
    if (e == cudaSuccess && b->kj_from > 0) {
      e = launch_kj_gate_cond(P<const WakeCase>(b->cases_d), P<const int>(b->step_d), h, s);
      if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &ndeps);
      ++l1;
    }
    // zero-filled storage: the parameter union has no usable default constructor
    union NodeParams {
      cudaGraphNodeParams p;
      unsigned char raw[sizeof(cudaGraphNodeParams)];
      NodeParams() { std::memset(raw, 0, sizeof(raw)); }
      ~NodeParams() {}
    } np;
    cudaGraphNodeParams &cp = np.p;
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, ndeps, &cp);
    if (e == cudaSuccess)
      e = cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(b->body_stream, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t e2 = enqueue_kj_iter(b, l2, b->body_stream, &h);
        e = cudaStreamEndCapture(b->body_stream, &body);
        if (e2 != cudaSuccess) e = e2;
      }
    }
  }
  if (e == cudaSuccess) e = enqueue_post(b, l3);
  if (capturing) {
    cudaGraph_t done = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(s, &done);
    if (e == cudaSuccess) e = e2;
    g = done;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec_step, g, 0);
  if (e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    b->exec_step = nullptr;
    b->g_step = nullptr;
    cudaGetLastError();
    return cuda_fail(e, "step graph with conditional iteration");
  }
  b->g_step = g;
  b->step_launches = l1 + l2 + l3;
  return WINDS_BS_OK;
}

int run_kj(winds_wake_batch *b, bool use_graph) {
  if (b->steps_done < b->kj_from) {  // the start-up's first step has no iteration
    b->kj_evals = 0;
    return WINDS_BS_OK;
  }
  cudaError_t e = enqueue_kj_begin(b);
  if (e != cudaSuccess) return cuda_fail(e, "kj begin");
  if (use_graph && !b->exec_kj) {
    int l = 0;
    e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    cudaError_t e2 = e == cudaSuccess ? enqueue_kj_iter(b, l, b->stream) : e;
    e = cudaStreamEndCapture(b->stream, &b->g_kj);
    if (e2 != cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec_kj, b->g_kj, 0);
    if (e != cudaSuccess) return cuda_fail(e, "kj capture");
  }
  b->kj_evals = 0;
  int active = 1;
  for (int it = 0; it < b->kjp.maxiter && active; ++it) {
    int l = 0;
    e = use_graph ? cudaGraphLaunch(b->exec_kj, b->stream) : enqueue_kj_iter(b, l, b->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&active, b->active.p, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "kj iteration");
    ++b->kj_evals;
  }
  return kj_step_errors(b);
}

// After a step's iteration: NaN Cl anywhere, or an error word of the network.
int kj_step_errors(winds_wake_batch *b) {
  std::vector<int> div(b->ncases);
  cudaError_t e = cudaMemcpy(div.data(), b->diverged.p, b->ncases * sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "kj flags");
  for (int k = 0; k < b->ncases; ++k)
    if (div[k]) return fail(WINDS_BS_ERR_DIVERGED, "case %d: Diverging soln!!! (Cl is NaN)", k);
  if (b->mlp) {
    unsigned word = 0;
    e = cudaMemcpy(&word, mlp_err_word(b->mlp), sizeof(word), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "mlp error word");
    if (word) {
      cudaMemset(mlp_err_word(b->mlp), 0, sizeof(unsigned));
      return fail(word & kErrWaitTimeout ? WINDS_BS_ERR_TIMEOUT : WINDS_BS_ERR_CUDA,
                  "mlp kernels reported error word 0x%x", word);
    }
  }
  return WINDS_BS_OK;
}

// Interactions of step s over all cases and evaluations (the live columns'
// nodes against the live filaments; the pcc prediction from its first step).
long long step_interactions(const winds_wake_batch *b, long long s) {
  long long n = 0;
  for (const WakeCase &c : b->cases) {
    const int m = live_cols(c, s);
    n += (long long)c.nst * m * c.nb * live_filaments(c, m);
    if (b->prm.integrator == WINDS_INTEG_PCC && s >= b->pcc_from) {
      const int m1 = live_cols(c, s + 1);
      n += (long long)c.nst * m1 * c.nb * live_filaments(c, m1);
    }
  }
  return n;
}

}  // namespace

extern "C" {

int winds_wake_create(const winds_wake_case *cases, int ncases, const winds_wake_params *prm,
                      winds_wake_batch **out) {
  if (!out || !prm || ncases <= 0 || !cases) return fail(WINDS_BS_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  winds_bs_params bp;
  std::memset(&bp, 0, sizeof(bp));
  bp.core_model = prm->core_model;
  bp.d = prm->d;
  bp.co = prm->co;
  bp.precision = prm->precision;
  int model, prec, rc;
  double dcut, nidx;
  if ((rc = resolve_model(&bp, &model, &dcut, &nidx, &prec))) return rc;
  if (prm->integrator < WINDS_INTEG_FE || prm->integrator > WINDS_INTEG_PCC)
    return fail(WINDS_BS_ERR_ARG, "unknown integrator %d", prm->integrator);
  if (prm->startup != WINDS_STARTUP_FULL && prm->startup != WINDS_STARTUP_REFERENCE)
    return fail(WINDS_BS_ERR_ARG, "unknown start-up %d", prm->startup);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    return fail(WINDS_BS_ERR_NODEV, "no CUDA device is visible");
  winds_wake_batch *b = new winds_wake_batch();
  cudaGetDevice(&b->dev);
  b->ncases = ncases;
  b->prm = *prm;
  b->model = model;
  b->prec = prec;
  b->dcut = dcut;
  b->nidx = nidx;
  const bool ref_startup = prm->startup == WINDS_STARTUP_REFERENCE;
  // time index p = s + 1: corrector when p > 2 (pcc.m:40), stretching when
  // p > 3 (filamentmod.m:26), no iteration at p = 1 (initials.m)
  b->pcc_from = ref_startup ? 2 : 0;
  b->kj_from = ref_startup ? 1 : 0;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&b->ev0)) != cudaSuccess || (e = cudaEventCreate(&b->ev1)) != cudaSuccess) {
    delete b;
    return cuda_fail(e, "wake stream/events");
  }
  long long node = 0, sh = 0, tr = 0, bd = 0, fil = 0, kin = 0, wnd = 0, ser = 0;
  for (int k = 0; k < ncases; ++k) {
    const winds_wake_case &h = cases[k];
    if (h.nst < 2 || h.nb < 1 || h.na < 3 || h.nsteps < 2 || !(h.dt > 0) || !h.quarter ||
        !h.trailing || !h.wind || !h.dom || !h.bound || !h.trail_gamma) {
      winds_wake_destroy(b);
      return fail(WINDS_BS_ERR_ARG, "case %d: bad sizes or null arrays", k);
    }
    if (h.na_start != 0 && (h.na_start < 2 || h.na_start > h.na)) {
      winds_wake_destroy(b);
      return fail(WINDS_BS_ERR_ARG, "case %d: na_start %d outside 2..na (%d)", k, h.na_start, h.na);
    }
    WakeCase c;
    std::memset(&c, 0, sizeof(c));
    c.nst = h.nst, c.nb = h.nb, c.na = h.na, c.nsteps = h.nsteps;
    c.node_off = node, c.shed_off = sh, c.trail_off = tr, c.bound_off = bd, c.fil_off = fil;
    c.fil_count = (long long)(h.nst - 1) * h.na * h.nb + (long long)h.nst * (h.na - 1) * h.nb;
    c.fil_pad = (c.fil_count + kFilamentPad - 1) / kFilamentPad * kFilamentPad;
    c.kin_off = kin, c.wind_off = wnd;
    c.dt = h.dt, c.t0 = h.t0, c.shear = h.shear, c.hub = h.hub_height > 0 ? h.hub_height : 1.0;
    c.r0 = h.r0, c.rc0 = h.rc0, c.alpha = h.alpha, c.nu = h.nu, c.a1 = h.a1, c.delta = h.delta;
    c.core_mode = h.core_mode;
    c.na0 = h.na_start ? h.na_start : h.na;
    c.ser_off = ser;
    c.has_time = h.time != nullptr;
    c.has_r0 = h.r0_step != nullptr;
    c.pcc_from = b->pcc_from;
    c.stretch_from = ref_startup ? 3 : 0;
    c.kj_from = b->kj_from;
    ser += 2LL * h.nsteps;
    const long long nn = (long long)h.nst * h.na * h.nb;
    node += nn;
    sh += (long long)(h.nst - 1) * h.na * h.nb;
    tr += (long long)h.nst * (h.na - 1) * h.nb;
    bd += (long long)(h.nst - 1) * h.nb;
    fil += c.fil_pad;
    kin += (long long)h.nst * 3 * h.nsteps * h.nb;
    wnd += 3LL * h.nsteps;
    b->max_nodes = std::max(b->max_nodes, nn);
    b->max_cols = std::max<long long>(b->max_cols, (long long)h.na * h.nb);
    b->max_nb = std::max(b->max_nb, h.nb);
    b->max_fil = std::max(b->max_fil, c.fil_pad);
    b->max_slots = std::max(b->max_slots, nn);
    b->min_nsteps = k == 0 ? h.nsteps : std::min<long long>(b->min_nsteps, h.nsteps);
    b->cases.push_back(c);
  }
  b->nodes = node, b->shed_n = sh, b->trail_n = tr, b->bound_n = bd, b->fil_pad = fil;
  b->kin_n = kin, b->wind_n = wnd, b->ser_n = ser;
  b->interactions = step_interactions(b, 0);
  bool grows = false;
  for (const WakeCase &c : b->cases) grows = grows || c.na0 < c.na;
  if (fil > (1ll << 30) || node > (1ll << 30)) {
    winds_wake_destroy(b);
    return fail(WINDS_BS_ERR_ARG, "batch too large");
  }
  b->ch = default_choice(node);
  b->ch.waves = 32.0;
  // a growing wake's first steps are no sample of its work: default tiling
  if (prec == WINDS_PREC_F32C && !grows) b->tuned = lookup_tune(model, node, fil, &b->ch);
  if ((rc = alloc_all(b)) || (rc = build_plans(b))) {
    winds_wake_destroy(b);
    return rc;
  }
  // upload cases and initial state
  std::vector<double> tmp;
  e = cudaMemcpy(b->cases_d.p, b->cases.data(), ncases * sizeof(WakeCase), cudaMemcpyHostToDevice);
  for (int k = 0; k < ncases && e == cudaSuccess; ++k) {
    const winds_wake_case &h = cases[k];
    const WakeCase &c = b->cases[k];
    const long long nn = (long long)h.nst * h.na * h.nb;
    const long long nkin = (long long)h.nst * 3 * h.nsteps * h.nb;
    const long long ntr = (long long)h.nst * (h.na - 1) * h.nb;
    e = cudaMemcpy(P<double>(b->dom) + c.node_off * 3, h.dom, nn * 3 * sizeof(double),
                   cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(P<double>(b->bound) + c.bound_off, h.bound,
                     (size_t)(h.nst - 1) * h.nb * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(P<double>(b->quarter) + c.kin_off, h.quarter, nkin * sizeof(double),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(P<double>(b->trailing) + c.kin_off, h.trailing, nkin * sizeof(double),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(P<double>(b->wind) + c.wind_off, h.wind, 3 * h.nsteps * sizeof(double),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h.time)
      e = cudaMemcpy(P<double>(b->ser) + c.ser_off, h.time, h.nsteps * sizeof(double),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h.r0_step)
      e = cudaMemcpy(P<double>(b->ser) + c.ser_off + h.nsteps, h.r0_step,
                     h.nsteps * sizeof(double), cudaMemcpyHostToDevice);
    // the stored trailing columns are those of the step before: trail_prev(:,k) = trail(:,k+1)
    if (e == cudaSuccess) {
      tmp.assign(ntr, 0.0);
      const int m = h.na - 1;
      for (int bl = 0; bl < h.nb; ++bl)
        for (int j = 0; j + 1 < m; ++j)
          for (int i = 0; i < h.nst; ++i)
            tmp[i + (long long)h.nst * (j + (long long)m * bl)] =
                h.trail_gamma[i + (long long)h.nst * ((j + 1) + (long long)m * bl)];
      e = cudaMemcpy(P<double>(b->trail_prev) + c.trail_off, tmp.data(), ntr * sizeof(double),
                     cudaMemcpyHostToDevice);
    }
  }
  const size_t n3 = (size_t)b->nodes * 3 * sizeof(double);
  for (DevBuf *x : {&b->uind_pred, &b->vel, &b->h1, &b->h2, &b->h3, &b->uind, &b->dom_new, &b->dom_pred})
    if (e == cudaSuccess) e = cudaMemset(x->p, 0, n3);
  // no previous lengths yet: copying the initial lengths makes the first strain zero
  if (e == cudaSuccess) e = cudaMemset(b->step_d.p, 0, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(b->err.p, 0, 64);
  if (e != cudaSuccess) {
    winds_wake_destroy(b);
    return cuda_fail(e, "wake upload");
  }
  {
    // initial lengths = current lengths (zero strain at the first step)
    int l = 0;
    cudaError_t e2 = launch_wake_bookkeep(P<const WakeCase>(b->cases_d), b->ncases, b->max_cols,
                                          P<const int>(b->step_d), 0, P<const double>(b->bound),
                                          P<const double>(b->trail_prev), P<double>(b->shed_cur),
                                          P<double>(b->trail_cur), b->stream);
    if (e2 == cudaSuccess)
      e2 = enqueue_eval(b, P<const double>(b->dom), P<const double>(b->shed_cur),
                        P<const double>(b->trail_cur), 0, P<const double>(b->len_old_s),
                        P<const double>(b->len_old_t), 0, P<double>(b->len_old_s),
                        P<double>(b->len_old_t), nullptr, nullptr, b->groups_pred, l);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(b->stream);
    // that evaluation wrote the predicted-induction buffer: no carry at step 0
    if (e2 == cudaSuccess) e2 = cudaMemset(b->uind_pred.p, 0, n3);
    if (e2 != cudaSuccess) {
      winds_wake_destroy(b);
      return cuda_fail(e2, "wake initial lengths");
    }
  }
  *out = b;
  return WINDS_BS_OK;
}

static int device_error_word(winds_wake_batch *b);

// First-step tiling choice for an FP32c batch the cache has no entry for:
// times the main evaluation of this batch for T in {3, 4}, KF in {32, 64}
// and 32 or 64 items per resident worker, keeps the fastest (cached for the
// batch's size bucket) and rebuilds the plan. The evaluations only write
// per-step scratch (velocities, cores, lengths) that the first step rewrites.
static int autotune_batch(winds_wake_batch *b) {
  int rc;
  Context *c = get_context(&rc);
  if (!c) return rc;
  b->tuned = true;
  if (!c->autotune) return build_plans(b);
  cudaStream_t s = b->stream;
  cudaError_t e = launch_wake_bookkeep(P<const WakeCase>(b->cases_d), b->ncases, b->max_cols,
                                       P<const int>(b->step_d), 0, P<const double>(b->bound),
                                       P<const double>(b->trail_prev), P<double>(b->shed_cur),
                                       P<double>(b->trail_cur), s);
  if (e != cudaSuccess) return cuda_fail(e, "autotune bookkeeping");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  TuneChoice best = b->ch;
  float best_ms = 1e30f;
  for (int T : {3, 4})
    for (int KF : {32, 64})
      for (double w : {32.0, 64.0}) {
        b->ch.T = T, b->ch.KF = KF, b->ch.waves = w;
        if ((rc = build_plans(b))) break;
        float ms = 0.f;
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {  // warm-up, then timed
          int l = 0;
          cudaEventRecord(e0, s);
          e = enqueue_eval(b, P<const double>(b->dom), P<const double>(b->shed_cur),
                           P<const double>(b->trail_cur), 0, P<const double>(b->len_old_s),
                           P<const double>(b->len_old_t), 1, P<double>(b->len_s),
                           P<double>(b->len_t), P<double>(b->rc_s), P<double>(b->rc_t),
                           b->groups_main, l);
          cudaEventRecord(e1, s);
          if (e == cudaSuccess) e = cudaEventSynchronize(e1);
          cudaEventElapsedTime(&ms, e0, e1);
        }
        if (e != cudaSuccess) break;
        if (ms < best_ms) best_ms = ms, best = b->ch;
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "wake autotune");
  if ((rc = device_error_word(b))) return rc;
  b->ch = best;
  store_tune(b->model, b->nodes, b->fil_pad, best);
  return build_plans(b);
}

// Error word of the direct-sum kernels (bounded waits that ran out).
static int device_error_word(winds_wake_batch *b) {
  unsigned word = 0;
  cudaError_t e = cudaMemcpy(&word, b->err.p, sizeof(word), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "error word read");
  if (word) {
    cudaMemset(b->err.p, 0, sizeof(unsigned));
    return fail(word & kErrWaitTimeout ? WINDS_BS_ERR_TIMEOUT : WINDS_BS_ERR_CUDA,
                "device reported error word 0x%x", word);
  }
  return WINDS_BS_OK;
}

static int step_impl(winds_wake_batch *b, int nsteps, int use_graph);

int winds_wake_step(winds_wake_batch *b, int nsteps, int use_graph) {
  if (!b || nsteps < 0) return fail(WINDS_BS_ERR_ARG, "bad step arguments");
  const long long s0 = b->steps_done;
  const int rc = step_impl(b, nsteps, use_graph);
  if (rc == WINDS_BS_OK && b->steps_done > s0) {
    long long n = 0;
    for (long long s = s0; s < b->steps_done; ++s) n += step_interactions(b, s);
    b->interactions = n / (b->steps_done - s0);
  }
  return rc;
}

int winds_wake_get_live(winds_wake_batch *b, int icase, int *na_live, long long *steps_done) {
  if (!b || icase < 0 || icase >= b->ncases) return fail(WINDS_BS_ERR_ARG, "bad case index");
  if (na_live) *na_live = live_cols(b->cases[icase], b->steps_done);
  if (steps_done) *steps_done = b->steps_done;
  return WINDS_BS_OK;
}

static int step_impl(winds_wake_batch *b, int nsteps, int use_graph) {
  if (b->steps_done + nsteps >= b->min_nsteps)
    return fail(WINDS_BS_ERR_ARG, "kinematics cover %lld steps; %lld done, %d more requested",
                b->min_nsteps - 1, b->steps_done, nsteps);
  cudaSetDevice(b->dev);
  if (!b->tuned && nsteps > 0) {
    int rc = autotune_batch(b);
    if (rc) return rc;
  }
  cudaError_t e = cudaSuccess;
  if (b->kj && use_graph && b->cond_ok) {
    // the whole step, iteration included, as one graph: one round trip per step
    if (!b->exec_step && build_step_graph(b) != WINDS_BS_OK) b->cond_ok = false;
  }
  if (b->kj && use_graph && b->exec_step) {
    b->launches = b->step_launches;
    cudaEventRecord(b->ev0, b->stream);
    for (int k = 0; k < nsteps; ++k) {
      e = cudaGraphLaunch(b->exec_step, b->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
      if (e != cudaSuccess) return cuda_fail(e, "wake step");
      int rc = kj_step_errors(b);
      if (!rc) rc = device_error_word(b);
      if (rc) return rc;
      ++b->steps_done;
      int it = 0;
      if ((e = cudaMemcpy(&it, b->kj_it.p, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "iteration count");
      b->kj_evals = it;
    }
    cudaEventRecord(b->ev1, b->stream);
    b->timed_steps = nsteps;
    e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "wake step sync");
  }
  if (b->kj) {
    // pre-commit part, the iteration (host loop on a device convergence flag), commit
    for (int k = 0; k < nsteps; ++k) {
      if (use_graph && !b->exec_pre) {
        int l1 = 0, l2 = 0;
        e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        cudaError_t e2 = e == cudaSuccess ? enqueue_pre(b, l1) : e;
        e = cudaStreamEndCapture(b->stream, &b->g_pre);
        if (e2 != cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec_pre, b->g_pre, 0);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        e2 = e == cudaSuccess ? enqueue_post(b, l2) : e;
        if (e == cudaSuccess) e = cudaStreamEndCapture(b->stream, &b->g_post);
        if (e2 != cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec_post, b->g_post, 0);
        b->launches = l1 + l2;
        if (e != cudaSuccess) return cuda_fail(e, "wake step capture");
      }
      if (k == 0) cudaEventRecord(b->ev0, b->stream);
      int l = 0;
      e = use_graph ? cudaGraphLaunch(b->exec_pre, b->stream) : enqueue_pre(b, l);
      if (e != cudaSuccess) return cuda_fail(e, "wake step");
      int rc = run_kj(b, use_graph != 0);
      if (!rc) rc = device_error_word(b);
      if (rc) return rc;
      int l2 = 0;
      e = use_graph ? cudaGraphLaunch(b->exec_post, b->stream) : enqueue_post(b, l2);
      if (!use_graph) b->launches = l + l2;
      if (e != cudaSuccess) return cuda_fail(e, "wake step commit");
    }
    b->timed_steps = nsteps;
    if (nsteps > 0) cudaEventRecord(b->ev1, b->stream);
    b->steps_done += nsteps;
    e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "wake step sync");
    return device_error_word(b);
  }
  if (use_graph && !b->exec && nsteps > 0) {
    // capture one step (launches nothing) before the timed steps
    e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    int l = 0;
    cudaError_t e2 = e == cudaSuccess ? enqueue_step(b, l) : e;
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->stream, &g);
    if (e2 != cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
    b->graph = g;
    b->launches = l;
    if (e != cudaSuccess) return cuda_fail(e, "wake step capture");
  }
  b->timed_steps = nsteps;
  if (nsteps > 0) cudaEventRecord(b->ev0, b->stream);
  for (int k = 0; k < nsteps && e == cudaSuccess; ++k) {
    if (use_graph) {
      e = cudaGraphLaunch(b->exec, b->stream);
    } else {
      e = enqueue_step(b, b->launches);
    }
  }
  if (nsteps > 0) cudaEventRecord(b->ev1, b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wake step");
  b->steps_done += nsteps;
  e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "wake step sync");
  return device_error_word(b);
}

int winds_wake_get_state(winds_wake_batch *b, int icase, double *dom, double *bound, double *shed,
                         double *trail, double *rc_shed, double *rc_trail, double *uind) {
  if (!b || icase < 0 || icase >= b->ncases) return fail(WINDS_BS_ERR_ARG, "bad case index");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  const WakeCase &c = b->cases[icase];
  const size_t nn = (size_t)c.nst * c.na * c.nb, ns = (size_t)(c.nst - 1) * c.na * c.nb,
               nt = (size_t)c.nst * (c.na - 1) * c.nb, nbd = (size_t)(c.nst - 1) * c.nb;
  cudaError_t e = cudaSuccess;
  auto get = [&](double *dst, DevBuf &src, long long off, size_t n) {
    if (dst && e == cudaSuccess)
      e = cudaMemcpy(dst, P<double>(src) + off, n * sizeof(double), cudaMemcpyDeviceToHost);
  };
  get(dom, b->dom, c.node_off * 3, nn * 3);
  get(bound, b->bound, c.bound_off, nbd);
  get(shed, b->shed_cur, c.shed_off, ns);
  get(trail, b->trail_cur, c.trail_off, nt);
  get(rc_shed, b->rc_s, c.shed_off, ns);
  get(rc_trail, b->rc_t, c.trail_off, nt);
  get(uind, b->uind, c.node_off * 3, nn * 3);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "wake state read");
}

int winds_wake_set_bound(winds_wake_batch *b, int icase, const double *bound) {
  if (!b || icase < 0 || icase >= b->ncases || !bound) return fail(WINDS_BS_ERR_ARG, "bad arguments");
  cudaSetDevice(b->dev);
  const WakeCase &c = b->cases[icase];
  cudaError_t e = cudaMemcpyAsync(P<double>(b->bound) + c.bound_off, bound,
                                  (size_t)(c.nst - 1) * c.nb * sizeof(double),
                                  cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "bound upload");
}

int winds_wake_stats(winds_wake_batch *b, double *step_ms, long long *interactions,
                     int *launches_per_step) {
  if (!b) return fail(WINDS_BS_ERR_ARG, "null batch");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  if (step_ms) {
    float ms = 0.f;
    if (b->timed_steps > 0) cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    *step_ms = b->timed_steps > 0 ? ms / b->timed_steps : 0.0;
  }
  if (interactions) *interactions = b->interactions;
  if (launches_per_step) *launches_per_step = b->launches;
  return WINDS_BS_OK;
}

int winds_wake_set_kj(winds_wake_batch *b, const winds_kj_case *kj, const winds_kj_params *prm) {
  if (!b || !kj || !prm || !(prm->relax > 0) || !(prm->tol >= 0) || prm->maxiter < 1)
    return fail(WINDS_BS_ERR_ARG, "bad lifting-line arguments");
  if (b->ncases > 1024) return fail(WINDS_BS_ERR_ARG, "at most 1024 cases with lifting lines");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  // graphs captured for an earlier attachment describe other buffers
  for (cudaGraphExec_t *x : {&b->exec_pre, &b->exec_kj, &b->exec_post, &b->exec_step})
    if (*x) cudaGraphExecDestroy(*x), *x = nullptr;
  for (cudaGraph_t *x : {&b->g_pre, &b->g_kj, &b->g_post, &b->g_step})
    if (*x) cudaGraphDestroy(*x), *x = nullptr;
  cudaStream_t s = b->stream;
  b->kjp = *prm;
  b->kjc.clear();
  long long fr = 0, tt = 0, st = 0, tab = 0, az = 0, rp = 0;
  bool all_inputs = true, have_twist = true, all_loads = true, any_pitch = false;
  std::vector<int> foil_off, foils, lift;
  std::vector<double2> stall;
  std::vector<double> aoa, cl, cd, chord;
  b->max_st = 0;
  b->max_bound_cols = 0;
  for (int k = 0; k < b->ncases; ++k) {
    const WakeCase &c = b->cases[k];
    const winds_kj_case &h = kj[k];
    const int ns = c.nst - 1;
    if (!h.ll || !h.bxn || !h.byn || !h.bzn || !h.vblade || !h.chord || !h.foil || h.n_foils < 1 ||
        !h.foil_points || !h.aoa || !h.cl || !h.cd)
      return fail(WINDS_BS_ERR_ARG, "case %d: null lifting-line array", k);
    KJCase q;
    q.frame_off = fr;
    q.t_off = tt;
    q.station_off = st;
    q.az_off = az;
    if (!h.r_over_R || !h.chord_over_R || !h.twist || !h.azimuth) all_inputs = false;
    if (!h.twist) have_twist = false;
    if (!h.r_station || !h.dr_station || !h.rpm || !(h.rho > 0)) all_loads = false;
    q.rpm_off = rp;
    q.rho = h.rho;
    q.has_pitch = h.pitch != nullptr;
    any_pitch = any_pitch || h.pitch;
    q.foil_base = (int)foil_off.size();
    q.n_foils = h.n_foils;
    long long o = 0;
    for (int f = 0; f < h.n_foils; ++f) {
      if (h.foil_points[f] < 2) return fail(WINDS_BS_ERR_ARG, "case %d: airfoil %d has < 2 points", k, f);
      foil_off.push_back((int)(tab + o));
      o += h.foil_points[f];
    }
    foil_off.push_back((int)(tab + o));
    for (long long j = 0; j < o; ++j) {
      aoa.push_back(h.aoa[j]);
      cl.push_back(h.cl[j]);
      cd.push_back(h.cd[j]);
    }
    // tables with lift (some Cl != 0); a station on a table without keeps its
    // previous circulation as the start value
    // and the stall bounds of each table: the AoA of its highest Cl above
    // 0 deg and of its lowest Cl below (within +-45 deg)
    std::vector<int> has_lift(h.n_foils, 0);
    std::vector<double2> bounds(h.n_foils);
    for (int f = 0, j = 0; f < h.n_foils; ++f) {
      double hi_cl = -1e300, lo_cl = 1e300, hi_a = 45.0, lo_a = -45.0;
      for (int e = 0; e < h.foil_points[f]; ++e, ++j) {
        if (h.cl[j] != 0.0) has_lift[f] = 1;
        const double a = h.aoa[j];
        if (a >= 0.0 && a <= 45.0 && h.cl[j] > hi_cl) hi_cl = h.cl[j], hi_a = a;
        if (a <= 0.0 && a >= -45.0 && h.cl[j] < lo_cl) lo_cl = h.cl[j], lo_a = a;
      }
      bounds[f] = make_double2(lo_a, hi_a);
    }
    for (int i = 0; i < ns; ++i) {
      if (h.foil[i] < 0 || h.foil[i] >= h.n_foils)
        return fail(WINDS_BS_ERR_ARG, "case %d: station %d uses airfoil %d of %d", k, i, h.foil[i], h.n_foils);
      foils.push_back(h.foil[i]);
      lift.push_back(has_lift[h.foil[i]]);
      stall.push_back(bounds[h.foil[i]]);
      chord.push_back(h.chord[i]);
    }
    tab += o;
    az += (long long)c.nsteps * c.nb;
    rp += c.nsteps;
    fr += (long long)ns * 3 * c.nsteps * c.nb;
    tt += (long long)ns * c.nb;
    st += ns;
    b->max_st = std::max(b->max_st, ns * c.nb);
    b->max_bound_cols = std::max<long long>(b->max_bound_cols, (long long)c.nb * (2 * ns + c.nst));
    b->kjc.push_back(q);
  }
  b->frames_n = fr, b->n_ll = tt, b->stations_n = st;
  int rc;
  for (DevBuf *x : {&b->ll, &b->bxn, &b->byn, &b->bzn, &b->vblade})
    if ((rc = x->ensure(fr * sizeof(double), s))) return rc;
  if ((rc = b->kjc_d.ensure(b->ncases * sizeof(KJCase), s)) ||
      (rc = b->chord.ensure(st * sizeof(double), s)) || (rc = b->foil.ensure(st * sizeof(int), s)) ||
      (rc = b->st_lift.ensure(st * sizeof(int), s)) ||
      (rc = b->st_stall.ensure(st * sizeof(double2), s)) ||
      (rc = b->foil_off.ensure(foil_off.size() * sizeof(int), s)) ||
      (rc = b->aoa_t.ensure(tab * sizeof(double), s)) || (rc = b->cl_t.ensure(tab * sizeof(double), s)) ||
      (rc = b->cd_t.ensure(tab * sizeof(double), s)) || (rc = b->tp_ll.ensure(tt * sizeof(double4), s)) ||
      (rc = b->perm_ll.ensure(tt * sizeof(int), s)) || (rc = b->uindb.ensure(tt * 3 * sizeof(double), s)))
    return rc;
  for (DevBuf *x : {&b->conv, &b->iters, &b->diverged, &b->res_max, &b->res_last, &b->active})
    if ((rc = x->ensure(std::max(b->ncases, 1) * 8 + 8, s))) return rc;
  if ((rc = b->kj_it.ensure(16, s))) return rc;
  for (DevBuf *x : {&b->cl_o, &b->cd_o, &b->aoa_o, &b->guess, &b->bound_last, &b->bound_last2})
    if ((rc = x->ensure(b->bound_n * sizeof(double), s))) return rc;
  // defined values before any iteration (a step without one reads them)
  for (DevBuf *x : {&b->conv, &b->iters, &b->diverged, &b->res_max, &b->res_last, &b->active})
    if (cudaError_t e0 = cudaMemset(x->p, 0, std::max(b->ncases, 1) * 8 + 8); e0 != cudaSuccess)
      return cuda_fail(e0, "lifting-line counters");
  for (DevBuf *x : {&b->cl_o, &b->cd_o, &b->aoa_o})
    if (cudaError_t e0 = cudaMemset(x->p, 0, b->bound_n * sizeof(double)); e0 != cudaSuccess)
      return cuda_fail(e0, "lifting-line outputs");
  // no change before the first step
  for (DevBuf *x : {&b->bound_last, &b->bound_last2})
    if (cudaError_t e0 = cudaMemcpy(x->p, b->bound.p, b->bound_n * sizeof(double),
                                    cudaMemcpyDeviceToDevice);
        e0 != cudaSuccess)
      return cuda_fail(e0, "bound copy");
  all_loads = all_loads && have_twist;
  b->mlp_inputs = all_inputs;
  b->loads = all_loads;
  if (have_twist) {
    if ((rc = b->st_tw.ensure(st * sizeof(double), s))) return rc;
    for (int k = 0; k < b->ncases; ++k) {
      cudaError_t e2 = cudaMemcpy(P<double>(b->st_tw) + b->kjc[k].station_off, kj[k].twist,
                                  (size_t)(b->cases[k].nst - 1) * 8, cudaMemcpyHostToDevice);
      if (e2 != cudaSuccess) return cuda_fail(e2, "twist upload");
    }
  }
  if (all_loads) {
    if ((rc = b->st_rr.ensure(st * sizeof(double), s)) || (rc = b->st_dr.ensure(st * sizeof(double), s)) ||
        (rc = b->rpm.ensure(rp * sizeof(double), s)) ||
        (rc = b->dl.ensure(std::max<long long>(tt, 1) * 3 * sizeof(double), s)) ||
        (rc = b->loads_out.ensure(std::max(b->ncases, 1) * 3 * sizeof(double), s)))
      return rc;
    for (int k = 0; k < b->ncases; ++k) {
      const size_t ns = (size_t)(b->cases[k].nst - 1), so = (size_t)b->kjc[k].station_off;
      cudaError_t e2 = cudaMemcpy(P<double>(b->st_rr) + so, kj[k].r_station, ns * 8, cudaMemcpyHostToDevice);
      if (e2 == cudaSuccess) e2 = cudaMemcpy(P<double>(b->st_dr) + so, kj[k].dr_station, ns * 8, cudaMemcpyHostToDevice);
      if (e2 == cudaSuccess)
        e2 = cudaMemcpy(P<double>(b->rpm) + b->kjc[k].rpm_off, kj[k].rpm,
                        (size_t)b->cases[k].nsteps * 8, cudaMemcpyHostToDevice);
      if (e2 != cudaSuccess) return cuda_fail(e2, "loads upload");
    }
    if ((rc = b->pitch.ensure(std::max<long long>(az, 1) * sizeof(double), s))) return rc;
    for (int k = 0; k < b->ncases && any_pitch; ++k) {
      if (!kj[k].pitch) continue;
      const WakeCase &c = b->cases[k];
      cudaError_t e2 = cudaMemcpy(P<double>(b->pitch) + b->kjc[k].az_off, kj[k].pitch,
                                  (size_t)c.nsteps * c.nb * 8, cudaMemcpyHostToDevice);
      if (e2 != cudaSuccess) return cuda_fail(e2, "pitch upload");
    }
    if (cudaError_t e0 = cudaMemset(b->loads_out.p, 0, b->ncases * 3 * sizeof(double)); e0 != cudaSuccess)
      return cuda_fail(e0, "loads reset");
  }
  // no induced velocity at the lifting line before the first step
  if (cudaError_t e0 = cudaMemset(b->uindb.p, 0, tt * 3 * sizeof(double)); e0 != cudaSuccess)
    return cuda_fail(e0, "lifting-line reset");
  if (all_inputs) {
    if ((rc = b->feat.ensure(std::max<long long>(tt, 1) * kKJFeatures * sizeof(float), s))) return rc;
    if ((rc = b->st_r.ensure(st * sizeof(double), s)) || (rc = b->st_c.ensure(st * sizeof(double), s)) ||
        (rc = b->azim.ensure(az * sizeof(double), s)))
      return rc;
    for (int k = 0; k < b->ncases; ++k) {
      const WakeCase &c = b->cases[k];
      const size_t ns = (size_t)(c.nst - 1);
      const size_t so = (size_t)b->kjc[k].station_off, ao = (size_t)b->kjc[k].az_off;
      cudaError_t e2 = cudaMemcpy(P<double>(b->st_r) + so, kj[k].r_over_R, ns * 8, cudaMemcpyHostToDevice);
      if (e2 == cudaSuccess) e2 = cudaMemcpy(P<double>(b->st_c) + so, kj[k].chord_over_R, ns * 8, cudaMemcpyHostToDevice);
      if (e2 == cudaSuccess)
        e2 = cudaMemcpy(P<double>(b->azim) + ao, kj[k].azimuth, (size_t)c.nsteps * c.nb * 8, cudaMemcpyHostToDevice);
      if (e2 != cudaSuccess) return cuda_fail(e2, "mlp station upload");
    }
  } else {
    b->mlp = nullptr;
  }
  cudaError_t e = cudaMemcpy(b->kjc_d.p, b->kjc.data(), b->ncases * sizeof(KJCase), cudaMemcpyHostToDevice);
  for (int k = 0; k < b->ncases && e == cudaSuccess; ++k) {
    const WakeCase &c = b->cases[k];
    const long long n = (long long)(c.nst - 1) * 3 * c.nsteps * c.nb;
    const long long off = b->kjc[k].frame_off;
    const double *src[5] = {kj[k].ll, kj[k].bxn, kj[k].byn, kj[k].bzn, kj[k].vblade};
    DevBuf *dst[5] = {&b->ll, &b->bxn, &b->byn, &b->bzn, &b->vblade};
    for (int a = 0; a < 5 && e == cudaSuccess; ++a)
      e = cudaMemcpy(P<double>(*dst[a]) + off, src[a], n * sizeof(double), cudaMemcpyHostToDevice);
  }
  std::vector<int> ident(std::max<long long>(tt, 1));
  for (long long i = 0; i < tt; ++i) ident[i] = (int)i;
  if (e == cudaSuccess) e = cudaMemcpy(b->chord.p, chord.data(), st * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->foil.p, foils.data(), st * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->st_lift.p, lift.data(), st * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->st_stall.p, stall.data(), st * sizeof(double2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->foil_off.p, foil_off.data(), foil_off.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->aoa_t.p, aoa.data(), tab * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->cl_t.p, cl.data(), tab * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->cd_t.p, cd.data(), tab * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->perm_ll.p, ident.data(), tt * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "lifting-line upload");
  // plan: each case's lifting-line points against its filaments
  std::vector<GroupSpec> gs;
  for (int k = 0; k < b->ncases; ++k) {
    const WakeCase &c = b->cases[k];
    GroupSpec g;
    g.out = P<double>(b->uindb) + 3 * b->kjc[k].t_off;
    g.t_begin = b->kjc[k].t_off;
    g.t_count = (long long)(c.nst - 1) * c.nb;
    g.ns_p = c.nst - 1;
    g.f_begin = (int)c.fil_off;
    g.f_end = (int)(c.fil_off + c.fil_pad);
    g.accumulate = 0;
    gs.push_back(g);
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
  int resident, quantum;
  if (b->prec == WINDS_PREC_F64 || b->kjp.ll_fp64) {
    b->kj_tile_cap = f64_threads();
    resident = f64_occupancy() * sms;
    quantum = f64_tile();
  } else {
    b->kj_tile_cap = f32c_threads() * b->kj_T;
    resident = f32c_occupancy(b->model, b->kj_T, b->kj_KF) * sms;
    quantum = kFilamentPad;
  }
  Plan pl;
  build_plan(pl, gs, b->kj_tile_cap, resident, 4.0, quantum);
  b->kj_ntiles = (int)pl.tiles.size();
  b->kj_nitems = (int)pl.items.size();
  b->kj_grid = std::max(1, std::min(b->kj_nitems, resident));
  if ((rc = b->kj_groups.ensure(pl.groups.size() * sizeof(Group), s)) ||
      (rc = b->kj_tiles.ensure(pl.tiles.size() * sizeof(Tile), s)) ||
      (rc = b->kj_items.ensure(pl.items.size() * sizeof(Item), s)) ||
      (rc = b->kj_order.ensure(pl.order.size() * sizeof(int), s)) ||
      (rc = b->kj_part.ensure((size_t)b->kj_nitems * 3 * b->kj_tile_cap * sizeof(double), s)))
    return rc;
  if ((e = cudaMemcpy(b->kj_groups.p, pl.groups.data(), pl.groups.size() * sizeof(Group), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->kj_tiles.p, pl.tiles.data(), pl.tiles.size() * sizeof(Tile), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->kj_items.p, pl.items.data(), pl.items.size() * sizeof(Item), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(b->kj_order.p, pl.order.data(), pl.order.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess)
    return cuda_fail(e, "lifting-line plan upload");
  // graphs captured without the iteration must be rebuilt
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  b->kj = true;
  return WINDS_BS_OK;
}

int winds_wake_set_mlp(winds_wake_batch *b, winds_mlp *m) {
  if (!b || !b->kj) return fail(WINDS_BS_ERR_ARG, "attach lifting lines before the MLP");
  // a captured step holds (or lacks) the network's launches
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  if (b->exec_step) cudaGraphExecDestroy(b->exec_step), b->exec_step = nullptr;
  if (b->g_step) cudaGraphDestroy(b->g_step), b->g_step = nullptr;
  if (!m) {
    b->mlp = nullptr;
    return WINDS_BS_OK;
  }
  if (!b->mlp_inputs)
    return fail(WINDS_BS_ERR_ARG, "every lifting line needs r_over_R, chord_over_R, twist, azimuth");
  if (mlp_n_in(m) != kKJFeatures)
    return fail(WINDS_BS_ERR_ARG, "the MLP has %d inputs, the start value uses %d", mlp_n_in(m),
                kKJFeatures);
  if (mlp_device(m) != b->dev) return fail(WINDS_BS_ERR_ARG, "MLP and batch on different devices");
  cudaSetDevice(b->dev);
  int rc = b->mw.ensure(std::max<long long>(b->n_ll, 1), false, b->stream);
  if (rc) return rc;
  b->mlp = m;
  return WINDS_BS_OK;
}

int winds_wake_get_kj_features(winds_wake_batch *b, int icase, float *x) {
  if (!b || !b->kj || !b->mlp_inputs || icase < 0 || icase >= b->ncases || !x)
    return fail(WINDS_BS_ERR_ARG, "no lifting-line features");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  const WakeCase &c = b->cases[icase];
  cudaError_t e = cudaMemcpy(x, P<float>(b->feat) + b->kjc[icase].t_off * kKJFeatures,
                             (size_t)(c.nst - 1) * c.nb * kKJFeatures * sizeof(float),
                             cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "feature read");
}

int winds_wake_get_loads(winds_wake_batch *b, double *thrust, double *torque, double *power) {
  if (!b || !b->kj || !b->loads) return fail(WINDS_BS_ERR_ARG, "no loads inputs attached");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  std::vector<double> h((size_t)b->ncases * 3);
  cudaError_t e = cudaMemcpy(h.data(), b->loads_out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "loads read");
  for (int k = 0; k < b->ncases; ++k) {
    if (thrust) thrust[k] = h[3 * k];
    if (torque) torque[k] = h[3 * k + 1];
    if (power) power[k] = h[3 * k + 2];
  }
  return WINDS_BS_OK;
}

int winds_wake_get_kj_guess(winds_wake_batch *b, int icase, double *guess) {
  if (!b || !b->kj || icase < 0 || icase >= b->ncases || !guess)
    return fail(WINDS_BS_ERR_ARG, "bad arguments");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  const WakeCase &c = b->cases[icase];
  cudaError_t e = cudaMemcpy(guess, P<double>(b->guess) + c.bound_off,
                             (size_t)(c.nst - 1) * c.nb * sizeof(double), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "guess read");
}

int winds_wake_kj_stats(winds_wake_batch *b, int *iterations, double *residual,
                        long long *ll_evaluations) {
  if (!b || !b->kj) return fail(WINDS_BS_ERR_ARG, "no lifting lines attached");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  cudaError_t e = cudaSuccess;
  if (iterations) e = cudaMemcpy(iterations, b->iters.p, b->ncases * sizeof(int), cudaMemcpyDeviceToHost);
  if (residual && e == cudaSuccess)
    e = cudaMemcpy(residual, b->res_last.p, b->ncases * sizeof(double), cudaMemcpyDeviceToHost);
  if (ll_evaluations) *ll_evaluations = b->kj_evals;
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "kj stats");
}

int winds_wake_get_perf(winds_wake_batch *b, int icase, double *cl, double *cd, double *aoa) {
  if (!b || !b->kj || icase < 0 || icase >= b->ncases) return fail(WINDS_BS_ERR_ARG, "bad arguments");
  cudaSetDevice(b->dev);
  cudaStreamSynchronize(b->stream);
  const WakeCase &c = b->cases[icase];
  const size_t n = (size_t)(c.nst - 1) * c.nb;
  cudaError_t e = cudaSuccess;
  if (cl) e = cudaMemcpy(cl, P<double>(b->cl_o) + c.bound_off, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (cd && e == cudaSuccess) e = cudaMemcpy(cd, P<double>(b->cd_o) + c.bound_off, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (aoa && e == cudaSuccess) e = cudaMemcpy(aoa, P<double>(b->aoa_o) + c.bound_off, n * sizeof(double), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? WINDS_BS_OK : cuda_fail(e, "perf read");
}

void winds_wake_destroy(winds_wake_batch *b) {
  if (!b) return;
  cudaSetDevice(b->dev);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaGraphExec_t x : {b->exec_pre, b->exec_kj, b->exec_post, b->exec_step})
    if (x) cudaGraphExecDestroy(x);
  for (cudaGraph_t x : {b->g_pre, b->g_kj, b->g_post, b->g_step})
    if (x) cudaGraphDestroy(x);
  if (b->body_stream) cudaStreamDestroy(b->body_stream);
  b->kj_it.release();
  b->st_lift.release();
  b->st_stall.release();
  for (DevBuf *x : {&b->kjc_d, &b->ll, &b->bxn, &b->byn, &b->bzn, &b->vblade, &b->chord, &b->foil,
                    &b->foil_off, &b->aoa_t, &b->cl_t, &b->cd_t, &b->tp_ll, &b->perm_ll, &b->uindb,
                    &b->kj_groups, &b->kj_tiles, &b->kj_items, &b->kj_order, &b->kj_part,
                    &b->conv, &b->iters,
                    &b->res_max, &b->res_last, &b->active, &b->diverged, &b->cl_o, &b->cd_o,
                    &b->aoa_o, &b->st_r, &b->st_c, &b->st_tw, &b->azim, &b->guess, &b->feat,
                    &b->bound_last, &b->bound_last2, &b->st_rr, &b->st_dr, &b->rpm, &b->pitch, &b->dl,
                    &b->loads_out})
    x->release();
  b->mw.release();
  for (DevBuf *x : {&b->cases_d, &b->step_d, &b->dom, &b->dom_pred, &b->dom_new, &b->vel, &b->h1,
                    &b->h2, &b->h3, &b->uind, &b->uind_pred, &b->bound, &b->trail_prev,
                    &b->shed_cur, &b->trail_cur, &b->shed_next, &b->trail_next, &b->rc_s,
                    &b->rc_t, &b->len_old_s, &b->len_old_t, &b->len_s, &b->len_t, &b->len_ps,
                    &b->len_pt, &b->quarter, &b->trailing, &b->wind, &b->pk, &b->ra, &b->rb, &b->tp, &b->tp_raw, &b->tgroup, &b->keys, &b->vals,
                    &b->perm, &b->sort_tmp, &b->groups_main, &b->groups_pred, &b->tiles,
                    &b->items, &b->order, &b->part, &b->bbox, &b->ctr, &b->err, &b->nearctr})
    x->release();
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

}  // extern "C"
