// bs_types.h -- plain structs shared by the host engine and the kernels.
//
// HBM layout of one evaluation (all per-context, grow-only buffers):
//   packed filaments, padded to the filament tile (KF) with inert entries, as
//   pair records: filaments 2j and 2j+1 share 32 floats (8 float4), field q of
//   filament 2j+h at float 2q+h, so every float4 holds two fields of both:
//     fields  0-3   x1_hi.x, x1_hi.y, x1_hi.z, |L|^2
//             4-7   x1_lo.x, x1_lo.y, x1_lo.z, Rn^2   (x1 = hi + lo to ~2^-48)
//             8-11  L.x, L.y, L.z, D                  (L = x2 - x1)
//            12-15  K L.x, K L.y, K L.z, rc           (K = gamma/4pi; rc the core
//                                                       radius, Vatistas with K != 0, else 0)
//   with D = (K^2 rc^2 |L|^2)^2 (Vatistas: the core term scaled like |K L x r1|^4,
//   so K cancels from the core factor and enters only through K L) or d |L|^2
//   (cut-off)
//   For the FP32c evaluations the records form a chained stream: the lines of
//   filaments of each family (the shed call's along the span, the trailing
//   call's along the wake age) fill the two lanes of consecutive records so
//   that x2 of a lane is x1 of the same lane one record earlier, except at the
//   records flagged in a head bit array (F32cArgs::heads).
//   raw FP64 filaments for near-singular terms and the FP64 path
//     ra[f] = (x1, y1, z1, gamma)  rb[f] = (x2, y2, z2, rc^2)   double4
//   targets  tp[t] = (x, y, z, 0) double4, sorted by (group, Morton code of the
//            position) so the T targets of a thread are close together;
//            perm[t] = index of sorted target t in the packed input order
//   partial sums per work item: part[item][3][tile_cap] double
#pragma once

#include <stdint.h>

namespace winds {

enum : int { kCoreCutoff = 0, kCoreVatistas = 1 };

enum : unsigned {
  kErrWaitTimeout = 1u,  // a bounded mbarrier wait ran out
  kErrBadItem = 2u,      // a work item pointed outside its tables
};

struct Group {          // one target set evaluated against one filament range
  double *out;          // MATLAB-layout output [ns_p, 3, ...]
  long long t_begin;    // first packed target
  long long t_count;
  long long ns_p;       // first dimension of the output layout
  int f_begin;          // packed filament range, multiples of the tile size
  int f_end;
  int accumulate;       // 1: out += result, 0: out = result
  int pad;
};

struct Tile {           // tile_cap consecutive targets of one group
  long long t_begin;
  int t_count;
  int group;
  int first_item;
  int n_items;
};

struct Item {           // one tile against one filament chunk
  int tile;
  int f_begin;
  int f_end;
  int pad;
};

// Live part of a group whose target and filament counts change on the device
// (a growing wake inside a fixed plan): sorted targets [Group.t_begin, t_end)
// and packed filaments [Group.f_begin, f_end) take part; tiles past t_end and
// items from f_end on are skipped, items crossing f_end are cut there. f_end
// is a multiple of the filament pad.
struct GroupLive {
  long long t_end;
  int f_end;
  int pad;
};

struct BBox {           // ordered-int keys of float bounds (see float_key)
  int tmin[3], tmax[3]; // targets
  int fmin[3], fmax[3]; // filament endpoints
};

struct F32cArgs {
  const float4 *pk;  // pair records, 8 float4 per two filaments
  const double4 *ra, *rb;
  const double4 *tp;
  const Group *groups;
  const Tile *tiles;
  const Item *items;
  const int *order;  // work queue: queue position -> item (nullptr: identity)
  const GroupLive *live = nullptr;  // per group (nullptr: every tile and item is live)
  // Chained stream (nullptr: unchained): bit (r & 31) of heads[r >> 5] is set
  // when pair record r starts a chain, i.e. when either of its filaments does
  // not end where the same lane's filament of record r - 1 begins.
  const unsigned *heads = nullptr;
  int n_items;
  int tile_cap;
  double *part;
  unsigned *work_ctr;
  unsigned *err;
  unsigned long long *near_ctr;
  const BBox *bbox;
  int model;
  double d, n, co;
  unsigned long long wait_limit_ns;
};

}  // namespace winds
