// bs_launch.h -- host-side launchers of the induced-velocity kernels.
#pragma once

#include <cuda_runtime.h>

#include "bs_types.h"

namespace winds {

struct PackedFilaments {
  float4 *pk;  // pair records: 4 float4 per filament (layout in bs_types.h)
  double4 *ra, *rb;
};

// Filament ranges of work items are multiples of this (a multiple of every
// FP32 tile size and of the FP64 stage).
constexpr int kFilamentPad = 128;

bool f32c_config_supported(int T, int KF);
// FP32c work runs on independent warp workers: a tile holds f32c_threads() * T
// targets, f32c_occupancy() counts resident workers per SM, and launch_f32c's
// grid counts workers.
int f32c_threads();
int f64_threads();
int f64_tile();
int f32c_occupancy(int model, int T, int KF, bool chain = false);
int f64_occupancy();
unsigned long long default_wait_limit_ns();

cudaError_t launch_bbox_init(BBox *bb, cudaStream_t s);
cudaError_t launch_pack_filaments(const double *F1, const double *F2, const double *gam,
                                  const double *rc, long long d0, long long nf, long long off,
                                  int model, double dcut, const PackedFilaments &pf, BBox *bb,
                                  cudaStream_t s);
cudaError_t launch_pad_filaments(long long from, long long to, const PackedFilaments &pf,
                                 cudaStream_t s);
// Chained filament stream (the FP32c path): records per [d0,3,d2,d3] family,
// and the packing of one family from record rec_off (cnt: 2 device words of
// scratch per family; heads zeroed beforehand, one bit per record).
long long chain_records(long long d0, long long d2, long long d3);
cudaError_t launch_pack_chains(const double *F1, const double *F2, const double *gam,
                               const double *rc, const long long d[4], long long rec_off,
                               unsigned long long *cnt, int model, double dcut,
                               const PackedFilaments &pf, unsigned *heads, BBox *bb,
                               cudaStream_t s);
cudaError_t launch_pad_chains(long long from, long long to, const PackedFilaments &pf,
                              unsigned *heads, cudaStream_t s);
cudaError_t launch_pack_targets(const double *P, long long ns, long long np, long long off,
                                int group, double4 *tp, int *tgroup, BBox *bb, cudaStream_t s);
cudaError_t launch_target_keys(const double4 *tp, const int *tgroup, long long n, const BBox *bb,
                               unsigned long long *keys, int *vals, cudaStream_t s);
cudaError_t launch_gather_targets(const double4 *src, const int *perm, long long n, double4 *dst,
                                  cudaStream_t s);
cudaError_t sort_target_keys(void *temp, size_t *temp_bytes, const unsigned long long *kin,
                             unsigned long long *kout, const int *vin, int *vout, long long n,
                             cudaStream_t s);
cudaError_t launch_f32c(const F32cArgs &a, int model, int T, int KF, int grid, cudaStream_t s);
cudaError_t launch_f64(const F32cArgs &a, int grid, cudaStream_t s);
// live (with the plan's items): only each group's live part (GroupLive).
cudaError_t launch_reduce(const Tile *tiles, int n_tiles, const Group *groups, const double *part,
                          const int *perm, int tile_cap, cudaStream_t s,
                          const Item *items = nullptr, const GroupLive *live = nullptr);
cudaError_t launch_ffma_peak(float *out, int blocks, int iters, cudaStream_t s);
cudaError_t launch_wait_selftest(unsigned *err, unsigned long long limit_ns, cudaStream_t s);
cudaError_t launch_length(const double *F1, const double *F2, long long d0, long long nf, double *L,
                          cudaStream_t s);

}  // namespace winds
