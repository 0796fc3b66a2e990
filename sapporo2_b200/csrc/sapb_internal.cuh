// Internal definitions shared by the device kernels and the C-ABI layer.
//
// HBM layout (one GPU, capacity `cap` j-particles):
//   j state, FP64 structure of arrays (written by the scatter kernel, read by
//   the predictor): t[cap], m[cap], x/v/a/j[3][cap], s/c[3][cap] (6th only),
//   eps[cap], id[cap].
//   Predicted j records, the force kernels' only j input, array of records:
//     mixed (DOUBLESINGLE): float4 per field, RS = 3 (4th) / 4 (6th):
//       {xh.x, xh.y, xh.z, m} {xl.x, xl.y, xl.z, id bits} {v, 0} {a, 0}
//     FP64 (DOUBLE): double4 per field, RS = 2 (4th) / 3 (6th):
//       {x, m} {v, id bits} {a, 0}
//   i records (packed by the host, one H2D copy per call), doubles:
//     {x0 x1 x2 h2 v0 v1 v2 id-bits} (+ {a0 a1 a2 0} for 6th)
//   results, one record of 12 doubles per i:
//     {acc0 acc1 acc2 pot jrk0 jrk1 jrk2 snp0 snp1 snp2 ds2min nnb|count}
//   partial sums (scratch, used when the j range is split over S slices):
//     12 doubles per (slice, i), same layout, NN stored as a 64-bit key.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sapb {

enum { GRAPE5 = 0, FOURTH = 1, SIXTH = 2 };
enum { FLOAT = 0, DOUBLESINGLE = 1, DOUBLE = 2 };

constexpr int kNgbPB = 256;     // neighbour slots per i (reference NGB_PB)
constexpr int kResStride = 12;  // doubles per result / partial record
constexpr float kNoNgbDs2 = 1.0e11f;  // initial nearest-neighbour distance

// Error bits written by kernels into the device status word.
enum { kErrWaitTimeout = 1, kErrBadConfig = 2 };

struct JState {
  double *t, *m, *eps;
  double *x[3], *v[3], *a[3], *j[3], *s[3], *c[3];
  int *id;
};

// Staging record written by the host for every j updated since the last
// push (doubles; the first slot holds two ints: address, id).
// 4th order: 16 doubles; 6th order: 22 doubles.
//   [0] addr|id  [1] t  [2] m  [3..5] x  [6..8] v  [9..11] a  [12..14] jerk
//   [15] eps     [16..18] snap  [19..21] crackle
constexpr int kStageStride4 = 16;
constexpr int kStageStride6 = 22;

__host__ __device__ constexpr int stage_stride(int order) {
  return order >= SIXTH ? kStageStride6 : kStageStride4;
}
__host__ __device__ constexpr int i_stride(int order) {  // doubles per i record
  return order >= SIXTH ? 12 : 8;
}
__host__ __device__ constexpr int pred_fields(int order) {  // records per j
  return order >= SIXTH ? 4 : 3;  // float4 fields (mixed)
}
__host__ __device__ constexpr int pred_fields64(int order) {
  return order >= SIXTH ? 3 : 2;  // double4 fields (FP64)
}

struct ForceArgs {
  const void *pred;   // predicted j records (float4 or double4 fields)
  int nj;             // number of j used as sources
  const double *irec; // i records
  int ni;
  double eps2;
  int nslices;        // S: j slices across blocks (slice s: tiles s, s+S, ...)
  int i_tiles;        // number of i tiles
  double *out;        // results (S == 1) or partials (S > 1)
  int write_partials; // 1: write 12-double partial records per (slice, i)
  int do_list;        // build neighbour lists
  int *ngb_count;     // [ni] (zeroed before launch)
  int *ngb_list;      // [ni * 256]
  int *status;        // device error word
  // Spatial mode (mixed precision; tbox == nullptr: off).  The j records of
  // `pred` are in Morton order; i position g of the launch is i record
  // iperm[g] (results and lists are written at iperm[g] too).
  const int *iperm;     // [ni] (nullptr: identity)
  const float *ibound;  // [ni] upper bound of the nearest-neighbour ds2 of i position g
  const float4 *tbox;   // [2 * tiles]: {min xyz, max |x|}, {max xyz, 0} of the high parts
  float far_c;          // 2^-23 / delta: far tiles are >= far_c * |x|max from every i
  unsigned long long *stats;  // [2]: += far (warp, tile) pairs, += all (warp, tile) pairs
  // Near pairs (mixed precision; 0: off): an i whose row of a tile holds a j
  // with ds2 < near_r2 has that row summed again in FP64 instead of FP32.
  float near_r2;
};

// ---- batched execution (block steps, ensembles of independent clusters) ----
// A cluster is a contiguous range of j addresses with its own prediction time
// and softening, plus a contiguous range of active i records.  Work items
// (cluster, i-tile, j-slice) are consumed by a persistent kernel from a queue
// in device memory, so one captured CUDA graph serves any step.
struct BatchCluster {
  int j_first, j_count;  // j addresses [j_first, j_first + j_count)
  int i_first, i_count;  // i records [i_first, i_first + i_count)
  int nslices;           // j-split of this cluster (1: items write results directly)
  int part_base;         // first partial record of this cluster
  double t_pred, eps2;
  float near_r2;         // mixed precision: near pairs (ds2 < near_r2) summed in FP64; 0 off
  int pad_;
};
struct BatchItem {
  int cluster;
  int i_begin, i_count;  // global i records of this tile
  int j_begin, j_count;  // j addresses of this slice
  int tpi;               // threads per i (1..32), i per thread is 2
  int slot;              // first partial record (-1: write final results)
};
struct BatchParams {
  int n_items, n_clusters, total_i, j_extent;
  int queue_head;        // next work item (reset to 0 before every run)
  int pad[3];
};
struct BatchArgs {
  const void *pred;
  JState js;
  void *pred_w;
  const BatchCluster *cl;
  const BatchItem *items;
  BatchParams *par;
  const double *irec;
  double *res;
  double *part;
  int *ngb_count, *ngb_list;
  int do_list, do_predict;
  int *status;
};

struct ReduceArgs {
  const double *part;
  int nslices;
  int ni;
  double *out;
  const int *ngb_count;
};

}  // namespace sapb
