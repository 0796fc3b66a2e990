// Device handle of the sapb_* C ABI (internal; shared by sapb_capi.cu and
// sapb_batch.cu).
#pragma once
#include "sapb_internal.cuh"
#include "../../include/sapporo_b200.h"

// Spatial mode of the mixed-precision force calls (sapb_spatial.cu): j
// records in Morton order with per-tile boxes, i positions in Morton order.
struct SpatialBufs {
  int mode = 1;          // 0 off, 1 on for large calls, 2 on for every call
  float far_c = 0.0f;    // 2^-23 / delta
  void *spred = nullptr;  // predicted j records in Morton order
  unsigned *jkey[2] = {nullptr, nullptr};
  int *jidx[2] = {nullptr, nullptr};
  float4 *tbox = nullptr;  // 2 per tile
  unsigned *tkey = nullptr;
  unsigned *ikey[2] = {nullptr, nullptr};
  int *iidx[2] = {nullptr, nullptr};
  float *ibound = nullptr;  // nearest-neighbour ds2 bound per sorted i
  int *frame = nullptr;  // bounding box of the j high parts, order-preserving ints
  unsigned long long *stats = nullptr;  // far / all (warp, tile) pairs since the last read
  void *temp = nullptr;  // radix-sort scratch
  size_t temp_bytes = 0;
  int jcap = 0, icap = 0;
  int valid_nj = -1;          // j count of the current ordering (-1: none)
  unsigned long long valid_gen = 0;  // pred_gen it was built from
  int order_age = 0;          // gathers with the current order since it was made
};

struct sapb_dev {
  using JState = sapb::JState;
  int device = 0;
  int order = SAPB_FOURTH;
  int prec = SAPB_DOUBLESINGLE;
  int n_pipes = SAPB_NPIPES;
  int num_sms = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;

  // j state
  int cap = 0;
  JState js{};
  void *pred = nullptr;
  unsigned long long pred_gen = 1;  // bumped whenever the predicted records change
  double *jpool = nullptr;  // one allocation holding the FP64 planes
  int *jid = nullptr;

  // j staging
  double *stage_h = nullptr;
  double *stage_d = nullptr;
  int stage_cap = 0;

  // i records, results
  double *irec_h = nullptr, *irec_d = nullptr;
  int i_cap = 0;
  double *res_h = nullptr, *res_d = nullptr;
  int *ngb_count_d = nullptr, *ngb_list_d = nullptr;
  double *part_d = nullptr;
  size_t part_cap = 0;  // doubles
  int *status_d = nullptr, *status_h = nullptr;
  int last_ni = 0;
  bool pending = false;

  // launch overrides (0 = planner)
  int tpi = 0, ip = 0, nslices = 0;

  // mixed precision: pairs with ds2 < near_k * eps2 are summed in FP64
  // (0: every pair in FP32)
  double near_k = 16.0;

  SpatialBufs sp;

  char err[512] = {0};
};


// Records an error message on the handle (or the global buffer) and returns
// `code`.
int sapb_fail(sapb_dev *d, int code, const char *fmt, ...);

// Spatial mode (sapb_spatial.cu): orders the predicted j records (when they
// changed since the last ordering) and the ni i records at i_dev, on the
// handle's stream.  spatial_free releases the buffers.
int spatial_prepare(sapb_dev *d, int nj, int ni, const double *i_dev);
void spatial_free(sapb_dev *d);
