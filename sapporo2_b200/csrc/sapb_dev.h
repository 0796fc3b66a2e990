// Device handle of the sapb_* C ABI (internal; shared by sapb_capi.cu and
// sapb_batch.cu).
#pragma once
#include "sapb_internal.cuh"
#include "../../include/sapporo_b200.h"

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

  char err[512] = {0};
};


// Records an error message on the handle (or the global buffer) and returns
// `code`.
int sapb_fail(sapb_dev *d, int code, const char *fmt, ...);
