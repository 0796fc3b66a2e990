// Batched execution of many force evaluations in one persistent launch:
// block-timestep steps with uneven active counts and ensembles of
// independent clusters, each cluster a contiguous range of j addresses with
// its own prediction time and softening.  Declared in include/sapporo_b200.h.
//
// Per run: one H2D copy of a packed host blob (parameters, cluster table,
// work items, i records), one CUDA graph launch (queue reset, list-count
// reset, per-cluster predictor, persistent force kernel, slice reduction;
// captured once and replayed while the capacities stay the same), one D2H
// copy of the results.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "../../include/sapporo_b200.h"
#include "sapb_dev.h"
#include "sapb_launch.h"

using namespace sapb;

struct sapb_batch {
  sapb_dev *d = nullptr;
  int max_clusters = 0, max_items = 0, max_i = 0;
  // packed blob: [BatchParams][BatchCluster x max_clusters][BatchItem x max_items][i records]
  size_t off_cl = 0, off_it = 0, off_i = 0, blob_bytes = 0;
  unsigned char *blob_h = nullptr, *blob_d = nullptr;
  double *res_h = nullptr, *res_d = nullptr;
  int *cnt_d = nullptr, *lst_d = nullptr;
  double *part_d = nullptr;
  size_t part_cap = 0;  // records
  int n_clusters = 0, n_items = 0, total_i = 0, j_extent = 0;
  size_t part_need = 0;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int g_flags = -1, g_cap = -1;
  const void *g_pred = nullptr;
  double *g_part = nullptr;
  int force_blocks = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
  int tpi_scale = 0;     // autotuner: log2 factor applied to the threads-per-i rule
  int split_factor = 4;  // autotuner: work items per resident block targeted by the j-split
  int runs = 0;
  // inputs of the last plan (re-planned by the autotuner)
  std::vector<int> p_jf, p_jc, p_ic;
  std::vector<double> p_t, p_e;

  BatchParams *par_h() { return reinterpret_cast<BatchParams *>(blob_h); }
  BatchCluster *cl_h() { return reinterpret_cast<BatchCluster *>(blob_h + off_cl); }
  BatchItem *it_h() { return reinterpret_cast<BatchItem *>(blob_h + off_it); }
  double *irec_h() { return reinterpret_cast<double *>(blob_h + off_i); }
};

#define BK(b, call)                                                                        \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return sapb_fail((b)->d, SAPB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                       __FILE__, __LINE__);                                                \
  } while (0)

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static void free_graph(sapb_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  b->g_flags = -1;
}

// threads per i for a cluster with `ni` active particles (2 i per thread):
// the smallest i-tile (256 / tpi) that still holds all of them, shifted by
// the autotuner's offset.
static int tpi_rule(int ni, int scale) {
  int tpi = 1;
  while (tpi < 32 && (256 / (tpi * 2)) >= ni) tpi *= 2;
  for (int s = scale; s > 0 && tpi < 32; s--) tpi *= 2;
  for (int s = scale; s < 0 && tpi > 1; s++) tpi /= 2;
  return tpi;
}

extern "C" {

int sapb_batch_create(sapb_dev *d, int max_clusters, int max_i, sapb_batch **out) {
  if (!d || !out || max_clusters <= 0 || max_i <= 0)
    return sapb_fail(d, SAPB_EINVAL, "sapb_batch_create: bad arguments");
  *out = nullptr;
  sapb_batch *b = new (std::nothrow) sapb_batch();
  if (!b) return sapb_fail(d, SAPB_ENOMEM, "host allocation");
  b->d = d;
  b->max_clusters = max_clusters;
  b->max_i = max_i;
  b->max_items = max_clusters * 8 + max_i / 16 + 4096;
  const int istr = i_stride(d->order);
  b->off_cl = align256(sizeof(BatchParams));
  b->off_it = b->off_cl + align256(sizeof(BatchCluster) * (size_t)max_clusters);
  b->off_i = b->off_it + align256(sizeof(BatchItem) * (size_t)b->max_items);
  b->blob_bytes = b->off_i + sizeof(double) * istr * (size_t)max_i;
  int rc = SAPB_OK;
  do {
    if (cudaSetDevice(d->device) != cudaSuccess) { rc = SAPB_ECUDA; break; }
    if (cudaHostAlloc(&b->blob_h, b->blob_bytes, cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc(&b->blob_d, b->blob_bytes) != cudaSuccess ||
        cudaHostAlloc(&b->res_h, sizeof(double) * kResStride * (size_t)max_i,
                      cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc(&b->res_d, sizeof(double) * kResStride * (size_t)max_i) != cudaSuccess ||
        cudaMalloc(&b->cnt_d, sizeof(int) * (size_t)max_i) != cudaSuccess ||
        cudaMalloc(&b->lst_d, sizeof(int) * kNgbPB * (size_t)max_i) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
      rc = SAPB_ENOMEM;
      break;
    }
    memset(b->blob_h, 0, b->blob_bytes);
    b->force_blocks = d->num_sms * batch_blocks_per_sm(d->order, d->prec);
  } while (0);
  if (rc) {
    cudaGetLastError();
    const size_t bytes = b->blob_bytes;
    sapb_batch_destroy(b);
    return sapb_fail(d, rc, "sapb_batch_create: device or pinned allocation failed (%zu-byte "
                     "table blob)", bytes);
  }
  *out = b;
  return SAPB_OK;
}

int sapb_batch_destroy(sapb_batch *b) {
  if (!b) return SAPB_OK;
  cudaSetDevice(b->d->device);
  if (b->pending) cudaEventSynchronize(b->done);
  free_graph(b);
  if (b->blob_h) cudaFreeHost(b->blob_h);
  if (b->res_h) cudaFreeHost(b->res_h);
  if (b->blob_d) cudaFree(b->blob_d);
  if (b->res_d) cudaFree(b->res_d);
  if (b->cnt_d) cudaFree(b->cnt_d);
  if (b->lst_d) cudaFree(b->lst_d);
  if (b->part_d) cudaFree(b->part_d);
  if (b->done) cudaEventDestroy(b->done);
  delete b;
  return SAPB_OK;
}

double *sapb_batch_i_stage(sapb_batch *b) {
  if (!b) return nullptr;
  if (b->pending) {
    cudaEventSynchronize(b->done);
    b->pending = false;
  }
  return b->irec_h();
}

int sapb_batch_plan(sapb_batch *b, int n_clusters, const int *j_first, const int *j_count,
                    const int *i_count, const double *t_pred, const double *eps2) {
  if (!b) return sapb_fail(nullptr, SAPB_EINVAL, "null batch");
  sapb_dev *d = b->d;
  if (n_clusters < 0 || n_clusters > b->max_clusters)
    return sapb_fail(d, SAPB_EINVAL, "%d clusters (capacity %d)", n_clusters, b->max_clusters);
  if (b->pending) {
    cudaEventSynchronize(b->done);
    b->pending = false;
  }
  BatchCluster *cl = b->cl_h();
  int i_first = 0, prev_end = 0, j_extent = 0;
  long long total_weight = 0;
  std::vector<int> tpi(n_clusters), tiles(n_clusters);
  for (int c = 0; c < n_clusters; c++) {
    if (j_count[c] < 0 || i_count[c] < 0 || j_first[c] < prev_end ||
        j_first[c] + j_count[c] > d->cap)
      return sapb_fail(d, SAPB_EINVAL,
                       "cluster %d: j range [%d, %d) must be in address order, disjoint and "
                       "within capacity %d", c, j_first[c], j_first[c] + j_count[c], d->cap);
    if (i_count[c] > 0 && j_count[c] == 0)
      return sapb_fail(d, SAPB_EINVAL, "cluster %d has active i but no j", c);
    prev_end = j_first[c] + j_count[c];
    j_extent = std::max(j_extent, prev_end);
    const double e2 = eps2 ? eps2[c] : 0.0;
    const float nr2 = (d->prec == SAPB_DOUBLE || d->order == SAPB_GRAPE5)
                          ? 0.0f : (float)(d->near_k * e2);
    cl[c] = BatchCluster{j_first[c], j_count[c], i_first, i_count[c], 1, 0,
                         t_pred ? t_pred[c] : 0.0, e2, nr2, 0};
    i_first += i_count[c];
    if (i_count[c] > 0) {
      tpi[c] = tpi_rule(i_count[c], b->tpi_scale);
      const int ti = 256 / tpi[c];
      tiles[c] = (i_count[c] + ti - 1) / ti;
      total_weight += (long long)tiles[c] * j_count[c];
    }
  }
  if (i_first > b->max_i)
    return sapb_fail(d, SAPB_EINVAL, "%d active i (capacity %d)", i_first, b->max_i);
  // j-split: aim at split_factor items per resident block for balance;
  // slices of at least 256 j
  const long long target = std::max<long long>(
      256, total_weight / std::max(1, b->split_factor * b->force_blocks));
  int n_items = 0;
  size_t part = 0;
  for (int c = 0; c < n_clusters; c++) {
    if (cl[c].i_count == 0) continue;
    const int max_s = std::max(1, (cl[c].j_count + 255) / 256);
    int s = (int)std::min<long long>(max_s, (cl[c].j_count + target - 1) / target);
    s = std::max(s, 1);
    const int sl = (cl[c].j_count + s - 1) / s;
    s = (cl[c].j_count + sl - 1) / sl;
    cl[c].nslices = s;
    cl[c].part_base = s > 1 ? (int)part : 0;
    if (s > 1) part += (size_t)s * cl[c].i_count;
    n_items += tiles[c] * s;
  }
  if (n_items > b->max_items)
    return sapb_fail(d, SAPB_EINVAL, "%d work items (capacity %d)", n_items, b->max_items);
  BatchItem *it = b->it_h();
  int k = 0;
  for (int c = 0; c < n_clusters; c++) {
    if (cl[c].i_count == 0) continue;
    const int ti = 256 / tpi[c];
    const int s_n = cl[c].nslices;
    const int sl = (cl[c].j_count + s_n - 1) / s_n;
    for (int t = 0; t < tiles[c]; t++) {
      const int ib = t * ti;
      const int ic = std::min(ti, cl[c].i_count - ib);
      for (int s = 0; s < s_n; s++) {
        const int jb = s * sl;
        const int jc = std::min(sl, cl[c].j_count - jb);
        it[k++] = BatchItem{c, cl[c].i_first + ib, ic, cl[c].j_first + jb, jc, tpi[c],
                            s_n > 1 ? cl[c].part_base + s * cl[c].i_count + ib : -1};
      }
    }
  }
  // longest items first
  std::stable_sort(it, it + n_items,
                   [](const BatchItem &a, const BatchItem &c) { return a.j_count > c.j_count; });
  b->p_jf.assign(j_first, j_first + n_clusters);
  b->p_jc.assign(j_count, j_count + n_clusters);
  b->p_ic.assign(i_count, i_count + n_clusters);
  b->p_t.assign(n_clusters, 0.0);
  b->p_e.assign(n_clusters, 0.0);
  for (int c = 0; c < n_clusters; c++) {
    b->p_t[c] = cl[c].t_pred;
    b->p_e[c] = cl[c].eps2;
  }
  b->n_clusters = n_clusters;
  b->n_items = n_items;
  b->total_i = i_first;
  b->j_extent = j_extent;
  b->part_need = part;
  *b->par_h() = BatchParams{n_items, n_clusters, i_first, j_extent, 0, {0, 0, 0}};
  return SAPB_OK;
}

int sapb_batch_run(sapb_batch *b, int flags) {
  if (!b) return sapb_fail(nullptr, SAPB_EINVAL, "null batch");
  sapb_dev *d = b->d;
  BK(b, cudaSetDevice(d->device));
  if (b->part_need > b->part_cap) {
    if (b->part_d) cudaFree(b->part_d);
    b->part_d = nullptr;
    const size_t want = b->part_need + b->part_need / 4 + 1024;
    if (cudaMalloc(&b->part_d, sizeof(double) * kResStride * want) != cudaSuccess) {
      cudaGetLastError();
      b->part_cap = 0;
      return sapb_fail(d, SAPB_ENOMEM, "batch partial sums (%zu records)", want);
    }
    b->part_cap = want;
  }
  const bool lists = (flags & SAPB_F_NGB_LIST) != 0;
  const bool predict = (flags & SAPB_F_PREDICT) != 0;
  if (!b->exec || b->g_flags != flags || b->g_cap != d->cap || b->g_pred != d->pred ||
      b->g_part != b->part_d) {
    free_graph(b);
    BatchArgs B{};
    B.pred = d->pred;
    B.js = d->js;
    B.pred_w = d->pred;
    B.par = reinterpret_cast<BatchParams *>(b->blob_d);
    B.cl = reinterpret_cast<const BatchCluster *>(b->blob_d + b->off_cl);
    B.items = reinterpret_cast<const BatchItem *>(b->blob_d + b->off_it);
    B.irec = reinterpret_cast<const double *>(b->blob_d + b->off_i);
    B.res = b->res_d;
    B.part = b->part_d;
    B.ngb_count = b->cnt_d;
    B.ngb_list = b->lst_d;
    B.do_list = lists ? 1 : 0;
    B.do_predict = predict ? 1 : 0;
    B.status = d->status_d;
    BK(b, cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaMemsetAsync(&B.par->queue_head, 0, sizeof(int), d->stream);
    if (e == cudaSuccess && lists)
      e = cudaMemsetAsync(b->cnt_d, 0, sizeof(int) * (size_t)b->max_i, d->stream);
    if (e == cudaSuccess)
      e = launch_batch(d->order, d->prec, B, predict ? d->cap : 0, b->force_blocks, b->max_i,
                       d->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(d->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return sapb_fail(d, SAPB_ECUDA, "batch graph capture: %s",
                       cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    b->graph = g;
    BK(b, cudaGraphInstantiate(&b->exec, g, 0));
    b->g_flags = flags;
    b->g_cap = d->cap;
    b->g_pred = d->pred;
    b->g_part = b->part_d;
  }
  const int istr = i_stride(d->order);
  // one copy: parameters, clusters, items, i records
  const size_t used_i = b->off_i + sizeof(double) * istr * (size_t)b->total_i;
  BK(b, cudaMemcpyAsync(b->blob_d, b->blob_h, used_i, cudaMemcpyHostToDevice, d->stream));
  BK(b, cudaGraphLaunch(b->exec, d->stream));
  if (predict) d->pred_gen++;  // the graph's predictor rewrote the records
  if (b->total_i > 0)
    BK(b, cudaMemcpyAsync(b->res_h, b->res_d, sizeof(double) * kResStride * (size_t)b->total_i,
                          cudaMemcpyDeviceToHost, d->stream));
  BK(b, cudaMemcpyAsync(d->status_h, d->status_d, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  BK(b, cudaEventRecord(b->done, d->stream));
  b->pending = true;
  b->runs++;
  return SAPB_OK;
}

int sapb_batch_results(sapb_batch *b, const double **results, int *total_i) {
  if (!b) return sapb_fail(nullptr, SAPB_EINVAL, "null batch");
  BK(b, cudaSetDevice(b->d->device));
  if (b->pending) {
    BK(b, cudaEventSynchronize(b->done));
    b->pending = false;
  }
  if (results) *results = b->res_h;
  if (total_i) *total_i = b->total_i;
  if (*b->d->status_h) {
    const int s = *b->d->status_h;
    *b->d->status_h = 0;
    cudaMemsetAsync(b->d->status_d, 0, sizeof(int), b->d->stream);
    return sapb_fail(b->d, s & 1 ? SAPB_ETIMEOUT : SAPB_EINVAL, "batch: device status 0x%x", s);
  }
  return SAPB_OK;
}

int sapb_batch_ngb_fetch(sapb_batch *b, int *counts, int *lists) {
  if (!b) return sapb_fail(nullptr, SAPB_EINVAL, "null batch");
  const int ni = b->total_i;
  BK(b, cudaSetDevice(b->d->device));
  if (counts && ni)
    BK(b, cudaMemcpyAsync(counts, b->cnt_d, sizeof(int) * (size_t)ni, cudaMemcpyDeviceToHost,
                          b->d->stream));
  if (lists && ni)
    BK(b, cudaMemcpyAsync(lists, b->lst_d, sizeof(int) * kNgbPB * (size_t)ni,
                          cudaMemcpyDeviceToHost, b->d->stream));
  BK(b, cudaStreamSynchronize(b->d->stream));
  return SAPB_OK;
}

int sapb_batch_info(sapb_batch *b, int *n_items, int *force_blocks, int *graph_runs) {
  if (!b) return sapb_fail(nullptr, SAPB_EINVAL, "null batch");
  if (n_items) *n_items = b->n_items;
  if (force_blocks) *force_blocks = b->force_blocks;
  if (graph_runs) *graph_runs = b->runs;
  return SAPB_OK;
}

int sapb_batch_set_tuning(sapb_batch *b, int tpi_scale) {
  if (!b || tpi_scale < -5 || tpi_scale > 5)
    return sapb_fail(b ? b->d : nullptr, SAPB_EINVAL, "tpi scale %d", tpi_scale);
  b->tpi_scale = tpi_scale;
  return SAPB_OK;
}

int sapb_batch_autotune(sapb_batch *b, int flags, int reps, int *best_scale, int *best_split,
                        float *best_ms) {
  if (!b || b->p_jf.empty() || reps < 1)
    return sapb_fail(b ? b->d : nullptr, SAPB_EINVAL, "autotune needs a plan and reps >= 1");
  sapb_dev *d = b->d;
  BK(b, cudaSetDevice(d->device));
  const int n = (int)b->p_jf.size();
  const std::vector<int> jf = b->p_jf, jc = b->p_jc, ic = b->p_ic;
  const std::vector<double> tp = b->p_t, ep = b->p_e;
  cudaEvent_t e0, e1;
  BK(b, cudaEventCreate(&e0));
  BK(b, cudaEventCreate(&e1));
  float best = 3.4e38f;
  int bs = b->tpi_scale, bf = b->split_factor;
  static const int scales[] = {-1, 0, 1, 2};
  static const int splits[] = {2, 4, 8};
  int rc = SAPB_OK;
  for (int sc : scales) {
    for (int sf : splits) {
      b->tpi_scale = sc;
      b->split_factor = sf;
      rc = sapb_batch_plan(b, n, jf.data(), jc.data(), ic.data(), tp.data(), ep.data());
      if (rc) break;
      rc = sapb_batch_run(b, flags);  // warm-up (and graph capture if needed)
      if (!rc) rc = sapb_batch_results(b, nullptr, nullptr);
      if (rc) break;
      if (cudaEventRecord(e0, d->stream) != cudaSuccess) { rc = SAPB_ECUDA; break; }
      for (int r = 0; r < reps && !rc; r++)
        if (cudaGraphLaunch(b->exec, d->stream) != cudaSuccess) rc = SAPB_ECUDA;
      if (rc || cudaEventRecord(e1, d->stream) != cudaSuccess ||
          cudaEventSynchronize(e1) != cudaSuccess) {
        rc = SAPB_ECUDA;
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= reps;
      if (ms < best) {
        best = ms;
        bs = sc;
        bf = sf;
      }
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->tpi_scale = bs;
  b->split_factor = bf;
  if (rc) return sapb_fail(d, rc, "autotune: a trial run failed");
  rc = sapb_batch_plan(b, n, jf.data(), jc.data(), ic.data(), tp.data(), ep.data());
  if (best_scale) *best_scale = bs;
  if (best_split) *best_split = bf;
  if (best_ms) *best_ms = best;
  return rc;
}

}  // extern "C"
