// C ABI over the device code: device state, staging, launch planning.
// Declared in include/sapporo_b200.h.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <new>

#include "../../include/sapporo_b200.h"
#include "sapb_dev.h"
#include "sapb_launch.h"

using namespace sapb;

static char g_err[512];

// Default accuracy bound of the single-float position difference on far
// tiles (relative to the pair distance).
constexpr double kSpatialDelta = 1e-6;

static int fail(sapb_dev *d, int code, const char *fmt, ...) {
  char *buf = d ? d->err : g_err;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, 512, fmt, ap);
  va_end(ap);
  return code;
}

int sapb_fail(sapb_dev *d, int code, const char *fmt, ...) {
  char *buf = d ? d->err : g_err;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, 512, fmt, ap);
  va_end(ap);
  return code;
}

#define CK(d, call)                                                                       \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail((d), SAPB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),       \
                  __FILE__, __LINE__);                                                    \
  } while (0)

static size_t pred_bytes_per_j(int order, int prec) {
  return prec == DOUBLE ? 32u * pred_fields64(order) : 16u * pred_fields(order);
}
static int nplanes(int order) {  // FP64 planes: t m eps + 3*(x v a j) [+ 3*(s c)]
  return 3 + 12 + (order >= SIXTH ? 6 : 0);
}

static void free_j(sapb_dev *d) {
  if (d->jpool) cudaFree(d->jpool);
  if (d->jid) cudaFree(d->jid);
  if (d->pred) cudaFree(d->pred);
  d->jpool = nullptr;
  d->jid = nullptr;
  d->pred = nullptr;
  d->cap = 0;
}

static void bind_planes(JState &js, double *pool, int *id, int cap, int order) {
  double *p = pool;
  js.t = p; p += cap;
  js.m = p; p += cap;
  js.eps = p; p += cap;
  for (int d = 0; d < 3; d++) { js.x[d] = p; p += cap; }
  for (int d = 0; d < 3; d++) { js.v[d] = p; p += cap; }
  for (int d = 0; d < 3; d++) { js.a[d] = p; p += cap; }
  for (int d = 0; d < 3; d++) { js.j[d] = p; p += cap; }
  for (int d = 0; d < 3; d++) {
    js.s[d] = order >= SIXTH ? p : nullptr;
    if (order >= SIXTH) p += cap;
  }
  for (int d = 0; d < 3; d++) {
    js.c[d] = order >= SIXTH ? p : nullptr;
    if (order >= SIXTH) p += cap;
  }
  js.id = id;
}

// Grows j storage to new_cap, copying the first old cap entries of every
// plane and of the predicted records.
static int grow_j(sapb_dev *d, int new_cap) {
  if (new_cap <= d->cap) return SAPB_OK;
  // grow the device store by at least half: callers that stage addresses in
  // order step their bound up by 10 % at a time (the reference's
  // increase_jMemory), which would otherwise reallocate and copy the whole
  // store ~44 times on the way from 16384 to 2^20
  if (d->cap > 0) new_cap = (int)std::min<long long>(INT_MAX / 2, std::max<long long>(new_cap, (long long)d->cap + d->cap / 2));
  const int np = nplanes(d->order);
  double *pool = nullptr;
  int *id = nullptr;
  void *pred = nullptr;
  const size_t pb = pred_bytes_per_j(d->order, d->prec);
  {  // refuse up front what cannot fit (no attempt, no partial allocation)
    const size_t need = ((size_t)np * 8 + 4 + pb) * (size_t)new_cap;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && need > free_b)
      return fail(d, SAPB_ENOMEM,
                  "cannot allocate j storage for %d particles: %.1f GB needed, %.1f GB free",
                  new_cap, need / 1e9, free_b / 1e9);
  }
  if (cudaMalloc(&pool, sizeof(double) * np * (size_t)new_cap) != cudaSuccess ||
      cudaMalloc(&id, sizeof(int) * (size_t)new_cap) != cudaSuccess ||
      cudaMalloc(&pred, pb * (size_t)new_cap) != cudaSuccess) {
    cudaGetLastError();
    if (pool) cudaFree(pool);
    if (id) cudaFree(id);
    if (pred) cudaFree(pred);
    return fail(d, SAPB_ENOMEM, "cannot allocate j storage for %d particles", new_cap);
  }
  CK(d, cudaMemsetAsync(pool, 0, sizeof(double) * np * (size_t)new_cap, d->stream));
  CK(d, cudaMemsetAsync(id, 0, sizeof(int) * (size_t)new_cap, d->stream));
  CK(d, cudaMemsetAsync(pred, 0, pb * (size_t)new_cap, d->stream));
  if (d->cap > 0) {
    for (int k = 0; k < np; k++)
      CK(d, cudaMemcpyAsync(pool + (size_t)k * new_cap, d->jpool + (size_t)k * d->cap,
                            sizeof(double) * d->cap, cudaMemcpyDeviceToDevice, d->stream));
    CK(d, cudaMemcpyAsync(id, d->jid, sizeof(int) * d->cap, cudaMemcpyDeviceToDevice, d->stream));
    CK(d, cudaMemcpyAsync(pred, d->pred, pb * d->cap, cudaMemcpyDeviceToDevice, d->stream));
    CK(d, cudaStreamSynchronize(d->stream));
  }
  free_j(d);
  d->jpool = pool;
  d->jid = id;
  d->pred = pred;
  d->pred_gen++;
  d->cap = new_cap;
  bind_planes(d->js, pool, id, new_cap, d->order);
  return SAPB_OK;
}

static int ensure_i(sapb_dev *d, int ni) {
  if (ni <= d->i_cap) return SAPB_OK;
  const int cap = std::max(ni, d->n_pipes);
  const int is = i_stride(d->order);
  double *ih = nullptr, *id = nullptr, *rh = nullptr, *rd = nullptr;
  int *cnt = nullptr, *lst = nullptr;
  bool ok = cudaHostAlloc(&ih, sizeof(double) * is * (size_t)cap, cudaHostAllocDefault) ==
                cudaSuccess &&
            cudaMalloc(&id, sizeof(double) * is * (size_t)cap) == cudaSuccess &&
            cudaHostAlloc(&rh, sizeof(double) * kResStride * (size_t)cap,
                          cudaHostAllocDefault) == cudaSuccess &&
            cudaMalloc(&rd, sizeof(double) * kResStride * (size_t)cap) == cudaSuccess &&
            cudaMalloc(&cnt, sizeof(int) * (size_t)cap) == cudaSuccess &&
            cudaMalloc(&lst, sizeof(int) * kNgbPB * (size_t)cap) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    if (ih) cudaFreeHost(ih);
    if (rh) cudaFreeHost(rh);
    if (id) cudaFree(id);
    if (rd) cudaFree(rd);
    if (cnt) cudaFree(cnt);
    if (lst) cudaFree(lst);
    return fail(d, SAPB_ENOMEM, "cannot allocate i buffers for %d particles", cap);
  }
  cudaStreamSynchronize(d->stream);  // a call in flight may still use the old buffers
  if (d->irec_h) {
    memcpy(ih, d->irec_h, sizeof(double) * is * (size_t)d->i_cap);
    cudaFreeHost(d->irec_h);
  }
  if (d->res_h) cudaFreeHost(d->res_h);
  if (d->irec_d) cudaFree(d->irec_d);
  if (d->res_d) cudaFree(d->res_d);
  if (d->ngb_count_d) cudaFree(d->ngb_count_d);
  if (d->ngb_list_d) cudaFree(d->ngb_list_d);
  d->irec_h = ih;
  d->irec_d = id;
  d->res_h = rh;
  d->res_d = rd;
  d->ngb_count_d = cnt;
  d->ngb_list_d = lst;
  d->i_cap = cap;
  CK(d, cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)cap, d->stream));
  return SAPB_OK;
}

static int ensure_part(sapb_dev *d, size_t doubles) {
  if (doubles <= d->part_cap) return SAPB_OK;
  if (d->part_d) cudaFree(d->part_d);
  d->part_d = nullptr;
  d->part_cap = 0;
  const size_t want = doubles + doubles / 4;
  if (cudaMalloc(&d->part_d, sizeof(double) * want) != cudaSuccess) {
    cudaGetLastError();
    return fail(d, SAPB_ENOMEM, "cannot allocate %zu bytes of partial sums", sizeof(double) * want);
  }
  d->part_cap = want;
  return SAPB_OK;
}

// ---------------------------------------------------------------------
// Launch planner: threads-per-i, i per thread and the number of j slices
// (cost model in make_plan below).
// ---------------------------------------------------------------------
struct Plan {
  int tpi, ip, ns, i_tiles, slice_tiles;
};

// resident blocks per SM of a force-kernel shape (occupancy API)
static int blocks_per_sm(int order, int prec, int tpi, int ip) {
  return std::max(1, force_blocks_per_sm(order, prec, tpi, ip));
}

// Launch shape for ni i-particles and nj j: threads-per-i, i per thread and
// the number of j-slices S.  Cost model: blocks of one shape run in waves
// of R = SMs x resident blocks per SM; a block of st tiles costs
// (st + 1) tile-times (prologue, nearest-neighbour rescan, epilogue), a
// tile-time being 128 x (i per block) x (blocks per SM) pair-times of one
// SM; S > 1 adds the slice reduction (S x ni records read).  The block
// count B = i-tiles x S is chosen near a whole number of waves: a last wave
// that holds a few blocks costs as much as a full one.
extern "C" {
static bool use_spatial(const sapb_dev *d, int ni, int nj);  // defined with the C ABI below
}

static Plan make_plan(const sapb_dev *d, int ni, int nj) {
  const int tj = force_tile_j();
  const int ntiles = std::max(1, (nj + tj - 1) / tj);
  // (threads per i, i per thread) and the shape's throughput relative to the
  // best one, measured on B200 at N = 2^20 (6th order, all i, where waves
  // cost nothing): mixed (1,4) 537.8, (2,4) 534.6, (1,2) 521.8, (2,2) 516.1,
  // (4,2) 510.4, (8,2) 491.2 G interactions/s; FP64 (2,2) 249.6, (4,2) 247.4,
  // (8,2) 244.8, (1,2) 243.9.  The one-i-per-thread shapes (only chosen for
  // very small ni) are estimates.
  static const int shapes_mix[][2] = {{1, 4}, {2, 4}, {1, 2}, {2, 2}, {4, 2}, {8, 2}, {16, 1}, {32, 1}};
  static const double eff_mix[] = {1.0, 0.994, 0.970, 0.960, 0.949, 0.913, 0.85, 0.85};
  static const int shapes_dp[][2] = {{2, 2}, {4, 2}, {8, 2}, {1, 2}, {16, 1}, {32, 1}};
  static const double eff_dp[] = {1.0, 0.991, 0.981, 0.977, 0.9, 0.9};
  const int nshape = d->prec == DOUBLE ? 6 : 8;
  // pair-times per SM and second (B200, measured order of magnitude): only
  // the balance between force and reduction depends on them
  const double sm_rate = d->prec == DOUBLE ? (d->order >= SIXTH ? 1.5e9 : 2.3e9)
                                           : (d->order >= SIXTH ? 3.6e9 : 5.6e9);
  const int max_ns = std::max(1, ntiles / 4);  // keep >= 4 tiles per slice
  // Mixed precision below 2^32 pairs and 2^19 j: the shape family comes from
  // the call size, the model above then picks the shape within it and the
  // j-split.  B200 sweeps of every shape and j-split (4th and 6th order, 256
  // to 65536 i on 16384 to 2^20 j) put the best shape at two i per thread
  // with about 65536 / ni threads per i (2 to 8) from 1024 i on (4th order,
  // 16384 x 16384: 0.45 ms against 0.66 ms for the model's free choice;
  // 6th order, 4096 i on 16384 j: 0.21 against 0.28 ms), and at 8 threads
  // per i or one i per thread below.  From 2^32 pairs, or with 2^19 j and
  // more, where the j-split alone fills the GPU, the model chooses freely:
  // (1,4) and (2,4) are then within 1 % of the best (2^20 j x 2048 i: (2,4)
  // 4 % ahead of (8,2)).  Calls in spatial mode keep the free choice too:
  // there these shapes gained only 0-7 %, and the 6th-order block steps of a
  // 262144-body system with tight binaries (200 steps, 10 % binaries
  // 1e-6..1e-4 apart) reached t = 5.7e-4 with them against 3.13e-3 with the
  // free choice and 3.25e-3 with FP64 forces (address order: 3.25e-3 with
  // either planner); the cause is not known.
  bool allow[8] = {true, true, true, true, true, true, true, true};
  if (d->prec != DOUBLE && !d->tpi && (double)ni * nj < 4294967296.0 && nj < (1 << 19) &&
      !use_spatial(d, ni, nj)) {
    for (bool &a : allow) a = false;
    if (ni < 1024) {
      allow[5] = allow[6] = allow[7] = true;  // (8,2), (16,1), (32,1)
    } else {
      int t = 2;
      while (t < 8 && (long)t * 2 * ni <= 65536) t *= 2;
      allow[t == 2 ? 3 : (t == 4 ? 4 : 5)] = true;  // (2,2), (4,2) or (8,2)
    }
  }
  // FP64 kernels, same call sizes (sweep of 4th and 6th order, 256 to 16384
  // i on 16384 and 131072 j): one i per thread with 16 or 32 threads per i
  // below 4096 i (16 from 1024 i on), (8,2) or (16,1) up to 16384 i, (8,2)
  // above; the model's free choice was up to 1.16x off (4th order, 4096 i on
  // 16384 j).
  if (d->prec == DOUBLE && !d->tpi && (double)ni * nj < 4294967296.0 && nj < (1 << 19)) {
    for (bool &a : allow) a = false;
    if (ni < 1024) {
      allow[4] = allow[5] = true;  // (16,1), (32,1)
    } else if (ni < 4096) {
      allow[4] = true;  // (16,1)
    } else if (ni < 16384) {
      allow[2] = allow[4] = true;  // (8,2), (16,1)
    } else {
      allow[2] = true;  // (8,2)
    }
  }
  Plan best{1, 2, 1, 1, ntiles};
  double best_t = 1e300;
  for (int q = 0; q < nshape; q++) {
    if (!d->tpi && !allow[q]) continue;
    const int *sh = d->prec == DOUBLE ? shapes_dp[q] : shapes_mix[q];
    const int tpi = d->tpi ? d->tpi : sh[0];
    const int ip = d->ip ? d->ip : sh[1];
    const int ti = force_tile_i(tpi, ip);
    const int i_tiles = (ni + ti - 1) / ti;
    const int bps = blocks_per_sm(d->order, d->prec, tpi, ip);
    const long R = (long)d->num_sms * bps;
    const double speed = d->tpi ? 1.0 : (d->prec == DOUBLE ? eff_dp[q] : eff_mix[q]);
    const double tile_time = 128.0 * ti * bps / (speed * sm_rate);
    auto consider = [&](int ns) {
      ns = std::max(1, std::min(ns, max_ns));
      const int st = (ntiles + ns - 1) / ns;
      const int nse = (ntiles + st - 1) / st;  // every slice non-empty
      const long B = (long)i_tiles * nse;
      const long waves = (B + R - 1) / R;
      double t = (double)waves * (st + 1.0) * tile_time;
      if (nse > 1) t += 5e-6 + (double)nse * ni * kResStride * 8.0 / 4.0e12;
      if (t < best_t * (1.0 - 1e-9)) {
        best_t = t;
        best = Plan{tpi, ip, nse, i_tiles, st};
      }
    };
    if (d->nslices) {
      consider(d->nslices);
    } else {
      consider(1);
      consider(max_ns);
      for (int k = 1; k <= 64; k++) {  // B just below k whole waves
        const long ns = (long)k * R / std::max(i_tiles, 1);
        if (ns < 1) continue;
        if (ns > max_ns) break;
        consider((int)ns);
      }
    }
    if (d->tpi) break;  // fixed shape
  }
  return best;
}

// ---------------------------------------------------------------------
// Fixed scratch of sapb_force_device_noalloc.  Every GPU that loads this
// library holds these 32 MiB until the process exits.  Host code must not
// use the symbol itself (in host code it names a host-side stand-in, not
// device memory): its device address is resolved once per device with
// cudaGetSymbolAddress, with that device current, and passed to the kernels.
// ---------------------------------------------------------------------
static __device__ __align__(256) double g_noalloc_scratch[SAPB_NOALLOC_SCRATCH_BYTES / 8];

constexpr int kMaxDevices = 64;
static double *g_noalloc_ptr[kMaxDevices];

// Resolves the scratch address for the current device (once per device).
static int noalloc_setup(sapb_dev *d) {
  if (d->device < 0 || d->device >= kMaxDevices)
    return fail(d, SAPB_EINVAL, "device ordinal %d beyond the no-allocation table", d->device);
  if (g_noalloc_ptr[d->device]) return SAPB_OK;
  CK(d, cudaSetDevice(d->device));
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr)
    return fail(d, SAPB_ECUDA, "cudaGetSymbolAddress(no-allocation scratch): %s",
                cudaGetErrorString(e));
  g_noalloc_ptr[d->device] = static_cast<double *>(ptr);
  return SAPB_OK;
}

// ---------------------------------------------------------------------
extern "C" {

const char *sapb_version(void) { return "sapporo-b200 0.1 (sm_100a)"; }

const char *sapb_error_string(int code) {
  switch (code) {
    case SAPB_OK: return "ok";
    case SAPB_ECUDA: return "CUDA runtime error";
    case SAPB_EINVAL: return "invalid argument";
    case SAPB_ENOMEM: return "out of memory";
    case SAPB_ETIMEOUT: return "device wait timed out";
    case SAPB_ENODEV: return "no CUDA device";
    default: return "unknown error";
  }
}

const char *sapb_last_error(const sapb_dev *d) { return d ? d->err : g_err; }

int sapb_device_count(int *count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *count = 0;
    return fail(nullptr, SAPB_ENODEV, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
  }
  *count = n;
  return SAPB_OK;
}

int sapb_open(sapb_dev **out, int device, int order, int precision, int n_pipes,
              int nj_reserve) {
  if (!out) return fail(nullptr, SAPB_EINVAL, "null handle pointer");
  *out = nullptr;
  if (order != GRAPE5 && order != FOURTH && order != SIXTH)
    return fail(nullptr, SAPB_EINVAL, "order %d not supported (GRAPE-5=0, 4th=1, 6th=2)",
                order);
  if (precision != DOUBLESINGLE && precision != DOUBLE)
    return fail(nullptr, SAPB_EINVAL, "precision %d not supported (DS=1, DOUBLE=2)", precision);
  int ndev = 0;
  if (sapb_device_count(&ndev) != SAPB_OK || ndev == 0)
    return fail(nullptr, SAPB_ENODEV, "no CUDA device available");
  if (device < 0 || device >= ndev)
    return fail(nullptr, SAPB_EINVAL, "device %d out of range (%d devices)", device, ndev);
  sapb_dev *d = new (std::nothrow) sapb_dev();
  if (!d) return fail(nullptr, SAPB_ENOMEM, "host allocation failed");
  d->device = device;
  d->order = order;
  d->prec = precision;
  d->n_pipes = n_pipes > 0 ? n_pipes : SAPB_NPIPES;
  d->sp.far_c = (float)(0x1p-23 / kSpatialDelta);
  if (const char *e = getenv("SAPPORO_B200_SPATIAL")) d->sp.mode = atoi(e) == 0 ? 0 : (atoi(e) >= 2 ? 2 : 1);
  if (const char *e = getenv("SAPPORO_B200_NEAR")) {
    const double k = atof(e);
    if (k >= 0.0 && k <= 1e6) d->near_k = k;
  }
  int rc = SAPB_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "cudaSetDevice(%d)", device); break; }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "cudaGetDeviceProperties"); break; }
    d->num_sms = prop.multiProcessorCount;
    if (prop.major < 10) {
      rc = fail(d, SAPB_ENODEV, "device %d is sm_%d%d; this library targets sm_100a", device,
                prop.major, prop.minor);
      break;
    }
    if (cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "stream"); break; }
    d->stream = d->own_stream;
    if (cudaEventCreateWithFlags(&d->done, cudaEventDisableTiming) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "event"); break; }
    if (cudaMalloc(&d->status_d, sizeof(int)) != cudaSuccess ||
        cudaHostAlloc(&d->status_h, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
      rc = fail(d, SAPB_ENOMEM, "status word");
      break;
    }
    *d->status_h = 0;
    if (cudaMemsetAsync(d->status_d, 0, sizeof(int), d->stream) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "memset"); break; }
    rc = grow_j(d, nj_reserve > 0 ? nj_reserve : 16384);
    if (rc) break;
    rc = ensure_i(d, d->n_pipes);
    if (rc) break;
    rc = noalloc_setup(d);
    if (rc) break;
    if (cudaStreamSynchronize(d->stream) != cudaSuccess) { rc = fail(d, SAPB_ECUDA, "sync"); break; }
  } while (0);
  if (rc != SAPB_OK) {
    snprintf(g_err, sizeof g_err, "%s", d->err);
    sapb_close(d);
    cudaGetLastError();
    return rc;
  }
  *out = d;
  return SAPB_OK;
}

int sapb_close(sapb_dev *d) {
  if (!d) return SAPB_OK;
  cudaSetDevice(d->device);
  if (d->stream) cudaStreamSynchronize(d->stream);
  free_j(d);
  spatial_free(d);
  if (d->stage_h) cudaFreeHost(d->stage_h);
  if (d->stage_d) cudaFree(d->stage_d);
  if (d->irec_h) cudaFreeHost(d->irec_h);
  if (d->irec_d) cudaFree(d->irec_d);
  if (d->res_h) cudaFreeHost(d->res_h);
  if (d->res_d) cudaFree(d->res_d);
  if (d->ngb_count_d) cudaFree(d->ngb_count_d);
  if (d->ngb_list_d) cudaFree(d->ngb_list_d);
  if (d->part_d) cudaFree(d->part_d);
  if (d->status_d) cudaFree(d->status_d);
  if (d->status_h) cudaFreeHost(d->status_h);
  if (d->done) cudaEventDestroy(d->done);
  if (d->own_stream) cudaStreamDestroy(d->own_stream);
  delete d;
  return SAPB_OK;
}

int sapb_info(const sapb_dev *d, int *order, int *precision, int *n_pipes, int *j_capacity,
              int *num_sms) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  if (order) *order = d->order;
  if (precision) *precision = d->prec;
  if (n_pipes) *n_pipes = d->n_pipes;
  if (j_capacity) *j_capacity = d->cap;
  if (num_sms) *num_sms = d->num_sms;
  return SAPB_OK;
}

int sapb_set_stream(sapb_dev *d, void *stream) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  CK(d, cudaStreamSynchronize(d->stream));
  d->stream = stream ? (cudaStream_t)stream : d->own_stream;
  return SAPB_OK;
}

int sapb_reserve_j(sapb_dev *d, int nj_capacity) {
  if (!d || nj_capacity < 0) return fail(d, SAPB_EINVAL, "bad capacity");
  CK(d, cudaSetDevice(d->device));
  return grow_j(d, nj_capacity);
}

int sapb_j_stage_stride(const sapb_dev *d) { return d ? stage_stride(d->order) : 0; }
int sapb_i_stage_stride(const sapb_dev *d) { return d ? i_stride(d->order) : 0; }

double *sapb_j_stage(sapb_dev *d, int n) {
  if (!d || n < 0) return nullptr;
  if (n <= d->stage_cap) return d->stage_h;
  const int ss = stage_stride(d->order);
  const int cap = std::max(n, d->stage_cap + d->stage_cap / 2 + 1024);
  double *h = nullptr, *dd = nullptr;
  cudaSetDevice(d->device);
  if (cudaHostAlloc(&h, sizeof(double) * ss * (size_t)cap, cudaHostAllocDefault) != cudaSuccess ||
      cudaMalloc(&dd, sizeof(double) * ss * (size_t)cap) != cudaSuccess) {
    cudaGetLastError();
    if (h) cudaFreeHost(h);
    fail(d, SAPB_ENOMEM, "cannot allocate staging for %d j records", cap);
    return nullptr;
  }
  if (d->stage_h) {
    cudaStreamSynchronize(d->stream);  // a pending push may still read the old buffer
    memcpy(h, d->stage_h, sizeof(double) * ss * (size_t)d->stage_cap);
    cudaFreeHost(d->stage_h);
    cudaFree(d->stage_d);
  }
  d->stage_h = h;
  d->stage_d = dd;
  d->stage_cap = cap;
  return h;
}

int sapb_push_j(sapb_dev *d, int n) {
  if (!d || n < 0 || n > d->stage_cap) return fail(d, SAPB_EINVAL, "push of %d records", n);
  if (n == 0) return SAPB_OK;
  CK(d, cudaSetDevice(d->device));
  // grow the j store to cover the highest staged address
  int maxaddr = -1;
  const int ss = stage_stride(d->order);
  for (int k = 0; k < n; k++) {
    int addr;
    memcpy(&addr, d->stage_h + (size_t)k * ss, sizeof(int));
    if (addr < 0) return fail(d, SAPB_EINVAL, "negative j address %d", addr);
    maxaddr = std::max(maxaddr, addr);
  }
  if (maxaddr >= d->cap) {
    int rc = grow_j(d, std::max(maxaddr + 1, (int)(d->cap * 1.1) + 1));
    if (rc) return rc;
  }
  CK(d, cudaMemcpyAsync(d->stage_d, d->stage_h, sizeof(double) * ss * (size_t)n,
                        cudaMemcpyHostToDevice, d->stream));
  CK(d, launch_scatter(d->order, d->prec, d->stage_d, n, d->cap, d->js, d->pred, d->status_d,
                       d->stream));
  d->pred_gen++;
  // the host may overwrite the staging buffer once the copy has been consumed
  CK(d, cudaStreamSynchronize(d->stream));
  return SAPB_OK;
}

int sapb_predict(sapb_dev *d, int nj, double ti) {
  if (!d || nj < 0 || nj > d->cap) return fail(d, SAPB_EINVAL, "predict of %d j (capacity %d)", nj, d ? d->cap : 0);
  CK(d, cudaSetDevice(d->device));
  CK(d, launch_predict(d->order, d->prec, nj, ti, d->js, d->pred, d->stream));
  d->pred_gen++;
  return SAPB_OK;
}

double *sapb_i_stage(sapb_dev *d, int ni) {
  if (!d || ni < 0) return nullptr;
  cudaSetDevice(d->device);
  if (d->pending) {  // do not hand out a buffer an in-flight copy still reads
    cudaEventSynchronize(d->done);
  }
  if (ensure_i(d, ni) != SAPB_OK) return nullptr;
  return d->irec_h;
}

// Spatial mode pays for its per-call work (the i sort and bounds, the j
// gather after each prediction) from about 2^28 pairs, 1024 i and 65536 j on
// (B200, predict + force per call, neighbour lists on, i a random subset of
// the j: 1.04-1.06 x at 2^28 with 65536 to 262144 j, 1.07-1.12 x from 2^31;
// 0.89-0.95 x at 2^28 with 16384 or 32768 j, 0.91-1.00 x at 2^26 and 2^27;
// block-step active sets, which are spatially clustered, gain more);
// smaller calls run in address order.
constexpr double kSpatialMinPairs = 268435456.0;  // 2^28
constexpr int kSpatialMinI = 1024;
constexpr int kSpatialMinJ = 65536;

static bool use_spatial(const sapb_dev *d, int ni, int nj) {
  if (d->prec != DOUBLESINGLE || d->sp.mode == 0) return false;
  if (d->sp.mode == 2) return true;
  return ni >= kSpatialMinI && nj >= kSpatialMinJ && (double)ni * nj >= kSpatialMinPairs;
}

// Near-pair radius^2 of a mixed-precision call (FP32, compared with the
// kernels' double-single ds2); 0 turns the FP64 near-pair sums off.
static float near_r2(const sapb_dev *d, double eps2) {
  if (d->prec == DOUBLE || d->order == GRAPE5) return 0.0f;
  return (float)(d->near_k * eps2);
}

static int run_force(sapb_dev *d, int nj, int ni, const double *i_dev, double eps2, int flags,
                     double *res_dev, int *cnt_dev, int *list_dev) {
  if (nj <= 0 || nj > d->cap) return fail(d, SAPB_EINVAL, "nj = %d (capacity %d)", nj, d->cap);
  const Plan P = make_plan(d, ni, nj);
  const bool list = (flags & SAPB_F_NGB_LIST) != 0;
  if (list) CK(d, cudaMemsetAsync(cnt_dev, 0, sizeof(int) * (size_t)ni, d->stream));
  ForceArgs A{};
  A.pred = d->pred;
  bool spatial = use_spatial(d, ni, nj);
  if (spatial) {
    const int rc = spatial_prepare(d, nj, ni, i_dev);
    if (rc == SAPB_ENOMEM) spatial = false;  // no room for its buffers: address order
    else if (rc) return rc;
  }
  if (spatial) {
    A.pred = d->sp.spred;
    A.iperm = d->sp.iidx[1];
    A.ibound = d->sp.ibound;
    A.tbox = d->sp.tbox;
    A.far_c = d->sp.far_c;
    A.stats = d->sp.stats;
  }
  A.nj = nj;
  A.irec = i_dev;
  A.ni = ni;
  A.eps2 = eps2;
  A.near_r2 = near_r2(d, eps2);
  A.nslices = P.ns;
  A.i_tiles = P.i_tiles;
  A.do_list = list ? 1 : 0;
  A.ngb_count = cnt_dev;
  A.ngb_list = list_dev;
  A.status = d->status_d;
  if (P.ns > 1) {
    int rc = ensure_part(d, (size_t)P.ns * ni * kResStride);
    if (rc) return rc;
    A.out = d->part_d;
    A.write_partials = 1;
  } else {
    A.out = res_dev;
    A.write_partials = 0;
  }
  CK(d, launch_force(d->order, d->prec, A, P.tpi, P.ip, d->stream));
  if (P.ns > 1) {
    ReduceArgs R{d->part_d, P.ns, ni, res_dev, cnt_dev};
    CK(d, launch_reduce(R, d->stream));
  }
  return SAPB_OK;
}

int sapb_force(sapb_dev *d, int nj, int ni, double eps2, double ti, int flags) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  if (ni < 0 || ni > d->i_cap) return fail(d, SAPB_EINVAL, "ni = %d (staged capacity %d)", ni, d->i_cap);
  CK(d, cudaSetDevice(d->device));
  if (flags & SAPB_F_PREDICT) {
    int rc = sapb_predict(d, nj, ti);
    if (rc) return rc;
  }
  d->last_ni = ni;
  if (ni == 0) return SAPB_OK;
  const int is = i_stride(d->order);
  CK(d, cudaMemcpyAsync(d->irec_d, d->irec_h, sizeof(double) * is * (size_t)ni,
                        cudaMemcpyHostToDevice, d->stream));
  int rc = run_force(d, nj, ni, d->irec_d, eps2, flags, d->res_d, d->ngb_count_d, d->ngb_list_d);
  if (rc) return rc;
  CK(d, cudaMemcpyAsync(d->res_h, d->res_d, sizeof(double) * kResStride * (size_t)ni,
                        cudaMemcpyDeviceToHost, d->stream));
  CK(d, cudaMemcpyAsync(d->status_h, d->status_d, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(d, cudaEventRecord(d->done, d->stream));
  d->pending = true;
  return SAPB_OK;
}

int sapb_results(sapb_dev *d, const double **results, int *ni) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  CK(d, cudaSetDevice(d->device));
  if (d->pending) {
    CK(d, cudaEventSynchronize(d->done));
    d->pending = false;
  }
  if (results) *results = d->res_h;
  if (ni) *ni = d->last_ni;
  if (*d->status_h) {
    const int s = *d->status_h;
    *d->status_h = 0;
    cudaMemsetAsync(d->status_d, 0, sizeof(int), d->stream);
    if (s & kErrWaitTimeout) return fail(d, SAPB_ETIMEOUT, "force kernel: bounded wait for a j tile timed out");
    return fail(d, SAPB_EINVAL, "device reported status 0x%x", s);
  }
  return SAPB_OK;
}

int sapb_ngb_fetch(sapb_dev *d, int *counts, int *lists, int ni) {
  if (!d || ni < 0 || ni > d->i_cap) return fail(d, SAPB_EINVAL, "bad ni %d", ni);
  CK(d, cudaSetDevice(d->device));
  if (ni == 0) return SAPB_OK;
  if (counts)
    CK(d, cudaMemcpyAsync(counts, d->ngb_count_d, sizeof(int) * (size_t)ni,
                          cudaMemcpyDeviceToHost, d->stream));
  if (lists)
    CK(d, cudaMemcpyAsync(lists, d->ngb_list_d, sizeof(int) * kNgbPB * (size_t)ni,
                          cudaMemcpyDeviceToHost, d->stream));
  CK(d, cudaStreamSynchronize(d->stream));
  return SAPB_OK;
}

int sapb_force_device(sapb_dev *d, int nj, int ni, const double *i_dev, double eps2, int flags,
                      double *res_dev, int *ngb_count_dev, int *ngb_list_dev) {
  if (!d || !i_dev || !res_dev || ni < 0) return fail(d, SAPB_EINVAL, "bad arguments");
  if ((flags & SAPB_F_NGB_LIST) && (!ngb_count_dev || !ngb_list_dev))
    return fail(d, SAPB_EINVAL, "neighbour lists requested without buffers");
  CK(d, cudaSetDevice(d->device));
  if (ni == 0) return SAPB_OK;
  return run_force(d, nj, ni, i_dev, eps2, flags, res_dev, ngb_count_dev, ngb_list_dev);
}

int sapb_wait_selftest(sapb_dev *d, int limit_ms) {
  if (!d || limit_ms < 1 || limit_ms > 2000)
    return fail(d, SAPB_EINVAL, "wait self-test limit %d ms (1..2000)", limit_ms);
  CK(d, cudaSetDevice(d->device));
  CK(d, cudaMemsetAsync(d->status_d, 0, sizeof(int), d->stream));
  CK(d, launch_wait_selftest((uint64_t)limit_ms * 1000000ull, d->status_d, d->stream));
  int s = 0;
  CK(d, cudaMemcpyAsync(&s, d->status_d, sizeof(int), cudaMemcpyDeviceToHost, d->stream));
  CK(d, cudaStreamSynchronize(d->stream));
  CK(d, cudaMemsetAsync(d->status_d, 0, sizeof(int), d->stream));
  if (s & kErrWaitTimeout)
    return fail(d, SAPB_ETIMEOUT, "self-test: the bounded device wait gave up after %d ms",
                limit_ms);
  return fail(d, SAPB_ECUDA, "self-test: the wait on a barrier nothing arrives at returned");
}

int sapb_force_device_noalloc(sapb_dev *d, int nj, int ni, const double *i_dev, double eps2,
                              int flags, double *res_dev, int *ngb_count_dev,
                              int *ngb_list_dev) {
  if (!d || !i_dev || !res_dev || ni < 0) return fail(d, SAPB_EINVAL, "bad arguments");
  if ((flags & SAPB_F_NGB_LIST) && (!ngb_count_dev || !ngb_list_dev))
    return fail(d, SAPB_EINVAL, "neighbour lists requested without buffers");
  const size_t cap_records = SAPB_NOALLOC_SCRATCH_BYTES / (sizeof(double) * kResStride);
  if ((size_t)ni > cap_records)
    return fail(d, SAPB_EINVAL,
                "sapb_force_device_noalloc: ni = %d exceeds the fixed scratch (at most %zu "
                "i-particles per call)", ni, cap_records);
  CK(d, cudaSetDevice(d->device));
  if (ni == 0) return SAPB_OK;  // as sapb_force_device: an empty call does nothing
  if (nj <= 0 || nj > d->cap) return fail(d, SAPB_EINVAL, "nj = %d (capacity %d)", nj, d->cap);
  int rc = noalloc_setup(d);  // normally already done by sapb_open
  if (rc) return rc;
  double *scratch = g_noalloc_ptr[d->device];
  // Same plan as sapb_force_device, with the j-split capped so that the
  // per-slice partial records fit the fixed scratch.
  Plan P = make_plan(d, ni, nj);
  const int tj = force_tile_j();
  const int ntiles = (nj + tj - 1) / tj;
  const int max_ns = (int)std::max<size_t>(1, cap_records / (size_t)ni);
  if (P.ns > max_ns) {
    P.slice_tiles = (ntiles + max_ns - 1) / max_ns;
    P.ns = (ntiles + P.slice_tiles - 1) / P.slice_tiles;
  }
  const bool list = (flags & SAPB_F_NGB_LIST) != 0;
  if (list) CK(d, cudaMemsetAsync(ngb_count_dev, 0, sizeof(int) * (size_t)ni, d->stream));
  ForceArgs A{};
  A.pred = d->pred;
  A.nj = nj;
  A.irec = i_dev;
  A.ni = ni;
  A.eps2 = eps2;
  A.near_r2 = near_r2(d, eps2);
  A.nslices = P.ns;
  A.i_tiles = P.i_tiles;
  A.do_list = list ? 1 : 0;
  A.ngb_count = ngb_count_dev;
  A.ngb_list = ngb_list_dev;
  A.status = d->status_d;
  A.out = scratch;  // every (slice, valid i) record is written before it is read
  A.write_partials = 1;
  CK(d, launch_force(d->order, d->prec, A, P.tpi, P.ip, d->stream));
  ReduceArgs R{scratch, P.ns, ni, res_dev, ngb_count_dev};
  CK(d, launch_reduce(R, d->stream));
  return SAPB_OK;
}

int sapb_set_spatial(sapb_dev *d, int mode, double delta) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  if (mode < 0 || mode > 2 || !(delta >= 0.0) || delta > 1e-4)
    return fail(d, SAPB_EINVAL, "spatial mode %d, delta %g (mode 0..2, delta 0..1e-4)", mode, delta);
  d->sp.mode = mode;
  d->sp.far_c = (float)(0x1p-23 / (delta > 0.0 ? delta : kSpatialDelta));
  return SAPB_OK;
}

int sapb_set_near(sapb_dev *d, double factor) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  if (!(factor >= 0.0) || factor > 1e6)
    return fail(d, SAPB_EINVAL, "near-pair factor %g (0..1e6)", factor);
  d->near_k = factor;
  return SAPB_OK;
}

int sapb_spatial_stats(sapb_dev *d, unsigned long long *far_tiles,
                       unsigned long long *warp_tiles, int reset) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  CK(d, cudaSetDevice(d->device));
  unsigned long long h[2] = {0, 0};
  if (d->sp.stats) {
    CK(d, cudaMemcpyAsync(h, d->sp.stats, sizeof h, cudaMemcpyDeviceToHost, d->stream));
    if (reset) CK(d, cudaMemsetAsync(d->sp.stats, 0, sizeof h, d->stream));
    CK(d, cudaStreamSynchronize(d->stream));
  }
  if (far_tiles) *far_tiles = h[0];
  if (warp_tiles) *warp_tiles = h[1];
  return SAPB_OK;
}

int sapb_set_launch(sapb_dev *d, int tpi, int ip, int nslices) {
  if (!d) return fail(nullptr, SAPB_EINVAL, "null device");
  const bool ok_tpi = tpi == 0 || ((tpi == 1 || tpi == 2 || tpi == 4 || tpi == 8) && ip <= 2) ||
                      ((tpi == 16 || tpi == 32) && ip == 1) ||
                      ((tpi == 1 || tpi == 2) && ip == 4 && d->prec != DOUBLE);
  if (!ok_tpi || (ip != 0 && ip != 1 && ip != 2 && ip != 4) || nslices < 0 || (tpi && !ip))
    return fail(d, SAPB_EINVAL, "unsupported launch shape tpi=%d ip=%d slices=%d", tpi, ip, nslices);
  d->tpi = tpi;
  d->ip = ip;
  d->nslices = nslices;
  return SAPB_OK;
}

int sapb_get_plan(sapb_dev *d, int ni, int nj, int *tpi, int *ip, int *nslices) {
  if (!d || ni <= 0 || nj <= 0) return fail(d, SAPB_EINVAL, "bad sizes");
  const Plan P = make_plan(d, ni, nj);
  if (tpi) *tpi = P.tpi;
  if (ip) *ip = P.ip;
  if (nslices) *nslices = P.ns;
  return SAPB_OK;
}

int sapb_read_j(sapb_dev *d, int first, int n, double ti, int predict, double *out) {
  if (!d || first < 0 || n < 0 || first + n > d->cap || (n > 0 && !out))
    return fail(d, SAPB_EINVAL, "read of j[%d, %d) (capacity %d)", first, first + n, d ? d->cap : 0);
  if (n == 0) return SAPB_OK;
  CK(d, cudaSetDevice(d->device));
  const size_t need = (size_t)n * 24;
  int rc = ensure_part(d, need);
  if (rc) return rc;
  CK(d, launch_readj(d->order, first, n, ti, predict, d->js, d->part_d, d->stream));
  CK(d, cudaMemcpyAsync(out, d->part_d, sizeof(double) * need, cudaMemcpyDeviceToHost, d->stream));
  CK(d, cudaStreamSynchronize(d->stream));
  return SAPB_OK;
}

}  // extern "C"
