/*
 * TEST INFRASTRUCTURE ONLY: a launcher for the reference's own CUDA kernels
 * (oracle/_ref/ref_kernels.cubin, built by oracle/Makefile from the
 * reference sources).  It is used by the GPU parity tests and by the
 * fixture generator to obtain the reference's answers on seeded inputs.
 * The product library never links or calls it.
 *
 * The launch geometry follows the reference host code:
 *   - dev_predictor: setWork_2D(128, nj) (lib/src/sapporohostclass.cpp:1281,
 *     lib/include/cudadev.h setWork_2D: ng = ceil(n/128) blocks arranged as
 *     nx = floor(sqrt(ng)), ny = ceil(ng/nx));
 *   - dev_reset_buffers: setWork_2D(256, ni_total) (:1487-1495);
 *   - dev_evaluate_gravity_*: one launch per 256-i chunk (:1499-1598) with
 *     p = ni (rounded to 32 for ni > 128, to 16 for ni > 96, 4th order only),
 *     q = min(512 / p, 32), NBLOCKS = SMs * 16 (lib/include/defines.h:117-120,
 *     lib/include/sapdevclass.h:139-142), dynamic shared memory p*q*perThreadSM
 *     (lib/include/defines.h:48-67) and nj per (block, row) from n_norm
 *     (:40-44, :1560-1561).
 *
 * Safety: the reference kernel returns early for padded i-threads
 * (kernels.cu:896) before later __syncthreads calls.  To keep every barrier
 * uniform this launcher only accepts 4th-order i-counts whose last chunk needs
 * no rounding (6th order never rounds); other counts return SAPREF_EBADSIZE
 * without launching anything.  i-buffers are padded to a multiple of 256
 * entries and zero-filled, so every read of the kernel stays in bounds.
 */
#include <cuda.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

namespace {

enum { GRAPE5 = 0, FOURTH = 1, SIXTH = 2 };
enum { FLOAT = 0, DOUBLESINGLE = 1, DOUBLE = 2 };

const int kNgbPB = 256;  // lib/include/defines.h:9
const int kNThreads = 256;  // lib/include/defines.h:18
const int kNThreads2 = 512;  // lib/include/defines.h:23

struct State {
  bool ready = false;
  CUdevice dev = 0;
  CUcontext ctx = nullptr;
  CUmodule mod = nullptr;
  CUfunction predictor = nullptr, reset = nullptr;
  CUfunction grav[3][3] = {};  // [order][precision]
  int nsm = 0;
  int warp = 32;
};
State g;
char g_err[512];

#define SAPREF_CHECK(call)                                              \
  do {                                                                  \
    CUresult r_ = (call);                                               \
    if (r_ != CUDA_SUCCESS) {                                           \
      const char *s_ = nullptr;                                         \
      cuGetErrorString(r_, &s_);                                        \
      snprintf(g_err, sizeof g_err, "%s failed: %s", #call, s_ ? s_ : "?"); \
      return -(int)r_ - 1000;                                           \
    }                                                                   \
  } while (0)

int per_thread_sm(int order, int precision) {
  // lib/include/defines.h:48-67
  if (order == FOURTH && precision == DOUBLESINGLE) return 48;
  if (order == FOURTH && precision == DOUBLE) return 64;
  if (order == SIXTH && precision == DOUBLESINGLE) return 60;
  if (order == SIXTH && precision == DOUBLE) return 88;
  return -1;
}

int n_norm(int n, int j) {  // lib/src/sapporohostclass.cpp:40-44
  n = ((n - 1) / j) * j + j;
  if (n == 0) n = j;
  return n;
}

void grid_2d(int n_threads, int items, unsigned *gx, unsigned *gy) {
  const int ng = (items - 1) / n_threads + 1;
  const int nx = (int)sqrt((double)ng);
  const int ny = (ng - 1) / nx + 1;
  *gx = (unsigned)nx;
  *gy = (unsigned)ny;
}

struct DevBuf {
  CUdeviceptr p = 0;
  ~DevBuf() {
    if (p) cuMemFree(p);
  }
};

}  // namespace

extern "C" {

const char *sapref_last_error(void) { return g_err; }

int sapref_open(const char *cubin_path, int device) {
  if (g.ready) return 0;
  SAPREF_CHECK(cuInit(0));
  SAPREF_CHECK(cuDeviceGet(&g.dev, device));
  SAPREF_CHECK(cuDevicePrimaryCtxRetain(&g.ctx, g.dev));
  SAPREF_CHECK(cuCtxSetCurrent(g.ctx));
  SAPREF_CHECK(cuDeviceGetAttribute(&g.nsm, CU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, g.dev));
  SAPREF_CHECK(cuDeviceGetAttribute(&g.warp, CU_DEVICE_ATTRIBUTE_WARP_SIZE, g.dev));
  SAPREF_CHECK(cuModuleLoad(&g.mod, cubin_path));
  SAPREF_CHECK(cuModuleGetFunction(&g.predictor, g.mod, "dev_predictor"));
  SAPREF_CHECK(cuModuleGetFunction(&g.reset, g.mod, "dev_reset_buffers"));
  SAPREF_CHECK(cuModuleGetFunction(&g.grav[FOURTH][DOUBLESINGLE], g.mod, "dev_evaluate_gravity_fourth_DS"));
  SAPREF_CHECK(cuModuleGetFunction(&g.grav[FOURTH][DOUBLE], g.mod, "dev_evaluate_gravity_fourth_double"));
  SAPREF_CHECK(cuModuleGetFunction(&g.grav[SIXTH][DOUBLESINGLE], g.mod, "dev_evaluate_gravity_sixth_DS"));
  SAPREF_CHECK(cuModuleGetFunction(&g.grav[SIXTH][DOUBLE], g.mod, "dev_evaluate_gravity_sixth_double"));
  g.ready = true;
  return 0;
}

int sapref_num_sms(void) { return g.nsm; }

/* Whether the reference geometry for this (order, ni_total) keeps every
 * barrier uniform; see the file comment. */
int sapref_size_ok(int order, int ni_total) {
  if (ni_total <= 0) return 0;
  if (order != FOURTH) return 1;
  const int last = ni_total - ((ni_total - 1) / kNThreads) * kNThreads;
  int mult = 1;
  if (last > 128) mult = 32;
  else if (last > 96) mult = 16;
  return (last % mult) == 0;
}

/* Runs dev_predictor.  Arrays use the reference layout: t = double2[nj]
 * (t, dt), pos = double4[nj] (x, y, z, m), vel/acc/jrk/snp/crk = double4[nj].
 * Outputs ppos/pvel/pacc are double4[nj].  snp/crk/pacc may be NULL for 4th
 * order. */
int sapref_predict(int order, int nj, double ti, const double *t,
                   const double *pos, const double *vel, const double *acc,
                   const double *jrk, const double *snp, const double *crk,
                   double *ppos, double *pvel, double *pacc) {
  if (!g.ready) return -1;
  if (nj <= 0) return 0;
  SAPREF_CHECK(cuCtxSetCurrent(g.ctx));
  const size_t b4 = sizeof(double) * 4 * (size_t)nj;
  DevBuf dt, dpos, dvel, dacc, djrk, dsnp, dcrk, dpp, dpv, dpa;
  SAPREF_CHECK(cuMemAlloc(&dt.p, sizeof(double) * 2 * (size_t)nj));
  CUdeviceptr *bufs[] = {&dpos.p, &dvel.p, &dacc.p, &djrk.p, &dsnp.p, &dcrk.p, &dpp.p, &dpv.p, &dpa.p};
  for (CUdeviceptr *b : bufs) {
    SAPREF_CHECK(cuMemAlloc(b, b4));
    SAPREF_CHECK(cuMemsetD8(*b, 0, b4));
  }
  SAPREF_CHECK(cuMemcpyHtoD(dt.p, t, sizeof(double) * 2 * (size_t)nj));
  SAPREF_CHECK(cuMemcpyHtoD(dpos.p, pos, b4));
  SAPREF_CHECK(cuMemcpyHtoD(dvel.p, vel, b4));
  SAPREF_CHECK(cuMemcpyHtoD(dacc.p, acc, b4));
  SAPREF_CHECK(cuMemcpyHtoD(djrk.p, jrk, b4));
  if (order >= SIXTH) {
    SAPREF_CHECK(cuMemcpyHtoD(dsnp.p, snp, b4));
    SAPREF_CHECK(cuMemcpyHtoD(dcrk.p, crk, b4));
  }
  int a_nj = nj, a_order = order;
  double a_ti = ti;
  void *args[] = {&a_nj, &a_ti, &a_order, &dt.p, &dpp.p, &dpos.p, &dpv.p,
                  &dvel.p, &dacc.p, &djrk.p, &dpa.p, &dsnp.p, &dcrk.p};
  unsigned gx, gy;
  grid_2d(128, nj, &gx, &gy);
  SAPREF_CHECK(cuLaunchKernel(g.predictor, gx, gy, 1, 128, 1, 1, 0, 0, args, nullptr));
  SAPREF_CHECK(cuCtxSynchronize());
  SAPREF_CHECK(cuMemcpyDtoH(ppos, dpp.p, b4));
  SAPREF_CHECK(cuMemcpyDtoH(pvel, dpv.p, b4));
  if (order >= SIXTH && pacc) SAPREF_CHECK(cuMemcpyDtoH(pacc, dpa.p, b4));
  return 0;
}

/* Runs dev_reset_buffers + the gravity kernel chunks exactly as
 * sapporo::evaluate_gravity does, `reps` times (timed with events; the mean
 * milliseconds per full sweep is written to *ms when ms != NULL).
 *
 * j arrays (predicted): jpos double4[nj] (x, y, z, m), jvel double4[nj]
 * (v, eps), jacc double4[nj] (6th only, else NULL), jid int[nj].
 * i arrays: ipos double4[ni] (x, y, z, h2), ivel double4[ni] (v, eps2),
 * iacc double4[ni] (6th only), iid int[ni].
 * Outputs: result double4[3*ni] (acc+pot | jerk+w | snap), ds float2[ni]
 * (nnb bits, ds2min), ngb_count int[ni], ngb_list int[ni*256] (may be NULL).
 */
int sapref_gravity(int order, int precision, int nj, const double *jpos,
                   const double *jvel, const double *jacc, const int *jid,
                   int ni, const double *ipos, const double *ivel,
                   const double *iacc, const int *iid, double eps2,
                   double *result, float *ds, int *ngb_count, int *ngb_list,
                   int reps, float *ms) {
  if (!g.ready) return -1;
  if (order != FOURTH && order != SIXTH) return -2;
  if (precision != DOUBLE && precision != DOUBLESINGLE) return -2;
  if (!sapref_size_ok(order, ni)) {
    snprintf(g_err, sizeof g_err, "i-count %d would make the reference kernel exit threads before a barrier", ni);
    return -3;
  }
  if (nj <= 0) return -2;
  if (reps < 1) reps = 1;
  SAPREF_CHECK(cuCtxSetCurrent(g.ctx));
  const int ni_pad = ((ni + kNThreads - 1) / kNThreads) * kNThreads;
  const size_t bj = sizeof(double) * 4 * (size_t)nj;
  const size_t bi = sizeof(double) * 4 * (size_t)ni_pad;
  DevBuf djp, djv, dja, djid, dip, div, dia, diid, dres, dds, dcnt, dlist;
  SAPREF_CHECK(cuMemAlloc(&djp.p, bj));
  SAPREF_CHECK(cuMemAlloc(&djv.p, bj));
  SAPREF_CHECK(cuMemAlloc(&dja.p, bj));
  SAPREF_CHECK(cuMemAlloc(&djid.p, sizeof(int) * (size_t)nj));
  SAPREF_CHECK(cuMemAlloc(&dip.p, bi));
  SAPREF_CHECK(cuMemAlloc(&div.p, bi));
  SAPREF_CHECK(cuMemAlloc(&dia.p, bi));
  SAPREF_CHECK(cuMemAlloc(&diid.p, sizeof(int) * (size_t)ni_pad));
  SAPREF_CHECK(cuMemAlloc(&dres.p, sizeof(double) * 4 * 3 * (size_t)ni_pad));
  SAPREF_CHECK(cuMemAlloc(&dds.p, sizeof(float) * 2 * (size_t)ni_pad));
  SAPREF_CHECK(cuMemAlloc(&dcnt.p, sizeof(int) * ((size_t)ni_pad + 1)));
  SAPREF_CHECK(cuMemAlloc(&dlist.p, sizeof(int) * (size_t)kNgbPB * ni_pad));
  SAPREF_CHECK(cuMemsetD8(dja.p, 0, bj));
  SAPREF_CHECK(cuMemsetD8(dip.p, 0, bi));
  SAPREF_CHECK(cuMemsetD8(div.p, 0, bi));
  SAPREF_CHECK(cuMemsetD8(dia.p, 0, bi));
  SAPREF_CHECK(cuMemsetD8(diid.p, 0, sizeof(int) * (size_t)ni_pad));
  SAPREF_CHECK(cuMemsetD8(dlist.p, 0, sizeof(int) * (size_t)kNgbPB * ni_pad));
  SAPREF_CHECK(cuMemcpyHtoD(djp.p, jpos, bj));
  SAPREF_CHECK(cuMemcpyHtoD(djv.p, jvel, bj));
  if (order >= SIXTH) SAPREF_CHECK(cuMemcpyHtoD(dja.p, jacc, bj));
  SAPREF_CHECK(cuMemcpyHtoD(djid.p, jid, sizeof(int) * (size_t)nj));
  SAPREF_CHECK(cuMemcpyHtoD(dip.p, ipos, sizeof(double) * 4 * (size_t)ni));
  SAPREF_CHECK(cuMemcpyHtoD(div.p, ivel, sizeof(double) * 4 * (size_t)ni));
  if (order >= SIXTH) SAPREF_CHECK(cuMemcpyHtoD(dia.p, iacc, sizeof(double) * 4 * (size_t)ni));
  SAPREF_CHECK(cuMemcpyHtoD(diid.p, iid, sizeof(int) * (size_t)ni));

  CUfunction kern = g.grav[order][precision];
  const int pts = per_thread_sm(order, precision);
  const int nblocks = g.nsm * 16;
  int max_dyn = 0;
  {
    // Largest launch below uses p*q <= 512 threads.
    const int need = kNThreads2 * pts;
    if (need > 48 * 1024) {
      SAPREF_CHECK(cuFuncSetAttribute(kern, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, need));
    }
    max_dyn = need;
  }
  (void)max_dyn;

  CUevent e0, e1;
  SAPREF_CHECK(cuEventCreate(&e0, CU_EVENT_DEFAULT));
  SAPREF_CHECK(cuEventCreate(&e1, CU_EVENT_DEFAULT));
  float total_ms = 0.f;
  for (int r = 0; r < reps; r++) {
    SAPREF_CHECK(cuEventRecord(e0, 0));
    {
      int a_ni = ni, a_ngb = 1, a_list = 1, a_order = order;
      void *args[] = {&a_ni, &a_ngb, &a_list, &a_order, &dres.p, &dds.p, &dcnt.p};
      unsigned gx, gy;
      grid_2d(256, ni, &gx, &gy);
      SAPREF_CHECK(cuLaunchKernel(g.reset, gx, gy, 1, 256, 1, 1, 0, 0, args, nullptr));
    }
    for (int ni_offset = 0; ni_offset < ni; ni_offset += kNThreads) {
      int nic = std::min(ni - ni_offset, kNThreads);
      int mult = 1;
      if (order <= FOURTH) {
        if (nic > 128) mult = g.warp;
        else if (nic > 96) mult = g.warp / 2;
      }
      nic = ((nic + mult - 1) / mult) * mult;
      const int p = nic;
      const int q = std::min(kNThreads2 / nic, 32);
      const int shmem = p * q * pts;
      const int nj_scaled = n_norm(nj, q * nblocks);
      int this_block = nj_scaled / (nblocks * q);
      int a_nj = nj, a_off = ni_offset, a_ni = ni;
      double a_eps = eps2;
      void *args[] = {&a_nj,   &this_block, &a_off,  &a_ni,   &djp.p,  &dip.p,
                      &dres.p, &a_eps,      &djv.p,  &djid.p, &div.p,  &diid.p,
                      &dds.p,  &dcnt.p,     &dlist.p, &dia.p, &dja.p};
      SAPREF_CHECK(cuLaunchKernel(kern, nblocks, 1, 1, p, q, 1, shmem, 0, args, nullptr));
    }
    SAPREF_CHECK(cuEventRecord(e1, 0));
    SAPREF_CHECK(cuEventSynchronize(e1));
    float t = 0.f;
    SAPREF_CHECK(cuEventElapsedTime(&t, e0, e1));
    total_ms += t;
  }
  cuEventDestroy(e0);
  cuEventDestroy(e1);
  if (ms) *ms = total_ms / reps;
  SAPREF_CHECK(cuMemcpyDtoH(result, dres.p, sizeof(double) * 4 * 3 * (size_t)ni));
  // result layout on the device is [acc ni_total][jrk ni_total][snp ni_total]
  SAPREF_CHECK(cuMemcpyDtoH(ds, dds.p, sizeof(float) * 2 * (size_t)ni));
  SAPREF_CHECK(cuMemcpyDtoH(ngb_count, dcnt.p, sizeof(int) * (size_t)ni));
  if (ngb_list) SAPREF_CHECK(cuMemcpyDtoH(ngb_list, dlist.p, sizeof(int) * (size_t)kNgbPB * ni));
  return 0;
}

}  // extern "C"
