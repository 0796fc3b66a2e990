// Spatial ordering for the mixed-precision force kernels.
//
// The force kernel takes the double-single position difference (9 FMA-pipe
// operations of the 56 of a 6th-order pair) because close pairs, binaries
// 1e-6 apart at |x| ~ 1, need it.  Far pairs do not: with both positions
// rounded to float, the difference of the high parts alone is within
// 2^-24 (|xi| + |xj|) of the exact one, i.e. within delta (relative) once the
// pair is at least |x|max * 2^-23 / delta apart.  When j records and i
// positions are both in Morton order, most (warp, j tile) pairs of a large
// call are that far apart as whole boxes, and the kernel runs those tiles
// with the 3-operation difference (pair_mix2_far).
//
// Per force call in spatial mode:
//   j (once per change of the predicted records; the first three steps only
//   for a new j count and after every 16 changes, otherwise the previous
//   order is reused):
//     frame_kernel   bounding box of the j high parts (ordered-int atomics)
//     jkey_kernel    30-bit Morton key of every j record in that box
//     radix sort     (key, record) pairs, CUB
//     gather_kernel  records in key order + per-tile box and first key
//   i (every call):
//     ikey_kernel    Morton key of every i record in the same box
//     radix sort     (key, i record) pairs, CUB
//     bound_kernel   for i position g, an upper bound of its nearest-neighbour
//                    ds2: the exact minimum over the j tile whose key range
//                    holds its key
// Neither ordering changes what is summed, only the order; nearest
// neighbours and neighbour lists stay exact (the kernel's far test).
#include <float.h>
#include <limits.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>

#include "sapb_dev.h"
#include "sapb_kernels.cuh"
#include "sapb_launch.h"
#include "sapb_pair.cuh"

namespace sapb {

// Float <-> int mapping that preserves order, for atomicMin/Max on floats.
__device__ __forceinline__ int ord_enc(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord_dec(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

// 10 bits spread to every third bit (bit interleaving of a Morton code).
__device__ __forceinline__ unsigned spread3(unsigned v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

struct Frame {
  float lo[3];
  float scale;  // cells per unit length (one scale for all axes: cubic cells)
};

__device__ __forceinline__ Frame load_frame(const int *f) {
  Frame F;
  float ext = 0.f;
  for (int d = 0; d < 3; d++) {
    F.lo[d] = ord_dec(f[d]);
    ext = fmaxf(ext, ord_dec(f[3 + d]) - F.lo[d]);
  }
  F.scale = ext > 0.f ? 1023.99f / ext : 0.f;
  return F;
}

// Positions outside the box (i not among the j) and NaNs clamp to its faces.
__device__ __forceinline__ unsigned morton30(const Frame &F, float x, float y, float z) {
  const float c[3] = {x, y, z};
  unsigned q[3];
  for (int d = 0; d < 3; d++) q[d] = (unsigned)fminf(fmaxf((c[d] - F.lo[d]) * F.scale, 0.f), 1023.f);
  return spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
}

__global__ void frame_init_kernel(int *frame) {
  const int t = threadIdx.x;
  if (t < 3) frame[t] = INT_MAX;
  else if (t < 6) frame[t] = INT_MIN;
}

// Bounding box of the j high parts (field 0 of each record).
template <int RS>
__global__ void __launch_bounds__(256) frame_kernel(const float4 *__restrict__ pred, int nj,
                                                    int *frame) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nj; k += gridDim.x * blockDim.x) {
    const float4 r = pred[(size_t)k * RS];
    lo[0] = fminf(lo[0], r.x); hi[0] = fmaxf(hi[0], r.x);
    lo[1] = fminf(lo[1], r.y); hi[1] = fmaxf(hi[1], r.y);
    lo[2] = fminf(lo[2], r.z); hi[2] = fmaxf(hi[2], r.z);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    for (int d = 0; d < 3; d++) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 3; d++) {
      atomicMin(frame + d, ord_enc(lo[d]));
      atomicMax(frame + 3 + d, ord_enc(hi[d]));
    }
}

template <int RS>
__global__ void __launch_bounds__(256) jkey_kernel(const float4 *__restrict__ pred, int nj,
                                                   const int *frame, unsigned *key, int *idx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nj) return;
  const Frame F = load_frame(frame);
  const float4 r = pred[(size_t)k * RS];
  key[k] = morton30(F, r.x, r.y, r.z);
  idx[k] = k;
}

// One block per tile of kTJ = 256 sorted records: copies the records into
// key order and writes the tile's box (high parts) and first key.
template <int RS>
__global__ void __launch_bounds__(256) gather_kernel(const float4 *__restrict__ pred,
                                                     const int *__restrict__ idx,
                                                     const unsigned *__restrict__ key, int nj,
                                                     float4 *__restrict__ spred, float4 *tbox,
                                                     unsigned *tkey) {
  static_assert(kTJ == 256, "one thread per record of a tile");
  __shared__ float red[8][7];
  const int tile = blockIdx.x;
  const int s = tile * kTJ + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX}, ab = 0.f;
  if (s < nj) {
    const int src = idx[s];
#pragma unroll
    for (int f = 0; f < RS; f++) spred[(size_t)s * RS + f] = pred[(size_t)src * RS + f];
    const float4 r = pred[(size_t)src * RS];
    lo[0] = hi[0] = r.x;
    lo[1] = hi[1] = r.y;
    lo[2] = hi[2] = r.z;
    ab = fmaxf(fabsf(r.x), fmaxf(fabsf(r.y), fabsf(r.z)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; d++) {
      lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    ab = fmaxf(ab, __shfl_xor_sync(0xffffffffu, ab, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; d++) {
      red[w][d] = lo[d];
      red[w][3 + d] = hi[d];
    }
    red[w][6] = ab;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int v = 1; v < 8; v++) {
      for (int d = 0; d < 3; d++) {
        lo[d] = fminf(lo[d], red[v][d]);
        hi[d] = fmaxf(hi[d], red[v][3 + d]);
      }
      ab = fmaxf(ab, red[v][6]);
    }
    tbox[2 * tile] = make_float4(lo[0], lo[1], lo[2], ab);
    tbox[2 * tile + 1] = make_float4(hi[0], hi[1], hi[2], 0.f);
    tkey[tile] = key[tile * kTJ];
  }
}

__global__ void __launch_bounds__(256) ikey_kernel(const double *__restrict__ irec, int ni,
                                                   int istride, const int *frame, unsigned *key,
                                                   int *idx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ni) return;
  const Frame F = load_frame(frame);
  const double *r = irec + (size_t)k * istride;
  key[k] = morton30(F, (float)r[0], (float)r[1], (float)r[2]);
  idx[k] = k;
}

// Upper bound of the nearest-neighbour ds2 of i position g: the exact
// minimum (the force kernel's double-single ds2, self pair masked by id) over
// the j tile whose key range holds the i key -- the last tile whose first
// key is <= it, tile 0 if none -- i.e. over spatial neighbours of the i.
// 2^lg lanes per i (1..32, aligned groups within a warp): the lanes take
// every 2^lg-th record of the tile and the minimum is reduced across the
// group.  Small calls take 32 lanes per i to fill the GPU; calls with enough
// i for one thread each take one (the whole warp then reads one tile).
template <int RS>
__global__ void __launch_bounds__(256) bound_kernel(const double *__restrict__ irec, int istride,
                                                    const int *__restrict__ iperm,
                                                    const unsigned *__restrict__ ikey, int ni,
                                                    int lg, const float4 *__restrict__ spred,
                                                    int nj, const unsigned *__restrict__ tkey,
                                                    float *bound) {
  const int L = 1 << lg;
  const int sub = threadIdx.x & (L - 1);
  const int gt = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> lg);
  const bool valid = gt < ni;  // uniform within a group
  const int g = valid ? gt : ni - 1;  // past the end: repeat the last i, write nothing
  const int ntiles = (nj + kTJ - 1) / kTJ;
  const unsigned k = ikey[g];
  int lo = 0, hi = ntiles;  // first tile with tkey > k lies in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tkey[mid] <= k) lo = mid + 1;
    else hi = mid;
  }
  const int t = max(lo - 1, 0);
  const double *r = irec + (size_t)iperm[g] * istride;
  IMix I{};
  I.xh = (float)r[0];
  I.yh = (float)r[1];
  I.zh = (float)r[2];
  I.xl = (float)(r[0] - (double)I.xh);
  I.yl = (float)(r[1] - (double)I.yh);
  I.zl = (float)(r[2] - (double)I.zh);
  I.id = __double2loint(r[7]);
  const int cnt = min(kTJ, nj - t * kTJ);
  const float4 *rec = spred + (size_t)t * kTJ * RS;
  float m = FLT_MAX;
  for (int q = sub; q < cnt; q += L) {
    float dx, dy, dz;
    m = fminf(m, pair_dr_mix(I, rec[q * RS + 0], rec[q * RS + 1], dx, dy, dz));
  }
  for (int o = L >> 1; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (valid && sub == 0) bound[g] = m;
}

}  // namespace sapb

using namespace sapb;

// ---------------------------------------------------------------------
// Buffers (grown on demand, freed by spatial_free).
// ---------------------------------------------------------------------
static size_t sort_temp_bytes(int n) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned *)nullptr, (unsigned *)nullptr,
                                  (const int *)nullptr, (int *)nullptr, n, 0, 30);
  return bytes;
}

void spatial_free(sapb_dev *d) {
  SpatialBufs &S = d->sp;
  void *ptrs[] = {S.spred, S.jkey[0], S.jkey[1], S.jidx[0], S.jidx[1], S.tbox, S.tkey,
                  S.ikey[0], S.ikey[1], S.iidx[0], S.iidx[1], S.ibound, S.frame, S.temp, S.stats};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  const int mode = S.mode;
  const float far_c = S.far_c;
  S = SpatialBufs{};
  S.mode = mode;
  S.far_c = far_c;
}

static cudaError_t grow_temp(SpatialBufs &S, int n) {
  const size_t need = sort_temp_bytes(n);
  if (need <= S.temp_bytes) return cudaSuccess;
  if (S.temp) cudaFree(S.temp);
  S.temp = nullptr;
  S.temp_bytes = 0;
  cudaError_t e = cudaMalloc(&S.temp, need);
  if (e == cudaSuccess) S.temp_bytes = need;
  return e;
}

static cudaError_t ensure_j(sapb_dev *d, size_t rec_bytes) {
  SpatialBufs &S = d->sp;
  if (!S.frame) {
    cudaError_t e = cudaMalloc(&S.frame, 8 * sizeof(int));
    if (e != cudaSuccess) return e;
  }
  if (!S.stats) {
    cudaError_t e = cudaMalloc(&S.stats, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(S.stats, 0, 2 * sizeof(unsigned long long), d->stream);
    if (e != cudaSuccess) return e;
  }
  if (S.jcap >= d->cap) return cudaSuccess;
  void *ptrs[] = {S.spred, S.jkey[0], S.jkey[1], S.jidx[0], S.jidx[1], S.tbox, S.tkey};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  S.spred = nullptr; S.jkey[0] = S.jkey[1] = nullptr; S.jidx[0] = S.jidx[1] = nullptr;
  S.tbox = nullptr; S.tkey = nullptr; S.jcap = 0;
  const int cap = d->cap;
  const int tiles = (cap + kTJ - 1) / kTJ;
  cudaError_t e = cudaMalloc(&S.spred, rec_bytes * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.jkey[0], sizeof(unsigned) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.jkey[1], sizeof(unsigned) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.jidx[0], sizeof(int) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.jidx[1], sizeof(int) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.tbox, 2 * sizeof(float4) * (size_t)tiles);
  if (e == cudaSuccess) e = cudaMalloc(&S.tkey, sizeof(unsigned) * (size_t)tiles);
  if (e == cudaSuccess) e = grow_temp(S, cap);
  if (e != cudaSuccess) return e;
  S.jcap = cap;
  S.valid_nj = -1;
  return cudaSuccess;
}

static cudaError_t ensure_i(SpatialBufs &S, int ni) {
  if (S.icap >= ni) return cudaSuccess;
  void *ptrs[] = {S.ikey[0], S.ikey[1], S.iidx[0], S.iidx[1], S.ibound};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  S.ikey[0] = S.ikey[1] = nullptr; S.iidx[0] = S.iidx[1] = nullptr; S.ibound = nullptr;
  S.icap = 0;
  const int cap = std::max(ni, 16384);
  cudaError_t e = cudaMalloc(&S.ikey[0], sizeof(unsigned) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.ikey[1], sizeof(unsigned) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.iidx[0], sizeof(int) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.iidx[1], sizeof(int) * (size_t)cap);
  if (e == cudaSuccess) e = cudaMalloc(&S.ibound, sizeof(float) * (size_t)cap);
  if (e == cudaSuccess) e = grow_temp(S, cap);
  if (e != cudaSuccess) return e;
  S.icap = cap;
  return cudaSuccess;
}

// Full ordering (full != 0): bounding box, keys, sort, then the gather.
// Otherwise only the gather, with the previous call's order and keys: the
// records are in the order of their positions some predictions ago, each
// tile's box is recomputed from the current positions (so the far test stays
// exact), and the first keys, which only pick the tile the nearest-neighbour
// bound is taken over, stay valid as an order.
template <int RS>
static cudaError_t order_j(sapb_dev *d, int nj, bool full, cudaStream_t st) {
  SpatialBufs &S = d->sp;
  const float4 *pred = static_cast<const float4 *>(d->pred);
  const int tiles = (nj + kTJ - 1) / kTJ;
  if (!full) {
    gather_kernel<RS><<<tiles, kTJ, 0, st>>>(pred, S.jidx[1], S.jkey[1], nj,
                                             static_cast<float4 *>(S.spred), S.tbox, S.tkey);
    return cudaGetLastError();
  }
  frame_init_kernel<<<1, 32, 0, st>>>(S.frame);
  const int blocks = std::min((nj + 255) / 256, std::max(d->num_sms, 1) * 8);
  frame_kernel<RS><<<blocks, 256, 0, st>>>(pred, nj, S.frame);
  jkey_kernel<RS><<<(nj + 255) / 256, 256, 0, st>>>(pred, nj, S.frame, S.jkey[0], S.jidx[0]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  size_t tb = S.temp_bytes;
  e = cub::DeviceRadixSort::SortPairs(S.temp, tb, S.jkey[0], S.jkey[1], S.jidx[0], S.jidx[1], nj,
                                      0, 30, st);
  if (e != cudaSuccess) return e;
  gather_kernel<RS><<<tiles, kTJ, 0, st>>>(pred, S.jidx[1], S.jkey[1], nj,
                                           static_cast<float4 *>(S.spred), S.tbox, S.tkey);
  return cudaGetLastError();
}

// Gathers with a previous order between two full orderings: the predicted
// records change every block step, while particles cross a Morton cell
// (~1/1000 of the cluster) in many steps.
constexpr int kReorderEvery = 16;

int spatial_prepare(sapb_dev *d, int nj, int ni, const double *i_dev) {
  SpatialBufs &S = d->sp;
  cudaStream_t st = d->stream;
  const int rs = pred_fields(d->order);
  cudaError_t e = ensure_j(d, 16u * rs);
  if (e == cudaSuccess) e = ensure_i(S, ni);
  if (e != cudaSuccess) {
    cudaGetLastError();
    spatial_free(d);
    return sapb_fail(d, SAPB_ENOMEM, "spatial ordering buffers: %s", cudaGetErrorString(e));
  }
  if (S.valid_nj != nj || d->pred_gen != S.valid_gen) {
    // a new order when the j count changed or after kReorderEvery reuses
    const bool full = S.valid_nj != nj || S.order_age >= kReorderEvery;
    S.order_age = full ? 0 : S.order_age + 1;
    e = rs == 4 ? order_j<4>(d, nj, full, st) : order_j<3>(d, nj, full, st);
    if (e != cudaSuccess)
      return sapb_fail(d, SAPB_ECUDA, "spatial ordering of j: %s", cudaGetErrorString(e));
    S.valid_nj = nj;
    S.valid_gen = d->pred_gen;
  }
  ikey_kernel<<<(ni + 255) / 256, 256, 0, st>>>(i_dev, ni, i_stride(d->order), S.frame, S.ikey[0],
                                                S.iidx[0]);
  e = cudaGetLastError();
  size_t tb = S.temp_bytes;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(S.temp, tb, S.ikey[0], S.ikey[1], S.iidx[0], S.iidx[1],
                                        ni, 0, 30, st);
  if (e == cudaSuccess) {
    const int is = i_stride(d->order);
    const float4 *sp4 = static_cast<const float4 *>(S.spred);
    // lanes per i: enough threads to fill every SM (2048 each), at most 32
    const long want = (long)d->num_sms * 2048;
    int lg = 0;
    while (lg < 5 && ((long)ni << lg) < want) lg++;
    const long threads = (long)ni << lg;
    const int nb = (int)((threads + 255) / 256);
    if (rs == 4)
      bound_kernel<4><<<nb, 256, 0, st>>>(i_dev, is, S.iidx[1], S.ikey[1], ni, lg, sp4, nj,
                                          S.tkey, S.ibound);
    else
      bound_kernel<3><<<nb, 256, 0, st>>>(i_dev, is, S.iidx[1], S.ikey[1], ni, lg, sp4, nj,
                                          S.tkey, S.ibound);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return sapb_fail(d, SAPB_ECUDA, "spatial ordering of i: %s", cudaGetErrorString(e));
  return SAPB_OK;
}
