// Batched execution: block-timestep steps and ensembles of independent
// clusters in one persistent launch (captured once in a CUDA graph by
// sapb_batch.cu).  Work is described in device memory (BatchParams,
// BatchCluster, BatchItem in sapb_internal.cuh), so the same graph runs any
// step; per-cluster prediction times and softening are supported.
#include "sapb_kernels.cuh"
#include "sapb_launch.h"
#include "sapb_pair.cuh"

namespace sapb {

// Cluster containing index x of a sorted-by-first range table (first/count
// fields selected by the accessor); -1 if none.
template <typename F>
__device__ __forceinline__ int find_cluster(const BatchCluster *cl, int n, int x, F first_of) {
  int lo = 0, hi = n - 1, c = -1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (first_of(cl[mid]) <= x) {
      c = mid;
      lo = mid + 1;
    } else {
      hi = mid - 1;
    }
  }
  return c;
}

// Predicts every j of every cluster to that cluster's own time.
template <int ORDER, int PREC>
__global__ void __launch_bounds__(256) batch_predict_kernel(BatchArgs B) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const BatchParams &P = *B.par;
  if (k >= P.j_extent) return;
  const int c = find_cluster(B.cl, P.n_clusters, k, [](const BatchCluster &q) { return q.j_first; });
  if (c < 0) return;
  const BatchCluster &CL = B.cl[c];
  if (k >= CL.j_first + CL.j_count) return;
  double p[3], v[3], a[3];
  taylor<ORDER>(B.js, k, CL.t_pred, p, v, a);
  store_record<ORDER, PREC>(B.pred_w, k, p[0], p[1], p[2], __ldg(B.js.m + k), __ldg(B.js.id + k),
                            v[0], v[1], v[2], a[0], a[1], a[2]);
}

// Persistent force kernel: each block repeatedly takes the next work item
// (cluster, i-tile, j-slice) from the queue and evaluates it like one block
// of force_kernel (2 i per thread, threads-per-i chosen per item).  The TMA
// ring keeps a block-wide tile counter across items, so its mbarrier phases
// continue from item to item without re-initialisation.
template <int ORDER, int PREC>
__global__ void __launch_bounds__(kBT, (PREC == DOUBLE ? 1 : (ORDER >= SIXTH ? 3 : 4)))
    batch_force_kernel(BatchArgs B) {
  using C = FCfg<ORDER, PREC, 2, 2>;  // shared-memory plan with a row reduction area
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + C::NS;
  unsigned char *tiles = smem + kHdr;
  double *tot = reinterpret_cast<double *>(tiles + C::BODY);
  __shared__ int s_item;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const unsigned char *pred = reinterpret_cast<const unsigned char *>(B.pred);
  const int istr = i_stride(ORDER);

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < C::NS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kBT / 32);
    }
    fence_barrier_init();
  }
  __syncthreads();

  int tbase = 0;  // tiles this block has streamed so far (ring position)
  bool broken = false;
  // thread 0: ring positions issued / seen arrived; after a timed-out wait
  // the copies in between are drained before the block exits
  int n_issued = 0, n_landed = 0;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(&B.par->queue_head, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= B.par->n_items) break;
    const BatchItem W = B.items[item];
    const float eps2f = (float)B.cl[W.cluster].eps2;
    const double eps2d = B.cl[W.cluster].eps2;
    const int tpi = W.tpi;
    const int tit = kBT / tpi;
    const int tx = tid % tit;
    const int ty = tid / tit;
    const int nt = (W.j_count + kTJ - 1) / kTJ;

    int li[2], gi[2];
    bool valid[2];
    IMix Im[2];
    IDp Id[2];
    float best[2];
    int best_tile[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      li[p] = p * tit + tx;
      valid[p] = li[p] < W.i_count;
      gi[p] = W.i_begin + (valid[p] ? li[p] : 0);
      const double *r = B.irec + (size_t)gi[p] * istr;
      const double x = r[0], y = r[1], z = r[2], h2 = r[3];
      const double vx = r[4], vy = r[5], vz = r[6];
      const int id = __double2loint(r[7]);
      double ax = 0, ay = 0, az = 0;
      if (ORDER >= SIXTH) {
        ax = r[8];
        ay = r[9];
        az = r[10];
      }
      if (PREC == DOUBLE) {
        Id[p] = IDp{x, y, z, vx, vy, vz, ax, ay, az, valid[p] ? h2 : -1.0, id};
      } else {
        const float hx = (float)x, hy = (float)y, hz = (float)z;
        Im[p] = IMix{hx, hy, hz, (float)(x - (double)hx), (float)(y - (double)hy),
                     (float)(z - (double)hz), (float)vx, (float)vy, (float)vz, (float)ax,
                     (float)ay, (float)az, valid[p] ? (float)h2 : -1.0f, id};
      }
      best[p] = valid[p] ? kNoNgbDs2 : -1.0f;
      best_tile[p] = -1;
    }
    AccDp D[2];
#pragma unroll
    for (int p = 0; p < 2; p++) D[p] = AccDp{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (PREC != DOUBLE) {
#pragma unroll
      for (int q = 0; q < 20; q++) tot[q * kBT + tid] = 0.0;
    }
    IMix2 I2;
    if (PREC != DOUBLE) I2 = pack_i2(Im[0], Im[1]);
    const float2 eps2v = make_float2(eps2f, eps2f);

    auto issue = [&](int t) {
      const int T = tbase + t;
      const int st = T % C::NS;
      const int cnt = min(kTJ, W.j_count - t * kTJ);
      const uint32_t bytes = (uint32_t)(cnt * C::REC);
      n_issued = T + 1;
      fence_proxy_async();
      mbar_expect_tx(&full[st], bytes);
      bulk_g2s(tiles + st * C::TILE_BYTES, pred + (size_t)(W.j_begin + t * kTJ) * C::REC, bytes,
               &full[st]);
    };
    if (tid == 0 && !broken) {
      for (int t = 0; t < C::NS && t < nt; t++) {
        const int T = tbase + t;
        if (T >= C::NS &&
            !mbar_wait_bounded(&empty[T % C::NS], (uint32_t)((T / C::NS - 1) & 1))) {
          broken = true;
          atomicOr(B.status, kErrWaitTimeout);
          break;
        }
        issue(t);
      }
    }

    for (int it = 0; it < nt; it++) {
      const int T = tbase + it;
      const int s = T % C::NS;
      if (!broken) {
        if (mbar_wait_bounded(&full[s], (uint32_t)((T / C::NS) & 1))) {
          n_landed = T + 1;
        } else {
          broken = true;
          atomicOr(B.status, kErrWaitTimeout);
        }
      }
      const int cnt = min(kTJ, W.j_count - it * kTJ);
      const unsigned char *buf = tiles + s * C::TILE_BYTES;
      if (PREC == DOUBLE) {
        const double4 *rec = reinterpret_cast<const double4 *>(buf);
        double tmin[2] = {DBL_MAX, DBL_MAX};
#pragma unroll 2
        for (int k = ty; k < cnt; k += tpi) {
          const double4 r0 = rec[k * C::RS + 0];
          const double4 r1 = rec[k * C::RS + 1];
          const double4 r2 = ORDER >= SIXTH ? rec[k * C::RS + 2] : r1;
          pair_dp<ORDER>(Id[0], r0, r1, r2, eps2d, D[0], tmin[0]);
          pair_dp<ORDER>(Id[1], r0, r1, r2, eps2d, D[1], tmin[1]);
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
          const float tf = (float)tmin[p];
          if (tf < best[p]) {
            best[p] = tf;
            best_tile[p] = it;
          }
          if (B.do_list)
            list_rescan_dp<C::RS>(Id[p], tmin[p] < Id[p].h2, gi[p], ty, tpi, rec, cnt, lane,
                                  B.ngb_count, B.ngb_list);
        }
      } else {
        const float4 *rec = reinterpret_cast<const float4 *>(buf);
        const float2 z2 = make_float2(0.f, 0.f);
        AccMix2 Q{z2, z2, z2, z2, z2, z2, z2, z2, z2, z2};
        float2 tm = make_float2(FLT_MAX, FLT_MAX);
#pragma unroll 2
        for (int k = ty; k < cnt; k += tpi) {
          const float4 r0 = rec[k * C::RS + 0];
          const float4 r1 = rec[k * C::RS + 1];
          const float4 r2 = rec[k * C::RS + 2];
          const float4 r3 = ORDER >= SIXTH ? rec[k * C::RS + 3] : r2;
          pair_mix2<ORDER>(I2, r0, r1, r2, r3, eps2v, Q, tm);
        }
        const float qv[2][10] = {
            {Q.ax.x, Q.ay.x, Q.az.x, -Q.pot.x, Q.jx.x, Q.jy.x, Q.jz.x, Q.sx.x, Q.sy.x, Q.sz.x},
            {Q.ax.y, Q.ay.y, Q.az.y, -Q.pot.y, Q.jx.y, Q.jy.y, Q.jz.y, Q.sx.y, Q.sy.y, Q.sz.y}};
        const float tmin[2] = {tm.x, tm.y};
        const float near_r2 = B.cl[W.cluster].near_r2;
#pragma unroll
        for (int p = 0; p < 2; p++) {
          double *t = tot + (size_t)p * 10 * kBT + tid;
          // a near pair in this row: the row is summed again in FP64
          // (near_rescan_mix) and its FP32 partial is dropped
          const bool nearp = ORDER != GRAPE5 && valid[p] && tmin[p] < near_r2;
          if (!nearp) {
#pragma unroll
            for (int f = 0; f < 10; f++) t[f * kBT] += (double)qv[p][f];
          }
          if (ORDER != GRAPE5) {
            const unsigned nm = __ballot_sync(0xffffffffu, nearp);
            if (nm) near_rescan_inl<ORDER, C::RS>(nm, gi[p], ty, tpi, rec, cnt, lane, B.irec,
                                                  eps2d, t);
          }
          if (tmin[p] < best[p]) {
            best[p] = tmin[p];
            best_tile[p] = it;
          }
          if (B.do_list)
            list_rescan_mix<C::RS>(Im[p], tmin[p] < Im[p].h2, gi[p], ty, tpi, rec, cnt, lane,
                                   B.ngb_count, B.ngb_list);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
      if (tid == 0 && !broken && it + C::NS < nt) {
        if (mbar_wait_bounded(&empty[s], (uint32_t)((T / C::NS) & 1))) {
          issue(it + C::NS);
        } else {
          broken = true;
          atomicOr(B.status, kErrWaitTimeout);
        }
      }
    }
    tbase += nt;

    if (PREC != DOUBLE) {
#pragma unroll
      for (int p = 0; p < 2; p++) {
        const double *t = tot + (size_t)p * 10 * kBT + tid;
        D[p] = AccDp{t[0], t[kBT], t[2 * kBT], t[3 * kBT], t[4 * kBT], t[5 * kBT], t[6 * kBT],
                     t[7 * kBT], t[8 * kBT], t[9 * kBT]};
      }
    }
    // nearest neighbour: one rescan of the best tile (from L2)
    unsigned long long key[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
      key[p] = nn_key(kNoNgbDs2, -1);
      if (best_tile[p] < 0) continue;
      const int j0 = W.j_begin + best_tile[p] * kTJ;
      const int cnt = min(kTJ, W.j_count - best_tile[p] * kTJ);
      if (PREC == DOUBLE) {
        const double4 *rec = reinterpret_cast<const double4 *>(pred + (size_t)j0 * C::REC);
        for (int k = ty; k < cnt; k += tpi) {
          double dx, dy, dz;
          const double4 r0 = rec[k * C::RS + 0];
          const double4 r1 = rec[k * C::RS + 1];
          const float f2 = (float)pair_dr_dp(Id[p], r0, r1, dx, dy, dz);
          if (f2 < kNoNgbDs2) key[p] = min(key[p], nn_key(f2, __double2loint(r1.w)));
        }
      } else {
        const float4 *rec = reinterpret_cast<const float4 *>(pred + (size_t)j0 * C::REC);
        for (int k = ty; k < cnt; k += tpi) {
          float dx, dy, dz;
          const float4 r0 = __ldg(rec + k * C::RS + 0);
          const float4 r1 = __ldg(rec + k * C::RS + 1);
          const float ds2 = pair_dr_mix(Im[p], r0, r1, dx, dy, dz);
          if (ds2 < kNoNgbDs2) key[p] = min(key[p], nn_key(ds2, __float_as_int(r1.w)));
        }
      }
    }
    // combine rows in fixed order (the ring stages are idle: use the tiles area)
    __syncthreads();
    if (tpi > 1) {
      double *red = reinterpret_cast<double *>(tiles);
#pragma unroll
      for (int p = 0; p < 2; p++) {
        double *o = red + ((size_t)(ty * tit + tx) * 2 + p) * kResStride;
        o[0] = D[p].ax; o[1] = D[p].ay; o[2] = D[p].az; o[3] = D[p].pot;
        o[4] = D[p].jx; o[5] = D[p].jy; o[6] = D[p].jz;
        o[7] = D[p].sx; o[8] = D[p].sy; o[9] = D[p].sz;
        o[10] = __longlong_as_double((long long)key[p]);
      }
      __syncthreads();
      if (ty == 0) {
#pragma unroll
        for (int p = 0; p < 2; p++) {
          for (int r = 1; r < tpi; r++) {
            const double *o = red + ((size_t)(r * tit + tx) * 2 + p) * kResStride;
            D[p].ax += o[0]; D[p].ay += o[1]; D[p].az += o[2]; D[p].pot += o[3];
            D[p].jx += o[4]; D[p].jy += o[5]; D[p].jz += o[6];
            D[p].sx += o[7]; D[p].sy += o[8]; D[p].sz += o[9];
            key[p] = min(key[p], (unsigned long long)__double_as_longlong(o[10]));
          }
        }
      }
    }
    if (ty == 0) {
#pragma unroll
      for (int p = 0; p < 2; p++) {
        if (!valid[p]) continue;
        double *o = W.slot >= 0 ? B.part + (size_t)(W.slot + li[p]) * kResStride
                                : B.res + (size_t)gi[p] * kResStride;
        o[0] = D[p].ax; o[1] = D[p].ay; o[2] = D[p].az; o[3] = D[p].pot;
        o[4] = D[p].jx; o[5] = D[p].jy; o[6] = D[p].jz;
        o[7] = D[p].sx; o[8] = D[p].sy; o[9] = D[p].sz;
        if (W.slot >= 0) {
          o[10] = __longlong_as_double((long long)key[p]);
          o[11] = 0.0;
        } else {
          o[10] = (double)__uint_as_float((unsigned int)(key[p] >> 32));
          o[11] = (double)(int)(unsigned int)(key[p] & 0xffffffffu);
        }
      }
    }
  }
  if (broken && tid == 0) {
    for (int T = n_landed; T < n_issued; T++)
      mbar_wait_bounded(&full[T % C::NS], (uint32_t)((T / C::NS) & 1));
  }
}

// Sums the j-slices of clusters that were split (fixed slice order).
__global__ void __launch_bounds__(256) batch_reduce_kernel(BatchArgs B) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const BatchParams &P = *B.par;
  if (i >= P.total_i) return;
  const int c = find_cluster(B.cl, P.n_clusters, i, [](const BatchCluster &q) { return q.i_first; });
  if (c < 0) return;
  const BatchCluster &CL = B.cl[c];
  if (i >= CL.i_first + CL.i_count || CL.nslices <= 1) return;
  const int li = i - CL.i_first;
  double acc[10];
#pragma unroll
  for (int f = 0; f < 10; f++) acc[f] = 0.0;
  unsigned long long key = nn_key(kNoNgbDs2, -1);
  for (int s = 0; s < CL.nslices; s++) {
    const double *o = B.part + ((size_t)CL.part_base + (size_t)s * CL.i_count + li) * kResStride;
#pragma unroll
    for (int f = 0; f < 10; f++) acc[f] += o[f];
    key = min(key, (unsigned long long)__double_as_longlong(o[10]));
  }
  double *w = B.res + (size_t)i * kResStride;
#pragma unroll
  for (int f = 0; f < 10; f++) w[f] = acc[f];
  w[10] = (double)__uint_as_float((unsigned int)(key >> 32));
  w[11] = (double)(int)(unsigned int)(key & 0xffffffffu);
}

// ---------------------------------------------------------------- launchers
template <int ORDER, int PREC>
static cudaError_t launch_batch_t(const BatchArgs &B, int j_grid, int force_blocks, int i_grid,
                                  cudaStream_t st) {
  using C = FCfg<ORDER, PREC, 2, 2>;
  static bool attr_done = false;
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(batch_force_kernel<ORDER, PREC>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  if (B.do_predict && j_grid > 0)
    batch_predict_kernel<ORDER, PREC><<<(j_grid + 255) / 256, 256, 0, st>>>(B);
  batch_force_kernel<ORDER, PREC><<<force_blocks, kBT, C::SMEM, st>>>(B);
  if (i_grid > 0) batch_reduce_kernel<<<(i_grid + 255) / 256, 256, 0, st>>>(B);
  return cudaGetLastError();
}

cudaError_t launch_batch(int order, int prec, const BatchArgs &B, int j_grid, int force_blocks,
                         int i_grid, cudaStream_t st) {
  if (order == GRAPE5) order = FOURTH;  // GRAPE-5 batches run the 4th-order kernels
  if (order == FOURTH && prec == DOUBLESINGLE)
    return launch_batch_t<FOURTH, DOUBLESINGLE>(B, j_grid, force_blocks, i_grid, st);
  if (order == FOURTH && prec == DOUBLE)
    return launch_batch_t<FOURTH, DOUBLE>(B, j_grid, force_blocks, i_grid, st);
  if (order == SIXTH && prec == DOUBLESINGLE)
    return launch_batch_t<SIXTH, DOUBLESINGLE>(B, j_grid, force_blocks, i_grid, st);
  if (order == SIXTH && prec == DOUBLE)
    return launch_batch_t<SIXTH, DOUBLE>(B, j_grid, force_blocks, i_grid, st);
  return cudaErrorInvalidValue;
}

template <int ORDER, int PREC>
static int batch_occ_t() {
  using C = FCfg<ORDER, PREC, 2, 2>;
  if (cudaFuncSetAttribute(batch_force_kernel<ORDER, PREC>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM) != cudaSuccess)
    return 1;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_force_kernel<ORDER, PREC>, kBT,
                                                    C::SMEM) != cudaSuccess || n < 1)
    return 1;
  return n;
}

int batch_blocks_per_sm(int order, int prec) {
  if (order == GRAPE5) order = FOURTH;
  if (order == FOURTH && prec == DOUBLESINGLE) return batch_occ_t<FOURTH, DOUBLESINGLE>();
  if (order == FOURTH && prec == DOUBLE) return batch_occ_t<FOURTH, DOUBLE>();
  if (order == SIXTH && prec == DOUBLESINGLE) return batch_occ_t<SIXTH, DOUBLESINGLE>();
  return batch_occ_t<SIXTH, DOUBLE>();
}

}  // namespace sapb
