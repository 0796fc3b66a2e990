// Device kernels of the direct-summation hot path and their host launchers.
// See sapb_kernels.cuh for the list and sapb_internal.cuh for the layouts.
#include <float.h>

#include <algorithm>

#include "sapb_kernels.cuh"
#include "sapb_launch.h"
#include "sapb_pair.cuh"

namespace sapb {

// ========================================================================
// Scatter: staged j -> FP64 state + unpredicted force record.
// The unpredicted copy is what the force uses when no prediction is asked
// for (reference: dev_copy_particles seeds Ppos/Pvel/Pacc,
// kernels.cu:281-297).
// ========================================================================
template <int ORDER, int PREC>
__global__ void __launch_bounds__(256) scatter_kernel(const double *__restrict__ stage, int n,
                                                      int cap, JState js, void *pred,
                                                      int *status) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double *r = stage + (size_t)k * stage_stride(ORDER);
  const int addr = __double2loint(r[0]);
  const int id = __double2hiint(r[0]);
  if (addr < 0 || addr >= cap) {
    atomicOr(status, kErrBadConfig);
    return;
  }
  js.t[addr] = r[1];
  js.m[addr] = r[2];
  js.eps[addr] = r[15];
  js.id[addr] = id;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    js.x[d][addr] = r[3 + d];
    js.v[d][addr] = r[6 + d];
    js.a[d][addr] = r[9 + d];
    js.j[d][addr] = r[12 + d];
    if (ORDER >= SIXTH) {
      js.s[d][addr] = r[16 + d];
      js.c[d][addr] = r[19 + d];
    }
  }
  store_record<ORDER, PREC>(pred, addr, r[3], r[4], r[5], r[2], id, r[6], r[7], r[8], r[9], r[10],
                            r[11]);
}

// ========================================================================
// Predictor: FP64 Taylor series in the Horner form of kernels.cu:331-383
// (4th order drops snap/crackle, which the reference does by dt4 = dt5 = 0).
// Reads the FP64 structure-of-arrays state with one coalesced 8-byte load
// per component and writes the force record of each j.
// ========================================================================
// The grid is one wave of resident blocks striding over the j (a grid of
// nj / 256 blocks would leave its last wave part-empty: 2^20 j are 3.5 waves).
template <int ORDER, int PREC>
__global__ void __launch_bounds__(256) predict_kernel(int nj, double ti, JState js, void *pred) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nj; k += gridDim.x * blockDim.x) {
    double p[3], v[3], a[3];
    taylor<ORDER>(js, k, ti, p, v, a);
    store_record<ORDER, PREC>(pred, k, p[0], p[1], p[2], __ldg(js.m + k), __ldg(js.id + k),
                              v[0], v[1], v[2], a[0], a[1], a[2]);
  }
}

// Readback of j[first, first+n): raw FP64 state and its FP64 prediction to
// ti (or the raw state again when predict == 0), 24 doubles per j:
//   x[3] m v[3] eps a[3] jerk[3] px[3] pv[3] pa[3] id
template <int ORDER>
__global__ void __launch_bounds__(256) readj_kernel(int first, int n, double ti, int predict,
                                                    JState js, double *out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int k = first + q;
  double p[3], v[3], a[3];
  if (predict) {
    taylor<ORDER>(js, k, ti, p, v, a);
  } else {
    for (int d = 0; d < 3; d++) {
      p[d] = js.x[d][k];
      v[d] = js.v[d][k];
      a[d] = js.a[d][k];
    }
  }
  double *o = out + (size_t)q * 24;
  for (int d = 0; d < 3; d++) {
    o[d] = js.x[d][k];
    o[4 + d] = js.v[d][k];
    o[8 + d] = js.a[d][k];
    o[11 + d] = js.j[d][k];
    o[14 + d] = p[d];
    o[17 + d] = v[d];
    o[20 + d] = a[d];
  }
  o[3] = js.m[k];
  o[7] = js.eps[k];
  o[23] = (double)js.id[k];
}

// ========================================================================
// Force kernel.
//
// Block = 4 warps, laid out as TPI rows x TIT = 128/TPI columns; each thread
// owns IP i-particles (columns tx, tx+TIT, ...), so a block covers an i-tile
// of TI = TIT*IP particles.  blockIdx.y selects j-slice s of S: the tiles
// s, s+S, s+2S, ... of kTJ = 256 records.  Lane 0 of warp 0 streams them
// into a 3-stage shared-memory ring with cp.async.bulk (TMA engine): `full`
// mbarriers signal arrival (complete_tx), `empty` mbarriers collect one
// arrival per warp; there is no block-wide barrier per tile, so warps drift
// up to two tiles apart instead of waiting for the slowest one.
// Row `ty` consumes records ty, ty+TPI, ... of each tile.
//
// Mixed precision (DOUBLESINGLE): dr = (xj_hi - xi_hi) + (xj_lo - xi_lo)
// in FP32 (double-single difference, kernels.cu:169-177), FP32 body with
// rsqrt on the MUFU pipe (two i per thread as packed FP32x2), FP32 sums per
// tile folded into FP64 totals (shared memory) after every tile.
// FP64 (DOUBLE): every step in double, rsqrt(double).
//
// The self pair (id_i == id_j, kernels.cu:565) is removed by replacing dx
// with a huge value, which makes ds2 ~ 1e36 (1e300 in FP64): its force
// underflows to zero and it can be neither nearest neighbour nor listed.
//
// Nearest neighbour and neighbour list cost one FMNMX per pair: the pair
// loop only keeps the tile's minimum ds2.  Neighbour list: when that minimum
// is below h2, the warp rescans the tile cooperatively (lanes split the j)
// and appends the hits.  Nearest neighbour: each thread remembers the tile
// where its smallest ds2 first appeared and rescans only that tile, from L2,
// after the loop.  Rescans recompute ds2 bit-identically (same rounded
// operations).
// ========================================================================
// Unroll depth of the packed j loop (B200, 6th order, N = 2^20: 1 -> 501,
// 2 -> 526, 4 -> 530 G interactions/s).
#ifndef SAPB_JUNROLL
#define SAPB_JUNROLL 4
#endif
#define SAPB_STR(x) #x
#define SAPB_UNROLL(n) _Pragma(SAPB_STR(unroll n))

template <int ORDER, int PREC, int TPI, int IP>
__global__ void __launch_bounds__(kBT, (FCfg<ORDER, PREC, TPI, IP>::MIN_BLOCKS))
    force_kernel(ForceArgs A) {
  using C = FCfg<ORDER, PREC, TPI, IP>;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smem);
  uint64_t *empty = full + C::NS;
  float4 *sbox = reinterpret_cast<float4 *>(smem + 64);  // spatial mode: box of each stage's tile
  unsigned char *tiles = smem + kHdr;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int itile = blockIdx.x;
  const int slice = blockIdx.y;

  // ---- j range of this slice ----
  const int ntiles_all = (A.nj + kTJ - 1) / kTJ;
  // slice s takes tiles s, s + S, s + 2S, ... (interleaved: in spatial mode
  // the tiles near a block's i, which run slower, are spread over all slices
  // instead of loading a few of them)
  const int S = A.nslices;
  const int nt = slice < ntiles_all ? (ntiles_all - slice + S - 1) / S : 0;
  const unsigned char *pred = reinterpret_cast<const unsigned char *>(A.pred);
  // spatial mode: far tiles take the single-float difference (pair_mix2_far)
  const bool spatial = PREC != DOUBLE && (IP % 2 == 0) && A.tbox != nullptr;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < C::NS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kBT / 32);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // ---- producer: lane 0 of warp 0 fills the ring ----
  // n_issued / n_landed (thread 0): tiles issued so far / tiles whose
  // arrival it has seen; after a timed-out wait the copies in between are
  // drained before the block exits
  int n_issued = 0, n_landed = 0;
  auto issue = [&](int it) {
    n_issued = it + 1;
    const int st = it % C::NS;
    const int tile = slice + it * S;
    const int cnt = min(kTJ, A.nj - tile * kTJ);
    const uint32_t bytes = (uint32_t)(cnt * C::REC);
    fence_proxy_async();
    mbar_expect_tx(&full[st], bytes + (spatial ? 32u : 0u));
    bulk_g2s(tiles + st * C::TILE_BYTES, pred + (size_t)tile * kTJ * C::REC, bytes, &full[st]);
    if (spatial) bulk_g2s(sbox + 2 * st, A.tbox + 2 * tile, 32u, &full[st]);
  };
  const bool producer = (tid == 0);
  if (producer)
    for (int it = 0; it < C::NS && it < nt; it++) issue(it);

  // ---- consumers: 128 threads = TPI rows x TIT columns, IP i each ----
  const int tx = tid % C::TIT;
  const int ty = tid / C::TIT;
  const int istr = i_stride(ORDER);
  int gi[IP];  // i position within the launch (Morton order in spatial mode)
  int oi[IP];  // its i record, result and list row
  bool valid[IP];
  IMix Im[IP];
  IDp Id[IP];
  float best[IP];     // smallest ds2 seen (float), -1 for padding i
  int best_tile[IP];  // tile (within the slice) where it was first seen
#pragma unroll
  for (int p = 0; p < IP; p++) {
    gi[p] = itile * C::TI + p * C::TIT + tx;
    valid[p] = gi[p] < A.ni;
    // (spatial mode is mixed precision only: the FP64 kernels keep address order)
    oi[p] = (PREC != DOUBLE && valid[p] && A.iperm) ? __ldg(A.iperm + gi[p]) : gi[p];
    const double *r = A.irec + (size_t)(valid[p] ? oi[p] : 0) * istr;
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

  AccDp D[IP];
#pragma unroll
  for (int p = 0; p < IP; p++) D[p] = AccDp{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  double *tot = reinterpret_cast<double *>(tiles + C::BODY);  // mixed: [p][field][tid]
  if (PREC != DOUBLE) {
#pragma unroll
    for (int q = 0; q < IP * 10; q++) tot[q * kBT + tid] = 0.0;
  }
  const float eps2f = (float)A.eps2;
  const float2 eps2v = make_float2(eps2f, eps2f);
  constexpr int NPAIR = IP / 2;  // packed i pairs per thread (mixed precision)
  IMix2 I2[NPAIR > 0 ? NPAIR : 1];
  if (PREC != DOUBLE) {
#pragma unroll
    for (int q = 0; q < NPAIR; q++) I2[q] = pack_i2(Im[2 * q], Im[(2 * q + 1) % IP]);
  }

  // ---- spatial mode: what a far tile must stay clear of, per i ----
  // A tile is far when, for every i of the warp, (1) its distance to the
  // tile's box is at least far_c * max(|xi|, |xj|) (single-float difference
  // accurate to delta) and (2) its squared distance, less a 1e-4 margin,
  // exceeds lim = the larger of an upper bound of its nearest-neighbour ds2
  // and near_r2: no pair of the tile can then be a nearest neighbour or a
  // near pair (FP64 rescan, below).  The warp votes, so the decision
  // is warp-uniform.  It does not depend on h2, so neither do the forces:
  // list members in far tiles are found by an exact rescan of the tile for
  // each i whose h2 reaches the tile's box (squared box distance, less the
  // same margin, below h2).
  float lim[IP];
#pragma unroll
  for (int p = 0; p < IP; p++) {
    lim[p] = -1.f;
    // a far tile must also hold no near pair (ds2 < near_r2)
    if (spatial && ORDER != GRAPE5 && valid[p])
      lim[p] = fmaxf(__ldg(A.ibound + gi[p]), A.near_r2);
  }
  // Margin of the far tests: a box distance from high parts, and a ds2 from
  // the single-float difference, are within 2 sqrt(3) delta (relative) of the
  // exact ones on a far tile.
  const float shrink = spatial ? fminf(0.9999f, 1.f - 8.f * (0x1p-23f / A.far_c)) : 1.f;
  bool broken = false;
  int nfar = 0;  // far tiles of this warp (spatial mode)

  for (int it = 0; it < nt; it++) {
    const int s = it % C::NS;
    if (!broken) {
      if (mbar_wait_bounded(&full[s], (uint32_t)((it / C::NS) & 1))) {
        n_landed = it + 1;
      } else {
        broken = true;
        atomicOr(A.status, kErrWaitTimeout);
      }
    }
    const int tile = slice + it * S;
    const int cnt = min(kTJ, A.nj - tile * kTJ);
    const unsigned char *buf = tiles + s * C::TILE_BYTES;

    if (PREC == DOUBLE) {
      const double4 *rec = reinterpret_cast<const double4 *>(buf);
      double tmin[IP];
#pragma unroll
      for (int p = 0; p < IP; p++) tmin[p] = DBL_MAX;
#pragma unroll 2
      for (int k = ty; k < cnt; k += TPI) {
        const double4 r0 = rec[k * C::RS + 0];
        const double4 r1 = rec[k * C::RS + 1];
        const double4 r2 = ORDER >= SIXTH ? rec[k * C::RS + 2] : r1;
#pragma unroll
        for (int p = 0; p < IP; p++) pair_dp<ORDER>(Id[p], r0, r1, r2, A.eps2, D[p], tmin[p]);
      }
#pragma unroll
      for (int p = 0; p < IP; p++) {
        const float tf = (float)tmin[p];
        if (tf < best[p]) {
          best[p] = tf;
          best_tile[p] = it;
        }
        if (A.do_list)
          list_rescan_dp<C::RS>(Id[p], tmin[p] < Id[p].h2, oi[p], ty, TPI, rec, cnt, lane,
                                A.ngb_count, A.ngb_list);
      }
    } else {
      const float4 *rec = reinterpret_cast<const float4 *>(buf);
      AccMix P[IP];
      float tmin[IP];
#pragma unroll
      for (int p = 0; p < IP; p++) {
        P[p] = AccMix{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        tmin[p] = FLT_MAX;
      }
      bool far = false;  // spatial mode: this tile took the single-float difference
      // far tiles: the i rows whose h2 reaches the tile's box (list rescan)
      unsigned lmask = 0;
      if constexpr (IP % 2 == 0) {
        AccMix2 Q[NPAIR];
        float2 tm[NPAIR];
        const float2 z2 = make_float2(0.f, 0.f);
#pragma unroll
        for (int q = 0; q < NPAIR; q++) {
          Q[q] = AccMix2{z2, z2, z2, z2, z2, z2, z2, z2, z2, z2};
          tm[q] = make_float2(FLT_MAX, FLT_MAX);
        }
        if (spatial) {
          const float4 bl = sbox[2 * s], bh = sbox[2 * s + 1];
          bool ok = true;
#pragma unroll
          for (int p = 0; p < IP; p++) {
            const float xh = Im[p].xh, yh = Im[p].yh, zh = Im[p].zh;
            const float gx = fmaxf(0.f, fmaxf(bl.x - xh, xh - bh.x));
            const float gy = fmaxf(0.f, fmaxf(bl.y - yh, yh - bh.y));
            const float gz = fmaxf(0.f, fmaxf(bl.z - zh, zh - bh.z));
            const float g2 = fmaf(gz, gz, fmaf(gy, gy, gx * gx));
            const float xa = fmaxf(fabsf(xh), fmaxf(fabsf(yh), fabsf(zh)));
            const float xm = fmaxf(bl.w, xa) * A.far_c;
            ok = ok && (!valid[p] || (g2 >= xm * xm && g2 * shrink > lim[p]));
            if (valid[p] && g2 * shrink < Im[p].h2) lmask |= 1u << p;
          }
          far = __all_sync(0xffffffffu, ok);
          nfar += far ? 1 : 0;
        }
        // The far loop is written out twice, for calls with and without
        // lists, although both copies are the same: with one shared copy the
        // kernel measured 1.5 % slower on B200, with lists and without (same
        // box, alternating runs).
        if (far && A.do_list) {
          SAPB_UNROLL(SAPB_JUNROLL)
          for (int k = ty; k < cnt; k += TPI) {
            const float4 r0 = rec[k * C::RS + 0];
            const float4 r2 = rec[k * C::RS + 2];
            const float4 r3 = ORDER >= SIXTH ? rec[k * C::RS + 3] : r2;
#pragma unroll
            for (int q = 0; q < NPAIR; q++) pair_mix2_far<ORDER>(I2[q], r0, r2, r3, eps2v, Q[q]);
          }
        } else if (far) {
          SAPB_UNROLL(SAPB_JUNROLL)
          for (int k = ty; k < cnt; k += TPI) {
            const float4 r0 = rec[k * C::RS + 0];
            const float4 r2 = rec[k * C::RS + 2];
            const float4 r3 = ORDER >= SIXTH ? rec[k * C::RS + 3] : r2;
#pragma unroll
            for (int q = 0; q < NPAIR; q++) pair_mix2_far<ORDER>(I2[q], r0, r2, r3, eps2v, Q[q]);
          }
        } else {
          SAPB_UNROLL(SAPB_JUNROLL)
          for (int k = ty; k < cnt; k += TPI) {
            const float4 r0 = rec[k * C::RS + 0];
            const float4 r1 = rec[k * C::RS + 1];
            const float4 r2 = rec[k * C::RS + 2];
            const float4 r3 = ORDER >= SIXTH ? rec[k * C::RS + 3] : r2;
#pragma unroll
            for (int q = 0; q < NPAIR; q++)
              pair_mix2<ORDER>(I2[q], r0, r1, r2, r3, eps2v, Q[q], tm[q]);
          }
        }
#pragma unroll
        for (int q = 0; q < NPAIR; q++) {
          P[2 * q] = AccMix{Q[q].ax.x, Q[q].ay.x, Q[q].az.x, -Q[q].pot.x, Q[q].jx.x, Q[q].jy.x,
                            Q[q].jz.x, Q[q].sx.x, Q[q].sy.x, Q[q].sz.x};
          P[2 * q + 1] = AccMix{Q[q].ax.y, Q[q].ay.y, Q[q].az.y, -Q[q].pot.y, Q[q].jx.y,
                                Q[q].jy.y, Q[q].jz.y, Q[q].sx.y, Q[q].sy.y, Q[q].sz.y};
          tmin[2 * q] = tm[q].x;
          tmin[2 * q + 1] = tm[q].y;
        }
      } else {
#pragma unroll 2
        for (int k = ty; k < cnt; k += TPI) {
          const float4 r0 = rec[k * C::RS + 0];
          const float4 r1 = rec[k * C::RS + 1];
          const float4 r2 = rec[k * C::RS + 2];
          const float4 r3 = ORDER >= SIXTH ? rec[k * C::RS + 3] : r2;
#pragma unroll
          for (int p = 0; p < IP; p++)
            pair_mix<ORDER>(Im[p], r0, r1, r2, r3, eps2f, P[p], tmin[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < IP; p++) {
        // a near pair in this row (never on a far tile): the row is summed
        // again in FP64 below, so its FP32 partial is dropped
        const bool nearp = ORDER != GRAPE5 && !far && valid[p] && tmin[p] < A.near_r2;
        double *t = tot + (size_t)p * 10 * kBT + tid;
        if (!nearp) {
          t[0 * kBT] += (double)P[p].ax;
          t[1 * kBT] += (double)P[p].ay;
          t[2 * kBT] += (double)P[p].az;
          t[3 * kBT] += (double)P[p].pot;
          t[4 * kBT] += (double)P[p].jx;
          t[5 * kBT] += (double)P[p].jy;
          t[6 * kBT] += (double)P[p].jz;
          if (ORDER >= SIXTH) {
            t[7 * kBT] += (double)P[p].sx;
            t[8 * kBT] += (double)P[p].sy;
            t[9 * kBT] += (double)P[p].sz;
          }
        }
        if (ORDER != GRAPE5) {
          const unsigned nm = __ballot_sync(0xffffffffu, nearp);
          if (nm) {
            // out of line where the register budget has room for the call,
            // inlined where the shape is held to 128 or 168 registers
            if constexpr (C::MIN_BLOCKS >= 3)
              near_rescan_inl<ORDER, C::RS>(nm, oi[p], ty, TPI, rec, cnt, lane, A.irec, A.eps2,
                                            t);
            else
              near_rescan_mix<ORDER, C::RS>(nm, oi[p], ty, TPI, rec, cnt, lane, A.irec, A.eps2,
                                            t);
          }
        }
        if (ORDER != GRAPE5) {  // GRAPE-5: no nearest neighbour, no lists
          // a far tile holds no nearest neighbour; its minimum is the
          // single-float ds2 (hence the margin on the rescan trigger; the
          // rescan itself is exact)
          if (!far && tmin[p] < best[p]) {
            best[p] = tmin[p];
            best_tile[p] = it;
          }
          // far tiles: no pair is closer than the tile's box, whose squared
          // distance from the high parts is, less the margin of the far test,
          // below the exact ds2 of every pair (lmask); the rescan itself is exact
          if (A.do_list)
            list_rescan_mix<C::RS>(Im[p], far ? ((lmask >> p) & 1u) != 0 : tmin[p] < Im[p].h2,
                                   oi[p], ty, TPI, rec, cnt, lane, A.ngb_count, A.ngb_list);
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with the stage
    // Refill the stage once all four warps released it; only warp 0 waits
    // here, the others may already be up to C::NS-1 tiles ahead.
    if (producer && !broken && it + C::NS < nt) {
      if (mbar_wait_bounded(&empty[s], (uint32_t)((it / C::NS) & 1))) {
        issue(it + C::NS);
      } else {
        broken = true;
        atomicOr(A.status, kErrWaitTimeout);
      }
    }
  }
  if (spatial && A.stats && lane == 0) {
    atomicAdd(A.stats, (unsigned long long)nfar);
    atomicAdd(A.stats + 1, (unsigned long long)nt);
  }
  if (broken && producer) {
    // let the copies still in flight land (bounded waits) before the block
    // exits and its shared memory is released
    for (int it = n_landed; it < n_issued; it++)
      mbar_wait_bounded(&full[it % C::NS], (uint32_t)((it / C::NS) & 1));
  }

  if (PREC != DOUBLE) {
#pragma unroll
    for (int p = 0; p < IP; p++) {
      const double *t = tot + (size_t)p * 10 * kBT + tid;
      D[p] = AccDp{t[0], t[kBT], t[2 * kBT], t[3 * kBT], t[4 * kBT], t[5 * kBT], t[6 * kBT],
                   t[7 * kBT], t[8 * kBT], t[9 * kBT]};
    }
  }

  // ---- nearest neighbour: one rescan of the best tile (from L2) ----
  unsigned long long key[IP];
#pragma unroll
  for (int p = 0; p < IP; p++) {
    key[p] = nn_key(kNoNgbDs2, -1);
    if (best_tile[p] < 0) continue;
    const int tile = slice + best_tile[p] * S;
    const int cnt = min(kTJ, A.nj - tile * kTJ);
    if (PREC == DOUBLE) {
      const double4 *rec = reinterpret_cast<const double4 *>(pred + (size_t)tile * kTJ * C::REC);
      for (int k = ty; k < cnt; k += TPI) {
        double dx, dy, dz;
        const double4 r0 = rec[k * C::RS + 0];
        const double4 r1 = rec[k * C::RS + 1];
        const float f2 = (float)pair_dr_dp(Id[p], r0, r1, dx, dy, dz);
        if (f2 < kNoNgbDs2) key[p] = min(key[p], nn_key(f2, __double2loint(r1.w)));
      }
    } else {
      const float4 *rec = reinterpret_cast<const float4 *>(pred + (size_t)tile * kTJ * C::REC);
      for (int k = ty; k < cnt; k += TPI) {
        float dx, dy, dz;
        const float4 r0 = __ldg(rec + k * C::RS + 0);
        const float4 r1 = __ldg(rec + k * C::RS + 1);
        const float ds2 = pair_dr_mix(Im[p], r0, r1, dx, dy, dz);
        if (ds2 < kNoNgbDs2) key[p] = min(key[p], nn_key(ds2, __float_as_int(r1.w)));
      }
    }
  }

  // ---- combine rows (threads-per-i > 1), fixed order ----
  if (TPI > 1) {
    named_barrier(1, kBT);  // all consumer warps are past their last tile
    double *red = reinterpret_cast<double *>(tiles);
#pragma unroll
    for (int p = 0; p < IP; p++) {
      double *o = red + ((size_t)(ty * C::TIT + tx) * IP + p) * kResStride;
      o[0] = D[p].ax; o[1] = D[p].ay; o[2] = D[p].az; o[3] = D[p].pot;
      o[4] = D[p].jx; o[5] = D[p].jy; o[6] = D[p].jz;
      o[7] = D[p].sx; o[8] = D[p].sy; o[9] = D[p].sz;
      o[10] = __longlong_as_double((long long)key[p]);
    }
    named_barrier(1, kBT);
    if (ty != 0) return;
#pragma unroll
    for (int p = 0; p < IP; p++) {
      for (int r = 1; r < TPI; r++) {
        const double *o = red + ((size_t)(r * C::TIT + tx) * IP + p) * kResStride;
        D[p].ax += o[0]; D[p].ay += o[1]; D[p].az += o[2]; D[p].pot += o[3];
        D[p].jx += o[4]; D[p].jy += o[5]; D[p].jz += o[6];
        D[p].sx += o[7]; D[p].sy += o[8]; D[p].sz += o[9];
        key[p] = min(key[p], (unsigned long long)__double_as_longlong(o[10]));
      }
    }
  }

  // ---- write this block's results ----
#pragma unroll
  for (int p = 0; p < IP; p++) {
    if (!valid[p]) continue;
    double *o = A.write_partials ? A.out + ((size_t)slice * A.ni + oi[p]) * kResStride
                                 : A.out + (size_t)oi[p] * kResStride;
    o[0] = D[p].ax; o[1] = D[p].ay; o[2] = D[p].az; o[3] = D[p].pot;
    o[4] = D[p].jx; o[5] = D[p].jy; o[6] = D[p].jz;
    o[7] = D[p].sx; o[8] = D[p].sy; o[9] = D[p].sz;
    if (A.write_partials) {
      o[10] = __longlong_as_double((long long)key[p]);
      o[11] = 0.0;
    } else {
      o[10] = (double)__uint_as_float((unsigned int)(key[p] >> 32));
      o[11] = (double)(int)(unsigned int)(key[p] & 0xffffffffu);
    }
  }
}

// ========================================================================
// Self-test of the bounded device wait: one thread waits on an mbarrier
// that nothing ever arrives at; the wait gives up after limit_ns and the
// kernel records kErrWaitTimeout and returns, leaving the context usable.
// ========================================================================
__global__ void wait_selftest_kernel(uint64_t limit_ns, int *status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0, limit_ns)) atomicOr(status, kErrWaitTimeout);
}

cudaError_t launch_wait_selftest(uint64_t limit_ns, int *status, cudaStream_t st) {
  wait_selftest_kernel<<<1, 32, 0, st>>>(limit_ns, status);
  return cudaGetLastError();
}

// ========================================================================
// Cross-slice reduction: fixed slice order, so results are bit-stable.
// ========================================================================
__global__ void __launch_bounds__(256) reduce_kernel(ReduceArgs R) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.ni) return;
  double acc[10];
#pragma unroll
  for (int f = 0; f < 10; f++) acc[f] = 0.0;
  unsigned long long key = nn_key(kNoNgbDs2, -1);
  for (int s = 0; s < R.nslices; s++) {
    const double *o = R.part + ((size_t)s * R.ni + i) * kResStride;
#pragma unroll
    for (int f = 0; f < 10; f++) acc[f] += o[f];
    key = min(key, (unsigned long long)__double_as_longlong(o[10]));
  }
  double *w = R.out + (size_t)i * kResStride;
#pragma unroll
  for (int f = 0; f < 10; f++) w[f] = acc[f];
  w[10] = (double)__uint_as_float((unsigned int)(key >> 32));
  w[11] = (double)(int)(unsigned int)(key & 0xffffffffu);
}

// ========================================================================
// Host launchers
// ========================================================================
template <int ORDER, int PREC>
static cudaError_t launch_scatter_t(const double *stage, int n, int cap, const JState &js,
                                   void *pred, int *status, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  scatter_kernel<ORDER, PREC><<<(n + 255) / 256, 256, 0, st>>>(stage, n, cap, js, pred, status);
  return cudaGetLastError();
}

cudaError_t launch_scatter(int order, int prec, const double *stage, int n, int cap,
                           const JState &js, void *pred, int *status, cudaStream_t st) {
  if (order == GRAPE5) order = FOURTH;  // GRAPE-5 keeps the 4th-order layout
  if (order == FOURTH && prec == DOUBLESINGLE)
    return launch_scatter_t<FOURTH, DOUBLESINGLE>(stage, n, cap, js, pred, status, st);
  if (order == FOURTH && prec == DOUBLE)
    return launch_scatter_t<FOURTH, DOUBLE>(stage, n, cap, js, pred, status, st);
  if (order == SIXTH && prec == DOUBLESINGLE)
    return launch_scatter_t<SIXTH, DOUBLESINGLE>(stage, n, cap, js, pred, status, st);
  if (order == SIXTH && prec == DOUBLE)
    return launch_scatter_t<SIXTH, DOUBLE>(stage, n, cap, js, pred, status, st);
  return cudaErrorInvalidValue;
}

template <int ORDER, int PREC>
static cudaError_t launch_predict_t(int nj, double ti, const JState &js, void *pred,
                                    cudaStream_t st) {
  if (nj <= 0) return cudaSuccess;
  static int wave = 0;  // resident blocks on the whole device (one per instantiation)
  if (!wave) {
    int dev = 0, sms = 0, occ = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, predict_kernel<ORDER, PREC>, 256, 0);
    if (e != cudaSuccess) return e;
    wave = std::max(1, sms * occ);
  }
  const int blocks = std::min((nj + 255) / 256, wave);
  predict_kernel<ORDER, PREC><<<blocks, 256, 0, st>>>(nj, ti, js, pred);
  return cudaGetLastError();
}

cudaError_t launch_predict(int order, int prec, int nj, double ti, const JState &js, void *pred,
                           cudaStream_t st) {
  if (order == GRAPE5) order = FOURTH;  // GRAPE-5 keeps the 4th-order layout
  if (order == FOURTH && prec == DOUBLESINGLE)
    return launch_predict_t<FOURTH, DOUBLESINGLE>(nj, ti, js, pred, st);
  if (order == FOURTH && prec == DOUBLE)
    return launch_predict_t<FOURTH, DOUBLE>(nj, ti, js, pred, st);
  if (order == SIXTH && prec == DOUBLESINGLE)
    return launch_predict_t<SIXTH, DOUBLESINGLE>(nj, ti, js, pred, st);
  if (order == SIXTH && prec == DOUBLE)
    return launch_predict_t<SIXTH, DOUBLE>(nj, ti, js, pred, st);
  return cudaErrorInvalidValue;
}

template <int ORDER, int PREC, int TPI, int IP>
static cudaError_t launch_force_t(const ForceArgs *A, cudaStream_t st, int *occ) {
  using C = FCfg<ORDER, PREC, TPI, IP>;
  static bool attr_done = false;  // one-time attribute per instantiation
  static int blocks_per_sm = 0;   // resident blocks per SM, from the occupancy API
  if (!attr_done) {
    cudaError_t e = cudaFuncSetAttribute(force_kernel<ORDER, PREC, TPI, IP>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    if (e != cudaSuccess) return e;
    attr_done = true;
  }
  if (occ) {  // query only
    if (!blocks_per_sm) {
      cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &blocks_per_sm, force_kernel<ORDER, PREC, TPI, IP>, kBT, C::SMEM);
      if (e != cudaSuccess) return e;
    }
    *occ = blocks_per_sm;
    return cudaSuccess;
  }
  dim3 grid(A->i_tiles, A->nslices);
  force_kernel<ORDER, PREC, TPI, IP><<<grid, kBT, C::SMEM, st>>>(*A);
  return cudaGetLastError();
}

// Launches (occ == nullptr) or reports the resident blocks per SM (occ) of
// one instantiation.
template <int ORDER, int PREC>
static cudaError_t launch_force_o(const ForceArgs *A, int tpi, int ip, cudaStream_t st, int *occ) {
  if (ip == 4) {
    if constexpr (PREC != DOUBLE) {  // 4 i per thread: mixed precision only
      switch (tpi) {
        case 1: return launch_force_t<ORDER, PREC, 1, 4>(A, st, occ);
        case 2: return launch_force_t<ORDER, PREC, 2, 4>(A, st, occ);
        default: break;
      }
    }
  } else if (ip == 2) {
    switch (tpi) {
      case 1: return launch_force_t<ORDER, PREC, 1, 2>(A, st, occ);
      case 2: return launch_force_t<ORDER, PREC, 2, 2>(A, st, occ);
      case 4: return launch_force_t<ORDER, PREC, 4, 2>(A, st, occ);
      case 8: return launch_force_t<ORDER, PREC, 8, 2>(A, st, occ);
      default: break;
    }
  } else if (ip == 1) {
    switch (tpi) {
      case 1: return launch_force_t<ORDER, PREC, 1, 1>(A, st, occ);
      case 2: return launch_force_t<ORDER, PREC, 2, 1>(A, st, occ);
      case 4: return launch_force_t<ORDER, PREC, 4, 1>(A, st, occ);
      case 8: return launch_force_t<ORDER, PREC, 8, 1>(A, st, occ);
      case 16: return launch_force_t<ORDER, PREC, 16, 1>(A, st, occ);
      case 32: return launch_force_t<ORDER, PREC, 32, 1>(A, st, occ);
      default: break;
    }
  }
  return cudaErrorInvalidConfiguration;
}

static cudaError_t force_dispatch(int order, int prec, const ForceArgs *A, int tpi, int ip,
                                  cudaStream_t st, int *occ) {
  if (order == GRAPE5 && prec == DOUBLESINGLE)
    return launch_force_o<GRAPE5, DOUBLESINGLE>(A, tpi, ip, st, occ);
  if (order == GRAPE5) order = FOURTH;  // FP64 GRAPE-5 calls run the 4th-order kernels
  if (order == FOURTH && prec == DOUBLESINGLE)
    return launch_force_o<FOURTH, DOUBLESINGLE>(A, tpi, ip, st, occ);
  if (order == FOURTH && prec == DOUBLE) return launch_force_o<FOURTH, DOUBLE>(A, tpi, ip, st, occ);
  if (order == SIXTH && prec == DOUBLESINGLE)
    return launch_force_o<SIXTH, DOUBLESINGLE>(A, tpi, ip, st, occ);
  if (order == SIXTH && prec == DOUBLE) return launch_force_o<SIXTH, DOUBLE>(A, tpi, ip, st, occ);
  return cudaErrorInvalidValue;
}

int force_blocks_per_sm(int order, int prec, int tpi, int ip) {
  int n = 0;
  if (force_dispatch(order, prec, nullptr, tpi, ip, 0, &n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int force_tile_i(int tpi, int ip) { return (kBT / tpi) * ip; }
int force_tile_j() { return kTJ; }

cudaError_t launch_force(int order, int prec, const ForceArgs &A, int tpi, int ip,
                         cudaStream_t st) {
  return force_dispatch(order, prec, &A, tpi, ip, st, nullptr);
}

cudaError_t launch_readj(int order, int first, int n, double ti, int predict, const JState &js,
                         double *out, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  if (order >= SIXTH)
    readj_kernel<SIXTH><<<(n + 255) / 256, 256, 0, st>>>(first, n, ti, predict, js, out);
  else
    readj_kernel<FOURTH><<<(n + 255) / 256, 256, 0, st>>>(first, n, ti, predict, js, out);
  return cudaGetLastError();
}

cudaError_t launch_reduce(const ReduceArgs &R, cudaStream_t st) {
  if (R.ni <= 0) return cudaSuccess;
  reduce_kernel<<<(R.ni + 255) / 256, 256, 0, st>>>(R);
  return cudaGetLastError();
}

}  // namespace sapb
