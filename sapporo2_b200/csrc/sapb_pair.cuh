// Pair arithmetic, tile geometry and rescan helpers shared by the grid force
// kernel (sapb_kernels.cu) and the persistent batch kernel
// (sapb_batch_kernels.cu).
#pragma once
#include <float.h>

#include "sapb_kernels.cuh"

namespace sapb {

// Force record of one predicted j (see sapb_internal.cuh for the layouts).
template <int ORDER, int PREC>
__device__ __forceinline__ void store_record(void *pred, int k, double px, double py, double pz,
                                             double m, int id, double vx, double vy, double vz,
                                             double ax, double ay, double az) {
  if (PREC == DOUBLE) {
    double4 *r = reinterpret_cast<double4 *>(pred) + (size_t)k * pred_fields64(ORDER);
    r[0] = make_double4(px, py, pz, m);
    r[1] = make_double4(vx, vy, vz, __hiloint2double(0, id));
    if (ORDER >= SIXTH) r[2] = make_double4(ax, ay, az, 0.0);
  } else {
    // Double-single split of the position: hi = (float)x, lo = (float)(x - hi)
    // (the DSX assignment of kernels.cu:163-167).
    const float hx = (float)px, hy = (float)py, hz = (float)pz;
    const float lx = (float)(px - (double)hx), ly = (float)(py - (double)hy),
                lz = (float)(pz - (double)hz);
    // The id goes into r[1].w and again into r[2].w, so that far tiles, which
    // need no low parts, read no r[1].
    float4 *r = reinterpret_cast<float4 *>(pred) + (size_t)k * pred_fields(ORDER);
    r[0] = make_float4(hx, hy, hz, (float)m);
    r[1] = make_float4(lx, ly, lz, __int_as_float(id));
    r[2] = make_float4((float)vx, (float)vy, (float)vz, __int_as_float(id));
    if (ORDER >= SIXTH) r[3] = make_float4((float)ax, (float)ay, (float)az, 0.f);
  }
}

// FP64 Taylor prediction in the Horner form of kernels.cu:331-383.
template <int ORDER>
__device__ __forceinline__ void taylor(const JState &js, int k, double ti, double p[3],
                                       double v[3], double a[3]) {
  const double dt = ti - __ldg(js.t + k);
  const double dt2 = (1. / 2.) * dt;
  const double dt3 = (1. / 3.) * dt;
  const double dt4 = (1. / 4.) * dt;
  const double dt5 = (1. / 5.) * dt;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double x = __ldg(js.x[d] + k), vv = __ldg(js.v[d] + k);
    const double aa = __ldg(js.a[d] + k), jj = __ldg(js.j[d] + k);
    if (ORDER >= SIXTH) {
      const double ss = __ldg(js.s[d] + k), cc = __ldg(js.c[d] + k);
      p[d] = x + dt * (vv + dt2 * (aa + dt3 * (jj + dt4 * (ss + dt5 * (cc)))));
      v[d] = vv + dt * (aa + dt2 * (jj + dt3 * (ss + dt4 * (cc))));
      a[d] = aa + dt * (jj + dt2 * (ss + dt3 * (cc)));
    } else {
      p[d] = x + dt * (vv + dt2 * (aa + dt3 * (jj)));
      v[d] = vv + dt * (aa + dt2 * (jj));
      a[d] = aa;
    }
  }
}

constexpr int kBT = 128;
constexpr int kTJ = 256;
constexpr int kNS = 3;
// Shared-memory header of the force kernel: full/empty mbarriers of the ring
// (bytes 0..47) and, in spatial mode, the box of the tile in each stage
// (2 float4 per stage, bytes 64..159); the tile ring starts at kHdr.
constexpr int kHdr = 256;

template <int ORDER, int PREC, int TPI, int IP>
struct FCfg {
  static constexpr int TIT = kBT / TPI;
  static constexpr int TI = TIT * IP;
  static constexpr int FB = PREC == DOUBLE ? 32 : 16;
  static constexpr int RS = PREC == DOUBLE ? pred_fields64(ORDER) : pred_fields(ORDER);
  static constexpr int REC = RS * FB;
  static constexpr int TILE_BYTES = kTJ * REC;
  static constexpr int RED_BYTES = TPI > 1 ? kBT * IP * kResStride * 8 : 0;
  // stages of the tile ring: two for 2 i per thread in mixed precision up to
  // 4th order, where three would hold the shape to 3 resident blocks per SM
  // by shared memory (57.6 KB) against the 4 its registers allow
  static constexpr int NS = (PREC != DOUBLE && ORDER <= FOURTH && IP == 2) ? 2 : kNS;
  static constexpr int BODY = NS * TILE_BYTES > RED_BYTES ? NS * TILE_BYTES : RED_BYTES;
  // mixed precision keeps its FP64 running totals in shared memory (10 per
  // i, [field][thread] so a warp's accesses are consecutive), which frees
  // 40 registers per thread and lets 4 blocks share an SM
  static constexpr int TOT_BYTES = PREC == DOUBLE ? 0 : IP * 10 * kBT * 8;
  static constexpr int SMEM = kHdr + BODY + TOT_BYTES;
  // resident blocks per SM the register budget is held to: FP64 kernels sit
  // at 168 registers, where one more allocation step (176) drops them from
  // 3 to 2 blocks per SM and costs 7 % at N = 2^20 (6th order)
  // (mixed 6th order with 2 i per thread: 3, since at 128 registers the FP64
  // near-pair rescan spills)
  static constexpr int MIN_BLOCKS =
      PREC == DOUBLE ? 3 : (IP >= 4 ? 2 : (ORDER >= SIXTH && IP == 2 ? 3 : 4));
};

// ---------------- mixed precision pair ----------------
// dr = (xj_hi - xi_hi) + (xj_lo - xi_lo) in FP32 (the double-single
// difference of kernels.cu:169-177), everything after it in FP32 with rsqrt
// on the MUFU pipe.  (A variant taking the difference in FP64 and rounding
// once moved 9 FMA-pipe operations per pair to the FP64 and XU pipes but was
// not faster: 3 FP64->FP32 conversions cost 24 XU cycles per warp and pair.)
struct IMix {
  float xh, yh, zh, xl, yl, zl, vx, vy, vz, ax, ay, az, h2;
  int id;
};
struct AccMix {
  float ax, ay, az, pot, jx, jy, jz, sx, sy, sz;
};

__device__ __forceinline__ float ds_sub(float jh, float jl, float ih, float il) {
  return __fadd_rn(__fsub_rn(jh, ih), __fsub_rn(jl, il));
}
// dr and ds2 of one pair, self pair masked; identical in the pair loop and
// in the rescans (explicitly rounded operations, no contraction freedom).
__device__ __forceinline__ float pair_dr_mix(const IMix &I, const float4 &r0, const float4 &r1,
                                             float &dx, float &dy, float &dz) {
  dx = ds_sub(r0.x, r1.x, I.xh, I.xl);
  dy = ds_sub(r0.y, r1.y, I.yh, I.yl);
  dz = ds_sub(r0.z, r1.z, I.zh, I.zl);
  dx = (__float_as_int(r1.w) == I.id) ? 1.0e18f : dx;
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

template <int ORDER>
__device__ __forceinline__ void pair_mix(const IMix &I, const float4 &r0, const float4 &r1,
                                         const float4 &r2, const float4 &r3, float eps2,
                                         AccMix &A, float &tmin) {
  float dx, dy, dz, ds2;
  if (ORDER == GRAPE5) {  // every pair, the self pair included (kernels.cu:565)
    dx = ds_sub(r0.x, r1.x, I.xh, I.xl);
    dy = ds_sub(r0.y, r1.y, I.yh, I.yl);
    dz = ds_sub(r0.z, r1.z, I.zh, I.zl);
    ds2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
  } else {
    ds2 = pair_dr_mix(I, r0, r1, dx, dy, dz);
    tmin = fminf(tmin, ds2);
  }
  const float inv = rsqrt_mufu(ds2 + eps2);
  const float inv2 = inv * inv;
  const float minv = r0.w * inv;
  const float minv3 = minv * inv2;
  A.ax = fmaf(minv3, dx, A.ax);
  A.ay = fmaf(minv3, dy, A.ay);
  A.az = fmaf(minv3, dz, A.az);
  A.pot -= minv;
  if (ORDER == GRAPE5) return;  // acceleration and potential only
  const float dvx = r2.x - I.vx, dvy = r2.y - I.vy, dvz = r2.z - I.vz;
  const float rv = fmaf(dz, dvz, fmaf(dy, dvy, dx * dvx));
  const float m3i2 = -3.0f * inv2;
  if (ORDER == FOURTH) {
    // jerk += m/r^3 (dv - 3 (dr.dv)/r^2 dr)   (kernels.cu:631-637)
    const float a3 = m3i2 * rv;
    A.jx = fmaf(minv3, fmaf(a3, dx, dvx), A.jx);
    A.jy = fmaf(minv3, fmaf(a3, dy, dvy), A.jy);
    A.jz = fmaf(minv3, fmaf(a3, dz, dvz), A.jz);
  } else {
    // kernels.cu:642-667 with a3 = -3 alpha, b3 = -3 beta:
    //   jerk_ij = minv3 (dv + a3 dr)
    //   snap   += minv3 (da + b3 dr) + 2 a3 jerk_ij = minv3 (da + b3 dr + 2 a3 t)
    const float dax = r3.x - I.ax, day = r3.y - I.ay, daz = r3.z - I.az;
    const float s = fmaf(dz, daz, fmaf(dy, day, fmaf(dx, dax, fmaf(dvz, dvz, fmaf(dvy, dvy, dvx * dvx)))));
    const float a3 = m3i2 * rv;
    const float b3 = fmaf(a3, a3 * (-1.0f / 3.0f), s * m3i2);
    const float a6 = a3 + a3;
    const float tx = fmaf(a3, dx, dvx), ty = fmaf(a3, dy, dvy), tz = fmaf(a3, dz, dvz);
    A.jx = fmaf(minv3, tx, A.jx);
    A.jy = fmaf(minv3, ty, A.jy);
    A.jz = fmaf(minv3, tz, A.jz);
    A.sx = fmaf(minv3, fmaf(a6, tx, fmaf(b3, dx, dax)), A.sx);
    A.sy = fmaf(minv3, fmaf(a6, ty, fmaf(b3, dy, day)), A.sy);
    A.sz = fmaf(minv3, fmaf(a6, tz, fmaf(b3, dz, daz)), A.sz);
  }
}

// ---------------- mixed precision, two i per thread, packed FP32x2 -------
// The two i-particles of a thread travel in the .x/.y halves of float2
// registers and every FP32 step is one sm_100 packed instruction
// (__fadd2_rn / __fmul2_rn / __ffma2_rn) for both; j operands are
// broadcast.  Per half the rounding is exactly that of the scalar path, so
// ds2 here is bit-identical to pair_dr_mix (used by the rescans).
struct IMix2 {
  float2 nxh, nyh, nzh, nxl, nyl, nzl;  // negated hi / lo position parts
  float2 nvx, nvy, nvz, nax, nay, naz;  // negated velocity, acceleration
  int ida, idb;
};
struct AccMix2 {
  float2 ax, ay, az, pot, jx, jy, jz, sx, sy, sz;  // pot accumulates +m/r
};

__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 neg2(float a, float b) { return make_float2(-a, -b); }

__device__ __forceinline__ IMix2 pack_i2(const IMix &a, const IMix &b) {
  IMix2 I;
  I.nxh = neg2(a.xh, b.xh); I.nyh = neg2(a.yh, b.yh); I.nzh = neg2(a.zh, b.zh);
  I.nxl = neg2(a.xl, b.xl); I.nyl = neg2(a.yl, b.yl); I.nzl = neg2(a.zl, b.zl);
  I.nvx = neg2(a.vx, b.vx); I.nvy = neg2(a.vy, b.vy); I.nvz = neg2(a.vz, b.vz);
  I.nax = neg2(a.ax, b.ax); I.nay = neg2(a.ay, b.ay); I.naz = neg2(a.az, b.az);
  I.ida = a.id;
  I.idb = b.id;
  return I;
}

// Two stages: (1) position difference, ds2 and rsqrt on the MUFU pipe,
// (2) the FMA-pipe bulk.  (Issuing stage 1 of record j+1 before stage 2 of
// record j by hand measured 6 % slower on B200 than letting the compiler
// interleave an unrolled loop.)
struct Pre2 {
  float2 dx, dy, dz, inv;
};

// The self pair is masked on every pair (two compares and selects on the
// ALU pipe): choosing an unmasked loop per tile from the tiles' id ranges
// measured 2 % slower on B200, the two loop copies costing more than the
// four ALU instructions they save.
template <bool NGB = true>  // false (GRAPE-5): no self-pair mask, no nearest-neighbour minimum
__device__ __forceinline__ Pre2 pair_mix2_pre(const IMix2 &I, const float4 &r0, const float4 &r1,
                                              float2 eps2, float2 &tmin) {
  Pre2 P;
  // x - y == x + (-y) exactly, so these equal ds_sub of the scalar path
  P.dx = __fadd2_rn(__fadd2_rn(bc2(r0.x), I.nxh), __fadd2_rn(bc2(r1.x), I.nxl));
  P.dy = __fadd2_rn(__fadd2_rn(bc2(r0.y), I.nyh), __fadd2_rn(bc2(r1.y), I.nyl));
  P.dz = __fadd2_rn(__fadd2_rn(bc2(r0.z), I.nzh), __fadd2_rn(bc2(r1.z), I.nzl));
  if (NGB) {
    const int idj = __float_as_int(r1.w);
    P.dx.x = (idj == I.ida) ? 1.0e18f : P.dx.x;
    P.dx.y = (idj == I.idb) ? 1.0e18f : P.dx.y;
  }
  const float2 ds2 = __ffma2_rn(P.dz, P.dz, __ffma2_rn(P.dy, P.dy, __fmul2_rn(P.dx, P.dx)));
  if (NGB) {
    tmin.x = fminf(tmin.x, ds2.x);
    tmin.y = fminf(tmin.y, ds2.y);
  }
  const float2 r2v = __fadd2_rn(ds2, eps2);
  P.inv = make_float2(rsqrt_mufu(r2v.x), rsqrt_mufu(r2v.y));
  return P;
}

template <int ORDER>
__device__ __forceinline__ void pair_mix2_post(const IMix2 &I, const Pre2 &P, float mj,
                                               const float4 &r2, const float4 &r3,
                                               AccMix2 &A) {
  const float2 dx = P.dx, dy = P.dy, dz = P.dz, inv = P.inv;
  const float2 inv2 = __fmul2_rn(inv, inv);
  const float2 minv = __fmul2_rn(bc2(mj), inv);
  const float2 minv3 = __fmul2_rn(minv, inv2);
  A.ax = __ffma2_rn(minv3, dx, A.ax);
  A.ay = __ffma2_rn(minv3, dy, A.ay);
  A.az = __ffma2_rn(minv3, dz, A.az);
  A.pot = __fadd2_rn(A.pot, minv);
  if (ORDER == GRAPE5) return;  // acceleration and potential only
  const float2 dvx = __fadd2_rn(bc2(r2.x), I.nvx);
  const float2 dvy = __fadd2_rn(bc2(r2.y), I.nvy);
  const float2 dvz = __fadd2_rn(bc2(r2.z), I.nvz);
  const float2 rv = __ffma2_rn(dz, dvz, __ffma2_rn(dy, dvy, __fmul2_rn(dx, dvx)));
  const float2 m3i2 = __fmul2_rn(bc2(-3.0f), inv2);
  if (ORDER == FOURTH) {
    const float2 a3 = __fmul2_rn(m3i2, rv);
    A.jx = __ffma2_rn(minv3, __ffma2_rn(a3, dx, dvx), A.jx);
    A.jy = __ffma2_rn(minv3, __ffma2_rn(a3, dy, dvy), A.jy);
    A.jz = __ffma2_rn(minv3, __ffma2_rn(a3, dz, dvz), A.jz);
  } else {
    const float2 dax = __fadd2_rn(bc2(r3.x), I.nax);
    const float2 day = __fadd2_rn(bc2(r3.y), I.nay);
    const float2 daz = __fadd2_rn(bc2(r3.z), I.naz);
    const float2 s = __ffma2_rn(dz, daz, __ffma2_rn(dy, day, __ffma2_rn(dx, dax,
                     __ffma2_rn(dvz, dvz, __ffma2_rn(dvy, dvy, __fmul2_rn(dvx, dvx))))));
    const float2 a3 = __fmul2_rn(m3i2, rv);
    const float2 b3 = __ffma2_rn(a3, __fmul2_rn(a3, bc2(-1.0f / 3.0f)), __fmul2_rn(s, m3i2));
    const float2 a6 = __fadd2_rn(a3, a3);
    const float2 tx = __ffma2_rn(a3, dx, dvx), ty = __ffma2_rn(a3, dy, dvy),
                 tz = __ffma2_rn(a3, dz, dvz);
    A.jx = __ffma2_rn(minv3, tx, A.jx);
    A.jy = __ffma2_rn(minv3, ty, A.jy);
    A.jz = __ffma2_rn(minv3, tz, A.jz);
    A.sx = __ffma2_rn(minv3, __ffma2_rn(a6, tx, __ffma2_rn(b3, dx, dax)), A.sx);
    A.sy = __ffma2_rn(minv3, __ffma2_rn(a6, ty, __ffma2_rn(b3, dy, day)), A.sy);
    A.sz = __ffma2_rn(minv3, __ffma2_rn(a6, tz, __ffma2_rn(b3, dz, daz)), A.sz);
  }
}

template <int ORDER>
__device__ __forceinline__ void pair_mix2(const IMix2 &I, const float4 &r0, const float4 &r1,
                                          const float4 &r2, const float4 &r3, float2 eps2,
                                          AccMix2 &A, float2 &tmin) {
  const Pre2 P = pair_mix2_pre<ORDER != GRAPE5>(I, r0, r1, eps2, tmin);
  pair_mix2_post<ORDER>(I, P, r0.w, r2, r3, A);
}

// Far tile (spatial mode): the j tile and the warp's i are at least
// |x|max * 2^-23 / delta apart, so the difference of the high parts alone,
// xj_hi - xi_hi, is within delta (relative) of the double-single one (each
// low part is below 2^-24 |x|): 3 FMA-pipe operations instead of 9, and the
// softening enters the first FMA of the squared distance (one operation
// less; no pair of a far tile is a nearest neighbour, so its unsoftened ds2
// is not needed: the caller checks that against the i's bounds).  No
// distance minimum is kept either: the caller rescans a far tile for list
// members when the tile's box comes within h2 of the i.  The self pair is
// still masked by id, read from the record's velocity row (r2.w), so a far
// pair reads three of the record's four float4 (6th order; two of three at 4th).
template <int ORDER>
__device__ __forceinline__ void pair_mix2_far(const IMix2 &I, const float4 &r0, const float4 &r2,
                                              const float4 &r3, float2 eps2, AccMix2 &A) {
  Pre2 P;
  P.dx = __fadd2_rn(bc2(r0.x), I.nxh);
  P.dy = __fadd2_rn(bc2(r0.y), I.nyh);
  P.dz = __fadd2_rn(bc2(r0.z), I.nzh);
  if (ORDER != GRAPE5) {
    const int idj = __float_as_int(r2.w);  // the id's copy beside the velocity
    P.dx.x = (idj == I.ida) ? 1.0e18f : P.dx.x;
    P.dx.y = (idj == I.idb) ? 1.0e18f : P.dx.y;
  }
  const float2 r2v = __ffma2_rn(P.dz, P.dz, __ffma2_rn(P.dy, P.dy, __ffma2_rn(P.dx, P.dx, eps2)));
  P.inv = make_float2(rsqrt_mufu(r2v.x), rsqrt_mufu(r2v.y));
  pair_mix2_post<ORDER>(I, P, r0.w, r2, r3, A);
}

// ---------------- FP64 pair ----------------
struct IDp {
  double x, y, z, vx, vy, vz, ax, ay, az, h2;
  int id;
};
struct AccDp {
  double ax, ay, az, pot, jx, jy, jz, sx, sy, sz;
};

__device__ __forceinline__ double pair_dr_dp(const IDp &I, const double4 &r0, const double4 &r1,
                                             double &dx, double &dy, double &dz) {
  dx = __dsub_rn(r0.x, I.x);
  dy = __dsub_rn(r0.y, I.y);
  dz = __dsub_rn(r0.z, I.z);
  dx = (__double2loint(r1.w) == I.id) ? 1.0e150 : dx;
  return __fma_rn(dz, dz, __fma_rn(dy, dy, __dmul_rn(dx, dx)));
}

// Same algebra as pair_mix: a3 = -3 alpha, b3 = -3 beta,
//   jerk_ij = minv3 t,  t = dv + a3 dr
//   snap_ij = minv3 (da + b3 dr + 2 a3 t)      (kernels.cu:642-667)
template <int ORDER>
__device__ __forceinline__ void pair_dp(const IDp &I, const double4 &r0, const double4 &r1,
                                        const double4 &r2, double eps2, AccDp &A, double &tmin) {
  double dx, dy, dz;
  const double ds2 = pair_dr_dp(I, r0, r1, dx, dy, dz);
  tmin = fmin(tmin, ds2);
  const double inv = rsqrt(ds2 + eps2);
  const double inv2 = inv * inv;
  const double minv = r0.w * inv;
  const double minv3 = minv * inv2;
  A.ax = fma(minv3, dx, A.ax);
  A.ay = fma(minv3, dy, A.ay);
  A.az = fma(minv3, dz, A.az);
  A.pot -= minv;
  const double dvx = r1.x - I.vx, dvy = r1.y - I.vy, dvz = r1.z - I.vz;
  const double rv = fma(dz, dvz, fma(dy, dvy, dx * dvx));
  const double m3i2 = -3.0 * inv2;
  const double a3 = m3i2 * rv;
  if (ORDER == FOURTH) {
    A.jx = fma(minv3, fma(a3, dx, dvx), A.jx);
    A.jy = fma(minv3, fma(a3, dy, dvy), A.jy);
    A.jz = fma(minv3, fma(a3, dz, dvz), A.jz);
  } else {
    const double dax = r2.x - I.ax, day = r2.y - I.ay, daz = r2.z - I.az;
    const double s = fma(dz, daz, fma(dy, day, fma(dx, dax, fma(dvz, dvz, fma(dvy, dvy, dvx * dvx)))));
    const double b3 = fma(a3, a3 * (-1.0 / 3.0), s * m3i2);
    const double a6 = a3 + a3;
    const double tx = fma(a3, dx, dvx), ty = fma(a3, dy, dvy), tz = fma(a3, dz, dvz);
    A.jx = fma(minv3, tx, A.jx);
    A.jy = fma(minv3, ty, A.jy);
    A.jz = fma(minv3, tz, A.jz);
    A.sx = fma(minv3, fma(a6, tx, fma(b3, dx, dax)), A.sx);
    A.sy = fma(minv3, fma(a6, ty, fma(b3, dy, day)), A.sy);
    A.sz = fma(minv3, fma(a6, tz, fma(b3, dz, daz)), A.sz);
  }
}

__device__ __forceinline__ void list_push(int *cnt, int *list, int gi, int idj) {
  const int pos = atomicAdd(cnt + gi, 1);
  if (pos < kNgbPB) list[(size_t)gi * kNgbPB + pos] = idj;
}

// Warp-cooperative neighbour-list rescan of one shared-memory tile: for every
// lane whose i saw a pair below h2 in this tile, the whole warp re-evaluates
// that i against the tile's j (lane-strided) and appends the hits.
template <int RS>
__device__ __forceinline__ void list_rescan_mix(const IMix &I, bool want, int gi, int row,
                                                int TPI, const float4 *rec, int cnt, int lane,
                                                int *ngb_count, int *ngb_list) {
  unsigned m = __ballot_sync(0xffffffffu, want);
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    IMix S;
    S.xh = __shfl_sync(0xffffffffu, I.xh, src);
    S.yh = __shfl_sync(0xffffffffu, I.yh, src);
    S.zh = __shfl_sync(0xffffffffu, I.zh, src);
    S.xl = __shfl_sync(0xffffffffu, I.xl, src);
    S.yl = __shfl_sync(0xffffffffu, I.yl, src);
    S.zl = __shfl_sync(0xffffffffu, I.zl, src);
    S.h2 = __shfl_sync(0xffffffffu, I.h2, src);
    S.id = __shfl_sync(0xffffffffu, I.id, src);
    const int sgi = __shfl_sync(0xffffffffu, gi, src);
    const int srow = __shfl_sync(0xffffffffu, row, src);
    for (int k = srow + lane * TPI; k < cnt; k += 32 * TPI) {
      float dx, dy, dz;
      const float4 r0 = rec[k * RS + 0];
      const float4 r1 = rec[k * RS + 1];
      const float ds2 = pair_dr_mix(S, r0, r1, dx, dy, dz);
      if (ds2 < S.h2) list_push(ngb_count, ngb_list, sgi, __float_as_int(r1.w));
    }
  }
}

// Near-pair rescan (mixed precision).  A pair closer than a few softening
// lengths can carry most of an i's jerk or snap while passing through zero
// (the radial snap of a softened pair vanishes at r^2 = 1.5 eps^2), and there
// the FP32 rounding of its terms, ~1e-7 of their size, becomes a large
// relative error of the small total.  So when an i's row of a tile holds a j
// with the exact double-single ds2 below near_r2, the caller drops that row's
// FP32 partial sum for the i and this routine sums the same records again in
// FP64: the warp splits the row's j, each lane evaluates pair_dp on the
// record widened to double (the double-single position hi + lo is exact in
// double; velocity, acceleration and mass as stored) against the i's own FP64
// record, and the warp sum is added to that i's FP64 totals by its lane.
// `nm` is the ballot of the lanes that asked.  near_rescan_mix keeps it out
// of line (the grid kernel, whose register budget has room for the call);
// near_rescan_inl is the same code inlined (the batch kernel, held to 128
// registers, where the call would spill).
template <int ORDER, int RS>
__device__ __forceinline__ void near_rescan_inl(unsigned nm, int oi, int row, int tpi,
                                                const float4 *rec, int cnt, int lane,
                                                const double *irec, double eps2, double *tot) {
  while (nm) {
    const int src = __ffs(nm) - 1;
    nm &= nm - 1;
    const int soi = __shfl_sync(0xffffffffu, oi, src);
    const int srow = __shfl_sync(0xffffffffu, row, src);
    const double *r = irec + (size_t)soi * i_stride(ORDER);
    IDp I;
    I.x = r[0]; I.y = r[1]; I.z = r[2]; I.h2 = 0.0;
    I.vx = r[4]; I.vy = r[5]; I.vz = r[6];
    I.id = __double2loint(r[7]);
    I.ax = I.ay = I.az = 0.0;
    if (ORDER >= SIXTH) {
      I.ax = r[8]; I.ay = r[9]; I.az = r[10];
    }
    AccDp S{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    double tmin = DBL_MAX;
    for (int k = srow + lane * tpi; k < cnt; k += 32 * tpi) {
      const float4 q0 = rec[k * RS + 0], q1 = rec[k * RS + 1], q2 = rec[k * RS + 2];
      const float4 q3 = ORDER >= SIXTH ? rec[k * RS + 3] : q2;
      const double4 j0 = make_double4((double)q0.x + (double)q1.x, (double)q0.y + (double)q1.y,
                                      (double)q0.z + (double)q1.z, (double)q0.w);
      const double4 j1 = make_double4(q2.x, q2.y, q2.z,
                                      __hiloint2double(0, __float_as_int(q1.w)));
      const double4 j2 = make_double4(q3.x, q3.y, q3.z, 0.0);
      pair_dp<ORDER>(I, j0, j1, j2, eps2, S, tmin);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      S.ax += __shfl_xor_sync(0xffffffffu, S.ax, o);
      S.ay += __shfl_xor_sync(0xffffffffu, S.ay, o);
      S.az += __shfl_xor_sync(0xffffffffu, S.az, o);
      S.pot += __shfl_xor_sync(0xffffffffu, S.pot, o);
      S.jx += __shfl_xor_sync(0xffffffffu, S.jx, o);
      S.jy += __shfl_xor_sync(0xffffffffu, S.jy, o);
      S.jz += __shfl_xor_sync(0xffffffffu, S.jz, o);
      if (ORDER >= SIXTH) {
        S.sx += __shfl_xor_sync(0xffffffffu, S.sx, o);
        S.sy += __shfl_xor_sync(0xffffffffu, S.sy, o);
        S.sz += __shfl_xor_sync(0xffffffffu, S.sz, o);
      }
    }
    if (lane == src) {
      tot[0 * kBT] += S.ax;
      tot[1 * kBT] += S.ay;
      tot[2 * kBT] += S.az;
      tot[3 * kBT] += S.pot;
      tot[4 * kBT] += S.jx;
      tot[5 * kBT] += S.jy;
      tot[6 * kBT] += S.jz;
      if (ORDER >= SIXTH) {
        tot[7 * kBT] += S.sx;
        tot[8 * kBT] += S.sy;
        tot[9 * kBT] += S.sz;
      }
    }
  }
}

template <int ORDER, int RS>
__device__ __noinline__ void near_rescan_mix(unsigned nm, int oi, int row, int tpi,
                                             const float4 *rec, int cnt, int lane,
                                             const double *irec, double eps2, double *tot) {
  near_rescan_inl<ORDER, RS>(nm, oi, row, tpi, rec, cnt, lane, irec, eps2, tot);
}

template <int RS>
__device__ __forceinline__ void list_rescan_dp(const IDp &I, bool want, int gi, int row,
                                               int TPI, const double4 *rec, int cnt, int lane,
                                               int *ngb_count, int *ngb_list) {
  unsigned m = __ballot_sync(0xffffffffu, want);
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    IDp S;
    S.x = __shfl_sync(0xffffffffu, I.x, src);
    S.y = __shfl_sync(0xffffffffu, I.y, src);
    S.z = __shfl_sync(0xffffffffu, I.z, src);
    S.h2 = __shfl_sync(0xffffffffu, I.h2, src);
    S.id = __shfl_sync(0xffffffffu, I.id, src);
    const int sgi = __shfl_sync(0xffffffffu, gi, src);
    const int srow = __shfl_sync(0xffffffffu, row, src);
    for (int k = srow + lane * TPI; k < cnt; k += 32 * TPI) {
      double dx, dy, dz;
      const double4 r0 = rec[k * RS + 0];
      const double4 r1 = rec[k * RS + 1];
      const double ds2 = pair_dr_dp(S, r0, r1, dx, dy, dz);
      if (ds2 < S.h2) list_push(ngb_count, ngb_list, sgi, __double2loint(r1.w));
    }
  }
}


}  // namespace sapb
