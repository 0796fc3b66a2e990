/*
 * FP64 CPU oracle for the Sapporo2 direct-summation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests,
 * the smoke check and the CPU-baseline leg of the benchmark link it.  The
 * product library never links, loads or calls it, and there is no CPU
 * fallback in the product path.
 *
 * It restates, in plain C with double precision everywhere, what the
 * reference computes:
 *   - the Taylor predictor of lib/CUDAKernels/kernels.cu:307-383
 *     (Horner form; 4th order forces dt4 = dt5 = 0 at :338-342), which is
 *     also the CPU form at lib/src/sapporohostclass.cpp:1287-1351;
 *   - the pair interaction of lib/CUDAKernels/kernels.cu:552-669
 *     (self pair skipped by id equality :565; dr = xj - xi; ds2 = |dr|^2
 *     without softening for the nearest neighbour and the list; strict
 *     "h2 > ds2" for the list :584; inv = 1/sqrt(ds2 + eps2) :591;
 *     acc += m inv^3 dr, pot += -m inv :616-619; 4th-order jerk :631-637;
 *     6th-order jerk and snap :642-667);
 *   - nearest neighbour as the first strict minimum of ds2 in j order
 *     (kernels.cu:539-546), initial state ds2min = 1e11, nnb = -1 (:522);
 *   - the 4th-order FP64 host loop of lib/src/sapporohostclass.cpp:1373-1438,
 *     which is the same arithmetic.
 *
 * Parity pin: the outputs of this oracle are compared with the reference's
 * own CUDA kernels (compiled from the reference sources into oracle/_ref)
 * on seeded inputs; the resulting fixtures live in tests/golden/.
 *
 * Neighbour lists: every j with h2_i > ds2 is counted; the first `ngb_cap`
 * ids in j order are stored.  The reference stores at most 256 per i and
 * flags overflow when the count reaches 256; callers compare sets only when
 * the count is below the capacity.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_GRAPE5 0
#define ORC_FOURTH 1
#define ORC_SIXTH 2

int orc_version(void) { return 1; }

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Predictor: kernels.cu:331-383.  Arrays are [n][3] (x, v, a, j, s, c);
 * s and c may be NULL for order <= 4th; pa may be NULL for order <= 4th. */
void orc_predict(int nj, double ti, int order, const double *t,
                 const double *x, const double *v, const double *a,
                 const double *j, const double *s, const double *c,
                 double *px, double *pv, double *pa, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
  for (int k = 0; k < nj; k++) {
    const double dt = ti - t[k];
    const double dt2 = (1. / 2.) * dt;
    const double dt3 = (1. / 3.) * dt;
    double dt4 = (1. / 4.) * dt;
    double dt5 = (1. / 5.) * dt;
    if (order <= ORC_FOURTH) {
      dt4 = 0;
      dt5 = 0;
    }
    for (int d = 0; d < 3; d++) {
      const double sn = (order >= ORC_SIXTH) ? s[3 * k + d] : 0.0;
      const double cr = (order >= ORC_SIXTH) ? c[3 * k + d] : 0.0;
      const double xx = x[3 * k + d], vv = v[3 * k + d];
      const double aa = a[3 * k + d], jj = j[3 * k + d];
      px[3 * k + d] = xx + dt * (vv + dt2 * (aa + dt3 * (jj + dt4 * (sn + dt5 * cr))));
      pv[3 * k + d] = vv + dt * (aa + dt2 * (jj + dt3 * (sn + dt4 * cr)));
      if (order >= ORC_SIXTH && pa)
        pa[3 * k + d] = aa + dt * (jj + dt2 * (sn + dt3 * cr));
    }
  }
  (void)nthreads;
}

/* Force on ni i-particles from nj predicted j-particles.
 * xi, vi, ai, acc, jrk, snp: [ni][3]; xj, vj, aj: [nj][3].
 * ai/aj/snp may be NULL unless order == 6th.  ngb_list: [ni][ngb_cap] or
 * NULL.  nnb/ds2min/ngb_count may be NULL. */
void orc_force(int order, int ni, const double *xi, const double *vi,
               const double *ai, const double *h2, const int *idi, int nj,
               const double *xj, const double *vj, const double *aj,
               const double *mj, const int *idj, double eps2, double *acc,
               double *jrk, double *snp, double *pot, int *nnb,
               double *ds2min, int *ngb_count, int *ngb_list, int ngb_cap,
               int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
  for (int i = 0; i < ni; i++) {
    const double px = xi[3 * i], py = xi[3 * i + 1], pz = xi[3 * i + 2];
    const double qx = vi[3 * i], qy = vi[3 * i + 1], qz = vi[3 * i + 2];
    double rx = 0, ry = 0, rz = 0;
    if (order >= ORC_SIXTH) {
      rx = ai[3 * i];
      ry = ai[3 * i + 1];
      rz = ai[3 * i + 2];
    }
    const double hh = h2 ? h2[i] : 0.0;
    const int myid = idi[i];
    double ax = 0, ay = 0, az = 0, ph = 0;
    double jx = 0, jy = 0, jz = 0;
    double sx = 0, sy = 0, sz = 0;
    double dmin = 1.0e11;
    int nn = -1;
    int cnt = 0;
    for (int k = 0; k < nj; k++) {
      if (idj[k] == myid && order != ORC_GRAPE5) continue; /* kernels.cu:565 */
      const double drx = xj[3 * k] - px;
      const double dry = xj[3 * k + 1] - py;
      const double drz = xj[3 * k + 2] - pz;
      const double ds2 = drx * drx + dry * dry + drz * drz;
      if (ds2 < dmin) { /* kernels.cu:539-546 */
        dmin = ds2;
        nn = idj[k];
      }
      if (hh > ds2) { /* kernels.cu:584-588 */
        if (ngb_list && cnt < ngb_cap) ngb_list[(size_t)i * ngb_cap + cnt] = idj[k];
        cnt++;
      }
      const double inv = 1.0 / sqrt(ds2 + eps2);
      const double minvr1 = mj[k] * inv;
      const double invr2 = inv * inv;
      const double minvr3 = minvr1 * invr2;
      ax += minvr3 * drx;
      ay += minvr3 * dry;
      az += minvr3 * drz;
      ph += -minvr1;
      if (order == ORC_GRAPE5) continue;
      const double dvx = vj[3 * k] - qx;
      const double dvy = vj[3 * k + 1] - qy;
      const double dvz = vj[3 * k + 2] - qz;
      const double rv = drx * dvx + dry * dvy + drz * dvz;
      if (order == ORC_FOURTH) { /* kernels.cu:631-637 */
        const double drdv = (-3.0) * (minvr3 * invr2) * rv;
        jx += minvr3 * dvx + drdv * drx;
        jy += minvr3 * dvy + drdv * dry;
        jz += minvr3 * dvz + drdv * drz;
        continue;
      }
      /* 6th order, kernels.cu:642-667 */
      const double dax = aj[3 * k] - rx;
      const double day = aj[3 * k + 1] - ry;
      const double daz = aj[3 * k + 2] - rz;
      const double v2 = dvx * dvx + dvy * dvy + dvz * dvz;
      const double ra = drx * dax + dry * day + drz * daz;
      double alpha = rv * invr2;
      double beta = (v2 + ra) * invr2 + alpha * alpha;
      alpha *= -3.0;
      const double ex = minvr3 * dvx + alpha * (minvr3 * drx);
      const double ey = minvr3 * dvy + alpha * (minvr3 * dry);
      const double ez = minvr3 * dvz + alpha * (minvr3 * drz);
      alpha *= 2.0;
      beta *= -3.0;
      sx += minvr3 * dax + alpha * ex + beta * (minvr3 * drx);
      sy += minvr3 * day + alpha * ey + beta * (minvr3 * dry);
      sz += minvr3 * daz + alpha * ez + beta * (minvr3 * drz);
      jx += ex;
      jy += ey;
      jz += ez;
    }
    acc[3 * i] = ax;
    acc[3 * i + 1] = ay;
    acc[3 * i + 2] = az;
    if (pot) pot[i] = ph;
    if (jrk) {
      jrk[3 * i] = jx;
      jrk[3 * i + 1] = jy;
      jrk[3 * i + 2] = jz;
    }
    if (snp && order >= ORC_SIXTH) {
      snp[3 * i] = sx;
      snp[3 * i + 1] = sy;
      snp[3 * i + 2] = sz;
    }
    if (nnb) nnb[i] = nn;
    if (ds2min) ds2min[i] = dmin;
    if (ngb_count) ngb_count[i] = cnt;
  }
  (void)nthreads;
}

/* The same pair sum for a subset of i given by index (for sampled checks at
 * large N): out arrays are [nsel][...] in the order of `sel`. */
void orc_force_subset(int order, int nsel, const int *sel, const double *xi,
                      const double *vi, const double *ai, const double *h2,
                      const int *idi, int nj, const double *xj,
                      const double *vj, const double *aj, const double *mj,
                      const int *idj, double eps2, double *acc, double *jrk,
                      double *snp, double *pot, int *nnb, double *ds2min,
                      int *ngb_count, int nthreads) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
  for (int q = 0; q < nsel; q++) {
    const int i = sel[q];
    double a3[3], j3[3], s3[3], p1, d1;
    int n1, c1;
    orc_force(order, 1, xi + 3 * (size_t)i, vi + 3 * (size_t)i,
              ai ? ai + 3 * (size_t)i : NULL, h2 ? h2 + i : NULL, idi + i, nj,
              xj, vj, aj, mj, idj, eps2, a3, j3, s3, &p1, &n1, &d1, &c1, NULL,
              0, 1);
    for (int d = 0; d < 3; d++) {
      acc[3 * q + d] = a3[d];
      if (jrk) jrk[3 * q + d] = j3[d];
      if (snp && order >= ORC_SIXTH) snp[3 * q + d] = s3[d];
    }
    if (pot) pot[q] = p1;
    if (nnb) nnb[q] = n1;
    if (ds2min) ds2min[q] = d1;
    if (ngb_count) ngb_count[q] = c1;
  }
  (void)nthreads;
}
