/*
 * sapporo6th.h -- 6th-order Hermite C interface, exported by
 * libsapporo6th_b200.so (a separate library because the names are generic;
 * the reference likewise builds lib/interfaces/sapporo6thlib.cpp outside
 * libsapporo.a, lib/Makefile:73-74).  Same names, arguments and behaviour as
 * lib/interfaces/sapporo6thlib.cpp; 6th order, all-FP64 kernels unless
 * SAPPORO_PRECISION=mixed.
 */
#ifndef SAPPORO6TH_H
#define SAPPORO6TH_H

#ifdef __cplusplus
extern "C" {
#endif

/* lib/interfaces/sapporo6thlib.cpp:18-40: open once with a device list. */
void initialize_special(int ndev, int *list);
/* :42-70: open once, devices from ./sapporo2.config. */
void initialize(void);
/* :84-93: stores a j-particle (true derivatives, not GRAPE-scaled). */
void set_j_particle(int add, double pos[3], double vel[3], double acc[3], double jrk[3],
                    double snp[3], double crk[3], double mass, double time, int id,
                    double eps2);
/* :103-111: predicts j[0, nj) to `time` now. */
void predict_all(double time, int nj);
/* :119-127: copies j[0, nj) into the force buffers without predicting. */
void no_predict_all(double time, int nj);
/* :167-201: acc, jerk, snap, potential and nearest neighbour of ni
 * i-particles from nj j-particles, in chunks of n_pipes; crackle is zeroed. */
void calc_force_on_predictors(int ni, int nj, int ids[], double pos[][3], double vel[][3],
                              double acc[][3], double mass[], double eps2[],
                              double accNew[][3], double jrkNew[][3], double snpNew[][3],
                              double crkNew[][3], double phi[], int nnb[], double nnb_r2[]);

#ifdef __cplusplus
/* :143-149: predicted state of the j-particle at addr (C++ reference args). */
void pick_up_predictor_2(int addr, int &id, double &mass, double &eps2, double pos[3],
                         double vel[3], double acc[3]);
#endif

#ifdef __cplusplus
}
#endif
#endif
