/*
 * sapporo_yebisu.h -- the 6th-order interface of lib/interfaces/sapporoYeblib.cpp
 * (written for the Yebisu N-body code), exported by libsapporoyeb_b200.so: a
 * library of its own because its generic names (initialize_special,
 * predict_all, calc_force_on_predictors, ...) are also those of the 6th-order
 * C interface (libsapporo6th_b200.so) with other arguments.  6th order,
 * all-FP64 kernels unless SAPPORO_PRECISION=mixed.
 */
#ifndef SAPPORO_YEBISU_H
#define SAPPORO_YEBISU_H

#ifdef __cplusplus
extern "C" {
#endif

/* The i-particle record of the reference (:17-28): 12 doubles. */
typedef struct sapporo_yeb_predictor {
  double pos[3], vel[3], acc[3];
  double mass;
  double id;
  double eps2;
} sapporo_yeb_predictor;

/* The result record of the reference (:31-52): acc, jerk, snap, phi =
 * -potential (positive), nearest neighbour id and squared distance. */
typedef struct sapporo_yeb_force {
  double acc[3], jrk[3], snp[3];
  double phi;
  int nnb_id;
  float nnb_r2;
} sapporo_yeb_force;

/* :182-216: open once with a device list. */
void initialize_special(int ndev, int *list);
/* :220-250: open once, devices from ./sapporo2.config (n unused). */
void initialize(int n);
/* :254-263: store a j-particle (true derivatives). */
void set_jp_2(int add, double pos[3], double vel[3], double acc[3], double jrk[3],
              double snp[3], double crk[3], double mass, double time, int id, double eps2);
/* :266-273: predict j[0, nj) to `time` now. */
void predict_all(double time, int nj);
/* :276-284: copy j[0, nj) to the force buffers without predicting. */
void no_predict_all(double time, int nj);
/* :288-295: predicted state of the j at addr into *pred. */
void pick_up_predictor_2(int addr, sapporo_yeb_predictor *pred);
/* :298-380: force on ni predicted i (eps2 of pred[0] for all), in chunks of
 * n_pipes, nearest neighbour on, lists off. */
void calc_force_on_predictors(int ni, sapporo_yeb_predictor pred[], sapporo_yeb_force force[],
                              int nj);
/* :383-396: individual softening -- not implemented by the reference either
 * (it prints a message and exits); here it prints the message and returns. */
void calc_force_on_predictors_epsj(int ni, sapporo_yeb_predictor pred[],
                                   sapporo_yeb_force force[], int nj);

#ifdef __cplusplus
}
#endif
#endif
