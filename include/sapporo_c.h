/*
 * sapporo_c.h -- C binding of the `sapporo` C++ class, for callers that
 * cannot use C++ (ctypes, cgo, Fortran ISO_C_BINDING).  Each function wraps
 * the class method of the same name (reference interface:
 * lib/include/sapporohostclass.h:125-175); array arguments are flat
 * row-major [n][3] doubles.  All return 0 on success or a negative
 * SAPB_E* code from sapporo_b200.h.
 */
#ifndef SAPPORO_C_H
#define SAPPORO_C_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sapporo_c sapporo_c;
struct sapb_dev;

sapporo_c *sapporo_c_new(void);
void sapporo_c_delete(sapporo_c *s);
/* sapporo::open with a one-device list {device}. */
int sapporo_c_open(sapporo_c *s, int device, int order, int precision);
/* sapporo::open(kernelFile, devices, ndev, order, precision): ndev > 0 uses
 * devices[0..ndev-1] (ids may repeat), 0 every visible device, < 0 the
 * first -ndev devices.  j are spread round-robin over them by address. */
int sapporo_c_open_devices(sapporo_c *s, int ndev, const int *devices, int order, int precision);
int sapporo_c_close(sapporo_c *s);
int sapporo_c_get_n_pipes(sapporo_c *s);
int sapporo_c_set_time(sapporo_c *s, double ti);
int sapporo_c_set_no_time(sapporo_c *s);
/* sapporo::set_j_particle for n particles; pointers for snap/crackle/eps
 * may be NULL.  x, v, a, jrk, snp, crk: [n][3]. */
int sapporo_c_set_j_particles(sapporo_c *s, int n, const int *address, const int *id,
                              const double *t, const double *mass, const double *x,
                              const double *v, const double *a, const double *jrk,
                              const double *snp, const double *crk, const double *eps);
/* sapporo::startGravCalc; ai may be NULL for 4th order, h2 NULL = 0. */
int sapporo_c_start(sapporo_c *s, int nj, int ni, const int *id, const double *xi,
                    const double *vi, const double *ai, double eps2, const double *h2);
/* sapporo::getGravResults; jrk/snp/nnb/dsmin may be NULL where the order or
 * `ngb` makes them unused. */
int sapporo_c_results(sapporo_c *s, int nj, int ni, double *acc, double *jrk, double *snp,
                      double *pot, int *nnb, double *dsmin, int ngb);
int sapporo_c_force_prediction(sapporo_c *s, int nj);
int sapporo_c_read_ngb_list(sapporo_c *s);
int sapporo_c_get_ngb_list(sapporo_c *s, int ipipe, int maxlength, int *nblen, int *nbl);
/* How many ids the last sapporo_c_get_ngb_list wrote to nbl (sorted): *nblen
 * capped at maxlength, less the ids beyond NGB_PB of an overflowing device's
 * list (which were not stored). */
int sapporo_c_ngb_list_copied(sapporo_c *s);
/* out: mass, id, eps2, pos[3], vel[3], acc[3] (10 doubles). */
int sapporo_c_retrieve_predicted(sapporo_c *s, int addr, double *out);
/* out: mass, id, eps2, pos[3], vel[3], acc[3], jrk[3], ppos[3], pvel[3], pacc[3] (24). */
int sapporo_c_retrieve_state(sapporo_c *s, int addr, double *out);
int sapporo_c_last_status(sapporo_c *s);
/* The device handle of the first device (sapporo_c_device) and of entry k
 * of the device list (null when k is out of range); their number. */
struct sapb_dev *sapporo_c_device(sapporo_c *s);
struct sapb_dev *sapporo_c_device_at(sapporo_c *s, int k);
int sapporo_c_n_devices(sapporo_c *s);

#ifdef __cplusplus
}
#endif
#endif
