/*
 * sapporo_g5.h -- GRAPE-5 C interface, exported by libsapporo_b200.so.
 * Same names, arguments and behaviour as lib/interfaces/sapporoG5lib.cpp:
 * positions and masses only, acceleration and potential out, no ids.  As on
 * GRAPE-5 the self pair is not skipped: it adds -m_i/eps to the potential of
 * an i that coincides with a j (and nothing to the acceleration).  Computed
 * by the GRAPE-5 mixed-precision kernels (double-single position
 * difference, no jerk, no neighbour search).  Void calls that the reference
 * ends with exit() (softening or nj not set) report on stderr and return
 * without computing.
 */
#ifndef SAPPORO_G5_H
#define SAPPORO_G5_H

#ifdef __cplusplus
extern "C" {
#endif

/* lib/interfaces/sapporoG5lib.cpp:39-53: open the devices of `list`. */
int g5_open_special(int ndev, int *list);
/* :55-85: open, devices from ./sapporo2.config. */
void g5_open(void);
/* :88: close. */
void g5_close(void);
/* :89: i-particles per force call. */
int g5_get_number_of_pipelines(void);
/* :91-94: number of j used by the force calls. */
void g5_set_n(int nj);
/* :96-99: softening eps^2 for all. */
void g5_set_eps2_to_all(double eps2);
/* :101-104: softening eps for all (squared here). */
void g5_set_eps_to_all(double eps);
/* :108-116: j [addr, addr+nj) from xj[addr..] and jmass[addr..]. */
void g5_set_xmj(int addr, int nj, double xj[][3], double jmass[]);
/* :118-121: same, arguments swapped. */
void g5_set_jp(int addr, int nj, double jmass[], double xj[][3]);
/* :126-145: stage ni <= n_pipes i-particles and start the force. */
void g5_set_xi(int ni, double xi[][3]);
/* :146: no-op (g5_set_xi starts the run). */
void g5_run(void);
/* :148-155: results of the force started by g5_set_xi. */
void g5_get_force(int ni, double a[][3], double *phi);
/* :159-194: force on any number of i, in chunks of n_pipes. */
void g5_calculate_force_on_x(double xi[][3], double a[][3], double *phi, int ni);
/* :198-202: no-op on a GPU. */
void g5_set_range(double xmin, double xmax, double mmin);
/* :205-218: constants of the reference. */
int g5_get_jmemsize(void);
int g5_get_number_of_real_pipelines(void);
int g5_get_pcibus_freq(void);

#ifdef __cplusplus
}
#endif
#endif
