/*
 * sapporo_g6.h -- GRAPE-6 C interface exported by libsapporo_b200.so.
 *
 * Exactly the symbols of the reference's lib/interfaces/sapporoG6lib.cpp
 * (Fortran-style trailing underscore, every argument by pointer), so an
 * integrator that links against the reference's libsapporo links against
 * this library unchanged.  Callers normally declare these themselves, as
 * the reference's testCodes/src/g6lib.h:4-50 does; this header is the same
 * list with the source of each.
 */
#ifndef SAPPORO_G6_H
#define SAPPORO_G6_H

#ifdef __cplusplus
extern "C" {
#endif

/* lib/interfaces/sapporoG6lib.cpp:25-44: open with an explicit device list. */
int g6_open_special(int ndev, int *list);
/* :46-77: open, reading ./sapporo2.config (device count, then ids). */
int g6_open_(int *id);
/* :80 */
int g6_close_(int *id);
/* :81-85: maximum i-particles per firsthalf/lasthalf call. */
int g6_npipes_(void);
/* :86-87: no-ops kept for GRAPE-6 compatibility. */
int g6_set_tunit_(double *);
int g6_set_xunit_(double *);
/* :88: prediction time of the next force call. */
int g6_set_ti_(int *id, double *ti);
/* :89-108: stores a j-particle; a2 = acc/2 and j6 = jerk/6 (GRAPE-6 scaling). */
int g6_set_j_particle_(int *cluster_id, int *address, int *index, double *tj, double *dtj,
                       double *mass, double k18[3], double j6[3], double a2[3], double v[3],
                       double x[3]);
/* :109-120: queues the force on ni i-particles from nj j-particles (async). */
void g6calc_firsthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                       double vi[][3], double aold[][3], double j6old[][3], double phiold[3],
                       double *eps2, double h2[]);
/* :121-134: waits and returns acc, jerk, pot. */
int g6calc_lasthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                     double vi[][3], double *eps2, double h2[], double acc[][3],
                     double jerk[][3], double pot[]);
/* :135-149: as lasthalf, plus the nearest-neighbour id in inn[]. */
int g6calc_lasthalf2_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                      double vi[][3], double *eps2, double h2[], double acc[][3],
                      double jerk[][3], double pot[], int *inn);
/* :176-179: no-ops. */
int g6_initialize_jp_buffer_(int *cluster_id, int *buf_size);
int g6_flush_jp_buffer_(int *cluster_id);
int g6_reset_(int *cluster_id);
int g6_reset_fofpga_(int *cluster_id);
/* :181-182: copies the neighbour lists of the last call; 1 on overflow. */
int g6_read_neighbour_list_(int *cluster_id);
/* :187-201: sorted neighbour ids of i-particle *ipipe; 1 on overflow. */
int g6_get_neighbour_list_(int *cluster_id, int *ipipe, int *maxlength, int *n_neighbours,
                           int neighbour_list[]);

#ifdef __cplusplus
/* :152-172: full stored state of the j-particle at addr (C++ linkage types). */
void get_j_part_data(int addr, int nj, double *pos, double *vel, double *acc, double *jrk,
                     double *ppos, double *pvel, double &mass, double &eps2, int &id);
#endif

#ifdef __cplusplus
}
#endif
#endif
