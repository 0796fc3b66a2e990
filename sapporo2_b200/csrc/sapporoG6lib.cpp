// GRAPE-6 C interface (Fortran-style names, all arguments by pointer) over
// one process-wide `sapporo` instance, as lib/interfaces/sapporoG6lib.cpp of
// the reference: 4th order, double-single precision by default.
// Declared in include/sapporo_g6.h.
//
// SAPPORO_PRECISION=double in the environment selects the all-FP64 kernels
// (the reference keeps that choice as a commented-out line, :36-37).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/sapporo_g6.h"
#include "../../include/sapporohostclass.h"

static sapporo grav;
static double *g6_dsmin_i = nullptr;  // nearest-neighbour distances (lasthalf2)

extern "C" {

int g6_open_special(int ndev, int *list) {
  int precision = DOUBLESINGLE;
  const char *p = getenv("SAPPORO_PRECISION");
  if (p && (!strcmp(p, "double") || !strcmp(p, "DOUBLE") || !strcmp(p, "2"))) precision = DOUBLE;
  const int res = grav.open("linked-in kernels", list, ndev, FOURTH, precision);
  const int n_pipes = grav.get_n_pipes();
  free(g6_dsmin_i);
  g6_dsmin_i = (double *)malloc(sizeof(double) * (size_t)(n_pipes > 0 ? n_pipes : 1));
  return res;
}

int g6_open_(int *id) {
  (void)id;
  // sapporo2.config in the working directory: first line = number of
  // devices, then one device id per line (lib/interfaces/sapporoG6lib.cpp:46-77).
  int *dev_list = nullptr;
  int how_many = 0;
  FILE *fd = fopen("sapporo2.config", "r");
  if (fd) {
    char line[256];
    if (fgets(line, sizeof line, fd) != nullptr) sscanf(line, "%d", &how_many);
    if (how_many > 0) {
      dev_list = new int[how_many];
      for (int i = 0; i < how_many; i++) {
        dev_list[i] = 0;
        if (fgets(line, sizeof line, fd) != nullptr) sscanf(line, "%d", &dev_list[i]);
      }
    }
    fclose(fd);
  }
  const int res = g6_open_special(how_many, dev_list);
  delete[] dev_list;
  return res;
}

int g6_close_(int *id) {
  (void)id;
  return grav.close();
}

int g6_npipes_() { return grav.get_n_pipes(); }
int g6_set_tunit_(double *) { return 0; }
int g6_set_xunit_(double *) { return 0; }

int g6_set_ti_(int *id, double *ti) {
  (void)id;
  return grav.set_time(*ti);
}

int g6_set_j_particle_(int *cluster_id, int *address, int *index, double *tj, double *dtj,
                       double *mass, double k18[3], double j6[3], double a2[3], double v[3],
                       double x[3]) {
  (void)cluster_id;
  // GRAPE-6 passes a/2 and j/6 (lib/interfaces/sapporoG6lib.cpp:102-104)
  double acc[3] = {a2[0] * 2, a2[1] * 2, a2[2] * 2};
  double jrk[3] = {j6[0] * 6, j6[1] * 6, j6[2] * 6};
  return grav.set_j_particle(*address, *index, *tj, *dtj, *mass, k18, jrk, acc, v, x, nullptr,
                             nullptr, 0);
}

void g6calc_firsthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                       double vi[][3], double aold[][3], double j6old[][3], double phiold[3],
                       double *eps2, double h2[]) {
  (void)cluster_id;
  grav.startGravCalc(*nj, *ni, index, xi, vi, aold, j6old, phiold, *eps2, h2, nullptr);
}

int g6calc_lasthalf_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                     double vi[][3], double *eps2, double h2[], double acc[][3],
                     double jerk[][3], double pot[]) {
  (void)cluster_id;
  return grav.getGravResults(*nj, *ni, index, xi, vi, *eps2, h2, acc, jerk, nullptr, nullptr,
                             pot, nullptr, nullptr, false);
}

int g6calc_lasthalf2_(int *cluster_id, int *nj, int *ni, int index[], double xi[][3],
                      double vi[][3], double *eps2, double h2[], double acc[][3],
                      double jerk[][3], double pot[], int *inn) {
  (void)cluster_id;
  return grav.getGravResults(*nj, *ni, index, xi, vi, *eps2, h2, acc, jerk, nullptr, nullptr,
                             pot, inn, g6_dsmin_i, true);
}

void get_j_part_data(int addr, int nj, double *pos, double *vel, double *acc, double *jrk,
                     double *ppos, double *pvel, double &mass, double &eps2, int &id) {
  (void)nj;
  double idt = 0;
  grav.retrieve_j_particle_state(addr, mass, idt, eps2, pos, vel, acc, jrk, ppos, pvel, nullptr);
  id = (int)idt;
}

int g6_initialize_jp_buffer_(int *cluster_id, int *buf_size) {
  (void)cluster_id;
  (void)buf_size;
  return 0;
}
int g6_flush_jp_buffer_(int *cluster_id) {
  (void)cluster_id;
  return 0;
}
int g6_reset_(int *cluster_id) {
  (void)cluster_id;
  return 0;
}
int g6_reset_fofpga_(int *cluster_id) {
  (void)cluster_id;
  return 0;
}

int g6_read_neighbour_list_(int *cluster_id) { return grav.read_ngb_list(*cluster_id); }

int g6_get_neighbour_list_(int *cluster_id, int *ipipe, int *maxlength, int *n_neighbours,
                           int neighbour_list[]) {
  return grav.get_ngb_list(*cluster_id, *ipipe, *maxlength, *n_neighbours, neighbour_list);
}

}  // extern "C"
