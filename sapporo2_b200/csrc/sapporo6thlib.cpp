// 6th-order Hermite C interface over one process-wide `sapporo` instance
// (6th order, all-FP64 kernels by default), as the reference's
// lib/interfaces/sapporo6thlib.cpp.  Built into its own library,
// libsapporo6th_b200.so, because its generic symbol names (initialize,
// set_j_particle, ...) would clash with callers of the GRAPE-6 library; the
// reference likewise leaves this file out of libsapporo.a (lib/Makefile:73-74).
// Declared in include/sapporo6th.h.
//
// SAPPORO_PRECISION=mixed selects the mixed-precision kernels.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/sapporo6th.h"
#include "../../include/sapporohostclass.h"

static sapporo grav6;
static std::vector<double> h2_zero;  // h2 = 0: no neighbour lists (:34-39)
static bool opened = false;

extern "C" {

void initialize_special(int ndev, int *list) {
  if (opened) return;  // "SHOULD BE CALLED FIRST! AND ONLY ONCE!" (:11-24)
  int precision = DOUBLE;
  const char *p = getenv("SAPPORO_PRECISION");
  if (p && (!strcmp(p, "mixed") || !strcmp(p, "doublesingle") || !strcmp(p, "1")))
    precision = DOUBLESINGLE;
  if (grav6.open("linked-in kernels", list, ndev, SIXTH, precision) != 0) return;
  h2_zero.assign((size_t)grav6.get_n_pipes(), 0.0);
  opened = true;
}

void initialize() {
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
  initialize_special(how_many, dev_list);
  delete[] dev_list;
}

void set_j_particle(int add, double pos[3], double vel[3], double acc[3], double jrk[3],
                    double snp[3], double crk[3], double mass, double time, int id,
                    double eps2) {
  double k18[3] = {0, 0, 0};
  grav6.set_j_particle(add, id, time, 0.0, mass, k18, jrk, acc, vel, pos, snp, crk, eps2);
}

void predict_all(double time, int nj) {
  grav6.set_time(time);
  grav6.forcePrediction(nj);
}

void no_predict_all(double time, int nj) {
  (void)time;
  grav6.set_no_time();
  grav6.forcePrediction(nj);
}

void pick_up_predictor_2(int addr, int &id, double &mass, double &eps2, double pos[3],
                         double vel[3], double acc[3]) {
  double id_d = 0;
  grav6.retrieve_predicted_j_particle(addr, mass, id_d, eps2, pos, vel, acc);
  id = (int)id_d;
}

void calc_force_on_predictors(int ni, int nj, int ids[], double pos[][3], double vel[][3],
                              double acc[][3], double mass[], double eps2[],
                              double accNew[][3], double jrkNew[][3], double snpNew[][3],
                              double crkNew[][3], double phi[], int nnb[], double nnb_r2[]) {
  (void)mass;
  const int n_pipes = grav6.get_n_pipes();
  for (int j = 0; j < ni; j += n_pipes) {  // :179-200
    const int tempni = ni - j < n_pipes ? ni - j : n_pipes;
    const double eps2_t = eps2[0];
    grav6.startGravCalc(nj, tempni, &ids[j], &pos[j], &vel[j], &acc[j], nullptr, nullptr, eps2_t,
                        h2_zero.data(), &eps2[j]);
    grav6.getGravResults(nj, tempni, &ids[j], &pos[j], &vel[j], 0, h2_zero.data(), &accNew[j],
                         &jrkNew[j], &snpNew[j], &crkNew[j], &phi[j], &nnb[j], &nnb_r2[j], true);
  }
}

}  // extern "C"
