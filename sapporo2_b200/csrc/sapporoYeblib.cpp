// The 6th-order interface of lib/interfaces/sapporoYeblib.cpp over one
// process-wide `sapporo` instance (6th order, all-FP64 kernels unless
// SAPPORO_PRECISION=mixed).  Built into libsapporoyeb_b200.so: its names are
// those of the 6th-order C interface with other arguments.  Declared in
// include/sapporo_yebisu.h.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/sapporo_yebisu.h"
#include "../../include/sapporohostclass.h"

static sapporo grav_yeb;
static bool opened = false;
// per-chunk host arrays of the reference (:163-178)
static std::vector<double> pos_i, vel_i, acc_i, jrk_i, snp_i, crk_i, eps2_i, h2_i, dsmin_i, pot_i;
static std::vector<int> id_i, nnb_i;

typedef double DB3[3];
static DB3 *v3(std::vector<double> &v) { return reinterpret_cast<DB3 *>(v.data()); }

extern "C" {

void initialize_special(int ndev, int *list) {
  if (opened) return;  // the reference opens once (:185-190)
  int precision = DOUBLE;
  const char *p = getenv("SAPPORO_PRECISION");
  if (p && (!strcmp(p, "mixed") || !strcmp(p, "doublesingle") || !strcmp(p, "1")))
    precision = DOUBLESINGLE;
  if (grav_yeb.open("linked-in kernels", list, ndev, SIXTH, precision) != 0) return;
  const size_t n = (size_t)grav_yeb.get_n_pipes();
  for (auto *v : {&pos_i, &vel_i, &acc_i, &jrk_i, &snp_i, &crk_i}) v->assign(3 * n, 0.0);
  for (auto *v : {&eps2_i, &h2_i, &dsmin_i, &pot_i}) v->assign(n, 0.0);
  id_i.assign(n, 0);
  nnb_i.assign(n, 0);
  opened = true;
}

void initialize(int n) {
  (void)n;
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

void set_jp_2(int add, double pos[3], double vel[3], double acc[3], double jrk[3],
              double snp[3], double crk[3], double mass, double time, int id, double eps2) {
  double k18[3] = {0, 0, 0};
  grav_yeb.set_j_particle(add, id, time, 0.0, mass, k18, jrk, acc, vel, pos, snp, crk, eps2);
}

void predict_all(double time, int nj) {
  grav_yeb.set_time(time);
  grav_yeb.forcePrediction(nj);
}

void no_predict_all(double time, int nj) {
  (void)time;
  grav_yeb.set_no_time();
  grav_yeb.forcePrediction(nj);
}

void pick_up_predictor_2(int addr, sapporo_yeb_predictor *pred) {
  grav_yeb.retrieve_predicted_j_particle(addr, pred->mass, pred->id, pred->eps2, pred->pos,
                                         pred->vel, pred->acc);
}

void calc_force_on_predictors(int ni, sapporo_yeb_predictor pred[], sapporo_yeb_force force[],
                              int nj) {
  if (!opened || ni <= 0) return;
  const int n_pipes = grav_yeb.get_n_pipes();
  for (int j = 0; j < ni; j += n_pipes) {  // :305-379
    const int tempni = ni - j < n_pipes ? ni - j : n_pipes;
    for (int i = 0; i < tempni; i++) {
      const sapporo_yeb_predictor &p = pred[j + i];
      for (int d = 0; d < 3; d++) {
        pos_i[3 * i + d] = p.pos[d];
        vel_i[3 * i + d] = p.vel[d];
        acc_i[3 * i + d] = p.acc[d];
      }
      id_i[i] = (int)p.id;
      eps2_i[i] = p.eps2;
      h2_i[i] = 0.0;  // lists off, nearest neighbour on
    }
    const double eps2 = pred[0].eps2;  // :332
    grav_yeb.startGravCalc(nj, tempni, id_i.data(), v3(pos_i), v3(vel_i), v3(acc_i), nullptr,
                           nullptr, eps2, h2_i.data(), eps2_i.data());
    grav_yeb.getGravResults(nj, tempni, id_i.data(), v3(pos_i), v3(vel_i), 0, h2_i.data(),
                            v3(acc_i), v3(jrk_i), v3(snp_i), v3(crk_i), pot_i.data(),
                            nnb_i.data(), dsmin_i.data(), true);
    for (int i = 0; i < tempni; i++) {
      sapporo_yeb_force &f = force[j + i];
      for (int d = 0; d < 3; d++) {
        f.acc[d] = acc_i[3 * i + d];
        f.jrk[d] = jrk_i[3 * i + d];
        f.snp[d] = snp_i[3 * i + d];
      }
      f.phi = -pot_i[i];  // :366
      f.nnb_id = nnb_i[i];
      f.nnb_r2 = (float)dsmin_i[i];
    }
  }
}

void calc_force_on_predictors_epsj(int ni, sapporo_yeb_predictor pred[],
                                   sapporo_yeb_force force[], int nj) {
  (void)ni;
  (void)pred;
  (void)force;
  (void)nj;
  fprintf(stderr,
          "sapporo calc_force_on_predictors_epsj: individual j softening is not implemented "
          "(nor in the reference); nothing computed\n");
}

}  // extern "C"
