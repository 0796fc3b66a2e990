// GRAPE-5 C interface over one process-wide `sapporo` instance, as the
// reference's lib/interfaces/sapporoG5lib.cpp (declared in
// include/sapporo_g5.h).  Opened in GRAPE5 order: the kernels compute
// acceleration and potential only, over every pair including the self pair
// (kernels.cu:565 does not skip it for GRAPE5: zero force, -m/eps potential).
#include <limits.h>
#include <stdio.h>

#include <vector>

#include "../../include/sapporo_g5.h"
#include "../../include/sapporohostclass.h"

static sapporo grav5;
static int nj_to_use = -1;       // :31
static double eps_to_use = -1;   // :32
static std::vector<double> h2_zero;  // h2 = 0: no neighbour lists

static void reserve_i(int ni) {
  if ((int)h2_zero.size() < ni) h2_zero.assign((size_t)ni, 0.0);
}

static bool ready(const char *what) {
  if (eps_to_use < 0) {  // reference: message and exit(-1) (:132-136, :172-176)
    fprintf(stderr, "sapporo %s: eps not set with g5_set_eps_to_all; nothing computed\n", what);
    return false;
  }
  if (nj_to_use <= 0) {  // :178-182
    fprintf(stderr, "sapporo %s: nj not set with g5_set_n; nothing computed\n", what);
    return false;
  }
  return true;
}

extern "C" {

int g5_open_special(int ndev, int *list) {
  nj_to_use = -1;
  eps_to_use = -1;
  const int rc = grav5.open("linked-in kernels", list, ndev, GRAPE5, DOUBLESINGLE);
  if (rc == 0) reserve_i(grav5.get_n_pipes());
  return rc;
}

void g5_open(void) {
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
  g5_open_special(how_many, dev_list);
  delete[] dev_list;
}

void g5_close(void) { grav5.close(); }
int g5_get_number_of_pipelines(void) { return grav5.get_n_pipes(); }
void g5_set_n(int nj) { nj_to_use = nj; }
void g5_set_eps2_to_all(double eps2) { eps_to_use = eps2; }
void g5_set_eps_to_all(double eps) { eps_to_use = eps * eps; }

void g5_set_xmj(int addr, int nj, double xj[][3], double jmass[]) {
  double z[3] = {0, 0, 0};
  for (int i = addr; i < addr + nj; i++)  // :111-115: arrays indexed by address
    grav5.set_j_particle(i, i, 0.0, 0.0, jmass[i], z, z, z, z, xj[i], z, z, 0.0);
}

void g5_set_jp(int addr, int nj, double jmass[], double xj[][3]) {
  g5_set_xmj(addr, nj, xj, jmass);
}

void g5_set_xi(int ni, double xi[][3]) {
  if (!ready("g5_set_xi") || ni <= 0) return;
  reserve_i(ni);
  grav5.startGravCalc(nj_to_use, ni, nullptr, xi, nullptr, nullptr, nullptr, nullptr,
                      eps_to_use, h2_zero.data(), nullptr);
}

void g5_run(void) {}

void g5_get_force(int ni, double a[][3], double *phi) {
  if (!ready("g5_get_force") || ni <= 0) return;
  reserve_i(ni);
  grav5.getGravResults(nj_to_use, ni, nullptr, nullptr, nullptr, 0, nullptr, a, nullptr,
                       nullptr, nullptr, phi, nullptr, nullptr, false);
}

void g5_calculate_force_on_x(double xi[][3], double a[][3], double *phi, int ni) {
  if (!ready("g5_calculate_force_on_x")) return;
  const int n_pipes = grav5.get_n_pipes();
  reserve_i(n_pipes);
  for (int j = 0; j < ni; j += n_pipes) {  // :185-193
    const int tempni = ni - j < n_pipes ? ni - j : n_pipes;
    g5_set_xi(tempni, &xi[j]);
    g5_get_force(tempni, &a[j], &phi[j]);
  }
}

void g5_set_range(double xmin, double xmax, double mmin) {
  (void)xmin;
  (void)xmax;
  (void)mmin;
}

int g5_get_jmemsize(void) { return INT_MAX; }
int g5_get_number_of_real_pipelines(void) { return 1; }
int g5_get_pcibus_freq(void) { return 1; }

}  // extern "C"
