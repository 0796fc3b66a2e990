// C binding of the sapporo class; declared in include/sapporo_c.h.
#include <new>
#include <vector>

#include "../../include/sapporo_b200.h"
#include "../../include/sapporo_c.h"
#include "../../include/sapporohostclass.h"

struct sapporo_c {
  sapporo obj;
};

namespace {
typedef double (*v3)[3];
inline v3 as3(const double *p) { return reinterpret_cast<v3>(const_cast<double *>(p)); }
}  // namespace

extern "C" {

sapporo_c *sapporo_c_new(void) { return new (std::nothrow) sapporo_c(); }
void sapporo_c_delete(sapporo_c *s) { delete s; }

int sapporo_c_open(sapporo_c *s, int device, int order, int precision) {
  if (!s) return SAPB_EINVAL;
  int list[1] = {device};
  return s->obj.open("linked-in kernels", list, 1, order, precision);
}
int sapporo_c_open_devices(sapporo_c *s, int ndev, const int *devices, int order, int precision) {
  if (!s || (ndev > 0 && !devices)) return SAPB_EINVAL;
  return s->obj.open("linked-in kernels", const_cast<int *>(devices), ndev, order, precision);
}
int sapporo_c_close(sapporo_c *s) { return s ? s->obj.close() : SAPB_EINVAL; }
int sapporo_c_get_n_pipes(sapporo_c *s) { return s ? s->obj.get_n_pipes() : 0; }
int sapporo_c_set_time(sapporo_c *s, double ti) { return s ? s->obj.set_time(ti) : SAPB_EINVAL; }
int sapporo_c_set_no_time(sapporo_c *s) { return s ? s->obj.set_no_time() : SAPB_EINVAL; }

int sapporo_c_set_j_particles(sapporo_c *s, int n, const int *address, const int *id,
                              const double *t, const double *mass, const double *x,
                              const double *v, const double *a, const double *jrk,
                              const double *snp, const double *crk, const double *eps) {
  if (!s || n < 0) return SAPB_EINVAL;
  return s->obj.set_j_particles(n, address, id, t, mass, x, v, a, jrk, snp, crk, eps);
}

int sapporo_c_start(sapporo_c *s, int nj, int ni, const int *id, const double *xi,
                    const double *vi, const double *ai, double eps2, const double *h2) {
  if (!s) return SAPB_EINVAL;
  std::vector<double> zeros;
  if (!ai) zeros.assign((size_t)3 * (ni > 0 ? ni : 1), 0.0);
  s->obj.startGravCalc(nj, ni, const_cast<int *>(id), as3(xi), as3(vi),
                       ai ? as3(ai) : as3(zeros.data()), nullptr, nullptr, eps2,
                       const_cast<double *>(h2), nullptr);
  return s->obj.last_status;
}

int sapporo_c_results(sapporo_c *s, int nj, int ni, double *acc, double *jrk, double *snp,
                      double *pot, int *nnb, double *dsmin, int ngb) {
  if (!s) return SAPB_EINVAL;
  std::vector<double> jtmp, stmp;
  std::vector<int> ntmp;
  if (!jrk) {
    jtmp.assign((size_t)3 * (ni > 0 ? ni : 1), 0.0);
    jrk = jtmp.data();
  }
  if (!snp) {
    stmp.assign((size_t)3 * (ni > 0 ? ni : 1), 0.0);
    snp = stmp.data();
  }
  if (ngb && !nnb) {
    ntmp.assign((size_t)(ni > 0 ? ni : 1), 0);
    nnb = ntmp.data();
  }
  return s->obj.getGravResults(nj, ni, nullptr, nullptr, nullptr, 0.0, nullptr, as3(acc),
                               as3(jrk), as3(snp), nullptr, pot, nnb, dsmin, ngb != 0);
}

int sapporo_c_force_prediction(sapporo_c *s, int nj) {
  if (!s) return SAPB_EINVAL;
  s->obj.forcePrediction(nj);
  return s->obj.last_status;
}
int sapporo_c_read_ngb_list(sapporo_c *s) { return s ? s->obj.read_ngb_list(0) : SAPB_EINVAL; }
int sapporo_c_get_ngb_list(sapporo_c *s, int ipipe, int maxlength, int *nblen, int *nbl) {
  if (!s || !nblen) return SAPB_EINVAL;
  return s->obj.get_ngb_list(0, ipipe, maxlength, *nblen, nbl);
}
int sapporo_c_ngb_list_copied(sapporo_c *s) { return s ? s->obj.ngb_list_copied() : 0; }

int sapporo_c_retrieve_predicted(sapporo_c *s, int addr, double *out) {
  if (!s || !out) return SAPB_EINVAL;
  double mass = 0, id = 0, eps2 = 0;
  s->obj.retrieve_predicted_j_particle(addr, mass, id, eps2, out + 3, out + 6, out + 9);
  out[0] = mass;
  out[1] = id;
  out[2] = eps2;
  return s->obj.last_status;
}

int sapporo_c_retrieve_state(sapporo_c *s, int addr, double *out) {
  if (!s || !out) return SAPB_EINVAL;
  double mass = 0, id = 0, eps2 = 0;
  s->obj.retrieve_j_particle_state(addr, mass, id, eps2, out + 3, out + 6, out + 9, out + 12,
                                   out + 15, out + 18, out + 21);
  out[0] = mass;
  out[1] = id;
  out[2] = eps2;
  return s->obj.last_status;
}

int sapporo_c_last_status(sapporo_c *s) { return s ? s->obj.last_status : SAPB_EINVAL; }
struct sapb_dev *sapporo_c_device(sapporo_c *s) { return s ? s->obj.device_handle() : nullptr; }
int sapporo_c_n_devices(sapporo_c *s) { return s ? s->obj.n_devices() : 0; }
struct sapb_dev *sapporo_c_device_at(sapporo_c *s, int k) {
  return s ? s->obj.device_handle(k) : nullptr;
}

}  // extern "C"
