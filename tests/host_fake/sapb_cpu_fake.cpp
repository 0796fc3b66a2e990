// A CPU stand-in for the device side of include/sapporo_b200.h, for tests of
// the host logic of the `sapporo` class (sapporohostclass.cpp) without a GPU:
// the j split over devices, address mapping, j-memory growth, staging, and
// the combination of the devices' results.  Each "device" keeps its j in FP64
// host arrays and computes with the FP64 oracle (orc_predict, orc_force of
// oracle/sapporo_oracle.c).  Test infrastructure only; it implements just the
// entry points the class and its C binding call.
//
// Result records follow the library's layout: the nearest-neighbour distance
// is rounded to float as the kernels report it, 1e11 / -1 when there is none.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sapporo_b200.h"

extern "C" {
void orc_predict(int nj, double ti, int order, const double *t, const double *x,
                 const double *v, const double *a, const double *j, const double *s,
                 const double *c, double *px, double *pv, double *pa, int nthreads);
void orc_force(int order, int ni, const double *xi, const double *vi, const double *ai,
               const double *h2, const int *idi, int nj, const double *xj, const double *vj,
               const double *aj, const double *mj, const int *idj, double eps2, double *acc,
               double *jrk, double *snp, double *pot, int *nnb, double *ds2min,
               int *ngb_count, int *ngb_list, int ngb_cap, int nthreads);
}

struct sapb_dev {
  int device = 0, order = SAPB_FOURTH, prec = SAPB_DOUBLESINGLE, n_pipes = SAPB_NPIPES;
  int cap = 0;
  // stored j (FP64), [cap][3] vectors
  std::vector<double> t, m, x, v, a, j, s, c, eps;
  std::vector<int> id;
  // force records: predicted state, or the raw copy written by a push
  std::vector<double> px, pv, pa;
  std::vector<double> stage, istage, res;
  std::vector<int> cnt, lst;
  int last_ni = 0;
  std::string err;
};

namespace {
int g_pushes = 0;  // pushes over all devices (the test reads it through fake_sapb_pushes)
std::vector<sapb_dev *> g_open;  // handles open now, in the order they were opened

int ndevices() {
  const char *e = getenv("FAKE_SAPB_DEVICES");
  return e ? atoi(e) : 4;
}
int jstride(int order) { return order >= SAPB_SIXTH ? 22 : 16; }
int istride(int order) { return order >= SAPB_SIXTH ? 12 : 8; }
int fail(sapb_dev *d, int rc, const char *msg) {
  if (d) d->err = msg;
  return rc;
}
void grow(sapb_dev *d, int n) {
  if (n <= d->cap) return;
  d->cap = n;
  const size_t n3 = (size_t)n * 3;
  for (auto *p : {&d->x, &d->v, &d->a, &d->j, &d->s, &d->c, &d->px, &d->pv, &d->pa})
    p->resize(n3, 0.0);
  for (auto *p : {&d->t, &d->m, &d->eps}) p->resize((size_t)n, 0.0);
  d->id.resize((size_t)n, -1);
}
void predict(sapb_dev *d, int first, int n, double ti, double *px, double *pv, double *pa) {
  const size_t o = (size_t)first * 3;
  orc_predict(n, ti, d->order, d->t.data() + first, d->x.data() + o, d->v.data() + o,
              d->a.data() + o, d->j.data() + o, d->s.data() + o, d->c.data() + o, px, pv,
              pa, 1);
}
}  // namespace

extern "C" {

int fake_sapb_pushes(void) { return g_pushes; }

// Device ids of the handles open now (up to max of them); returns their number.
int fake_sapb_open_devices(int *ids, int max) {
  const int n = (int)g_open.size();
  for (int k = 0; k < n && k < max; k++) ids[k] = g_open[k]->device;
  return n;
}

const char *sapb_error_string(int code) {
  switch (code) {
    case SAPB_OK: return "ok";
    case SAPB_EINVAL: return "invalid argument";
    case SAPB_ENOMEM: return "out of memory";
    case SAPB_ENODEV: return "no device";
    default: return "error";
  }
}
const char *sapb_last_error(const sapb_dev *d) { return d ? d->err.c_str() : ""; }

int sapb_device_count(int *count) {
  *count = ndevices();
  return SAPB_OK;
}

int sapb_open(sapb_dev **out, int device, int order, int precision, int n_pipes,
              int nj_reserve) {
  if (!out || device < 0 || device >= ndevices()) return SAPB_ENODEV;
  sapb_dev *d = new sapb_dev();
  d->device = device;
  d->order = order;
  d->prec = precision;
  d->n_pipes = n_pipes > 0 ? n_pipes : SAPB_NPIPES;
  grow(d, nj_reserve > 0 ? nj_reserve : 16384);
  g_open.push_back(d);
  *out = d;
  return SAPB_OK;
}

int sapb_close(sapb_dev *d) {
  g_open.erase(std::remove(g_open.begin(), g_open.end(), d), g_open.end());
  delete d;
  return SAPB_OK;
}

int sapb_info(const sapb_dev *d, int *order, int *precision, int *n_pipes, int *j_capacity,
              int *num_sms) {
  if (!d) return SAPB_EINVAL;
  if (order) *order = d->order;
  if (precision) *precision = d->prec;
  if (n_pipes) *n_pipes = d->n_pipes;
  if (j_capacity) *j_capacity = d->cap;
  if (num_sms) *num_sms = 148;
  return SAPB_OK;
}

int sapb_reserve_j(sapb_dev *d, int nj_capacity) {
  if (!d || nj_capacity < 0) return SAPB_EINVAL;
  grow(d, nj_capacity);
  return SAPB_OK;
}

int sapb_j_stage_stride(const sapb_dev *d) { return d ? jstride(d->order) : 0; }
int sapb_i_stage_stride(const sapb_dev *d) { return d ? istride(d->order) : 0; }

double *sapb_j_stage(sapb_dev *d, int n) {
  if (!d || n < 0) return nullptr;
  const size_t need = (size_t)n * jstride(d->order);
  if (d->stage.size() < need) d->stage.resize(need, 0.0);
  return d->stage.data();
}

int sapb_push_j(sapb_dev *d, int n) {
  if (!d || n < 0 || (size_t)n * jstride(d->order) > d->stage.size())
    return fail(d, SAPB_EINVAL, "push beyond the staging");
  const int ss = jstride(d->order);
  const bool six = d->order >= SAPB_SIXTH;
  for (int k = 0; k < n; k++) {
    const double *r = d->stage.data() + (size_t)k * ss;
    int32_t w[2];
    memcpy(w, &r[0], sizeof w);
    const int addr = w[0];
    if (addr < 0) return fail(d, SAPB_EINVAL, "negative address");
    if (addr >= d->cap) grow(d, std::max(addr + 1, (int)(d->cap * 1.1) + 1));
    d->id[addr] = w[1];
    d->t[addr] = r[1];
    d->m[addr] = r[2];
    d->eps[addr] = r[15];
    for (int q = 0; q < 3; q++) {
      const size_t o = (size_t)addr * 3 + q;
      d->x[o] = r[3 + q];
      d->v[o] = r[6 + q];
      d->a[o] = r[9 + q];
      d->j[o] = r[12 + q];
      d->s[o] = six ? r[16 + q] : 0.0;
      d->c[o] = six ? r[19 + q] : 0.0;
      d->px[o] = d->x[o];
      d->pv[o] = d->v[o];
      d->pa[o] = d->a[o];
    }
  }
  if (n > 0) g_pushes++;
  return SAPB_OK;
}

int sapb_predict(sapb_dev *d, int nj, double ti) {
  if (!d || nj < 0 || nj > d->cap) return fail(d, SAPB_EINVAL, "predict beyond capacity");
  predict(d, 0, nj, ti, d->px.data(), d->pv.data(), d->pa.data());
  return SAPB_OK;
}

double *sapb_i_stage(sapb_dev *d, int ni) {
  if (!d || ni < 0) return nullptr;
  const size_t need = (size_t)std::max(ni, 1) * istride(d->order);
  if (d->istage.size() < need) d->istage.resize(need, 0.0);
  return d->istage.data();
}

int sapb_force(sapb_dev *d, int nj, int ni, double eps2, double ti, int flags) {
  if (!d || nj < 0 || ni < 0 || nj > d->cap || ni > d->n_pipes)
    return fail(d, SAPB_EINVAL, "bad force call");
  if (flags & SAPB_F_PREDICT) sapb_predict(d, nj, ti);
  const int is = istride(d->order);
  const bool six = d->order >= SAPB_SIXTH;
  std::vector<double> xi((size_t)ni * 3), vi((size_t)ni * 3), ai((size_t)ni * 3), h2(ni);
  std::vector<int> idi(ni);
  for (int i = 0; i < ni; i++) {
    const double *r = d->istage.data() + (size_t)i * is;
    for (int q = 0; q < 3; q++) {
      xi[3 * i + q] = r[q];
      vi[3 * i + q] = r[4 + q];
      ai[3 * i + q] = six ? r[8 + q] : 0.0;
    }
    h2[i] = r[3];
    int32_t w[2];
    memcpy(w, &r[7], sizeof w);
    idi[i] = w[0];
  }
  std::vector<double> acc((size_t)ni * 3), jrk((size_t)ni * 3), snp((size_t)ni * 3), pot(ni),
      ds2(ni);
  std::vector<int> nnb(ni);
  d->cnt.assign((size_t)ni, 0);
  d->lst.assign((size_t)ni * SAPB_NGB_PB, 0);
  orc_force(d->order, ni, xi.data(), vi.data(), ai.data(), h2.data(), idi.data(), nj,
            d->px.data(), d->pv.data(), d->pa.data(), d->m.data(), d->id.data(), eps2,
            acc.data(), jrk.data(), snp.data(), pot.data(), nnb.data(), ds2.data(),
            d->cnt.data(), (flags & SAPB_F_NGB_LIST) ? d->lst.data() : nullptr, SAPB_NGB_PB,
            1);
  d->res.assign((size_t)std::max(ni, 1) * SAPB_RES_STRIDE, 0.0);
  for (int i = 0; i < ni; i++) {
    double *r = d->res.data() + (size_t)i * SAPB_RES_STRIDE;
    for (int q = 0; q < 3; q++) {
      r[q] = acc[3 * i + q];
      r[4 + q] = jrk[3 * i + q];
      r[7 + q] = six ? snp[3 * i + q] : 0.0;
    }
    r[3] = pot[i];
    r[10] = nnb[i] < 0 ? 1.0e11 : (double)(float)ds2[i];
    r[11] = nnb[i];
  }
  d->last_ni = ni;
  return SAPB_OK;
}

int sapb_results(sapb_dev *d, const double **results, int *ni) {
  if (!d) return SAPB_EINVAL;
  if (results) *results = d->res.data();
  if (ni) *ni = d->last_ni;
  return SAPB_OK;
}

int sapb_ngb_fetch(sapb_dev *d, int *counts, int *lists, int ni) {
  if (!d || ni < 0 || ni > d->last_ni) return fail(d, SAPB_EINVAL, "bad ni");
  if (counts) memcpy(counts, d->cnt.data(), sizeof(int) * (size_t)ni);
  if (lists) memcpy(lists, d->lst.data(), sizeof(int) * (size_t)ni * SAPB_NGB_PB);
  return SAPB_OK;
}

int sapb_read_j(sapb_dev *d, int first, int n, double ti, int do_predict, double *out) {
  if (!d || first < 0 || n < 0 || first + n > d->cap) return fail(d, SAPB_EINVAL, "bad read");
  std::vector<double> px((size_t)n * 3), pv((size_t)n * 3), pa((size_t)n * 3);
  if (do_predict) predict(d, first, n, ti, px.data(), pv.data(), pa.data());
  for (int k = 0; k < n; k++) {
    const int g = first + k;
    double *o = out + (size_t)k * 24;
    for (int q = 0; q < 3; q++) {
      const size_t s3 = (size_t)g * 3 + q;
      o[q] = d->x[s3];
      o[4 + q] = d->v[s3];
      o[8 + q] = d->a[s3];
      o[11 + q] = d->j[s3];
      o[14 + q] = do_predict ? px[3 * k + q] : d->x[s3];
      o[17 + q] = do_predict ? pv[3 * k + q] : d->v[s3];
      o[20 + q] = do_predict ? pa[3 * k + q] : d->a[s3];
    }
    o[3] = d->m[g];
    o[7] = d->eps[g];
    o[23] = d->id[g];
  }
  return SAPB_OK;
}

}  // extern "C"
