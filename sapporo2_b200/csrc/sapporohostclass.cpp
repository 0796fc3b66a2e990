// The `sapporo` class on top of the sapb_* C ABI, one device handle per
// device given to open.
//
// Behaviour follows lib/src/sapporohostclass.cpp of the reference:
//   - set_j_particle stages into host memory only; j travel to the GPU at the
//     next startGravCalc / forcePrediction (:434-558, :669-676);
//   - set_time makes the next force call predict all j to t_i (:405-415);
//   - startGravCalc returns after queueing the work, getGravResults blocks
//     (README.extended:154-171);
//   - nearest neighbour: taken only when ds2 < 1e10, nnbindex zeroed first,
//     dsmin_i written only when taken (:722-775);
//   - neighbour lists: overflow when a count reaches NGB_PB (:804-835),
//     get_ngb_list copies and sorts (:837-880);
//   - several devices: j address a on device a % G at a / G (:473-474), the
//     first nj addresses split as nj / G plus one on the first nj % G devices
//     (:687-691), the i broadcast, forces and potentials summed over the
//     devices in device order, the nearest neighbour the closest over the
//     devices, lists concatenated in device order (:749-799, :837-880).
// Deviations: fatal exits become error returns; get_ngb_list never copies
// more than NGB_PB entries of a device and flags overflow when a device's
// count reaches NGB_PB; of nearest neighbours at the same distance on two
// devices the lower id is taken (the rule inside one device), so the result
// does not depend on the number of devices.
#include "../../include/sapporohostclass.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/sapporo_b200.h"

namespace {
bool verbose() {
  static int v = -1;
  if (v < 0) {
    const char *e = getenv("SAPPORO_VERBOSE");
    v = (e && *e && *e != '0') ? 1 : 0;
  }
  return v == 1;
}
void report(const char *what, int rc, sapb_dev *d) {
  fprintf(stderr, "sapporo: %s failed: %s (%s)\n", what, sapb_error_string(rc), sapb_last_error(d));
}
inline void put_int_pair(double *slot, int lo, int hi) {
  int32_t w[2] = {lo, hi};
  memcpy(slot, w, sizeof(double));
}
}  // namespace

sapporo::sapporo()
    : dev_(nullptr),
      n_pipes(NPIPES),
      nj_max(0),
      integrationOrder(FOURTH),
      integrationPrecision(DOUBLESINGLE),
      EPS2(0.0),
      t_i(0.0),
      predict(false),
      nj_updated(false),
      predJOnHost(false),
      jcache_n_(0),
      dev_ni(0),
      nj_last_(0),
      ngb_fetched_(false),
      ngb_copied_(0),
      last_status(0) {}

sapporo::~sapporo() { close(); }

// lib/src/sapporohostclass.cpp:90-163: |nprocs| devices (all visible ones
// when 0); ids from `devices` when nprocs > 0, else 0, 1, ... (the reference
// lets the driver choose when nprocs < 0).  A device id may repeat: each
// entry gets its own handle, stream and memory.
int sapporo::open(std::string kernelFile, int *devices, int nprocs, int order, int precision) {
  (void)kernelFile;  // kernels are linked into the library
  if (!devs_.empty()) close();
  integrationOrder = order;
  integrationPrecision = precision;
  int visible = 0;
  if (sapb_device_count(&visible) != SAPB_OK) visible = 0;
  int G = nprocs < 0 ? -nprocs : nprocs;
  if (G == 0) G = std::max(visible, 1);
  std::vector<int> ids((size_t)G);
  for (int k = 0; k < G; k++)
    ids[k] = (nprocs > 0 && devices) ? devices[k] : (visible > 0 ? k % visible : k);
  const char *np = getenv("SAPPORO_NPIPES");
  const int pipes = np ? atoi(np) : NPIPES;
  for (int k = 0; k < G; k++) {
    sapb_dev *d = nullptr;
    const int rc = sapb_open(&d, ids[k], order, precision, pipes, 16384);
    if (rc != SAPB_OK) {
      fprintf(stderr, "sapporo: device %d (entry %d of %d): ", ids[k], k, G);
      report("open", rc, nullptr);
      close();
      return last_status = rc;
    }
    devs_.push_back(d);
  }
  last_status = 0;
  dev_ = devs_[0];
  n_pipes = INT_MAX;
  for (sapb_dev *d : devs_) {
    int p = 0;
    sapb_info(d, nullptr, nullptr, &p, nullptr, nullptr);
    n_pipes = std::min(n_pipes, p);
  }
  nj_max = 16384;  // lib/src/sapporohostclass.cpp:161-162
  stage_slot_.assign(nj_max, -1);
  pred_time_.assign(nj_max, NAN);
  staged_addr_.assign((size_t)G, std::vector<int>());
  dev_nj_.assign((size_t)G, 0);
  ngb_count_h_.assign((size_t)G, std::vector<int>());
  ngb_list_h_.assign((size_t)G, std::vector<int>());
  predict = false;
  nj_updated = false;
  predJOnHost = false;
  ngb_fetched_ = false;
  dev_ni = 0;
  nj_last_ = 0;
  if (verbose())
    for (int k = 0; k < G; k++)
      fprintf(stderr, "sapporo: opened device %d (entry %d of %d), order %d, precision %d, %d pipes\n",
              ids[k], k, G, order, precision, n_pipes);
  return 0;
}

int sapporo::close() {
  for (sapb_dev *d : devs_) sapb_close(d);
  devs_.clear();
  dev_ = nullptr;
  return 0;
}

int sapporo::nj_on(int g, int nj) const {
  // lib/src/sapporohostclass.cpp:687-691
  const int G = ndev();
  return nj / G + (g < nj % G ? 1 : 0);
}

int sapporo::get_n_pipes() { return n_pipes; }

int sapporo::set_time(double time) {
  t_i = time;
  predict = true;
  predJOnHost = false;
  return 0;
}

int sapporo::set_no_time() {
  predict = false;
  predJOnHost = false;
  return 0;
}

void sapporo::increase_jMemory() {
  // lib/src/sapporohostclass.cpp:560-583: +10 %, rounded up to a multiple of
  // the device count; each device holds nj_max / G
  const int G = std::max(ndev(), 1);
  int temp = (int)(nj_max * 1.1);
  temp = (temp / G + 1) * G;
  nj_max = temp;
  stage_slot_.resize(nj_max, -1);
  pred_time_.resize(nj_max, NAN);
  for (sapb_dev *d : devs_) {
    const int rc = sapb_reserve_j(d, nj_max / G);
    if (rc) report("reserve_j", rc, d);
  }
}

// The staging record of `address` on its device (a new slot when the address
// is not staged yet), with the local address and id to be written by the
// caller; null with rc set when the staging cannot grow.
double *sapporo::stage_record(int address, int &rc) {
  const int G = ndev();
  const int g = address % G;
  int slot = stage_slot_[address];
  if (slot < 0) {
    slot = (int)staged_addr_[g].size();
    stage_slot_[address] = slot;
    staged_addr_[g].push_back(address);
  }
  double *base = sapb_j_stage(devs_[g], (int)staged_addr_[g].size());
  if (!base) {
    rc = SAPB_ENOMEM;
    report("j staging", rc, devs_[g]);
    return nullptr;
  }
  rc = 0;
  return base + (size_t)slot * sapb_j_stage_stride(devs_[g]);
}

int sapporo::set_j_particle(int address, int id, double tj, double dtj, double mass,
                            double k18[3], double j6[3], double a2[3], double v[3], double x[3],
                            double snp[3], double crk[3], double eps) {
  (void)k18;
  (void)dtj;
  if (devs_.empty()) return last_status = SAPB_EINVAL;
  if (address < 0) {
    fprintf(stderr, "sapporo::set_j_particle: negative address %d\n", address);
    return last_status = SAPB_EINVAL;
  }
  predJOnHost = false;
  nj_updated = true;
  if (address >= nj_max) {
    increase_jMemory();
    if (address >= nj_max) {
      // reference: exit(-1) (lib/src/sapporohostclass.cpp:463-466)
      fprintf(stderr,
              "sapporo::set_j_particle: address %d beyond %d after growing; send particles in "
              "address order\n",
              address, nj_max);
      return last_status = SAPB_EINVAL;
    }
  }
  int rc = 0;
  double *r = stage_record(address, rc);
  if (!r) return last_status = rc;
  put_int_pair(&r[0], address / ndev(), id);
  r[1] = tj;
  r[2] = mass;
  for (int d = 0; d < 3; d++) {
    r[3 + d] = x[d];
    r[6 + d] = v ? v[d] : 0.0;
    r[9 + d] = a2 ? a2[d] : 0.0;
    r[12 + d] = j6 ? j6[d] : 0.0;
  }
  r[15] = eps;
  if (integrationOrder > FOURTH) {
    for (int d = 0; d < 3; d++) {
      r[16 + d] = snp ? snp[d] : 0.0;
      r[19 + d] = crk ? crk[d] : 0.0;
    }
  }
  return 0;
}

// fn(begin, end) over [0, n): chunks of at least kFillChunk on up to 16
// threads (a bulk j upload of 2^20 records packs 185 MB); a thread that cannot
// be started runs its chunk inline.
static const int kFillChunk = 32768;
template <class F>
static void parallel_chunks(int n, F fn) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::max(1, std::min((int)std::min(hw, 16u), n / kFillChunk));
  if (nt <= 1) {
    fn(0, n);
    return;
  }
  const int step = (n + nt - 1) / nt;
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 1; t < nt; t++) {
    const int b = t * step, e = std::min(n, b + step);
    if (b >= e) continue;
    try {
      th.emplace_back(fn, b, e);
    } catch (const std::system_error &) {
      fn(b, e);
    }
  }
  fn(0, std::min(n, step));
  for (auto &x : th) x.join();
}

int sapporo::set_j_particles(int n, const int *address, const int *id, const double *t,
                             const double *mass, const double *x, const double *v,
                             const double *a, const double *jrk, const double *snp,
                             const double *crk, const double *eps) {
  if (devs_.empty() || n < 0 || (n && (!address || !id || !mass || !x)))
    return last_status = SAPB_EINVAL;
  if (n == 0) return 0;
  // the address rules of set_j_particle, in the given order; on a bad address
  // nothing of this call is staged
  for (int k = 0; k < n; k++) {
    const int addr = address[k];
    if (addr < 0) {
      fprintf(stderr, "sapporo::set_j_particles: negative address %d\n", addr);
      return last_status = SAPB_EINVAL;
    }
    if (addr >= nj_max) {
      increase_jMemory();
      if (addr >= nj_max) {
        fprintf(stderr,
                "sapporo::set_j_particles: address %d beyond %d after growing; send particles "
                "in address order\n",
                addr, nj_max);
        return last_status = SAPB_EINVAL;
      }
    }
  }
  predJOnHost = false;
  nj_updated = true;
  // slots, then one staging reservation per device and a tight fill.  An
  // address named twice in one call keeps its later entry, as with
  // set_j_particle one by one; the fill of such a call runs on one thread
  // (on several, two threads would write the same record)
  const int G = ndev();
  std::vector<int> slots((size_t)n);
  std::vector<unsigned char> seen;
  if (n >= 2 * kFillChunk) seen.assign((size_t)nj_max, 0);  // smaller fills run on one thread
  bool repeats = false;
  for (int k = 0; k < n; k++) {
    const int addr = address[k];
    const int g = G == 1 ? 0 : addr % G;
    int slot = stage_slot_[addr];
    if (slot < 0) {
      slot = (int)staged_addr_[g].size();
      stage_slot_[addr] = slot;
      staged_addr_[g].push_back(addr);
    }
    slots[k] = slot;
    if (!seen.empty()) {
      repeats |= seen[addr] != 0;
      seen[addr] = 1;
    }
  }
  std::vector<double *> bases((size_t)G, nullptr);
  for (int g = 0; g < G; g++) {
    if (staged_addr_[g].empty()) continue;
    bases[g] = sapb_j_stage(devs_[g], (int)staged_addr_[g].size());
    if (!bases[g]) {
      report("j staging", SAPB_ENOMEM, devs_[g]);
      return last_status = SAPB_ENOMEM;
    }
  }
  const int ss = sapb_j_stage_stride(devs_[0]);
  const bool six = integrationOrder > FOURTH;
  const int *sl = slots.data();
  double *const *bs = bases.data();
  auto fill = [=](int k0, int k1) {
    for (int k = k0; k < k1; k++) {
      const int addr = address[k];
      double *r = (G == 1 ? bs[0] : bs[addr % G]) + (size_t)sl[k] * ss;
      put_int_pair(&r[0], G == 1 ? addr : addr / G, id[k]);
      r[1] = t ? t[k] : 0.0;
      r[2] = mass[k];
      for (int d = 0; d < 3; d++) {
        r[3 + d] = x[3 * k + d];
        r[6 + d] = v ? v[3 * k + d] : 0.0;
        r[9 + d] = a ? a[3 * k + d] : 0.0;
        r[12 + d] = jrk ? jrk[3 * k + d] : 0.0;
      }
      r[15] = eps ? eps[k] : 0.0;
      if (six)
        for (int d = 0; d < 3; d++) {
          r[16 + d] = snp ? snp[3 * k + d] : 0.0;
          r[19 + d] = crk ? crk[3 * k + d] : 0.0;
        }
    }
  };
  if (repeats)
    fill(0, n);
  else
    parallel_chunks(n, fill);
  return 0;
}

int sapporo::push_staged() {
  if (!nj_updated) return 0;
  int rc = 0;
  for (int g = 0; g < ndev(); g++) {
    std::vector<int> &staged = staged_addr_[g];
    if (staged.empty()) continue;
    const int r = sapb_push_j(devs_[g], (int)staged.size());
    for (int a : staged) {
      stage_slot_[a] = -1;
      pred_time_[a] = NAN;
    }
    staged.clear();
    if (r) {
      report("push_j", r, devs_[g]);
      if (!rc) rc = r;
    }
  }
  nj_updated = false;
  return rc;
}

void sapporo::send_j_particles_to_device() {
  if (!devs_.empty()) last_status = push_staged();
}

void sapporo::send_i_particles_to_device(int i) {
  (void)i;  // i records are uploaded together with the force launch
}

void sapporo::startGravCalc(int nj, int ni, int id[], double xi[][3], double vi[][3],
                            double a[][3], double j6old[][3], double phiold[3], double eps2,
                            double h2[], double eps2_i[]) {
  (void)j6old;
  (void)phiold;
  (void)eps2_i;  // stored by the reference (vel_i.w) but unused by its kernels
  last_status = 0;
  if (ni == 0 || nj == 0) return;
  if (devs_.empty() || ni < 0 || nj < 0) {
    last_status = SAPB_EINVAL;
    return;
  }
  EPS2 = eps2;
  double *rec = sapb_i_stage(dev_, ni);
  if (!rec) {
    last_status = SAPB_ENOMEM;
    report("i staging", last_status, dev_);
    return;
  }
  const int is = sapb_i_stage_stride(dev_);
  for (int i = 0; i < ni; i++) {
    double *r = rec + (size_t)i * is;
    r[0] = xi[i][0];
    r[1] = xi[i][1];
    r[2] = xi[i][2];
    r[3] = h2 ? h2[i] : 0.0;
    // GRAPE-5 callers pass no velocities and no ids (sapporohostclass.cpp:617-633)
    r[4] = vi ? vi[i][0] : 0.0;
    r[5] = vi ? vi[i][1] : 0.0;
    r[6] = vi ? vi[i][2] : 0.0;
    put_int_pair(&r[7], id ? id[i] : INT_MIN, 0);
    if (integrationOrder > FOURTH) {
      r[8] = a[i][0];
      r[9] = a[i][1];
      r[10] = a[i][2];
      r[11] = 0.0;
    }
  }
  // the same i on every device (lib/src/sapporohostclass.cpp:651-660)
  int rc = 0;
  for (int g = 1; g < ndev() && !rc; g++) {
    double *copy = sapb_i_stage(devs_[g], ni);
    if (!copy) {
      rc = SAPB_ENOMEM;
      report("i staging", rc, devs_[g]);
    } else {
      memcpy(copy, rec, sizeof(double) * (size_t)ni * is);
    }
  }
  if (!rc) rc = push_staged();
  int flags = SAPB_F_NGB_LIST;
  if (predict) flags |= SAPB_F_PREDICT;
  for (int g = 0; g < ndev(); g++) dev_nj_[g] = 0;
  for (int g = 0; g < ndev() && !rc; g++) {
    const int njg = nj_on(g, nj);
    if (njg == 0) continue;  // no j on this device: it adds nothing
    rc = sapb_force(devs_[g], njg, ni, eps2, t_i, flags);
    if (rc) {
      report("startGravCalc", rc, devs_[g]);
    } else {
      dev_nj_[g] = njg;
    }
  }
  if (!rc && predict)
    for (int k = 0; k < nj && k < (int)pred_time_.size(); k++) pred_time_[k] = t_i;
  last_status = rc;
  dev_ni = ni;
  nj_last_ = nj;
  ngb_fetched_ = false;
  predict = false;
  predJOnHost = false;
}

int sapporo::getGravResults(int nj, int ni, int index[], double xi[][3], double vi[][3],
                            double eps2, double h2[], double acc[][3], double jerk[][3],
                            double snp[][3], double crk[][3], double pot[], int nnbindex[],
                            double dsmin_i[], bool ngb) {
  (void)index; (void)xi; (void)vi; (void)eps2; (void)h2;
  if (ni == 0 || nj == 0) return 0;
  for (int i = 0; i < ni; i++) {
    pot[i] = acc[i][0] = acc[i][1] = acc[i][2] = 0;
    if (integrationOrder > GRAPE5) jerk[i][0] = jerk[i][1] = jerk[i][2] = 0;
    if (ngb) nnbindex[i] = 0;
    if (integrationOrder > FOURTH) {
      snp[i][0] = snp[i][1] = snp[i][2] = 0;
      if (crk) crk[i][0] = crk[i][1] = crk[i][2] = 0;
    }
  }
  if (devs_.empty()) return last_status = SAPB_EINVAL;
  if (last_status) return last_status;
  // nearest neighbour over the devices: ds2 < 1e10 (lib/src/sapporohostclass.cpp:732,
  // 767-774), the lower id at equal ds2
  std::vector<double> best_ds(ngb ? (size_t)ni : 0, 1.0e10);
  for (int g = 0; g < ndev(); g++) {
    if (dev_nj_[g] == 0) continue;
    const double *res = nullptr;
    int nres = 0;
    const int rc = sapb_results(devs_[g], &res, &nres);
    if (rc) {
      report("getGravResults", rc, devs_[g]);
      return last_status = rc;
    }
    const int n = std::min(ni, nres);
    for (int i = 0; i < n; i++) {
      const double *r = res + (size_t)i * SAPB_RES_STRIDE;
      acc[i][0] += r[0];
      acc[i][1] += r[1];
      acc[i][2] += r[2];
      pot[i] += r[3];
      if (integrationOrder > GRAPE5) {
        jerk[i][0] += r[4];
        jerk[i][1] += r[5];
        jerk[i][2] += r[6];
        if (ngb) {
          const double ds = r[10];
          const int id = (int)r[11];
          if (ds < best_ds[i] ||
              (ds == best_ds[i] && ds < 1.0e10 && (unsigned)id < (unsigned)nnbindex[i])) {
            best_ds[i] = ds;
            nnbindex[i] = id;
            if (dsmin_i) dsmin_i[i] = ds;
          }
        }
      }
      if (integrationOrder > FOURTH) {
        snp[i][0] += r[7];
        snp[i][1] += r[8];
        snp[i][2] += r[9];
      }
    }
  }
  return 0;
}

int sapporo::fetch_ngb_list_from_device(int) {
  if (devs_.empty()) return 0;
  const size_t n = (size_t)std::max(dev_ni, 1);
  for (int g = 0; g < ndev(); g++) {
    std::vector<int> &cnt = ngb_count_h_[g];
    std::vector<int> &lst = ngb_list_h_[g];
    cnt.assign(n, 0);
    lst.resize(n * NGB_PB);
    if (dev_nj_[g] == 0) continue;  // no j on this device: no neighbours
    const double *res = nullptr;
    sapb_results(devs_[g], &res, nullptr);  // the lists belong to the last force call
    const int rc = sapb_ngb_fetch(devs_[g], cnt.data(), lst.data(), dev_ni);
    if (rc) {
      report("ngb fetch", rc, devs_[g]);
      return 0;
    }
  }
  ngb_fetched_ = true;
  return dev_ni;
}

int sapporo::read_ngb_list(int cluster_id) {
  // lib/src/sapporohostclass.cpp:804-835: overflow when a device's count
  // reaches NGB_PB
  const int ni = fetch_ngb_list_from_device(cluster_id);
  bool overflow = false;
  for (int g = 0; g < ndev() && ni > 0; g++)
    for (int j = 0; j < ni; j++)
      if (ngb_count_h_[g][j] >= NGB_PB) overflow = true;
  return overflow;
}

int sapporo::get_ngb_list(int cluster_id, int ipipe, int maxlength, int &nblen, int nbl[]) {
  // lib/src/sapporohostclass.cpp:837-880: the devices' lists in device order,
  // overflow once the total reaches maxlength; then sorted
  nblen = 0;
  ngb_copied_ = 0;
  if (!ngb_fetched_) fetch_ngb_list_from_device(cluster_id);
  if (ipipe < 0 || ipipe >= dev_ni || !ngb_fetched_) return 1;
  bool overflow = false;
  int copied = 0;
  for (int g = 0; g < ndev(); g++) {
    const int len = ngb_count_h_[g][ipipe];
    const int to_copy = std::max(0, std::min(std::min(len, NGB_PB), maxlength - copied));
    memcpy(nbl + copied, &ngb_list_h_[g][(size_t)ipipe * NGB_PB], sizeof(int) * to_copy);
    copied += to_copy;
    nblen += len;
    if (len >= NGB_PB) overflow = true;  // ids beyond NGB_PB were not stored
    if (nblen >= maxlength) {
      overflow = true;
      break;
    }
  }
  std::sort(nbl, nbl + copied);
  ngb_copied_ = copied;
  if (overflow && verbose())
    fprintf(stderr, "sapporo::get_ngb_list(..) - overflow for ipipe= %d, ngb= %d\n", ipipe, nblen);
  return overflow;
}

void sapporo::forcePrediction(int nj) {
  if (devs_.empty()) return;
  int rc = push_staged();
  for (int g = 0; g < ndev() && !rc && predict && nj > 0; g++) {
    const int njg = nj_on(g, nj);
    if (njg == 0) continue;
    rc = sapb_predict(devs_[g], njg, t_i);
    if (rc) report("forcePrediction", rc, devs_[g]);
  }
  if (!rc && predict && nj > 0)
    for (int k = 0; k < nj && k < (int)pred_time_.size(); k++) pred_time_[k] = t_i;
  last_status = rc;
  predict = false;
}

// Reads the FP64 state of every stored j once per modification (like the
// reference's full readback guarded by predJOnHost), predicted to the time
// of the most recent prediction; addresses pushed after that prediction or
// predicted at an older time are handled one by one.
int sapporo::refresh_jcache(int addr) {
  if (devs_.empty() || addr < 0) return SAPB_EINVAL;
  const int G = ndev();
  int cap = 0;
  sapb_info(devs_[addr % G], nullptr, nullptr, nullptr, &cap, nullptr);
  if (addr / G >= cap) return SAPB_EINVAL;
  if (!predJOnHost) {
    push_staged();
    // all addresses below nj_max that the devices hold, device by device
    std::vector<int> caps((size_t)G, 0);
    int n = 0;
    for (int g = 0; g < G; g++) {
      sapb_info(devs_[g], nullptr, nullptr, nullptr, &caps[g], nullptr);
      n = std::max(n, std::min(nj_max, caps[g] * G));
    }
    jcache_.assign((size_t)n * 24, 0.0);
    std::vector<double> part;
    for (int g = 0; g < G; g++) {
      const int ng = std::min(caps[g], n > g ? (n - g + G - 1) / G : 0);
      if (ng == 0) continue;
      double *out = jcache_.data();
      if (G > 1) {
        part.resize((size_t)ng * 24);
        out = part.data();
      }
      const int rc = sapb_read_j(devs_[g], 0, ng, t_i, 1, out);
      if (rc) return rc;
      if (G > 1)
        for (int la = 0; la < ng; la++)
          memcpy(&jcache_[(size_t)(la * G + g) * 24], &part[(size_t)la * 24], 24 * sizeof(double));
    }
    jcache_n_ = n;
    predJOnHost = true;
  }
  if (addr >= jcache_n_) return SAPB_EINVAL;
  const double pt = addr < (int)pred_time_.size() ? pred_time_[addr] : NAN;
  if (std::isnan(pt) || pt != t_i) {
    double one[24];
    const int rc = sapb_read_j(devs_[addr % G], addr / G, 1, std::isnan(pt) ? 0.0 : pt,
                               std::isnan(pt) ? 0 : 1, one);
    if (rc) return rc;
    memcpy(&jcache_[(size_t)addr * 24], one, sizeof one);
  }
  return 0;
}

void sapporo::retrieve_predicted_j_particle(int addr, double &mass, double &id, double &eps2,
                                            double pos[3], double vel[3], double acc[3]) {
  last_status = refresh_jcache(addr);
  if (last_status) {
    report("retrieve_predicted_j_particle", last_status, dev_);
    return;
  }
  const double *o = &jcache_[(size_t)addr * 24];
  for (int d = 0; d < 3; d++) {
    pos[d] = o[14 + d];
    vel[d] = o[17 + d];
    if (integrationOrder > FOURTH && acc) acc[d] = o[20 + d];
  }
  mass = o[3];
  eps2 = o[7];
  id = o[23];
}

void sapporo::retrieve_j_particle_state(int addr, double &mass, double &id, double &eps2,
                                        double pos[3], double vel[3], double acc[3],
                                        double jrk[3], double ppos[3], double pvel[3],
                                        double pacc[3]) {
  last_status = refresh_jcache(addr);
  if (last_status) {
    report("retrieve_j_particle_state", last_status, dev_);
    return;
  }
  const double *o = &jcache_[(size_t)addr * 24];
  mass = o[3];
  for (int d = 0; d < 3; d++) {
    pos[d] = o[d];
    if (integrationOrder > GRAPE5) {
      ppos[d] = o[14 + d];
      pvel[d] = o[17 + d];
      vel[d] = o[4 + d];
      acc[d] = o[8 + d];
      jrk[d] = o[11 + d];
    }
    if (integrationOrder > FOURTH && pacc) pacc[d] = o[20 + d];
  }
  if (integrationOrder > GRAPE5) {
    eps2 = o[7];
    id = o[23];
  }
}
