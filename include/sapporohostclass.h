/*
 * sapporohostclass.h -- the `sapporo` C++ class of the B200 build.
 *
 * Source-compatible with the reference's public interface
 * (lib/include/sapporohostclass.h:37-176): same class name, method names,
 * argument order and meaning, default arguments and enum values, so callers
 * written against the reference compile and link unchanged.  The private
 * part is this library's own (one sapb_* device handle of sapporo_b200.h per
 * device given to open); no binary layout compatibility is implied.
 *
 * Like the reference header it pulls in <iostream>, <vector>, <map>,
 * <string>, <cmath> and `using namespace std`, which its callers rely on.
 */
#ifndef _SAPPORO_H_
#define _SAPPORO_H_

#include <assert.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <algorithm>
#include <iostream>
#include <map>
#include <string>
#include <vector>

using namespace std;

// lib/include/defines.h:9-31
#ifndef NGB_PB
#define NGB_PB 256
#endif
#ifndef NGB
#define NGB
#endif
#ifndef NPIPES
#define NPIPES 16384
#endif
enum { GRAPE5 = 0, FOURTH, SIXTH, EIGHT };
enum { FLOAT = 0, DOUBLESINGLE, DOUBLE };

struct sapb_dev;

class sapporo {
 protected:
  // One handle per device of open(); j address a lives on devs_[a % G] at
  // local address a / G (G = devs_.size()), as the reference distributes j
  // round-robin over its devices (lib/src/sapporohostclass.cpp:473-474).
  std::vector<sapb_dev *> devs_;
  sapb_dev *dev_;       // devs_[0]
  int n_pipes;
  int nj_max;           // allocated j capacity (addresses below it are accepted)
  int integrationOrder;
  int integrationPrecision;
  double EPS2;
  double t_i;
  bool predict;         // predict j to t_i at the next force / forcePrediction
  bool nj_updated;      // j staged since the last push
  bool predJOnHost;     // host cache of the predicted j state is current

  // j staging: slot of each address staged since the last push (in the
  // staging of its device), -1 if none; per device the staged addresses
  std::vector<int> stage_slot_;
  std::vector<std::vector<int> > staged_addr_;

  // per-address prediction time of the force records (NaN: unpredicted copy)
  std::vector<double> pred_time_;
  std::vector<double> jcache_;   // 24 doubles per address, see sapb_read_j
  int jcache_n_;

  int dev_ni;                    // i count of the last force call
  int nj_last_;
  std::vector<int> dev_nj_;      // per device: j of the last force call
  std::vector<std::vector<int> > ngb_count_h_;  // per device
  std::vector<std::vector<int> > ngb_list_h_;
  bool ngb_fetched_;
  int ngb_copied_;               // ids written by the last get_ngb_list

  int ndev() const { return (int)devs_.size(); }
  int nj_on(int g, int nj) const;  // j among the first nj addresses held by device g
  double *stage_record(int address, int &rc);
  int push_staged();
  void increase_jMemory();
  int refresh_jcache(int addr);

 public:
  sapporo();
  ~sapporo();

  // lib/include/sapporohostclass.h:121-122
  void send_j_particles_to_device();
  void send_i_particles_to_device(int i);

  // lib/include/sapporohostclass.h:125-175
  int open(std::string kernelFile, int *devices, int nprocs = 1, int order = FOURTH,
           int precision = DOUBLESINGLE);
  int close();
  int get_n_pipes();
  int set_time(double ti);
  int set_no_time();

  int set_j_particle(int address, int index, double tj, double dtj, double mass, double k18[3],
                     double j6[3], double a2[3], double v[3], double x[3], double snp[3],
                     double crk[3], double eps);

  void startGravCalc(int nj, int ni, int index[], double xi[][3], double vi[][3],
                     double aold[][3], double j6old[][3], double phiold[3], double eps2,
                     double h2[], double eps2_i[]);

  int getGravResults(int nj, int ni, int index[], double xi[][3], double vi[][3], double eps2,
                     double h2[], double acc[][3], double jerk[][3], double snp[][3],
                     double crk[][3], double pot[], int nnbindex[], double dsmin_i[], bool ngb);

  void forcePrediction(int nj);
  void retrieve_predicted_j_particle(int addr, double &mass, double &id, double &eps2,
                                     double pos[3], double vel[3], double acc[3]);

  void retrieve_j_particle_state(int addr, double &mass, double &id, double &eps2, double pos[3],
                                 double vel[3], double acc[3], double jrk[3], double ppos[3],
                                 double pvel[3], double pacc[3]);

  int fetch_ngb_list_from_device(int);
  int read_ngb_list(int);
  int get_ngb_list(int cluster_id, int ipipe, int maxlength, int &nblen, int nbl[]);

  // Additions of this library (not in the reference): the underlying device
  // handles, the status of the last call that can fail (0 = ok), and n calls
  // of set_j_particle in one (arrays of n, vectors [n][3]; a, jrk, snp, crk,
  // eps, t may be null for zeros): the same address rules, one staging
  // reservation per device for all; an address given twice keeps its later
  // entry, as with n calls of set_j_particle.
  sapb_dev *device_handle() { return dev_; }
  sapb_dev *device_handle(int k) { return k >= 0 && k < ndev() ? devs_[k] : nullptr; }
  int n_devices() const { return ndev(); }
  // the number of ids the last get_ngb_list wrote to nbl (sorted): nblen
  // capped at maxlength, less any ids beyond NGB_PB of a device's list
  int ngb_list_copied() const { return ngb_copied_; }
  int last_status;
  int set_j_particles(int n, const int *address, const int *id, const double *t,
                      const double *mass, const double *x, const double *v, const double *a,
                      const double *jrk, const double *snp, const double *crk,
                      const double *eps);
};

#endif
