/*
 * sapporo_b200.h -- the thin C ABI between the host library (the sapporo
 * class and the GRAPE-6 g6_* interface) and the B200 device code.
 *
 * Plain C types only; every function returns 0 on success or a negative
 * SAPB_E* code (see sapb_error_string).  One sapb_dev owns one GPU's state
 * and one CUDA stream.  Not thread-safe per handle.
 *
 * Each entry point names the reference interface whose role it takes
 * (reference file:line, paths relative to the reference tree).
 */
#ifndef SAPPORO_B200_H
#define SAPPORO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SAPB_OK 0
#define SAPB_ECUDA (-1)     /* a CUDA runtime call failed */
#define SAPB_EINVAL (-2)    /* invalid argument or state */
#define SAPB_ENOMEM (-3)    /* device or pinned allocation failed */
#define SAPB_ETIMEOUT (-4)  /* a device-side bounded wait gave up */
#define SAPB_ENODEV (-5)    /* no usable CUDA device */

/* integration order / precision, same values as lib/include/defines.h:30-31 */
#define SAPB_GRAPE5 0
#define SAPB_FOURTH 1
#define SAPB_SIXTH 2
#define SAPB_FLOAT 0
#define SAPB_DOUBLESINGLE 1
#define SAPB_DOUBLE 2

#define SAPB_NGB_PB 256      /* neighbour slots per i, lib/include/defines.h:9 */
#define SAPB_NPIPES 16384    /* default i per call, lib/include/defines.h:14 */
#define SAPB_RES_STRIDE 12   /* doubles per result record */

/* result record (SAPB_RES_STRIDE doubles per i):
 *   [0..2] acc  [3] pot  [4..6] jerk  [7..9] snap  [10] ds2 of the nearest
 *   neighbour (float precision, 1e11 if none)  [11] its id (-1 if none)   */

/* flags for sapb_force */
#define SAPB_F_PREDICT 1    /* run the predictor to t_i first */
#define SAPB_F_NGB_LIST 2   /* build neighbour lists */

typedef struct sapb_dev sapb_dev;

/* Library build / error helpers. */
const char *sapb_version(void);
const char *sapb_error_string(int code);
const char *sapb_last_error(const sapb_dev *d); /* detail of the last failure */
int sapb_device_count(int *count);

/* Opens `device` for the given order/precision.  Replaces
 * sapporo::open (lib/src/sapporohostclass.cpp:90-372) together with
 * device::assignDevice / allocateMemory (lib/include/sapdevclass.h:122-273).
 * n_pipes: maximum i per force call (<= 0: SAPB_NPIPES);
 * nj_reserve: initial j capacity (<= 0: 16384, as the reference).
 * order SAPB_GRAPE5 (mixed precision): acceleration and potential only, every
 * pair including the self pair, no nearest neighbour or lists (the
 * reference's GRAPE5 kernels, kernels.cu:565, :1096-1098); with DOUBLE it
 * runs the 4th-order FP64 kernels.  Storage is the 4th-order layout. */
int sapb_open(sapb_dev **out, int device, int order, int precision, int n_pipes,
              int nj_reserve);
int sapb_close(sapb_dev *d);
int sapb_info(const sapb_dev *d, int *order, int *precision, int *n_pipes, int *j_capacity,
              int *num_sms);

/* Uses an external cudaStream_t (passed as void*) for all work; NULL
 * restores the library's own stream. */
int sapb_set_stream(sapb_dev *d, void *stream);

/* Grows the device j capacity, keeping the stored j.  Replaces
 * sapporo::increase_jMemory / device::reallocJParticles
 * (lib/src/sapporohostclass.cpp:560-583, lib/include/sapdevclass.h:275-325). */
int sapb_reserve_j(sapb_dev *d, int nj_capacity);

/* Pinned host staging for updated j-particles: returns a pointer to room for
 * `n` records of sapb_j_stage_stride() doubles (contents preserved on
 * growth), or NULL.  Record layout:
 *   [0] address (low 32 bits) | id (high 32 bits)  [1] t  [2] mass
 *   [3..5] x  [6..8] v  [9..11] acc  [12..14] jerk  [15] eps
 *   [16..18] snap  [19..21] crackle   (6th order only)
 * Plays the role of the *_temp host mirrors written by
 * sapporo::set_j_particle (lib/src/sapporohostclass.cpp:500-516). */
double *sapb_j_stage(sapb_dev *d, int n);
int sapb_j_stage_stride(const sapb_dev *d);

/* Copies the first n staged records to the device and scatters them to their
 * addresses (asynchronous).  The n records name distinct addresses: of two
 * records for one address either may land.  The sapporo class keeps one
 * record per address, the later values overwriting the earlier, as the
 * reference's address map does (lib/src/sapporohostclass.cpp:476-494).
 * Replaces send_j_particles_to_device + copyJInDev
 * (lib/src/sapporohostclass.cpp:889-923, 1204-1248). */
int sapb_push_j(sapb_dev *d, int n);

/* Predicts j[0, nj) to t_i (asynchronous).  Replaces predictJParticles
 * (lib/src/sapporohostclass.cpp:1250-1284). */
int sapb_predict(sapb_dev *d, int nj, double ti);

/* Pinned host buffer for `ni` i records (8 doubles each for 4th order:
 * x0 x1 x2 h2 v0 v1 v2 id-bits; 12 for 6th: + a0 a1 a2 0).  The id is
 * stored in the low 32 bits of slot 7. */
double *sapb_i_stage(sapb_dev *d, int ni);
int sapb_i_stage_stride(const sapb_dev *d);

/* Force on the ni staged i-particles from j[0, nj): H2D of the i records,
 * optional prediction to ti, force kernels, D2H of the results into pinned
 * memory -- all asynchronous on the device stream.  Replaces the launch part
 * of sapporo::startGravCalc / evaluate_gravity
 * (lib/src/sapporohostclass.cpp:586-703, 1442-1602). */
int sapb_force(sapb_dev *d, int nj, int ni, double eps2, double ti, int flags);

/* Waits for the last sapb_force and returns its pinned result records
 * (SAPB_RES_STRIDE doubles per i).  Replaces the blocking readback of
 * sapporo::getGravResults (lib/src/sapporohostclass.cpp:705-802, 949-966). */
int sapb_results(sapb_dev *d, const double **results, int *ni);

/* Copies the neighbour counts and lists of the last force call to the host.
 * counts: ni ints; lists: ni*SAPB_NGB_PB ints (may be NULL).  Replaces
 * fetch_ngb_list_from_device (lib/src/sapporohostclass.cpp:1149-1162). */
int sapb_ngb_fetch(sapb_dev *d, int *counts, int *lists, int ni);

/* Device-resident variants for callers that keep i-data on the GPU
 * (no host copies; `i_dev`, `res_dev` are device pointers with the record
 * layouts above; asynchronous on the device stream). */
int sapb_force_device(sapb_dev *d, int nj, int ni, const double *i_dev, double eps2, int flags,
                      double *res_dev, int *ngb_count_dev, int *ngb_list_dev);

/* Self-test of the device-side failure path (no reference counterpart; the
 * reference has no bounded waits).  Launches one thread that waits on a
 * shared-memory barrier nothing ever arrives at, with the same bounded wait
 * the force kernels use but a limit of limit_ms (1..2000).  Returns
 * SAPB_ETIMEOUT when the wait gave up and the kernel returned -- the
 * expected outcome, after which the device stays usable. */
int sapb_wait_selftest(sapb_dev *d, int limit_ms);

/* Force call that allocates nothing: no cudaMalloc, cudaFree or other
 * allocating routine, on any call.  It is for callers that cannot allocate
 * device memory while they integrate -- codes that hand the whole GPU to
 * their own pool allocator, or that must not take the device-wide
 * synchronisation cudaFree implies in the middle of a time step -- whereas
 * sapb_force_device grows its partial-sum buffer with cudaMalloc/cudaFree
 * when a larger active set arrives.  This entry point of this library has no
 * counterpart in the reference.
 *
 * Same arguments, layouts and results as sapb_force_device.  The j-split
 * partial sums go to one fixed 32 MiB device array (SAPB_NOALLOC_SCRATCH_
 * BYTES) that every GPU loading the library holds until exit; ni is limited
 * to SAPB_NOALLOC_SCRATCH_BYTES / (8 * SAPB_RES_STRIDE) = 349525 per call
 * (larger ni returns SAPB_EINVAL with a message), and the j-split is capped
 * to fit.  The array's device address is resolved once per device by
 * sapb_open (or by the first call on that device, which should then come
 * before any stream capture).  All calls on a device share the array and it
 * keeps the last call's contents (each call overwrites every record it
 * reads, so nothing needs clearing); calls that overlap on the GPU --
 * different streams or handles on one device -- race on it. */
#define SAPB_NOALLOC_SCRATCH_BYTES (32u << 20)
int sapb_force_device_noalloc(sapb_dev *d, int nj, int ni, const double *i_dev, double eps2,
                              int flags, double *res_dev, int *ngb_count_dev,
                              int *ngb_list_dev);

/* FP64 state of j[first, first+n), 24 doubles per j:
 *   x[3] mass v[3] eps acc[3] jerk[3] px[3] pv[3] pa[3] id
 * where px/pv/pa are the FP64 prediction to ti (predict != 0) or the raw
 * state (predict == 0).  Synchronous.  Backs retrieve_predicted_j_particle
 * and retrieve_j_particle_state (lib/src/sapporohostclass.cpp:969-1147). */
int sapb_read_j(sapb_dev *d, int first, int n, double ti, int predict, double *out);

/* ---- Batched force evaluation: many independent force calls in one
 * persistent launch inside a captured CUDA graph.  Replaces the reference's
 * one-launch-per-256-i loop (lib/src/sapporohostclass.cpp:1499-1598) for
 * block-timestep steps with uneven active counts and for ensembles of
 * independent clusters.  A cluster is a contiguous, address-ordered range
 * of j addresses [j_first, j_first + j_count) of this device's j store, with
 * its own prediction time and softening, and i_count active i records
 * (layout of sapb_i_stage) stored consecutively, cluster after cluster, in
 * sapb_batch_i_stage().  Self pairs are skipped by id within a cluster. */
typedef struct sapb_batch sapb_batch;
int sapb_batch_create(sapb_dev *d, int max_clusters, int max_i, sapb_batch **out);
int sapb_batch_destroy(sapb_batch *b);
/* pinned i-record staging for max_i records */
double *sapb_batch_i_stage(sapb_batch *b);
/* Work plan of the next run: threads per i and j-split per cluster (the
 * planner's rule, shifted by sapb_batch_set_tuning), work items in
 * longest-first order. */
int sapb_batch_plan(sapb_batch *b, int n_clusters, const int *j_first, const int *j_count,
                    const int *i_count, const double *t_pred, const double *eps2);
/* Asynchronous run: one H2D copy, one graph launch (queue reset, list-count
 * reset, per-cluster predictor if SAPB_F_PREDICT, persistent force kernel,
 * slice reduction), one D2H copy of the results. */
int sapb_batch_run(sapb_batch *b, int flags);
/* Waits; results in i-record order, SAPB_RES_STRIDE doubles each. */
int sapb_batch_results(sapb_batch *b, const double **results, int *total_i);
int sapb_batch_ngb_fetch(sapb_batch *b, int *counts, int *lists);
int sapb_batch_info(sapb_batch *b, int *n_items, int *force_blocks, int *graph_runs);
/* Autotuner knob: log2 factor on the threads-per-i rule (-5..5). */
int sapb_batch_set_tuning(sapb_batch *b, int tpi_scale);
/* Measures the last plan's workload under each threads-per-i scale
 * (-1..2) and j-split density (2, 4, 8 items per resident block), `reps`
 * graph replays each, keeps the fastest and re-plans with it. */
int sapb_batch_autotune(sapb_batch *b, int flags, int reps, int *best_scale, int *best_split,
                        float *best_ms);

/* ---- Neighbour-radius network (no counterpart in the reference; the
 * reference's h2 comes from the caller).  A 5 -> 64 -> 64 -> 64 -> 1 ReLU
 * perceptron with FP32 weights, run and trained on this device by the
 * library's own CUDA kernels.  Host arrays: x [n][5] floats, t and y [n].
 * Parameters: sapb_mlp_num_params() floats in the order W1[64][5] b1 W2[64][64]
 * b2 W3[64][64] b3 W4[64] b4. */
typedef struct sapb_mlp sapb_mlp;
int sapb_mlp_num_params(void);
/* He/Glorot-uniform initialisation from `seed` (splitmix64 stream). */
int sapb_mlp_create(sapb_dev *d, unsigned long long seed, sapb_mlp **out);
int sapb_mlp_destroy(sapb_mlp *m);
int sapb_mlp_set_params(sapb_mlp *m, const float *params);  /* also resets Adam state */
int sapb_mlp_get_params(sapb_mlp *m, float *params);
/* y = net(x) for n samples (synchronous). */
int sapb_mlp_forward(sapb_mlp *m, int n, const float *x, float *y);
/* Gradient of 1/(2n) sum (net(x) - t)^2 (grad may be NULL) and the loss. */
int sapb_mlp_gradient(sapb_mlp *m, int n, const float *x, const float *t, float *grad,
                      float *loss);
/* `epochs` full-batch Adam steps (lr, beta 0.9/0.999); loss before the last. */
/* Radius proposal in one call: in = n records of 9 floats (previous
 * neighbour count, previous h2, acceleration[3], jerk[3], L = the particle's
 * running mean of log density over its past evaluations); the features
 * (log rho with the density estimate rho = n/(4/3 pi h^3), n = max(count,
 * 1/2), log |a|, log |jerk|, L - log rho, log h2) are standardised with mu[5],
 * sd[5]; the network's correction, clipped to [-max_down, max_up], is added
 * to the count-scaled step 2/3 log(target/n); h2_out = h2 * exp(step clipped
 * to +-clip). */
int sapb_mlp_propose(sapb_mlp *m, int n, const float *in, const float *mu, const float *sd,
                     float target, float max_down, float max_up, float clip, float *h2_out);
int sapb_mlp_train(sapb_mlp *m, int n, const float *x, const float *t, int epochs, float lr,
                   float *loss);

/* Launch-shape override for the force kernel: threads per i (1,2,4,8,16,32),
 * i per thread (1,2) and j slices (>= 1).  Zeros restore the built-in
 * planner.  Replaces the compile-time NTHREADS / NBLOCKS_PER_MULTI tables
 * (lib/include/defines.h:13-122). */
int sapb_set_launch(sapb_dev *d, int tpi, int ip, int nslices);
int sapb_get_plan(sapb_dev *d, int ni, int nj, int *tpi, int *ip, int *nslices);

/* Spatial mode of the mixed-precision (DOUBLESINGLE) force calls: j records
 * and i positions are taken in Morton order, and (warp, j tile) pairs whose
 * boxes are at least |x|max * 2^-23 / delta apart use the single-float
 * difference of the high position parts instead of the double-single one of
 * the reference (kernels.cu:169-177), which is then accurate to delta
 * relative.  Tiles that could hold a nearest neighbour always take the
 * double-single path and list members on far tiles are found by an exact
 * rescan, so neighbours and lists are unchanged; the force sums change only
 * at the rounding level (the summation order too) and do not depend on h2.
 * mode 0: off (address order, the reference's arithmetic for every pair),
 * 1: on for calls of >= 2^28 pairs, >= 1024 i and >= 65536 j (the default), 2: on for
 * every call.
 * delta 0 keeps the default 1e-6; at most 1e-4.  The environment variable
 * SAPPORO_B200_SPATIAL (0, 1, 2) sets the mode at open.  A call for whose
 * sort buffers the device has no room runs in address order.  Not used by
 * sapb_force_device_noalloc or the batch calls. */
int sapb_set_spatial(sapb_dev *d, int mode, double delta);
/* Work of the spatial-mode calls since the last reset: (warp, j tile) pairs
 * that took the far path and all (warp, j tile) pairs of those calls (the
 * packed shapes; 0 and 0 before any spatial call).  Synchronises the
 * handle's stream; reset != 0 zeroes the counters. */
int sapb_spatial_stats(sapb_dev *d, unsigned long long *far_tiles,
                       unsigned long long *warp_tiles, int reset);

/* Near pairs of the mixed-precision (DOUBLESINGLE) force calls, an addition
 * to the reference's double-single kernels (kernels.cu:552-669, which take
 * every pair in FP32 after the position difference): when an i's share of a
 * j tile holds a pair with ds2 < factor * eps2, that share is summed in FP64
 * instead (positions hi + lo, velocity, acceleration and mass as stored).
 * Softened pairs a few softening lengths apart can dominate an i's jerk or
 * snap while their sum passes through zero, and there FP32 rounding would
 * leave large relative errors; tight binaries are such pairs.  factor 0 turns
 * it off (every pair in FP32, as the reference); the default is 16 (pairs
 * within 4 softening lengths).  The environment variable SAPPORO_B200_NEAR
 * sets the factor at open.  No effect with eps2 = 0 or on the FP64 and
 * GRAPE-5 kernels.  Batch calls take the factor in force when they are
 * planned (sapb_batch_plan). */
int sapb_set_near(sapb_dev *d, double factor);

#ifdef __cplusplus
}
#endif
#endif
