// Host-side launchers of the device kernels (implemented in sapb_kernels.cu).
#pragma once
#include "sapb_internal.cuh"

namespace sapb {

cudaError_t launch_scatter(int order, int prec, const double *stage, int n, int cap,
                           const JState &js, void *pred, int *status, cudaStream_t st);
cudaError_t launch_predict(int order, int prec, int nj, double ti, const JState &js, void *pred,
                           cudaStream_t st);
cudaError_t launch_force(int order, int prec, const ForceArgs &A, int tpi, int ip,
                         cudaStream_t st);
cudaError_t launch_reduce(const ReduceArgs &R, cudaStream_t st);
cudaError_t launch_wait_selftest(uint64_t limit_ns, int *status, cudaStream_t st);
cudaError_t launch_readj(int order, int first, int n, double ti, int predict, const JState &js,
                         double *out, cudaStream_t st);

// Batched step: per-cluster predictor (if B.do_predict), persistent force
// kernel over the work queue, slice reduction.  Grids are fixed by the
// capacities (j_grid threads, force_blocks blocks, i_grid threads) so the
// launch sequence can be captured once in a CUDA graph.
cudaError_t launch_batch(int order, int prec, const BatchArgs &B, int j_grid, int force_blocks,
                         int i_grid, cudaStream_t st);
int batch_blocks_per_sm(int order, int prec);  // resident persistent blocks per SM

int force_tile_i(int tpi, int ip);  // i-particles per block
// resident blocks per SM of one force-kernel instantiation (occupancy API,
// cached; 0 if the shape does not exist)
int force_blocks_per_sm(int order, int prec, int tpi, int ip);
int force_tile_j();                  // j records per tile

}  // namespace sapb
