/*
 * TEST INFRASTRUCTURE ONLY: compiles the reference's own device kernels,
 * unchanged, from the reference tree (include path given by oracle/Makefile)
 * into oracle/_ref/ref_kernels.cubin.  Nothing in the product links this.
 *
 * lib/CUDAKernels/kernels.cu:210-222 defines a CAS-loop
 * atomicAdd(double*, double) for pre-sm_60 GPUs, which collides with the
 * builtin on sm_60 and newer.  The rename below keeps the reference's own
 * CAS loop (same semantics) and forwards the int overload, which the
 * neighbour-list reservation at kernels.cu:1007 uses, to the builtin.
 */
__device__ __forceinline__ int sapref_builtin_int_add(int *a, int v) {
  return atomicAdd(a, v);
}
#define atomicAdd sapref_atomicAdd
__device__ __forceinline__ int sapref_atomicAdd(int *a, int v) {
  return sapref_builtin_int_add(a, v);
}
#include "CUDAKernels/kernels.cu"
