// fma_ceiling -- a measurement probe, not part of the library: what the FP32
// pipe of this GPU sustains for instruction mixes like the force kernel's, so
// the force kernel's fraction of the nominal FP32 peak can be read against a
// measured ceiling.  Compiled and run by
//
//   python bench.py --workload fma_ceiling
//
// Each test runs independent chains of FP32 FMAs (scalar FFMA or packed
// FP32x2 __ffma2_rn) for a fixed count and reports FMA lane-operations/s as
// TFLOP/s (2 flops per FMA), at 8, 4, 3 and 2 resident 128-thread blocks per
// SM (the force kernel runs 2 or 3).  Mixes:
//   ffma        scalar FFMA, 16 chains
//   ffma2       packed FFMA2, 8 float2 chains
//   ffma2+mufu  one rsqrt.approx (MUFU) per 16 FFMA2 (+2 FADD feeding it)
//   ffma2+lds   one broadcast LDS.128 per 32 FFMA2, j operand broadcast
// All indexes stay inside a 256-entry shared array; no waits.
#include <cstdio>
#include <cuda_runtime.h>

namespace {

constexpr int kThreads = 128;

template <int MODE>
__global__ void __launch_bounds__(kThreads) chains(float *out, int iters) {
  __shared__ float4 srec[256];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    const float v = 0.999f + 1e-6f * i;
    srec[i] = make_float4(v, v * 0.5f, v * 0.25f, v * 0.125f);
  }
  __syncthreads();
  const float s = 0.9999f;
  if (MODE == 0) {
    float c[16];
#pragma unroll
    for (int k = 0; k < 16; k++) c[k] = 1.0f + t * 1e-7f + k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
      for (int r = 0; r < 8; r++)
#pragma unroll
        for (int k = 0; k < 16; k++) c[k] = fmaf(c[k], s, 0.5f);
    }
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) sum += c[k];
    out[t] = sum;
    return;
  }
  float2 c[8];
#pragma unroll
  for (int k = 0; k < 8; k++) c[k] = make_float2(1.0f + t * 1e-7f + k, 1.0f - k);
  const float2 s2 = make_float2(s, s * 0.999f), h2 = make_float2(0.5f, 0.25f);
  float acc = 0.f;
  for (int i = 0; i < iters; i++) {
    if (MODE == 3) {
      // 2 x (one LDS.128, 4 broadcast operands x 8 chains) = 64 FFMA2
#pragma unroll
      for (int half = 0; half < 2; half++) {
        const float4 v = srec[(2 * i + half) & 255];
        const float q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
          for (int k = 0; k < 8; k++) c[k] = __ffma2_rn(c[k], make_float2(q[r], q[r]), h2);
      }
      continue;
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
#pragma unroll
      for (int k = 0; k < 8; k++) c[k] = __ffma2_rn(c[k], s2, h2);
      if (MODE == 2 && (r & 1)) {
        float y;
        asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(c[r & 7].x + 2.0f));
        acc += y;
      }
    }
  }
  float sum = acc;
#pragma unroll
  for (int k = 0; k < 8; k++) sum += c[k].x + c[k].y;
  out[t] = sum;
}

template <int MODE>
float run(float *out, int blocks, int iters) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  chains<MODE><<<blocks, kThreads>>>(out, iters);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    cudaEventRecord(e0);
    chains<MODE><<<blocks, kThreads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    best = ms < best ? ms : best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

int main() {
  int dev = 0, nsm = 0, clk_khz = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, dev);
  const double nominal = nsm * 128.0 * 2.0 * clk_khz * 1e3 / 1e12;
  printf("SMs %d, max clock %.0f MHz, nominal FP32 %.2f TFLOP/s\n", nsm, clk_khz / 1e3, nominal);
  const int iters = 20000;
  float *out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * nsm * 8 * kThreads) != cudaSuccess) return 1;
  const char *names[4] = {"ffma", "ffma2", "ffma2+mufu", "ffma2+lds"};
  for (int bps : {8, 4, 3, 2}) {
    const int blocks = nsm * bps;
    // FMA lane-operations per thread: 128 per iteration in every mode
    const double ops = (double)blocks * kThreads * iters * 128.0;
    for (int mode = 0; mode < 4; mode++) {
      float ms = 0.f;
      if (mode == 0) ms = run<0>(out, blocks, iters);
      if (mode == 1) ms = run<1>(out, blocks, iters);
      if (mode == 2) ms = run<2>(out, blocks, iters);
      if (mode == 3) ms = run<3>(out, blocks, iters);
      const double tf = 2.0 * ops / (ms * 1e-3) / 1e12;
      printf("%d blocks/SM  %-11s %8.3f ms  %6.2f TFLOP/s  %5.1f %% of nominal\n", bps,
             names[mode], ms, tf, 100.0 * tf / nominal);
    }
  }
  const cudaError_t e = cudaGetLastError();
  printf("status: %s\n", cudaGetErrorString(e));
  cudaFree(out);
  return e == cudaSuccess ? 0 : 1;
}
