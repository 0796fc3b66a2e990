// Neighbour-radius network: a 5 -> 64 -> 64 -> 64 -> 1 perceptron with ReLU
// hidden layers, FP32 weights, trained on the GPU with hand-written forward,
// backward and Adam kernels.  It proposes log(h2) for each i-particle from
// five features of its previous evaluation; the host side (Python) builds
// features and targets from the neighbour counts the force kernel reports.
// Declared in include/sapporo_b200.h (sapb_mlp_*).
//
// Parameter layout (floats): W1[64][5] b1[64] W2[64][64] b2[64] W3[64][64]
// b3[64] W4[64] b4[1]  -- 8769 parameters.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "../../include/sapporo_b200.h"
#include "sapb_dev.h"

namespace {

constexpr int kIn = 5, kH = 64;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH,
              oW3 = oB2 + kH, oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kH,
              kNP = oB4 + 1;
constexpr int kMB = 128;  // samples per block in the backward kernel

// y = W4 relu(W3 relu(W2 relu(W1 x + b1) + b2) + b3) + b4 for one sample;
// h1/h2/h3 receive the post-ReLU activations when non-null.
__device__ __forceinline__ float mlp_eval(const float *__restrict__ P, const float *x, float *h1,
                                          float *h2, float *h3) {
  float a1[kH], a2[kH];
#pragma unroll
  for (int o = 0; o < kH; o++) {
    float s = P[oB1 + o];
#pragma unroll
    for (int k = 0; k < kIn; k++) s = fmaf(P[oW1 + o * kIn + k], x[k], s);
    a1[o] = fmaxf(s, 0.f);
  }
#pragma unroll 4
  for (int o = 0; o < kH; o++) {
    float s = P[oB2 + o];
#pragma unroll
    for (int k = 0; k < kH; k++) s = fmaf(P[oW2 + o * kH + k], a1[k], s);
    a2[o] = fmaxf(s, 0.f);
  }
  if (h1)
    for (int k = 0; k < kH; k++) h1[k] = a1[k];
  float y = P[oB4];
#pragma unroll 4
  for (int o = 0; o < kH; o++) {
    float s = P[oB3 + o];
#pragma unroll
    for (int k = 0; k < kH; k++) s = fmaf(P[oW3 + o * kH + k], a2[k], s);
    s = fmaxf(s, 0.f);
    if (h3) h3[o] = s;
    y = fmaf(P[oW4 + o], s, y);
  }
  if (h2)
    for (int k = 0; k < kH; k++) h2[k] = a2[k];
  return y;
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float *__restrict__ P, int n,
                                                          const float *__restrict__ X,
                                                          float *__restrict__ Y) {
  __shared__ float sp[kNP];
  for (int k = threadIdx.x; k < kNP; k += blockDim.x) sp[k] = P[k];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[kIn];
#pragma unroll
  for (int k = 0; k < kIn; k++) x[k] = X[(size_t)i * kIn + k];
  Y[i] = mlp_eval(sp, x, nullptr, nullptr, nullptr);
}

// Proposal: the five features of each particle from its raw previous state
// (n_prev, h2_prev, a[3], jerk[3], L; features: log rho with the density
// estimate rho = n / (4/3 pi h^3), n = max(n_prev, 1/2), log |a|, log |jerk|,
// L - log rho with L the particle's running mean of log rho over its past
// evaluations, log h2), standardised with (mu, sd), the network's correction
// clipped to [-max_down, max_up] and added to the count-scaled step
// 2/3 log(target/n); out: h2_prev * exp(clip(step, -clip, clip)).
struct MlpScale {
  float mu[kIn], sd[kIn];
  float target, max_down, max_up, clip;
};
constexpr int kPropIn = 9;

__global__ void __launch_bounds__(128) mlp_propose_kernel(const float *__restrict__ P, int n,
                                                          const float *__restrict__ IN,
                                                          MlpScale sc, float *__restrict__ H2) {
  __shared__ float sp[kNP];
  for (int k = threadIdx.x; k < kNP; k += blockDim.x) sp[k] = P[k];
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float *r = IN + (size_t)i * kPropIn;
  const float np = fmaxf(r[0], 0.5f), h2 = r[1];
  const float an = sqrtf(r[2] * r[2] + r[3] * r[3] + r[4] * r[4]) + 1e-30f;
  const float jn = sqrtf(r[5] * r[5] + r[6] * r[6] + r[7] * r[7]) + 1e-30f;
  const float lh2 = logf(h2);
  const float lrho = logf(np) - logf(4.18879020f) - 1.5f * lh2;
  const float f[kIn] = {lrho, logf(an), logf(jn), r[8] - lrho, lh2};
  float x[kIn];
#pragma unroll
  for (int k = 0; k < kIn; k++) x[k] = (f[k] - sc.mu[k]) / sc.sd[k];
  const float corr = fminf(fmaxf(mlp_eval(sp, x, nullptr, nullptr, nullptr), -sc.max_down),
                           sc.max_up);
  const float step = (2.f / 3.f) * logf(sc.target / np) + corr;
  H2[i] = h2 * expf(fminf(fmaxf(step, -sc.clip), sc.clip));
}

// Gradient of L = 1/(2n) sum (y - t)^2 over the n samples, accumulated into
// G (zeroed by the caller), loss accumulated into *loss.
//
// Persistent: each block loops over chunks of 128 samples (one per thread)
// and keeps its share of the gradient in registers until the end, so G
// receives one atomic per parameter per block (not per chunk).  Within a
// chunk the activations and deltas sit in shared memory as [sample][unit]
// rows padded to kS floats; every weight gradient is a sum over samples of
// outer products, computed as register tiles (4 output units x 8 input units
// per thread for the 64x64 layers: 3 vector shared loads per 32 FMA), and the
// back-propagated deltas read the weight rows as float4 (one vector load per
// 4 FMA, broadcast to the warp).
constexpr int kS = 68;  // padded row: float4-aligned, conflict-free columns
constexpr int kNPp = (kNP + 3) / 4 * 4;
constexpr int kBwdFloats = kNPp + kMB * 8 + 4 * kMB * kS + kMB;

__device__ __forceinline__ float4 ld4(const float *p) {
  return *reinterpret_cast<const float4 *>(p);
}

__global__ void __launch_bounds__(kMB, 1) mlp_backward_kernel(const float *__restrict__ P, int n,
                                                              const float *__restrict__ X,
                                                              const float *__restrict__ T,
                                                              float *__restrict__ G,
                                                              float *__restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  float *sp = sm;                  // parameters (kNP, padded)
  float *XS = sp + kNPp;           // [128][8]
  float *A1 = XS + kMB * 8;        // [128][kS] post-ReLU layer 1
  float *A2 = A1 + kMB * kS;       // [128][kS] post-ReLU layer 2
  float *A3 = A2 + kMB * kS;       // [128][kS] post-ReLU layer 3, then delta 2
  float *D3 = A3 + kMB * kS;       // [128][kS] delta 3, then delta 1
  float *DY = D3 + kMB * kS;       // [128]
  const int t = threadIdx.x;
  const int lane = t & 31;
  for (int k = t; k < kNP; k += kMB) sp[k] = P[k];

  // register-tile owners: 4 output rows x 8 input columns of W2 and W3
  const int o0 = (t >> 3) * 4, k0 = (t & 7) * 8;
  float gW3[4][8], gW2[4][8];
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 8; c++) gW3[r][c] = gW2[r][c] = 0.f;
  float gW1[kIn] = {0, 0, 0, 0, 0};  // row t (t < 64)
  float gB1 = 0.f, gB2 = 0.f, gB3 = 0.f, gW4 = 0.f, gB4 = 0.f;
  float lsum = 0.f;
  __syncthreads();

  const int nchunks = (n + kMB - 1) / kMB;
  for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int i = chunk * kMB + t;
    const bool valid = i < n;
    // ---- forward for this thread's sample ----
    float x[kIn];
#pragma unroll
    for (int k = 0; k < kIn; k++) x[k] = valid ? X[(size_t)i * kIn + k] : 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) XS[t * 8 + k] = k < kIn ? x[k] : 0.f;
#pragma unroll 4
    for (int o = 0; o < kH; o++) {
      float s = sp[oB1 + o];
#pragma unroll
      for (int k = 0; k < kIn; k++) s = fmaf(sp[oW1 + o * kIn + k], x[k], s);
      A1[t * kS + o] = fmaxf(s, 0.f);
    }
    // layers 2 and 3 read this thread's previous-layer row back as float4
    // (activations stay out of the registers, which hold the gradient tiles)
#pragma unroll 2
    for (int o = 0; o < kH; o++) {
      float s = sp[oB2 + o];
#pragma unroll
      for (int k = 0; k < kH; k += 4) {
        const float4 w = ld4(sp + oW2 + o * kH + k);
        const float4 h = ld4(A1 + t * kS + k);
        s = fmaf(w.x, h.x, fmaf(w.y, h.y, fmaf(w.z, h.z, fmaf(w.w, h.w, s))));
      }
      A2[t * kS + o] = fmaxf(s, 0.f);
    }
    float y = sp[oB4];
#pragma unroll 2
    for (int o = 0; o < kH; o++) {
      float s = sp[oB3 + o];
#pragma unroll
      for (int k = 0; k < kH; k += 4) {
        const float4 w = ld4(sp + oW3 + o * kH + k);
        const float4 h = ld4(A2 + t * kS + k);
        s = fmaf(w.x, h.x, fmaf(w.y, h.y, fmaf(w.z, h.z, fmaf(w.w, h.w, s))));
      }
      s = fmaxf(s, 0.f);
      A3[t * kS + o] = s;
      y = fmaf(sp[oW4 + o], s, y);
    }
    const float err = valid ? y - T[i] : 0.f;
    const float dy = err / (float)n;
    lsum += 0.5f * err * err / (float)n;
    DY[t] = dy;
#pragma unroll 8
    for (int o = 0; o < kH; o++) D3[t * kS + o] = A3[t * kS + o] > 0.f ? dy * sp[oW4 + o] : 0.f;
    __syncthreads();

    // ---- W3 (tile), W4, b3, b4 ----
#pragma unroll 2
    for (int b = 0; b < kMB; b++) {
      const float4 d = ld4(D3 + b * kS + o0);
      const float4 h0 = ld4(A2 + b * kS + k0), h1 = ld4(A2 + b * kS + k0 + 4);
      const float dv[4] = {d.x, d.y, d.z, d.w};
      const float hv[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 8; c++) gW3[r][c] = fmaf(dv[r], hv[c], gW3[r][c]);
    }
    if (t < kH) {
      for (int b = 0; b < kMB; b++) {
        gW4 = fmaf(DY[b], A3[b * kS + t], gW4);
        gB3 += D3[b * kS + t];
      }
    } else if (t == kH) {
      for (int b = 0; b < kMB; b++) gB4 += DY[b];
    }
    // ---- delta 2 of this thread's sample: (W3^T d3) * relu'(a2) ----
    float d2[kH];
#pragma unroll
    for (int k = 0; k < kH; k++) d2[k] = 0.f;
#pragma unroll 2
    for (int o = 0; o < kH; o++) {
      const float d = D3[t * kS + o];
#pragma unroll
      for (int k = 0; k < kH; k += 4) {
        const float4 w = ld4(sp + oW3 + o * kH + k);
        d2[k] = fmaf(w.x, d, d2[k]);
        d2[k + 1] = fmaf(w.y, d, d2[k + 1]);
        d2[k + 2] = fmaf(w.z, d, d2[k + 2]);
        d2[k + 3] = fmaf(w.w, d, d2[k + 3]);
      }
    }
    __syncthreads();  // A3 and D3 are read by every thread above
    float *D2 = A3;
#pragma unroll
    for (int k = 0; k < kH; k += 4) {
      const float4 a = ld4(A2 + t * kS + k);
      *reinterpret_cast<float4 *>(D2 + t * kS + k) =
          make_float4(a.x > 0.f ? d2[k] : 0.f, a.y > 0.f ? d2[k + 1] : 0.f,
                      a.z > 0.f ? d2[k + 2] : 0.f, a.w > 0.f ? d2[k + 3] : 0.f);
    }
    __syncthreads();

    // ---- W2 (tile), b2 ----
#pragma unroll 2
    for (int b = 0; b < kMB; b++) {
      const float4 d = ld4(D2 + b * kS + o0);
      const float4 h0 = ld4(A1 + b * kS + k0), h1 = ld4(A1 + b * kS + k0 + 4);
      const float dv[4] = {d.x, d.y, d.z, d.w};
      const float hv[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
#pragma unroll
      for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 8; c++) gW2[r][c] = fmaf(dv[r], hv[c], gW2[r][c]);
    }
    if (t < kH)
      for (int b = 0; b < kMB; b++) gB2 += D2[b * kS + t];
    // ---- delta 1 of this thread's sample: (W2^T d2) * relu'(a1) ----
    float d1[kH];
#pragma unroll
    for (int k = 0; k < kH; k++) d1[k] = 0.f;
#pragma unroll 2
    for (int o = 0; o < kH; o++) {
      const float d = D2[t * kS + o];
#pragma unroll
      for (int k = 0; k < kH; k += 4) {
        const float4 w = ld4(sp + oW2 + o * kH + k);
        d1[k] = fmaf(w.x, d, d1[k]);
        d1[k + 1] = fmaf(w.y, d, d1[k + 1]);
        d1[k + 2] = fmaf(w.z, d, d1[k + 2]);
        d1[k + 3] = fmaf(w.w, d, d1[k + 3]);
      }
    }
    float *D1 = D3;  // D3 is no longer read: every thread passed the barrier above
#pragma unroll
    for (int k = 0; k < kH; k += 4) {
      const float4 a = ld4(A1 + t * kS + k);
      *reinterpret_cast<float4 *>(D1 + t * kS + k) =
          make_float4(a.x > 0.f ? d1[k] : 0.f, a.y > 0.f ? d1[k + 1] : 0.f,
                      a.z > 0.f ? d1[k + 2] : 0.f, a.w > 0.f ? d1[k + 3] : 0.f);
    }
    __syncthreads();

    // ---- W1, b1 (row t) ----
    if (t < kH) {
      for (int b = 0; b < kMB; b++) {
        const float d = D1[b * kS + t];
        gB1 += d;
#pragma unroll
        for (int k = 0; k < kIn; k++) gW1[k] = fmaf(d, XS[b * 8 + k], gW1[k]);
      }
    }
    __syncthreads();  // the next chunk overwrites every array
  }

  // ---- one atomic per parameter per block ----
#pragma unroll
  for (int r = 0; r < 4; r++)
#pragma unroll
    for (int c = 0; c < 8; c++) {
      atomicAdd(G + oW3 + (o0 + r) * kH + k0 + c, gW3[r][c]);
      atomicAdd(G + oW2 + (o0 + r) * kH + k0 + c, gW2[r][c]);
    }
  if (t < kH) {
#pragma unroll
    for (int k = 0; k < kIn; k++) atomicAdd(G + oW1 + t * kIn + k, gW1[k]);
    atomicAdd(G + oB1 + t, gB1);
    atomicAdd(G + oB2 + t, gB2);
    atomicAdd(G + oB3 + t, gB3);
    atomicAdd(G + oW4 + t, gW4);
  } else if (t == kH) {
    atomicAdd(G + oB4, gB4);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
  if (lane == 0) atomicAdd(loss, lsum);
}

// Adam step (bias-corrected) on all parameters.
__global__ void mlp_adam_kernel(float *P, const float *G, float *M, float *V, int np, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float g = G[k];
  const float m = b1 * M[k] + (1.f - b1) * g;
  const float v = b2 * V[k] + (1.f - b2) * g * g;
  M[k] = m;
  V[k] = v;
  P[k] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

constexpr size_t kBwdSmem = sizeof(float) * kBwdFloats;

uint64_t splitmix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

struct sapb_mlp {
  sapb_dev *d = nullptr;
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr, *loss = nullptr;
  float *X = nullptr, *T = nullptr, *Y = nullptr;  // device staging
  int cap = 0;
  int steps = 0;
};

#define MK(m, call)                                                                        \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return sapb_fail((m)->d, SAPB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));       \
  } while (0)

// persistent backward grid: one block per SM at most (its shared memory
// allows one), never more blocks than chunks of 128 samples
static int bwd_grid(const sapb_mlp *m, int n) {
  const int chunks = (n + kMB - 1) / kMB;
  return std::max(1, std::min(chunks, m->d->num_sms));
}

static int mlp_reserve(sapb_mlp *m, int n) {
  if (n <= m->cap) return SAPB_OK;
  const int cap = n + n / 2 + 1024;
  cudaFree(m->X);
  cudaFree(m->T);
  cudaFree(m->Y);
  m->X = m->T = m->Y = nullptr;
  m->cap = 0;
  if (cudaMalloc(&m->X, sizeof(float) * kPropIn * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&m->T, sizeof(float) * (size_t)cap) != cudaSuccess ||
      cudaMalloc(&m->Y, sizeof(float) * (size_t)cap) != cudaSuccess) {
    cudaGetLastError();
    return sapb_fail(m->d, SAPB_ENOMEM, "mlp staging for %d samples", cap);
  }
  m->cap = cap;
  return SAPB_OK;
}

extern "C" {

int sapb_mlp_num_params(void) { return kNP; }

int sapb_mlp_create(sapb_dev *d, unsigned long long seed, sapb_mlp **out) {
  if (!d || !out) return sapb_fail(d, SAPB_EINVAL, "bad arguments");
  *out = nullptr;
  sapb_mlp *m = new (std::nothrow) sapb_mlp();
  if (!m) return sapb_fail(d, SAPB_ENOMEM, "host allocation");
  m->d = d;
  if (cudaSetDevice(d->device) != cudaSuccess ||
      cudaMalloc(&m->P, sizeof(float) * kNP) != cudaSuccess ||
      cudaMalloc(&m->G, sizeof(float) * kNP) != cudaSuccess ||
      cudaMalloc(&m->M, sizeof(float) * kNP) != cudaSuccess ||
      cudaMalloc(&m->V, sizeof(float) * kNP) != cudaSuccess ||
      cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess ||
      cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kBwdSmem) != cudaSuccess) {
    cudaGetLastError();
    sapb_mlp_destroy(m);
    return sapb_fail(d, SAPB_ENOMEM, "mlp parameter buffers");
  }
  // He-uniform hidden layers, Glorot-uniform output layer, zero biases,
  // from a seeded splitmix64 stream.
  std::vector<float> p(kNP, 0.f);
  uint64_t s = seed;
  auto uni = [&](float lim) {
    const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
    return (float)((2.0 * u - 1.0) * lim);
  };
  for (int k = 0; k < kH * kIn; k++) p[oW1 + k] = uni(sqrtf(6.f / kIn));
  for (int k = 0; k < kH * kH; k++) p[oW2 + k] = uni(sqrtf(6.f / kH));
  for (int k = 0; k < kH * kH; k++) p[oW3 + k] = uni(sqrtf(6.f / kH));
  for (int k = 0; k < kH; k++) p[oW4 + k] = uni(sqrtf(6.f / (kH + 1)));
  int rc = sapb_mlp_set_params(m, p.data());
  if (rc) {
    sapb_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return SAPB_OK;
}

int sapb_mlp_destroy(sapb_mlp *m) {
  if (!m) return SAPB_OK;
  cudaFree(m->P);
  cudaFree(m->G);
  cudaFree(m->M);
  cudaFree(m->V);
  cudaFree(m->loss);
  cudaFree(m->X);
  cudaFree(m->T);
  cudaFree(m->Y);
  delete m;
  return SAPB_OK;
}

int sapb_mlp_set_params(sapb_mlp *m, const float *params) {
  if (!m || !params) return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  MK(m, cudaSetDevice(m->d->device));
  MK(m, cudaMemcpy(m->P, params, sizeof(float) * kNP, cudaMemcpyHostToDevice));
  MK(m, cudaMemset(m->M, 0, sizeof(float) * kNP));
  MK(m, cudaMemset(m->V, 0, sizeof(float) * kNP));
  m->steps = 0;
  return SAPB_OK;
}

int sapb_mlp_get_params(sapb_mlp *m, float *params) {
  if (!m || !params) return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  MK(m, cudaSetDevice(m->d->device));
  MK(m, cudaMemcpy(params, m->P, sizeof(float) * kNP, cudaMemcpyDeviceToHost));
  return SAPB_OK;
}

int sapb_mlp_forward(sapb_mlp *m, int n, const float *x, float *y) {
  if (!m || n < 0 || (n && (!x || !y))) return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  if (n == 0) return SAPB_OK;
  MK(m, cudaSetDevice(m->d->device));
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  cudaStream_t st = m->d->stream;
  MK(m, cudaMemcpyAsync(m->X, x, sizeof(float) * kIn * (size_t)n, cudaMemcpyHostToDevice, st));
  mlp_forward_kernel<<<(n + 127) / 128, 128, 0, st>>>(m->P, n, m->X, m->Y);
  MK(m, cudaGetLastError());
  MK(m, cudaMemcpyAsync(y, m->Y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st));
  MK(m, cudaStreamSynchronize(st));
  return SAPB_OK;
}

int sapb_mlp_propose(sapb_mlp *m, int n, const float *in, const float *mu, const float *sd,
                     float target, float max_down, float max_up, float clip, float *h2_out) {
  if (!m || n < 0 || (n && (!in || !mu || !sd || !h2_out)) || !(target > 0.f))
    return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  if (n == 0) return SAPB_OK;
  MK(m, cudaSetDevice(m->d->device));
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  MlpScale sc;
  for (int k = 0; k < kIn; k++) {
    sc.mu[k] = mu[k];
    sc.sd[k] = sd[k];
  }
  sc.target = target;
  sc.max_down = max_down;
  sc.max_up = max_up;
  sc.clip = clip;
  cudaStream_t st = m->d->stream;
  MK(m, cudaMemcpyAsync(m->X, in, sizeof(float) * kPropIn * (size_t)n, cudaMemcpyHostToDevice, st));
  mlp_propose_kernel<<<(n + 127) / 128, 128, 0, st>>>(m->P, n, m->X, sc, m->Y);
  MK(m, cudaGetLastError());
  MK(m, cudaMemcpyAsync(h2_out, m->Y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, st));
  MK(m, cudaStreamSynchronize(st));
  return SAPB_OK;
}

int sapb_mlp_gradient(sapb_mlp *m, int n, const float *x, const float *t, float *grad,
                      float *loss) {
  if (!m || n <= 0 || !x || !t) return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  MK(m, cudaSetDevice(m->d->device));
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  cudaStream_t st = m->d->stream;
  MK(m, cudaMemcpyAsync(m->X, x, sizeof(float) * kIn * (size_t)n, cudaMemcpyHostToDevice, st));
  MK(m, cudaMemcpyAsync(m->T, t, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st));
  MK(m, cudaMemsetAsync(m->G, 0, sizeof(float) * kNP, st));
  MK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), st));
  mlp_backward_kernel<<<bwd_grid(m, n), kMB, kBwdSmem, st>>>(m->P, n, m->X, m->T, m->G,
                                                                 m->loss);
  MK(m, cudaGetLastError());
  if (grad) MK(m, cudaMemcpyAsync(grad, m->G, sizeof(float) * kNP, cudaMemcpyDeviceToHost, st));
  float l = 0.f;
  MK(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  MK(m, cudaStreamSynchronize(st));
  if (loss) *loss = l;
  return SAPB_OK;
}

int sapb_mlp_train(sapb_mlp *m, int n, const float *x, const float *t, int epochs, float lr,
                   float *loss) {
  if (!m || n <= 0 || epochs <= 0) return sapb_fail(m ? m->d : nullptr, SAPB_EINVAL, "bad arguments");
  MK(m, cudaSetDevice(m->d->device));
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  cudaStream_t st = m->d->stream;
  MK(m, cudaMemcpyAsync(m->X, x, sizeof(float) * kIn * (size_t)n, cudaMemcpyHostToDevice, st));
  MK(m, cudaMemcpyAsync(m->T, t, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st));
  for (int e = 0; e < epochs; e++) {
    MK(m, cudaMemsetAsync(m->G, 0, sizeof(float) * kNP, st));
    MK(m, cudaMemsetAsync(m->loss, 0, sizeof(float), st));
    mlp_backward_kernel<<<bwd_grid(m, n), kMB, kBwdSmem, st>>>(m->P, n, m->X, m->T, m->G,
                                                                   m->loss);
    m->steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)m->steps), c2 = 1.f - powf(b2, (float)m->steps);
    mlp_adam_kernel<<<(kNP + 255) / 256, 256, 0, st>>>(m->P, m->G, m->M, m->V, kNP, lr, b1, b2,
                                                       1e-8f, c1, c2);
    MK(m, cudaGetLastError());
  }
  float l = 0.f;
  MK(m, cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  MK(m, cudaStreamSynchronize(st));
  if (loss) *loss = l;  // loss before the last update
  return SAPB_OK;
}

}  // extern "C"
