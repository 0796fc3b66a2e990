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

// Gradient of L = 1/(2n) sum (y - t)^2 over the n samples, accumulated into
// G (zeroed by the caller), loss accumulated into *loss.  Block b handles
// samples [128 b, 128 b + 128): activations and deltas are kept transposed
// in shared memory ([unit][sample]) and each weight gradient is the block's
// sum of outer products, added to G with one atomic per parameter.
__global__ void __launch_bounds__(kMB) mlp_backward_kernel(const float *__restrict__ P, int n,
                                                           const float *__restrict__ X,
                                                           const float *__restrict__ T,
                                                           float *__restrict__ G,
                                                           float *__restrict__ loss) {
  extern __shared__ float sm[];
  float *sp = sm;                  // parameters  kNP
  float *XS = sp + kNP;            // [5][128]
  float *H1 = XS + kIn * kMB;      // [64][128]
  float *H2 = H1 + kH * kMB;       // [64][128]
  float *H3 = H2 + kH * kMB;       // [64][128]  (later: delta of layer 2)
  float *D3 = H3 + kH * kMB;       // [64][128]  (later: delta of layer 1)
  float *DY = D3 + kH * kMB;       // [128]
  const int tid = threadIdx.x;
  for (int k = tid; k < kNP; k += kMB) sp[k] = P[k];
  const int i = blockIdx.x * kMB + tid;
  const bool valid = i < n;
  float x[kIn] = {0, 0, 0, 0, 0};
  if (valid)
    for (int k = 0; k < kIn; k++) x[k] = X[(size_t)i * kIn + k];
  __syncthreads();
  float h1[kH], h2[kH], h3[kH];
  const float y = mlp_eval(sp, x, h1, h2, h3);
  const float dy = valid ? (y - T[i]) / (float)n : 0.f;
  if (valid) atomicAdd(loss, 0.5f * (y - T[i]) * (y - T[i]) / (float)n);
  for (int k = 0; k < kIn; k++) XS[k * kMB + tid] = valid ? x[k] : 0.f;
  for (int k = 0; k < kH; k++) {
    H1[k * kMB + tid] = valid ? h1[k] : 0.f;
    H2[k * kMB + tid] = valid ? h2[k] : 0.f;
    H3[k * kMB + tid] = valid ? h3[k] : 0.f;
    // delta of layer 3 pre-activation: dy * W4 * relu'
    D3[k * kMB + tid] = (valid && h3[k] > 0.f) ? dy * sp[oW4 + k] : 0.f;
  }
  DY[tid] = dy;
  __syncthreads();
  // ---- layer 4: W4, b4 ----
  if (tid < kH) {
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s = fmaf(DY[b], H3[tid * kMB + b], s);
    atomicAdd(G + oW4 + tid, s);
  }
  if (tid == kH) {
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s += DY[b];
    atomicAdd(G + oB4, s);
  }
  // ---- layer 3: W3[o][k] += sum_b D3[o][b] H2[k][b], b3 ----
  for (int q = tid; q < kH * kH; q += kMB) {
    const int o = q / kH, k = q % kH;
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s = fmaf(D3[o * kMB + b], H2[k * kMB + b], s);
    atomicAdd(G + oW3 + q, s);
  }
  if (tid < kH) {
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s += D3[tid * kMB + b];
    atomicAdd(G + oB3 + tid, s);
  }
  // delta of layer 2 for this thread's sample: (W3^T d3) * relu'(h2)
  float d2[kH];
  for (int k = 0; k < kH; k++) {
    float s = 0.f;
    for (int o = 0; o < kH; o++) s = fmaf(sp[oW3 + o * kH + k], D3[o * kMB + tid], s);
    d2[k] = h2[k] > 0.f ? s : 0.f;
  }
  __syncthreads();  // everyone is done reading H3 / D3
  float *D2 = H3;
  for (int k = 0; k < kH; k++) D2[k * kMB + tid] = d2[k];
  __syncthreads();
  // ---- layer 2 ----
  for (int q = tid; q < kH * kH; q += kMB) {
    const int o = q / kH, k = q % kH;
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s = fmaf(D2[o * kMB + b], H1[k * kMB + b], s);
    atomicAdd(G + oW2 + q, s);
  }
  if (tid < kH) {
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s += D2[tid * kMB + b];
    atomicAdd(G + oB2 + tid, s);
  }
  float d1[kH];
  for (int k = 0; k < kH; k++) {
    float s = 0.f;
    for (int o = 0; o < kH; o++) s = fmaf(sp[oW2 + o * kH + k], D2[o * kMB + tid], s);
    d1[k] = h1[k] > 0.f ? s : 0.f;
  }
  __syncthreads();
  float *D1 = D3;
  for (int k = 0; k < kH; k++) D1[k * kMB + tid] = d1[k];
  __syncthreads();
  // ---- layer 1 ----
  for (int q = tid; q < kH * kIn; q += kMB) {
    const int o = q / kIn, k = q % kIn;
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s = fmaf(D1[o * kMB + b], XS[k * kMB + b], s);
    atomicAdd(G + oW1 + q, s);
  }
  if (tid < kH) {
    float s = 0.f;
    for (int b = 0; b < kMB; b++) s += D1[tid * kMB + b];
    atomicAdd(G + oB1 + tid, s);
  }
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

constexpr size_t kBwdSmem = sizeof(float) * (kNP + kIn * kMB + 4 * kH * kMB + kMB);

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

static int mlp_reserve(sapb_mlp *m, int n) {
  if (n <= m->cap) return SAPB_OK;
  const int cap = n + n / 2 + 1024;
  cudaFree(m->X);
  cudaFree(m->T);
  cudaFree(m->Y);
  m->X = m->T = m->Y = nullptr;
  m->cap = 0;
  if (cudaMalloc(&m->X, sizeof(float) * kIn * (size_t)cap) != cudaSuccess ||
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
  mlp_backward_kernel<<<(n + kMB - 1) / kMB, kMB, kBwdSmem, st>>>(m->P, n, m->X, m->T, m->G,
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
    mlp_backward_kernel<<<(n + kMB - 1) / kMB, kMB, kBwdSmem, st>>>(m->P, n, m->X, m->T, m->G,
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
