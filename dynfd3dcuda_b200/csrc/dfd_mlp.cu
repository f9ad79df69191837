// Training and batch inference of the learned initial guess of the rate-and-state Newton
// solve (the reference solves f(x) = 2 V0 e^{-psi/a} sinh x + coef x - Vhat = 0 from a
// guess built on the previous slip rate, trial_ratestate.cu:20-57 and :695).
//
// Network: 4 -> 32 -> 32 -> 1, tanh hidden layers, FP32.  Inputs (psi/a, log10 Vhat,
// log10 coef, a) are standardised by stored means/scales; the output, de-standardised,
// is the residual x* - asinh(Vhat e^{psi/a} / (2 V0)), i.e. the correction of the exact
// root of the problem without the radiation-damping term coef*x.
//
// Parameter vector (DFD_MLP_PARAMS floats):
//   W1[32][4] b1[32] W2[32][32] b2[32] W3[32] b3 | mu[4] sd[4] ymu ysd
// the first DFD_MLP_TRAINABLE are trained; the last 10 are the standardisation.
//
// Training is plain minibatch Adam on the mean squared error of the standardised
// residual.  One block of 64 threads takes 64 samples: each thread runs the forward and
// backward pass of its sample and keeps its activations and deltas in shared memory; the
// weight gradients are then batch contractions over those shared arrays (dW2 = dH2^T H1
// etc.), accumulated into the global gradient with one atomic add per parameter and block.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/dfd_b200.h"
#include "dfd_mlp.cuh"

namespace dfd {
namespace mlp {

constexpr int H = 32;
constexpr int OW1 = 0, OB1 = 128, OW2 = 160, OB2 = 1184, OW3 = 1216, OB3 = 1248;
constexpr int NTRAIN = 1249;  // == DFD_MLP_TRAINABLE
constexpr int OMU = 1249, OSD = 1253, OYMU = 1257, OYSD = 1258;
constexpr int NPAR = 1259;  // == DFD_MLP_PARAMS
constexpr int BS = 64;  // samples per block (its activations and deltas fit the static shared memory)
static_assert(NTRAIN == DFD_MLP_TRAINABLE && NPAR == DFD_MLP_PARAMS, "parameter layout");

// forward of one sample; h1, h2 are the hidden activations, returns the standardised output
__device__ __forceinline__ float forward(const float* __restrict__ w, const float* xin, float* h1, float* h2) {
  float x[4];
#pragma unroll
  for (int c = 0; c < 4; c++) x[c] = (xin[c] - w[OMU + c]) / w[OSD + c];
#pragma unroll
  for (int r = 0; r < H; r++) {
    float s = w[OB1 + r];
#pragma unroll
    for (int c = 0; c < 4; c++) s = fmaf(w[OW1 + r * 4 + c], x[c], s);
    h1[r] = tanhf(s);
  }
  float out = w[OB3];
  for (int r = 0; r < H; r++) {
    float s = w[OB2 + r];
#pragma unroll
    for (int c = 0; c < H; c++) s = fmaf(w[OW2 + r * H + c], h1[c], s);
    h2[r] = tanhf(s);
    out = fmaf(w[OW3 + r], h2[r], out);
  }
  return out;
}

__global__ void forward_kernel(const float* __restrict__ w, const float* __restrict__ X, int n, float* y) {
  __shared__ float sw[NPAR];
  for (int p = threadIdx.x; p < NPAR; p += blockDim.x) sw[p] = w[p];
  __syncthreads();
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float h1[H], h2[H];
  float xin[4] = {X[4 * t], X[4 * t + 1], X[4 * t + 2], X[4 * t + 3]};
  y[t] = forward(sw, xin, h1, h2);  // standardised output
}

// The node kernel's inference paths on a batch (n a multiple of 32): tc 0 the per-thread
// network, tc 1 the tensor-core network of a full warp; de-standardised residuals.
__global__ void __launch_bounds__(128) forward_node_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                            int n, int tc, float* y) {
  __shared__ __align__(16) float sw[NPAR];
  for (int p = threadIdx.x; p < NPAR; p += blockDim.x) sw[p] = w[p];
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;  // n is a multiple of 32: warps stay whole
  const float xin[4] = {X[4 * t], X[4 * t + 1], X[4 * t + 2], X[4 * t + 3]};
  y[t] = tc ? mlp_residual_warp(sw, xin) : mlp_residual(sw, xin);
}

// Gradient of the mean squared error over n samples (sample s = idx[s0 + b] for b < nb)
// accumulated into g[NTRAIN] (scaled by 1/n_total) and the loss sum into *loss.
__global__ void __launch_bounds__(BS) grad_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                  const float* __restrict__ Y, const int* __restrict__ idx, int s0,
                                                  int nb, float inv_n, float* g, double* loss) {
  __shared__ float sw[NPAR];
  __shared__ float xs[BS][4];    // standardised inputs
  __shared__ float a1[BS][H];    // hidden 1 activations
  __shared__ float a2[BS][H];    // hidden 2 activations
  __shared__ float d1[BS][H];    // deltas of hidden 1 pre-activations
  __shared__ float d2[BS][H];    // deltas of hidden 2 pre-activations
  __shared__ float dout[BS];     // output deltas
  __shared__ float red[BS / 32];
  for (int p = threadIdx.x; p < NPAR; p += BS) sw[p] = w[p];
  __syncthreads();
  const int b = threadIdx.x;
  const int gb = blockIdx.x * BS + b;  // position in the batch
  float l = 0.0f;
  if (gb < nb) {
    const int s = idx ? idx[s0 + gb] : s0 + gb;
    float xin[4] = {X[4 * s], X[4 * s + 1], X[4 * s + 2], X[4 * s + 3]};
    float h1[H], h2[H];
    float out = forward(sw, xin, h1, h2);
    float yt = (Y[s] - sw[OYMU]) / sw[OYSD];
    float e = out - yt;
    l = e * e;
    float go = 2.0f * e * inv_n;
    dout[b] = go;
#pragma unroll
    for (int c = 0; c < 4; c++) xs[b][c] = (xin[c] - sw[OMU + c]) / sw[OSD + c];
    float g2[H];
#pragma unroll
    for (int r = 0; r < H; r++) {
      a1[b][r] = h1[r];
      a2[b][r] = h2[r];
      g2[r] = go * sw[OW3 + r] * (1.0f - h2[r] * h2[r]);
      d2[b][r] = g2[r];
    }
#pragma unroll
    for (int c = 0; c < H; c++) {
      float s = 0.0f;
#pragma unroll
      for (int r = 0; r < H; r++) s = fmaf(sw[OW2 + r * H + c], g2[r], s);
      d1[b][c] = s * (1.0f - h1[c] * h1[c]);
    }
  } else {
    dout[b] = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; c++) xs[b][c] = 0.0f;
    for (int r = 0; r < H; r++) { a1[b][r] = 0.0f; a2[b][r] = 0.0f; d1[b][r] = 0.0f; d2[b][r] = 0.0f; }
  }
  // loss: warp then block reduction
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((b & 31) == 0) red[b >> 5] = l;
  __syncthreads();
  if (b == 0) {
    float t = 0.0f;
    for (int i = 0; i < BS / 32; i++) t += red[i];
    atomicAdd(loss, (double)t);
  }
  // weight gradients as contractions over the block's samples; parameter p per thread
  for (int p = b; p < NTRAIN; p += BS) {
    float acc = 0.0f;
    if (p < OB1) {                      // W1[r][c] = sum d1[r] x[c]
      int r = p / 4, c = p % 4;
      for (int i = 0; i < BS; i++) acc = fmaf(d1[i][r], xs[i][c], acc);
    } else if (p < OW2) {               // b1[r]
      int r = p - OB1;
      for (int i = 0; i < BS; i++) acc += d1[i][r];
    } else if (p < OB2) {               // W2[r][c] = sum d2[r] h1[c]
      int q = p - OW2, r = q / H, c = q % H;
      for (int i = 0; i < BS; i++) acc = fmaf(d2[i][r], a1[i][c], acc);
    } else if (p < OW3) {               // b2[r]
      int r = p - OB2;
      for (int i = 0; i < BS; i++) acc += d2[i][r];
    } else if (p < OB3) {               // W3[r] = sum dout h2[r]
      int r = p - OW3;
      for (int i = 0; i < BS; i++) acc = fmaf(dout[i], a2[i][r], acc);
    } else {                            // b3
      for (int i = 0; i < BS; i++) acc += dout[i];
    }
    atomicAdd(g + p, acc);
  }
}

__global__ void adam_kernel(float* w, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NTRAIN) return;
  float gp = g[p];
  float mp = b1 * m[p] + (1.0f - b1) * gp;
  float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
  m[p] = mp;
  v[p] = vp;
  w[p] -= lr * (mp / c1) / (sqrtf(vp / c2) + eps);
}

}  // namespace mlp
}  // namespace dfd

using namespace dfd::mlp;

namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  template <typename T>
  T* get() { return static_cast<T*>(p); }
};
#define MCK(call)                                   \
  do {                                              \
    if ((call) != cudaSuccess) return DFD_ERR_CUDA; \
  } while (0)
}  // namespace

extern "C" {

int dfd_mlp_init(float* w, unsigned seed, const float* x_mean, const float* x_scale, float y_mean, float y_scale) {
  if (!w || !x_mean || !x_scale || !(y_scale > 0)) return DFD_ERR_PARAM;
  // Xavier-uniform weights from a 64-bit LCG, zero biases
  uint64_t s = 0x9E3779B97F4A7C15ull ^ (uint64_t)seed;
  auto uni = [&]() {
    s = s * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((s >> 40) * (1.0 / 16777216.0)) * 2.0f - 1.0f;
  };
  memset(w, 0, sizeof(float) * NPAR);
  float a1 = sqrtf(6.0f / (4 + H)), a2 = sqrtf(6.0f / (H + H)), a3 = sqrtf(6.0f / (H + 1));
  for (int i = 0; i < 128; i++) w[OW1 + i] = a1 * uni();
  for (int i = 0; i < 1024; i++) w[OW2 + i] = a2 * uni();
  for (int i = 0; i < 32; i++) w[OW3 + i] = a3 * uni();
  for (int c = 0; c < 4; c++) {
    if (!(x_scale[c] > 0)) return DFD_ERR_PARAM;
    w[OMU + c] = x_mean[c];
    w[OSD + c] = x_scale[c];
  }
  w[OYMU] = y_mean;
  w[OYSD] = y_scale;
  return DFD_OK;
}

int dfd_mlp_forward(const float* w, const float* x, int n, float* y) {
  if (!w || !x || !y || n <= 0) return DFD_ERR_PARAM;
  DevBuf dw, dx, dy;
  MCK(cudaMalloc(&dw.p, sizeof(float) * NPAR));
  MCK(cudaMalloc(&dx.p, sizeof(float) * 4 * (size_t)n));
  MCK(cudaMalloc(&dy.p, sizeof(float) * (size_t)n));
  MCK(cudaMemcpy(dw.p, w, sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dx.p, x, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice));
  forward_kernel<<<(n + 255) / 256, 256>>>(dw.get<float>(), dx.get<float>(), n, dy.get<float>());
  MCK(cudaGetLastError());
  MCK(cudaMemcpy(y, dy.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
  // de-standardise
  for (int i = 0; i < n; i++) y[i] = y[i] * w[OYSD] + w[OYMU];
  return DFD_OK;
}

int dfd_mlp_forward_node(const float* w, const float* x, int n, int tensor_cores, float* y) {
  if (!w || !x || !y || n <= 0) return DFD_ERR_PARAM;
  const int np = (n + 31) / 32 * 32;  // whole warps: the rows past n repeat the last input
  std::vector<float> xp(4 * (size_t)np);
  memcpy(xp.data(), x, sizeof(float) * 4 * (size_t)n);
  for (int i = n; i < np; i++) memcpy(&xp[4 * (size_t)i], x + 4 * (size_t)(n - 1), 4 * sizeof(float));
  DevBuf dw, dx, dy;
  MCK(cudaMalloc(&dw.p, sizeof(float) * NPAR));
  MCK(cudaMalloc(&dx.p, sizeof(float) * 4 * (size_t)np));
  MCK(cudaMalloc(&dy.p, sizeof(float) * (size_t)np));
  MCK(cudaMemcpy(dw.p, w, sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dx.p, xp.data(), sizeof(float) * 4 * (size_t)np, cudaMemcpyHostToDevice));
  forward_node_kernel<<<(np + 127) / 128, 128>>>(dw.get<float>(), dx.get<float>(), np, tensor_cores ? 1 : 0,
                                                 dy.get<float>());
  MCK(cudaGetLastError());
  MCK(cudaMemcpy(y, dy.p, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost));
  return DFD_OK;
}

int dfd_mlp_loss_grad(const float* w, const float* x, const float* y, int n, double* loss, float* grad) {
  if (!w || !x || !y || n <= 0) return DFD_ERR_PARAM;
  DevBuf dw, dx, dy, dg, dl;
  MCK(cudaMalloc(&dw.p, sizeof(float) * NPAR));
  MCK(cudaMalloc(&dx.p, sizeof(float) * 4 * (size_t)n));
  MCK(cudaMalloc(&dy.p, sizeof(float) * (size_t)n));
  MCK(cudaMalloc(&dg.p, sizeof(float) * NTRAIN));
  MCK(cudaMalloc(&dl.p, sizeof(double)));
  MCK(cudaMemcpy(dw.p, w, sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dx.p, x, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dy.p, y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
  MCK(cudaMemset(dg.p, 0, sizeof(float) * NTRAIN));
  MCK(cudaMemset(dl.p, 0, sizeof(double)));
  grad_kernel<<<(n + BS - 1) / BS, BS>>>(dw.get<float>(), dx.get<float>(), dy.get<float>(), nullptr, 0, n,
                                         1.0f / (float)n, dg.get<float>(), dl.get<double>());
  MCK(cudaGetLastError());
  double l = 0;
  MCK(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
  if (loss) *loss = l / n;
  if (grad) MCK(cudaMemcpy(grad, dg.p, sizeof(float) * NTRAIN, cudaMemcpyDeviceToHost));
  return DFD_OK;
}

int dfd_mlp_train(const float* x, const float* y, int n, int epochs, int batch, float lr, unsigned seed, float* w,
                  float* loss_per_epoch) {
  if (!x || !y || !w || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0)) return DFD_ERR_PARAM;
  DevBuf dw, dx, dy, dg, dm, dv, dl, di;
  MCK(cudaMalloc(&dw.p, sizeof(float) * NPAR));
  MCK(cudaMalloc(&dx.p, sizeof(float) * 4 * (size_t)n));
  MCK(cudaMalloc(&dy.p, sizeof(float) * (size_t)n));
  MCK(cudaMalloc(&dg.p, sizeof(float) * NTRAIN));
  MCK(cudaMalloc(&dm.p, sizeof(float) * NTRAIN));
  MCK(cudaMalloc(&dv.p, sizeof(float) * NTRAIN));
  MCK(cudaMalloc(&dl.p, sizeof(double)));
  MCK(cudaMalloc(&di.p, sizeof(int) * (size_t)n));
  MCK(cudaMemcpy(dw.p, w, sizeof(float) * NPAR, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dx.p, x, sizeof(float) * 4 * (size_t)n, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(dy.p, y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
  MCK(cudaMemset(dm.p, 0, sizeof(float) * NTRAIN));
  MCK(cudaMemset(dv.p, 0, sizeof(float) * NTRAIN));
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  uint64_t s = 0xD1B54A32D192ED03ull ^ (uint64_t)seed;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  long long t = 0;
  for (int e = 0; e < epochs; e++) {
    for (int i = n - 1; i > 0; i--) {  // Fisher-Yates shuffle
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      int j = (int)((s >> 33) % (uint64_t)(i + 1));
      std::swap(perm[i], perm[j]);
    }
    MCK(cudaMemcpy(di.p, perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    MCK(cudaMemset(dl.p, 0, sizeof(double)));
    for (int s0 = 0; s0 < n; s0 += batch) {
      int nb = std::min(batch, n - s0);
      MCK(cudaMemsetAsync(dg.p, 0, sizeof(float) * NTRAIN));
      grad_kernel<<<(nb + BS - 1) / BS, BS>>>(dw.get<float>(), dx.get<float>(), dy.get<float>(), di.get<int>(), s0,
                                              nb, 1.0f / (float)nb, dg.get<float>(), dl.get<double>());
      t++;
      float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
      adam_kernel<<<(NTRAIN + 255) / 256, 256>>>(dw.get<float>(), dg.get<float>(), dm.get<float>(), dv.get<float>(),
                                                 lr, b1, b2, eps, c1, c2);
    }
    MCK(cudaGetLastError());
    double l = 0;
    MCK(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
    if (loss_per_epoch) loss_per_epoch[e] = (float)(l / n);
  }
  MCK(cudaMemcpy(w, dw.p, sizeof(float) * NTRAIN, cudaMemcpyDeviceToHost));
  return DFD_OK;
}

}  // extern "C"
