// Inference of the learned initial guess of the rate-and-state Newton solve, shared by
// the fault node kernel (dfd_fault.cu) and the batch inference entry (dfd_mlp.cu).
#pragma once
#include <cuda_fp16.h>

namespace dfd {

// Learned initial guess: MLP 4 -> 32 -> 32 -> 1 (tanh) on the standardised inputs; the
// de-standardised output is the residual x* - asinh(Vhat e^{psi/a} / (2 V0)).  Weight
// layout (dfd_mlp.cu): W1[32][4] b1[32] W2[32][32] b2[32] W3[32] b3 mu[4] sd[4] ymu ysd.
// The hidden activations use the hardware tanh approximation (absolute error ~5e-4): the
// output is scaled by the residual's small standard deviation, and the Newton correction
// evaluated at the guess (the residual test of the node kernel) removes what is left.
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float mlp_residual(const float* w, const float* xin) {
  const float4* W1 = reinterpret_cast<const float4*>(w);  // rows of 4
  const float* b1 = w + 128;
  const float4* W2 = reinterpret_cast<const float4*>(w + 160);
  const float* b2 = w + 1184;
  const float* W3 = w + 1216;
  const float* b3 = w + 1248;
  const float* mu = b3 + 1;
  const float* sd = mu + 4;
  const float* ys = sd + 4;
  float x[4];
#pragma unroll
  for (int c = 0; c < 4; c++) x[c] = (xin[c] - mu[c]) / sd[c];
  float h1[32];
#pragma unroll
  for (int r = 0; r < 32; r++) {
    const float4 wr = W1[r];
    float s = b1[r];
    s = fmaf(wr.x, x[0], s); s = fmaf(wr.y, x[1], s); s = fmaf(wr.z, x[2], s); s = fmaf(wr.w, x[3], s);
    h1[r] = tanh_fast(s);
  }
  float out = *b3;
#pragma unroll 4
  for (int r = 0; r < 32; r++) {
    float s = b2[r];
#pragma unroll
    for (int c = 0; c < 8; c++) {
      const float4 wv = W2[r * 8 + c];
      s = fmaf(wv.x, h1[4 * c], s); s = fmaf(wv.y, h1[4 * c + 1], s);
      s = fmaf(wv.z, h1[4 * c + 2], s); s = fmaf(wv.w, h1[4 * c + 3], s);
    }
    out = fmaf(W3[r], tanh_fast(s), out);
  }
  return out * ys[1] + ys[0];
}

// The same network for the 32 nodes of a full warp at once, every layer on the tensor
// cores: mma.sync m16n8k16 with FP16 operands and FP32 accumulation, the warp's 32 nodes
// as the two 16-row tiles of A.
//   layer 1: A = standardised inputs with a constant 1 for the bias (k = 0..4 of 16),
//            B[k][n] = W1[n][k], b1[n] at k = 4;
//   layer 2: A = tanh of the layer-1 accumulators (an m16n8 accumulator pair is laid out
//            exactly as the A fragment of the next k16 step, so no data moves between
//            lanes), B[k][n] = W2[n][k], accumulators start at b2;
//   layer 3: B[k][0] = W3[k], the other seven columns zero; column 0 of the accumulator
//            (lanes 4 g) holds the outputs of rows g and g + 8 of each tile.
// Lane 4 g + t holds rows g, g+8 (tile 0) and g+16, g+24 (tile 1).  The FP16 rounding of
// activations and weights (relative 2^-11) matches the tanh approximation the per-thread
// network already carries.  All 32 lanes must be here together (the caller checks the
// warp is full).
__device__ __forceinline__ unsigned pack_h2(float lo, float hi) {
  const __half2 h = __floats2half2_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&h);
}
__device__ __forceinline__ void mma16816(float* c, const unsigned* a, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ float mlp_residual_warp(const float* w, const float* xin) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const float* W1 = w;
  const float* b1 = w + 128;
  const float* W2 = w + 160;
  const float* b2 = w + 1184;
  const float* W3 = w + 1216;
  const float* b3 = w + 1248;
  const float* mu = b3 + 1;
  const float* sd = mu + 4;
  const float* ys = sd + 4;
  float x[4];
#pragma unroll
  for (int c = 0; c < 4; c++) x[c] = (xin[c] - mu[c]) / sd[c];
  // ---- layer 1.  A fragment of tile mi: reg 0 row g (k = 2t, 2t+1), reg 1 row g+8,
  // regs 2, 3 (k = 2t+8, 2t+9) zero.  Lanes t = 0, 1 carry inputs 2t, 2t+1, lane t = 2 the
  // bias input 1.
  // every lane offers its inputs as two FP16 pairs; a shuffle returns the source lane's
  // pair, and lane t keeps the one it holds (t = 0: inputs 0, 1; t = 1: inputs 2, 3)
  const unsigned p01 = pack_h2(x[0], x[1]), p23 = pack_h2(x[2], x[3]);
  unsigned a1[2][4];
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int src = g + 8 * h + 16 * mi;
      const unsigned u01 = __shfl_sync(FULL, p01, src), u23 = __shfl_sync(FULL, p23, src);
      a1[mi][h] = t == 0 ? u01 : t == 1 ? u23 : t == 2 ? pack_h2(1.0f, 0.0f) : 0u;
      a1[mi][h + 2] = 0u;
    }
  float c1[2][4][4];
#pragma unroll
  for (int ni = 0; ni < 4; ni++) {
    const int n = 8 * ni + g;
    const unsigned bq = t < 2 ? pack_h2(W1[4 * n + 2 * t], W1[4 * n + 2 * t + 1]) : t == 2 ? pack_h2(b1[n], 0.0f) : 0u;
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
      c1[mi][ni][0] = c1[mi][ni][1] = c1[mi][ni][2] = c1[mi][ni][3] = 0.0f;
      mma16816(c1[mi][ni], a1[mi], bq, 0u);
    }
  }
  // ---- layer 2: the layer-1 accumulators of columns 16 ki .. 16 ki + 15 become the A
  // fragment of k step ki (column tile 2 ki -> regs 0, 1, tile 2 ki + 1 -> regs 2, 3)
  unsigned a2[2][2][4];
#pragma unroll
  for (int mi = 0; mi < 2; mi++)
#pragma unroll
    for (int ki = 0; ki < 2; ki++)
#pragma unroll
      for (int hh = 0; hh < 2; hh++) {
        const float* cc = c1[mi][2 * ki + hh];
        a2[mi][ki][2 * hh] = pack_h2(tanh_fast(cc[0]), tanh_fast(cc[1]));
        a2[mi][ki][2 * hh + 1] = pack_h2(tanh_fast(cc[2]), tanh_fast(cc[3]));
      }
  float c2[2][4][4];
#pragma unroll
  for (int ni = 0; ni < 4; ni++) {
    const float bb0 = b2[8 * ni + 2 * t], bb1 = b2[8 * ni + 2 * t + 1];
#pragma unroll
    for (int mi = 0; mi < 2; mi++) { c2[mi][ni][0] = bb0; c2[mi][ni][1] = bb1; c2[mi][ni][2] = bb0; c2[mi][ni][3] = bb1; }
  }
  // B[k][n] = W2[n][k]: lane holds n = 8 ni + g, k = 16 ki + 2t (+1), (+8, +9)
#pragma unroll
  for (int ni = 0; ni < 4; ni++)
#pragma unroll
    for (int ki = 0; ki < 2; ki++) {
      const float* r = W2 + (8 * ni + g) * 32 + 16 * ki + 2 * t;
      const unsigned bq0 = pack_h2(r[0], r[1]), bq1 = pack_h2(r[8], r[9]);
#pragma unroll
      for (int mi = 0; mi < 2; mi++) mma16816(c2[mi][ni], a2[mi][ki], bq0, bq1);
    }
  // ---- layer 3: tanh of the layer-2 accumulators as A again, W3 in column 0 of B
  float c3[2][4];
#pragma unroll
  for (int mi = 0; mi < 2; mi++) c3[mi][0] = c3[mi][1] = c3[mi][2] = c3[mi][3] = 0.0f;
#pragma unroll
  for (int ki = 0; ki < 2; ki++) {
    const unsigned bq0 = g == 0 ? pack_h2(W3[16 * ki + 2 * t], W3[16 * ki + 2 * t + 1]) : 0u;
    const unsigned bq1 = g == 0 ? pack_h2(W3[16 * ki + 2 * t + 8], W3[16 * ki + 2 * t + 9]) : 0u;
#pragma unroll
    for (int mi = 0; mi < 2; mi++) {
      unsigned a3[4];
#pragma unroll
      for (int hh = 0; hh < 2; hh++) {
        const float* cc = c2[mi][2 * ki + hh];
        a3[2 * hh] = pack_h2(tanh_fast(cc[0]), tanh_fast(cc[1]));
        a3[2 * hh + 1] = pack_h2(tanh_fast(cc[2]), tanh_fast(cc[3]));
      }
      mma16816(c3[mi], a3, bq0, bq1);
    }
  }
  // row L (this lane's node) = 16 mi + 8 hf + g' sits in lane 4 g', element 2 hf of tile mi
  const int src = (lane & 7) * 4, mi = lane >> 4, hf = (lane >> 3) & 1;
  const float r00 = __shfl_sync(FULL, c3[0][0], src), r01 = __shfl_sync(FULL, c3[0][2], src);
  const float r10 = __shfl_sync(FULL, c3[1][0], src), r11 = __shfl_sync(FULL, c3[1][2], src);
  const float out = mi ? (hf ? r11 : r10) : (hf ? r01 : r00);
  return (out + *b3) * ys[1] + ys[0];
}

}  // namespace dfd
