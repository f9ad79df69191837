// Device helpers shared by the volume kernels (dfd_volume.cu, dfd_tile.cu): the
// per-axis velocity-stress terms, the ADE PML update of one face and the RK4 store.
#pragma once
#include "dfd_internal.cuh"

namespace dfd {

// axis contribution of the velocity-stress system for one set of derivatives d[9]
// (Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz) and metric row e (wave.cu:133-141)
__device__ __forceinline__ void axis_terms(const float* d, float e0, float e1, float e2, float lam, float mu,
                                           float rrho, float* D) {
  float l2m = lam + 2.0f * mu;
  D[0] = (d[3] * e0 + d[6] * e1 + d[7] * e2) * rrho;
  D[1] = (d[6] * e0 + d[4] * e1 + d[8] * e2) * rrho;
  D[2] = (d[7] * e0 + d[8] * e1 + d[5] * e2) * rrho;
  D[3] = d[0] * e0 * l2m + d[1] * e1 * lam + d[2] * e2 * lam;
  D[4] = d[0] * e0 * lam + d[1] * e1 * l2m + d[2] * e2 * lam;
  D[5] = d[0] * e0 * lam + d[1] * e1 * lam + d[2] * e2 * l2m;
  D[6] = (d[0] * e1 + d[1] * e0) * mu;
  D[7] = (d[0] * e2 + d[2] * e0) * mu;
  D[8] = (d[1] * e2 + d[2] * e1) * mu;
}

// CALL(K) with the stage irk as the compile-time constant K
#define DFD_BY_STAGE(irk, CALL) \
  do {                          \
    switch (irk) {              \
      case 0: CALL(0); break;   \
      case 1: CALL(1); break;   \
      case 2: CALL(2); break;   \
      default: CALL(3); break;  \
    }                           \
  } while (0)

// Classic RK4 without storing the accumulator at stages 0 and 1.  With step-start value y0
// and stage inputs y1 = y0 + (dt/2) k1, y2 = y0 + (dt/2) k2,
//   y0 + (dt/6) k1 + (dt/3) k2 = y0 + (u + 2 v) / 3,   u = y1 - y0, v = y2 - y0,
// is the accumulator after stage 1, so after stage 2 it is y0 + (u + 2 v) / 3 + rkb h with
// rkb h = (dt/3) k3.  Stages 0 and 1 therefore write no accumulator and stage 1 reads
// none; stage 2 re-reads its node's stage-1 input (the buffer it is about to overwrite)
// and writes the accumulator that stage 3 completes (rk4.cu:20-33 forms the same sums term
// by term).  The increments, not y0, are scaled by the rounded 1/3: (y1 + 2 y2) / 3 would
// scale y0 itself by 1 + 3e-8 every step.  Stored stage inputs carry the sponge factor
// damp, so they are scaled back by rd = 1 / damp (exactly 1 outside the sponge).
__device__ __forceinline__ float rk_rd(float damp) { return damp == 1.0f ? 1.0f : __frcp_rn(damp); }
__device__ __forceinline__ float rk_sum(float y0, float y1, float y2, float rd) {
  return fmaf(2.0f, fmaf(y2, rd, -y0), fmaf(y1, rd, -y0));  // u + 2 v
}
__device__ __forceinline__ float rk_acc(float y0, float s, float rkb, float h) {
  return fmaf(rkb, h, fmaf(s, 1.0f / 3.0f, y0));
}

// The ADE state of a PML face is pointwise, so its three 9-field blocks cycle like the
// volume buffers with the accumulator in the block the stage no longer needs:
//   stage 0: current block 0 (y0)                   -> block 1 = y0 + rka h
//   stage 1: current block 1, y0 in block 0         -> block 2 = y0 + rka h
//   stage 2: current block 2, y0 in 0, y1 in 1      -> block 1 = y0 + rka h, block 2 = acc
//   stage 3: current block 1, acc in block 2        -> block 0 = acc + rkb h
// Between steps block 0 holds the state.  Block of the current value at stage irk:
__host__ __device__ constexpr int aux_cur(int irk) { return irk == 0 ? 0 : irk == 2 ? 2 : 1; }

// ADE state of one PML face for this node, loaded ahead of its use: the current value
// and the registers the stage needs (y0 at stages 1 and 2, y1 at stage 2, the accumulator
// at stage 3), blocks st * 9 apart.
struct PmlState {
  float w[9], s[9], y1[9];
};
// IRK: the stage as a compile-time constant, or -1 to take it from a.irk
template <int IRK>
__device__ __forceinline__ void pml_load(const VolArgs& a, int face, long long qa, long long st, PmlState& ps) {
  const int irk = IRK >= 0 ? IRK : a.irk;
  const long long b9 = 9 * st;
#pragma unroll
  for (int f = 0; f < 9; f++) {
    // the blocks of each stage spelled out: constant multiples of the block stride
    const float* x = a.aux[face] + f * st + qa;
    if (irk == 0) {
      ps.w[f] = x[0];
    } else if (irk == 1) {
      ps.w[f] = x[b9];
      ps.s[f] = x[0];
    } else if (irk == 2) {
      ps.w[f] = x[2 * b9];
      ps.s[f] = x[0];
      ps.y1[f] = x[b9];
    } else {
      ps.w[f] = x[b9];
      ps.s[f] = x[2 * b9];
    }
  }
}

// PML auxiliary update of one face for this node from its loaded state: accumulates
// -aux/beta into p[] and advances the state with the RK4 blocks above (pmlx.cu:165-208,
// rk4.cu:208-255).
template <int IRK>
__device__ __forceinline__ void pml_update(const VolArgs& a, int face, long long qa, long long st, float rb, float b,
                                           float dd, float al, const float* Dv, const float* dzv, float ez0,
                                           float ez1, float ez2, float lam, float mu, const PmlState& ps,
                                           float* p) {
  const int irk = IRK >= 0 ? IRK : a.irk;
  const long long b9 = 9 * st;
  float ad = -(al + dd);
  float add[6];
  if (dzv) {
    float l2m = lam + 2.0f * mu, c = dd * b;
    add[0] = c * (l2m * ez0 * dzv[0] + lam * ez1 * dzv[1] + lam * ez2 * dzv[2]);
    add[1] = c * (lam * ez0 * dzv[0] + l2m * ez1 * dzv[1] + lam * ez2 * dzv[2]);
    add[2] = c * (lam * ez0 * dzv[0] + lam * ez1 * dzv[1] + l2m * ez2 * dzv[2]);
    add[3] = c * mu * (ez1 * dzv[0] + ez0 * dzv[1]);
    add[4] = c * mu * (ez2 * dzv[0] + ez0 * dzv[2]);
    add[5] = c * mu * (ez2 * dzv[1] + ez1 * dzv[2]);
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    float* x = a.aux[face] + f * st + qa;
    p[f] += -ps.w[f] * rb;
    float h = ad * ps.w[f] + dd * Dv[f];
    if (dzv && f >= 3) h += add[f - 3];
    if (irk == 0) {
      x[b9] = fmaf(a.rka, h, ps.w[f]);
    } else if (irk == 1) {
      x[2 * b9] = fmaf(a.rka, h, ps.s[f]);
    } else if (irk == 2) {
      x[2 * b9] = rk_acc(ps.s[f], rk_sum(ps.s[f], ps.y1[f], ps.w[f], 1.0f), a.rkb, h);
      x[b9] = fmaf(a.rka, h, ps.s[f]);
    } else {
      x[0] = fmaf(a.rkb, h, ps.s[f]);
    }
  }
}

// Both steps at once: every load of the face precedes every store (the compiler cannot
// prove the blocks distinct, and a load issued after a store would wait for a full
// memory round trip per field).
template <int IRK>
__device__ __forceinline__ void pml_face(const VolArgs& a, int face, long long qa, long long st, float rb, float b,
                                         float dd, float al, const float* Dv, const float* dzv, float ez0,
                                         float ez1, float ez2, float lam, float mu, float* p) {
  PmlState ps;
  pml_load<IRK>(a, face, qa, st, ps);
  pml_update<IRK>(a, face, qa, st, rb, b, dd, al, Dv, dzv, ez0, ez1, ez2, lam, mu, ps, p);
}

// RK4 update of the nine fields of node q with right-hand side h (+ p), then the sponge
// factor (rk4.cu:20-33, cerjan.cu:166-200); the accumulator only at stages 2 and 3 (rk_acc).
// Every load precedes every store.
template <int IRK>
__device__ __forceinline__ void rk_store(const VolArgs& a, long long q, const float* h, const float* p,
                                         float damp) {
  const int irk = IRK >= 0 ? IRK : a.irk;
  const long long n = a.d.nxyz;
  const float rd = irk == 2 ? rk_rd(damp) : 1.0f;
  float r0[9], r1[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    if (irk == 0) {
      r0[f] = __ldg(a.Win + x);
    } else if (irk == 1) {
      r0[f] = __ldg(a.W0 + x);
    } else if (irk == 2) {
      r0[f] = __ldg(a.W0 + x);
      r1[f] = rk_sum(r0[f], a.Wout[x], __ldg(a.Win + x), rd);  // the stage-1 input, overwritten below
    } else {
      r1[f] = a.T[x];
    }
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    const float hf = p ? h[f] + p[f] : h[f];
    float w;
    if (irk < 2) {
      w = fmaf(a.rka, hf, r0[f]);
    } else if (irk == 2) {
      a.T[x] = rk_acc(r0[f], r1[f], a.rkb, hf);
      w = fmaf(a.rka, hf, r0[f]);
    } else {
      w = fmaf(a.rkb, hf, r1[f]);
    }
    a.Wout[x] = w * damp;
  }
}

}  // namespace dfd
