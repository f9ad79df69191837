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

// ADE state of one PML face for this node, loaded ahead of its use: current value, and the
// RK registers the stage needs (accumulator for stages 1..3, step start for stages 1, 2).
struct PmlState {
  float w[9], t[9], w0[9];
};
__device__ __forceinline__ void pml_load(const VolArgs& a, int face, long long qa, long long st, PmlState& ps) {
  const float* aux = a.aux[face];
  const float* aux0 = a.aux0[face];
  const float* auxT = a.auxT[face];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * st + qa;
    ps.w[f] = aux[x];
    if (a.irk >= 1) ps.t[f] = auxT[x];
    if (a.irk == 1 || a.irk == 2) ps.w0[f] = aux0[x];
  }
}

// PML auxiliary update of one face for this node from its loaded state: accumulates
// -aux/beta into p[] and advances aux in place with the RK4 registers (pmlx.cu:165-208,
// rk4.cu:208-255).
__device__ __forceinline__ void pml_update(const VolArgs& a, int face, long long qa, long long st, float rb, float b,
                                           float dd, float al, const float* Dv, const float* dzv, float ez0,
                                           float ez1, float ez2, float lam, float mu, const PmlState& ps,
                                           float* p) {
  float* aux = a.aux[face];
  float* aux0 = a.aux0[face];
  float* auxT = a.auxT[face];
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
    const long long x = f * st + qa;
    p[f] += -ps.w[f] * rb;
    float h = ad * ps.w[f] + dd * Dv[f];
    if (dzv && f >= 3) h += add[f - 3];
    if (a.irk == 0) {
      aux0[x] = ps.w[f];
      auxT[x] = fmaf(a.rkb, h, ps.w[f]);
      aux[x] = fmaf(a.rka, h, ps.w[f]);
    } else if (a.irk < 3) {
      auxT[x] = fmaf(a.rkb, h, ps.t[f]);
      aux[x] = fmaf(a.rka, h, ps.w0[f]);
    } else {
      aux[x] = fmaf(a.rkb, h, ps.t[f]);
    }
  }
}

// Both steps at once: every load of the face precedes every store (the compiler cannot
// prove the three buffers distinct, and a load issued after a store would wait for a full
// memory round trip per field).
__device__ __forceinline__ void pml_face(const VolArgs& a, int face, long long qa, long long st, float rb, float b,
                                         float dd, float al, const float* Dv, const float* dzv, float ez0,
                                         float ez1, float ez2, float lam, float mu, float* p) {
  PmlState ps;
  pml_load(a, face, qa, st, ps);
  pml_update(a, face, qa, st, rb, b, dd, al, Dv, dzv, ez0, ez1, ez2, lam, mu, ps, p);
}

// RK4 register update of the nine fields of node q with right-hand side h (+ p), then the
// sponge factor (rk4.cu:20-33, cerjan.cu:166-200).  Every load precedes every store.
__device__ __forceinline__ void rk_store(const VolArgs& a, long long q, const float* h, const float* p,
                                         float damp) {
  const long long n = a.d.nxyz;
  float r0[9], r1[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    if (a.irk == 0) {
      r0[f] = __ldg(a.Win + x);
    } else if (a.irk < 3) {
      r0[f] = __ldg(a.W0 + x);
      r1[f] = a.T[x];
    } else {
      r1[f] = a.T[x];
    }
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    const float hf = p ? h[f] + p[f] : h[f];
    float w;
    if (a.irk == 0) {
      a.T[x] = fmaf(a.rkb, hf, r0[f]);
      w = fmaf(a.rka, hf, r0[f]);
    } else if (a.irk < 3) {
      a.T[x] = fmaf(a.rkb, hf, r1[f]);
      w = fmaf(a.rka, hf, r0[f]);
    } else {
      w = fmaf(a.rkb, hf, r1[f]);
    }
    a.Wout[x] = w * damp;
  }
}

}  // namespace dfd
