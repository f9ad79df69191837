// Split-node fault kernels of one RK stage.
//
// fault_node_kernel (one thread per non-united fault node, numbered row by row over their
//   rectangle), first in the stage:
//   state and slip RK4 with the rate-and-state evolution law in FP64 (rk4.cu:791-938),
//   trial traction + slip-weakening (trial_slipweakening.cu:23-732) or rate-and-state
//   FP64 Newton solve (trial_ratestate.cu:20-893), then the split-node -> volume transfer
//   of the fault plane (transform.cu:224-403).
// fault_band_kernel (seven threads per non-united fault node: one per off-fault layer,
//   one for the split nodes), after the volume kernels: velocity RHS on the six off-fault
//   layers and both split sides
//   (fault_dvelo.cu:17-389), stress RHS (fault_dstrs_f.cu / fault_dstrs_b.cu), the RK4
//   update of those band nodes and of the split nodes (rk4.cu:573-789), the RK-weighted
//   on-fault outputs (rk4.cu:466-571), the end-of-stage transfer and the sponge.
#include "dfd_internal.cuh"
#include "dfd_mlp.cuh"
#include "../../include/dfd_b200.h"

namespace dfd {

__device__ __forceinline__ float L5(const float* v, int c, int F) {  // 7-point register line
  return F == 1 ? -DFD_C1 * v[c - 1] - DFD_C2 * v[c] + DFD_C3 * v[c + 1] - DFD_C4 * v[c + 2] + DFD_C5 * v[c + 3]
                : -DFD_C5 * v[c - 3] + DFD_C4 * v[c - 2] - DFD_C3 * v[c - 1] + DFD_C2 * v[c] + DFD_C1 * v[c + 1];
}
__device__ __forceinline__ float L2(const float* v, int c, int F) { return F == 1 ? v[c + 1] - v[c] : v[c] - v[c - 1]; }
__device__ __forceinline__ float L3(const float* v, int c, int F) {
  return F == 1 ? -DFD_C24_1 * v[c] + DFD_C24_2 * v[c + 1] - DFD_C24_3 * v[c + 2]
                : DFD_C24_3 * v[c - 2] - DFD_C24_2 * v[c - 1] + DFD_C24_1 * v[c];
}
// strided global versions
__device__ __forceinline__ float G5(const float* v, long long q, long long s, int F) {
  return F == 1 ? -DFD_C1 * v[q - s] - DFD_C2 * v[q] + DFD_C3 * v[q + s] - DFD_C4 * v[q + 2 * s] + DFD_C5 * v[q + 3 * s]
                : -DFD_C5 * v[q - 3 * s] + DFD_C4 * v[q - 2 * s] - DFD_C3 * v[q - s] + DFD_C2 * v[q] + DFD_C1 * v[q + s];
}
__device__ __forceinline__ float G2(const float* v, long long q, long long s, int F) {
  return F == 1 ? v[q + s] - v[q] : v[q] - v[q - s];
}
__device__ __forceinline__ float G3(const float* v, long long q, long long s, int F) {
  return F == 1 ? -DFD_C24_1 * v[q] + DFD_C24_2 * v[q + s] - DFD_C24_3 * v[q + 2 * s]
                : DFD_C24_3 * v[q - 2 * s] - DFD_C24_2 * v[q - s] + DFD_C24_1 * v[q];
}

__device__ __forceinline__ void trac3(const float* W, const float* M, long long n, long long q, int mo, float* t) {
  float e0 = M[mo * n + q], e1 = M[(mo + 1) * n + q], e2 = M[(mo + 2) * n + q], jac = M[9 * n + q];
  float txx = W[3 * n + q], tyy = W[4 * n + q], tzz = W[5 * n + q];
  float txy = W[6 * n + q], txz = W[7 * n + q], tyz = W[8 * n + q];
  t[0] = (e0 * txx + e1 * txy + e2 * txz) * jac;
  t[1] = (e0 * txy + e1 * tyy + e2 * tyz) * jac;
  t[2] = (e0 * txz + e1 * tyz + e2 * tzz) * jac;
}
// 3x3 table times vector, table t stored as planes (t*9+e)*nyz + pf
__device__ __forceinline__ void tmv(const float* tab, int t, long long nyz, long long pf, const float* v, float* o) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float* m = tab + (long long)(t * 9 + 3 * r) * nyz + pf;
    o[r] = m[0] * v[0] + m[nyz] * v[1] + m[2 * nyz] * v[2];
  }
}
__device__ __forceinline__ void tfmv(const float* tab, int t, int ny, int j1, const float* v, float* o) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const float* m = tab + (long long)(t * 9 + 3 * r) * ny + j1;
    o[r] = m[0] * v[0] + m[ny] * v[1] + m[2 * ny] * v[2];
  }
}
__device__ __forceinline__ void inv3(const float m[3][3], float r[3][3]) {
  float c00 = m[1][1] * m[2][2] - m[2][1] * m[1][2], c01 = m[2][1] * m[0][2] - m[0][1] * m[2][2];
  float c02 = m[0][1] * m[1][2] - m[0][2] * m[1][1], c10 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
  float c11 = m[0][0] * m[2][2] - m[2][0] * m[0][2], c12 = m[1][0] * m[0][2] - m[0][0] * m[1][2];
  float c20 = m[1][0] * m[2][1] - m[1][1] * m[2][0], c21 = m[2][0] * m[0][1] - m[0][0] * m[2][1];
  float c22 = m[0][0] * m[1][1] - m[0][1] * m[1][0];
  float det = 1.0f / (c00 * m[0][0] + c01 * m[1][0] + c02 * m[2][0]);
  r[0][0] = c00 * det; r[0][1] = c01 * det; r[0][2] = c02 * det;
  r[1][0] = c10 * det; r[1][1] = c11 * det; r[1][2] = c12 * det;
  r[2][0] = c20 * det; r[2][1] = c21 * det; r[2][2] = c22 * det;
}

// Split nodes -> volume at the fault plane: velocity average and stress from the
// traction matrix [T1 | avg T2 | avg T3] times the inverse metric (transform.cu:310-385).
__device__ void fault_to_volume(const FaultArgs& a, const float* FW, float* Wdst, int j1, int k1, float damp) {
  const Dims& d = a.d;
  long long n = d.nxyz, nyz = d.nyz, pf = j1 + (long long)k1 * d.ny;
  long long q = idx3(d, d.i0, j1, k1);
  float met[3][3], im[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) met[r][c] = a.M[(3 * c + r) * n + q];
  float rj = 1.0f / a.M[9 * n + q];
  float tr[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    tr[c][0] = a.T1[(c * 7 + 3) * nyz + pf];
    tr[c][1] = (FW[(3 + c) * 2 * nyz + pf] + FW[(3 + c) * 2 * nyz + nyz + pf]) * 0.5f;
    tr[c][2] = (FW[(6 + c) * 2 * nyz + pf] + FW[(6 + c) * 2 * nyz + nyz + pf]) * 0.5f;
  }
  inv3(met, im);
  float sg[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) sg[r][c] = (tr[r][0] * im[0][c] + tr[r][1] * im[1][c] + tr[r][2] * im[2][c]) * rj;
#pragma unroll
  for (int c = 0; c < 3; c++) Wdst[c * n + q] = (FW[c * 2 * nyz + pf] + FW[c * 2 * nyz + nyz + pf]) * 0.5f * damp;
  Wdst[3 * n + q] = sg[0][0] * damp;
  Wdst[4 * n + q] = sg[1][1] * damp;
  Wdst[5 * n + q] = sg[2][2] * damp;
  Wdst[6 * n + q] = (sg[0][1] + sg[1][0]) * 0.5f * damp;
  Wdst[7 * n + q] = (sg[0][2] + sg[2][0]) * 0.5f * damp;
  Wdst[8 * n + q] = (sg[1][2] + sg[2][1]) * 0.5f * damp;
}

// fault_to_volume with the split-node values of the stage (fw[field][side]) in registers
// and every load issued before the first store
__device__ __forceinline__ void fault_to_volume_r(const FaultArgs& a, const float (*fw)[2], float* Wdst, int j1,
                                                  int k1, float damp) {
  const Dims& d = a.d;
  long long n = d.nxyz, nyz = d.nyz, pf = j1 + (long long)k1 * d.ny;
  long long q = idx3(d, d.i0, j1, k1);
  float met[3][3], im[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) met[r][c] = a.M[(3 * c + r) * n + q];
  float rj = 1.0f / a.M[9 * n + q];
  float tr[3][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    tr[c][0] = a.T1[(c * 7 + 3) * nyz + pf];
    tr[c][1] = (fw[3 + c][0] + fw[3 + c][1]) * 0.5f;
    tr[c][2] = (fw[6 + c][0] + fw[6 + c][1]) * 0.5f;
  }
  inv3(met, im);
  float sg[3][3];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) sg[r][c] = (tr[r][0] * im[0][c] + tr[r][1] * im[1][c] + tr[r][2] * im[2][c]) * rj;
#pragma unroll
  for (int c = 0; c < 3; c++) Wdst[c * n + q] = (fw[c][0] + fw[c][1]) * 0.5f * damp;
  Wdst[3 * n + q] = sg[0][0] * damp;
  Wdst[4 * n + q] = sg[1][1] * damp;
  Wdst[5 * n + q] = sg[2][2] * damp;
  Wdst[6 * n + q] = (sg[0][1] + sg[1][0]) * 0.5f * damp;
  Wdst[7 * n + q] = (sg[0][2] + sg[2][0]) * 0.5f * damp;
  Wdst[8 * n + q] = (sg[1][2] + sg[2][1]) * 0.5f * damp;
}

// compensated sum s + inc with the running compensation term *c (Kahan summation)
__device__ __forceinline__ float kahan_add(float s, float inc, float* c) {
  const float y = __fsub_rn(inc, *c);
  const float t = __fadd_rn(s, y);
  *c = __fsub_rn(__fsub_rn(t, s), y);
  return t;
}

__device__ __forceinline__ double gt_func(double t, double T) {  // device.cu:134-143
  if (t < T) {
    double t1 = t - T, t2 = t - 2.0 * T;
    return exp(t1 * t1 / t / t2);
  }
  return 1.0;
}

// 16-byte pieces of the learned-guess weight vector (its last piece runs past the
// vector's end into the allocation's slack)
constexpr int NET_PIECES = (DFD_MLP_PARAMS + 3) / 4;

// Base of the learned guess: the root asinh(Vhat e^{psi/a} / (2 V0)) of the solve without
// the radiation-damping term, V0 = 1e-6; from its logarithm where the argument is above
// e^18 (asinh y = ln 2y + 1/(4 y^2) + ..., the rest below FP64 rounding there), which
// also keeps e^{psi/a} from overflowing.  Takes ln Vhat and psi/a.
__device__ __forceinline__ double guess_base(double lnVhat, double psi_over_a) {
  const double ly = lnVhat + psi_over_a + 13.122363377404328;  // ln(1 / 2e-6)
  return ly > 18.0 ? ly + 0.6931471805599453 : asinh(exp(ly));
}

// Bounded Newton on f(x) = 2 V0 e^{-psi/a} sinh x + coef x - Vhat (trial_ratestate.cu:20-57);
// returns the iterate and the iteration count, sets *ok when |dx|/|x| < 1e-12 was reached.
__device__ double newton_rs(double x, double psi, double ra, double Vhat, double coef, int cap, int* iters,
                            bool* ok) {
  const double V0 = 1e-6;
  double e = 2.0 * exp(-psi / ra) * V0;
  int it = 0;
  *ok = false;
  double xn = x;
  while (it < cap) {
    double fv = e * sinh(x) + coef * x - Vhat;
    double df = e * cosh(x) + coef;
    double dd = -fv / (df + 1e-100);
    xn = x + dd;
    double err = fabs(dd) / (fabs(x) + 1e-100);
    x = xn;
    it++;
    if (err < 1e-12) { *ok = true; break; }
  }
  *iters = it;
  return xn;
}

// Body of the fault node kernel for the block (bx, by) of a (32, 4) grid over (NY, NZ);
// snet is the block's shared copy of the learned-guess weights.
template <int FY, int FZ>
__device__ __forceinline__ void fault_node_body(const FaultArgs& a, int blk, float* snet) {
  const Dims& d = a.d;
  // learned-guess weights to shared memory (the network's lanes then read the same weight
  // at the same time: a broadcast), copied asynchronously in 16-byte pieces so that they
  // land while the node's state update and trial traction run.  The block meets once at
  // a barrier before the network: a thread whose node is not live arrives at once, the
  // others before their solve; the barrier has no .aligned, which lets threads arrive from
  // the two places.  (The weight vector's allocation and snet both extend to a whole
  // 16-byte piece.)
  const bool learned = a.friction_type != 0 && a.rs_guess && a.guess_net;
  if (learned) {
    const int tid = threadIdx.x + threadIdx.y * blockDim.x, nt = blockDim.x * blockDim.y;
    for (int p = tid; p < NET_PIECES; p += nt)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(snet + 4 * p)),
                   "l"(a.guess_net + 4 * p)
                   : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  auto net_ready = [&]() {
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("barrier.sync 0;" ::: "memory");
  };
  // node t of the non-united rectangle, numbered row by row
  const NodeRect rc = node_rect(a.NY, a.NZ, a.freenode, a.jg0, d.nj);
  const long long tn = (long long)blk * blockDim.x + threadIdx.x;
  const bool inr = tn < rc.count();
  const int j = inr ? rc.j0 + (int)(tn % rc.w) : 0, k = inr ? rc.k0 + (int)(tn / rc.w) : 0;
  const int q2 = j + k * d.nj;
  const bool live = inr && !a.united[q2];
  // the tensor-core network takes a whole warp (32 consecutive nodes of the rectangle):
  // it runs where every lane's node is live (all warps but the last), the per-thread
  // network elsewhere
  const bool warp_full = __all_sync(0xffffffffu, live);
  if (!live) {
    if (learned) net_ready();
    return;
  }
  const long long n = d.nxyz, nyz = d.nyz;
  const int j1 = j + 3, k1 = k + 3, km = d.nk - k;
  const long long pf = j1 + (long long)k1 * d.ny;
  const float* FW = a.FWin;
  float s1[3], s2[3], nv[3];
#pragma unroll
  for (int c = 0; c < 3; c++) { s1[c] = a.vecs1[c * nyz + pf]; s2[c] = a.vecs2[c * nyz + pf]; }

  // ---- state and slip (rk4.cu:833-935)
  {
    float dV[3];
#pragma unroll
    for (int c = 0; c < 3; c++) dV[c] = FW[c * 2 * nyz + nyz + pf] - FW[c * 2 * nyz + pf];
    float vs1 = dV[0] * s1[0] + dV[1] * s1[1] + dV[2] * s1[2];
    float vs2 = dV[0] * s2[0] + dV[1] * s2[1] + dV[2] * s2[2];
    float hs = sqrtf(vs2 * vs2 + vs1 * vs1);
    a.hslip[q2] = hs;
    float hState = 0.0f;
    if (a.friction_type >= 1) {
      double V = fmax((double)hs, 1e-30), st = a.State[q2];
      double ra = a.a[q2], rb = a.b[q2], rl = a.L[q2];
      if (a.friction_type == 1) {
        hState = (float)(rb * a.V0 / rl * (exp((a.f0 - st) / rb) - V / a.V0));
      } else {
        double flv = a.f0 - (rb - ra) * log(V / a.V0);
        double fss = a.fw + (flv - a.fw) / pow(1. + pow(V / (double)a.Vw[q2], 8), 0.125);
        double psiss = ra * (log(sinh(fss / ra)) + log(2. * (a.V0 / V)));
        hState = (float)(-V / rl * (st - psiss));
      }
    }
    // the accumulator holds the step's increment only; the last stage adds it to the
    // step-start value with a compensation term (Kahan), so that FP32 rounding does not
    // build up over the thousands of steps of a rupture (the reference sums into the value
    // itself, rk4.cu:833-935)
    if (a.irk == 0) {
      float st0 = a.State[q2], sl0 = a.slip[q2];
      a.mState[q2] = st0; a.tState[q2] = a.rkb * hState;
      a.mslip[q2] = sl0; a.tslip[q2] = a.rkb * hs;
    } else if (a.irk < 3) {
      a.tState[q2] = fmaf(a.rkb, hState, a.tState[q2]);
      a.tslip[q2] = fmaf(a.rkb, hs, a.tslip[q2]);
    }
    if (a.irk == 3) {
      a.State[q2] = kahan_add(a.mState[q2], fmaf(a.rkb, hState, a.tState[q2]), a.cState + q2);
      a.slip[q2] = kahan_add(a.mslip[q2], fmaf(a.rkb, hs, a.tslip[q2]), a.cslip + q2);
    } else {
      a.State[q2] = fmaf(a.rka, hState, a.mState[q2]);
      a.slip[q2] = fmaf(a.rka, hs, a.mslip[q2]);
    }
  }

  // ---- trial traction: T1 layers, split-node DyT2/DzT3, residuals of the half cells
  if (a.irk == 0)
#pragma unroll
    for (int c = 0; c < 3; c++) a.mT1[c * nyz + pf] = a.T1[(c * 7 + 3) * nyz + pf];
  float Mrho[2], R[3][2], jac_last = 1.0f, rho_last = 1.0f;
  const float DH = a.DH, DH2 = DH * DH;
#pragma unroll
  for (int m = 0; m < 2; m++) {
    float jac = 1.0f;
    float rho = a.rhof[m * nyz + pf];
#pragma unroll
    for (int l = 1; l <= 3; l++) {
      int ii = d.i0 + (2 * m - 1) * l;
      long long q = idx3(d, ii, j1, k1);
      float t[3];
      trac3(a.Win, a.M, n, q, 0, t);
      jac = a.M[9 * n + q];  // the i0 -/+ 3 value feeds the half-cell mass (reference quirk)
      int lay = 3 + (2 * m - 1) * l;
#pragma unroll
      for (int c = 0; c < 3; c++) a.T1[(c * 7 + lay) * nyz + pf] = t[c];
    }
    float DyT[3], DzT[3];
    const bool ry = a.rupy[q2] % 7, rz = a.rupz[q2] % 7;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* t2 = FW + (3 + c) * 2 * nyz + m * nyz;
      DyT[c] = (ry ? G2(t2, pf, 1, FY) : G5(t2, pf, 1, FY)) * a.rDH;
      float v3[7];
      const float* t3 = FW + (6 + c) * 2 * nyz + m * nyz;
#pragma unroll
      for (int l = 0; l < 7; l++) v3[l] = t3[pf + (long long)(l - 3) * d.ny];
      if (a.freenode && km <= 3) {
        v3[km + 2] = 0.0f;
        for (int l = km + 3; l < 7; l++) v3[l] = -v3[2 * (km + 2) - l];
      }
      DzT[c] = (rz ? L2(v3, 3, FZ) : L5(v3, 3, FZ)) * a.rDH;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* T = a.T1 + c * 7 * nyz + pf;
      float r_ = m == 0 ? DFD_A1 * T[2 * nyz] + DFD_A2 * T[1 * nyz] + DFD_A3 * T[0]
                        : DFD_A1 * T[4 * nyz] + DFD_A2 * T[5 * nyz] + DFD_A3 * T[6 * nyz];
      R[c][m] = 0.5f * ((2 * m - 1) * r_ + (DyT[c] + DzT[c]) * DH) * DH2;
    }
    Mrho[m] = 0.5f * jac * rho * DH * DH2;
    jac_last = jac;
    rho_last = rho;
  }
  long long qm = idx3(d, d.i0, j1, k1);
#pragma unroll
  for (int c = 0; c < 3; c++) nv[c] = a.M[c * n + qm];
  float n0 = sqrtf(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
  float jacvec = a.M[9 * n + qm] * n0;
#pragma unroll
  for (int c = 0; c < 3; c++) nv[c] /= n0;
  const int it = *a.it_dev;
  double t = a.irk == 0 ? it * a.dDT : (a.irk == 3 ? (it + 1) * a.dDT : (it + 0.5) * a.dDT);
  float G = (float)gt_func(t, a.smooth_load_T);
  float dV[3];
#pragma unroll
  for (int c = 0; c < 3; c++) dV[c] = a.Fm[c * 2 * nyz + nyz + pf] - a.Fm[c * 2 * nyz + pf];

  float Tau[3], Tau_n, Vcheck;
  float T1new[3];
  bool from_tau;
  if (a.friction_type == 0) {
    // ---- slip weakening (trial_slipweakening.cu:322-615)
    if (a.inport_stress == 1) {
      a.sx[q2] = a.T0x[q2] + G * a.dT0x[q2];
      a.sy[q2] = a.T0y[q2] + G * a.dT0y[q2];
      a.sz[q2] = a.T0z[q2] + G * a.dT0z[q2];
    }
    float si[3] = {a.sx[q2], a.sy[q2], a.sz[q2]};
    float den = DH2 * (Mrho[0] * DFD_A0P - DFD_A0M * Mrho[1]);
    float TL[3], Ts[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      T1new[c] = -(Mrho[0] * Mrho[1] * dV[c] / a.DT + Mrho[0] * R[c][1] - Mrho[1] * R[c][0]) / den * 2.0f;
      TL[c] = T1new[c] / jacvec + si[c];
    }
    float Trn = TL[0] * nv[0] + TL[1] * nv[1] + TL[2] * nv[2];
#pragma unroll
    for (int c = 0; c < 3; c++) Ts[c] = TL[c] - nv[c] * Trn;
    float Ts0 = sqrtf(Ts[0] * Ts[0] + Ts[1] * Ts[1] + Ts[2] * Ts[2]);
    bool change = false;
    float Tau_s;
    if (Trn >= 0.0f) { Tau_n = 0.0f; change = true; } else Tau_n = Trn;
    float mus = a.str_peak[q2], sl = a.slip[q2], dc = a.Dc[q2];
    float fr = sl <= dc ? mus - (mus - a.mu_d) * sl / dc : a.mu_d;
    float Tau_c = -fr * Tau_n + a.C0[q2];
    if (Ts0 >= Tau_c) { Tau_s = Tau_c; a.flag_rup[q2] = 1; change = true; }
    else { Tau_s = Ts0; a.flag_rup[q2] = 0; }
    if (change) {
      if (fabsf(Ts0) < 1e-1f) {
#pragma unroll
        for (int c = 0; c < 3; c++) Tau[c] = Tau_n * nv[c];
      } else {
#pragma unroll
        for (int c = 0; c < 3; c++) Tau[c] = Tau_n * nv[c] + (Tau_s / Ts0) * Ts[c];
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) Tau[c] = TL[c];
    }
    from_tau = change;
    Vcheck = a.hslip[q2];
  } else {
    // ---- rate and state (trial_ratestate.cu:374-802), FP64
    double Rr[3][2];
#pragma unroll
    for (int m = 0; m < 2; m++) {
      Rr[0][m] = nv[0] * R[0][m] + nv[1] * R[1][m] + nv[2] * R[2][m];
      Rr[1][m] = s1[0] * R[0][m] + s1[1] * R[1][m] + s1[2] * R[2][m];
      Rr[2][m] = s2[0] * R[0][m] + s2[1] * R[1][m] + s2[2] * R[2][m];
    }
    double y1 = j + a.jg0 - a.NY / 2;
    double z1 = a.freenode ? (double)((a.NZ - 1 - k) - (int)(7.5e3 / a.DH)) : (double)(k - a.NZ / 2);
    double r = sqrt(y1 * y1 + z1 * z1) * (double)a.DH;
    double Fr = r < 3.0e3 ? exp(r * r / (r * r - 9.0e6)) : 0.0;
    a.sx[q2] = -120e6f;
    a.sy[q2] = (float)(-25e6 * Fr * (double)G + -75e6);
    a.sz[q2] = 0.0f;
    if (a.inport_stress == 1) {
      a.sx[q2] = a.T0x[q2] + G * a.dT0x[q2];
      a.sy[q2] = a.T0y[q2] + G * a.dT0y[q2];
      a.sz[q2] = a.T0z[q2] + G * a.dT0z[q2];
    }
    double T0[3] = {a.sx[q2], a.sy[q2], a.sz[q2]};
    double T0l[3] = {nv[0] * T0[0] + nv[1] * T0[1] + nv[2] * T0[2], s1[0] * T0[0] + s1[1] * T0[1] + s1[2] * T0[2],
                     s2[0] * T0[0] + s2[1] * T0[1] + s2[2] * T0[2]};
    double dt1 = a.dDT;
    double Rl[3] = {nv[0] * (double)dV[0] + nv[1] * (double)dV[1] + nv[2] * (double)dV[2],
                    s1[0] * (double)dV[0] + s1[1] * (double)dV[1] + s1[2] * (double)dV[2],
                    s2[0] * (double)dV[0] + s2[1] * (double)dV[1] + s2[2] * (double)dV[2]};
    Rl[1] -= a.Vini;
    double M0 = Mrho[0], M1 = Mrho[1], dDH = DH;
    double den = dDH * dDH * (M0 * (double)DFD_A0P - (double)DFD_A0M * M1) * (double)jacvec;
    double Tl[3];
#pragma unroll
    for (int c = 0; c < 3; c++) Tl[c] = T0l[c] - 2.0 * (M0 * M1 * Rl[c] / dt1 + M0 * Rr[c][1] - M1 * Rr[c][0]) / den;
    double cc = -((double)DFD_A0P - (double)DFD_A0M) * dt1 * jacvec / ((double)jac_last * rho_last * dDH);
    double tn = Tl[0] >= -1e-1 ? -1e-1 : Tl[0];
    // thermal pressurisation: the friction law sees the effective normal stress tn + P at
    // the fault; the traction put back keeps (tn + P) - P (trial_ratestate.cu:636-643, 787-790)
    const float Pf = a.tpP ? a.tpP[q2] : 0.0f;
    tn += Pf;
    double Vt1 = cc * Tl[1], Vt2 = cc * Tl[2];
    double ra = a.a[q2], st = a.State[q2];
    double coef = cc * ra * fabs(tn);
    double Vtn = sqrt(Vt1 * Vt1 + Vt2 * Vt2);
    double Ttn = sqrt(Tl[1] * Tl[1] + Tl[2] * Tl[2]);
    double Rn = sqrt(Rl[1] * Rl[1] + Rl[2] * Rl[2]);
    const double psi_a = st / ra;
    const double es = exp(psi_a);
    int its = 0, its2 = 0;
    bool ok = false;
    double xn;
    // network inputs (FP32, as the network computes), needed by the learned guess and by
    // the sample recording only
    // network inputs (FP32, as the network computes), from ln Vhat, which the guess's base
    // needs too
    auto features = [&](double lnV, float* fin) {
      fin[0] = (float)psi_a;
      fin[1] = (float)fmax(lnV * 0.4342944819032518, -30.0);  // log10 max(Vhat, 1e-30)
      fin[2] = log10f(fmaxf((float)coef, 1e-30f));
      fin[3] = (float)ra;
    };
    long long clk0 = 0;
    if (a.prof) clk0 = clock64();
    bool accepted = false;
    if (a.rs_guess && a.guess_net) {
      // learned guess: the root without radiation damping corrected by the network.  Newton
      // corrections are evaluated from the guess (sinh and cosh from one expm1), and after
      // each the residual test bounds the error left, |f''| dd^2 / (2 f') with f'' taken at
      // its largest over the step (the iteration converges quadratically): the corrected
      // guess is accepted when that bound is at most guess_tol |x|.  After two corrections
      // without acceptance the plain solve from the reference's guess runs.
      const double lnV = log(fmax(Vtn, 1e-300));
      float fin[4];
      features(lnV, fin);
      net_ready();
      float res;
      if (warp_full) {
        __syncwarp();
        res = mlp_residual_warp(snet, fin);
      } else {
        res = mlp_residual(snet, fin);
      }
      const double e = 2e-6 / es;
      double x = guess_base(lnV, psi_a) + (double)res;
      its = 0;
      for (int c = 0; c < 2 && !accepted; c++) {
        const double em = expm1(x), r = 1.0 / (1.0 + em);
        const double sh = 0.5 * (em + em * r), ch = sh + r;
        const double rfp = 1.0 / (e * ch + coef + 1e-100);
        const double dd = -(e * sh + coef * x - Vtn) * rfp;
        const double bound = e * (fabs(sh) + 2.0 * fabs(dd) * ch) * dd * dd * rfp;
        its++;
        x += dd;
        if (!isfinite(x)) break;
        accepted = fabs(dd) <= 1e-2 * (1.0 + fabs(x)) && bound <= a.guess_tol * fabs(x);
      }
      if (accepted) {
        xn = x;
        ok = true;
      } else {
        xn = newton_rs(asinh(es * Rn / (2.0 * 1e-6)), st, ra, Vtn, coef, 100, &its2, &ok);
      }
      if (a.judge) {
        // the plain solve as the judge of the accepted value (a measurement aid)
        int itj;
        bool okj;
        const double xp = newton_rs(asinh(es * Rn / (2.0 * 1e-6)), st, ra, Vtn, coef, 100, &itj, &okj);
        const float rel = (float)(fabs(xn - xp) / fmax(fabs(xp), 1e-300));
        atomicMax(reinterpret_cast<unsigned*>(a.newton + 6), __float_as_uint(rel));
      }
    } else {
      xn = newton_rs(asinh(es * Rn / (2.0 * 1e-6)), st, ra, Vtn, coef, 100, &its, &ok);
      if (a.rec && ok && ((unsigned)q2 * 7919u + (unsigned)it * 4u + (unsigned)a.irk) % (unsigned)a.rec_every == 0) {
        // training sample: inputs and the residual target of the converged solve
        unsigned slot = atomicAdd(a.rec_n, 1u);
        if (slot < (unsigned)a.rec_cap) {
          const double lnV = log(fmax(Vtn, 1e-300));
          float fin[4];
          features(lnV, fin);
          float* o = a.rec + 5ull * slot;
          o[0] = fin[0]; o[1] = fin[1]; o[2] = fin[2]; o[3] = fin[3];
          o[4] = (float)(xn - guess_base(lnV, psi_a));
        }
      }
    }
    {
      // Newton statistics, one atomic per warp: iterations, capped solves, accepted learned
      // guesses, learned guesses that fell back, and with solve timing on the clock cycles
      // of the solve (guess, network, Newton) and the solves timed
      const unsigned m = __activemask();
      const unsigned sum_it = __reduce_add_sync(m, (unsigned)(its + its2));
      const unsigned n_bad = __reduce_add_sync(m, ok ? 0u : 1u);
      const unsigned n_acc = __reduce_add_sync(m, accepted ? 1u : 0u);
      const unsigned n_all = __popc(m);
      const unsigned cyc = a.prof ? __reduce_add_sync(m, (unsigned)(clock64() - clk0)) : 0u;
      if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == __ffs(m) - 1) {
        atomicAdd(a.newton, (unsigned long long)sum_it);
        if (n_bad) atomicAdd(a.newton + 1, (unsigned long long)n_bad);
        if (a.rs_guess && a.guess_net) {
          atomicAdd(a.newton + 2, (unsigned long long)n_acc);
          atomicAdd(a.newton + 3, (unsigned long long)(n_all - n_acc));
        }
        if (a.prof) {
          atomicAdd(a.newton + 4, (unsigned long long)cyc);
          atomicAdd(a.newton + 5, (unsigned long long)n_all);
        }
      }
    }
    double V = 2.0 * 1e-6 * exp(-st / ra) * sinh(xn);
    double T = ra * xn * fabs(tn);
    a.friction[q2] = (float)(ra * xn);
    Ttn = fmax(Ttn, 1e-8);
    double ts1 = Tl[1] / Ttn * T, ts2 = Tl[2] / Ttn * T;
    float Vf = fmaxf((float)V, 1e-30f);
#pragma unroll
    tn -= Pf;
    for (int c = 0; c < 3; c++) Tau[c] = (float)(tn * nv[c] + ts1 * s1[c] + ts2 * s2[c]);
    Tau[0] = a.sx[q2];  // the normal-traction perturbation is forced to zero (:797)
    Tau_n = Tau[0] * nv[0] + Tau[1] * nv[1] + Tau[2] * nv[2];
    from_tau = true;
    Vcheck = Vf;
  }
  // ---- store T1 at the fault, its rate, outputs (trial_slipweakening.cu:629-709)
  float si[3] = {a.sx[q2], a.sy[q2], a.sz[q2]};
  float vis = a.viscosity * a.DT;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float v = from_tau ? (Tau[c] - si[c]) * jacvec : T1new[c];
    float hv = (v - a.mT1[c * nyz + pf]) / a.DT;
    if (a.irk == 3) a.hT1[c * nyz + pf] = hv;
    a.T1[(c * 7 + 3) * nyz + pf] = v + vis * hv;
  }
  a.tTs1[q2] = Tau[0] * s1[0] + Tau[1] * s1[1] + Tau[2] * s1[2];
  a.tTs2[q2] = Tau[0] * s2[0] + Tau[1] * s2[1] + Tau[2] * s2[2];
  a.tTn[q2] = Tau_n;
  if (!a.init_t0_flag[q2] && Vcheck > 1e-3f) {
    a.init_t0[q2] = (float)(it * a.dDT);
    a.init_t0_flag[q2] = 1;
    a.flag_rup[q2] = 1;
  }
  // ---- fault plane into the stage input (transform.cu:224-403)
  fault_to_volume(a, FW, a.Win, j1, k1, 1.0f);
}

// stress RHS of a volume node from its velocity gradient (fault_dstrs_f.cu:1213-1248)
__device__ __forceinline__ void hooke(const float* M, long long n, long long q, const float* X, const float* Y,
                                      const float* Z, float* hT) {
  float lam = M[10 * n + q], mu = M[11 * n + q], l2m = lam + 2.0f * mu;
  float ex0 = M[q], ex1 = M[n + q], ex2 = M[2 * n + q];
  float ey0 = M[3 * n + q], ey1 = M[4 * n + q], ey2 = M[5 * n + q];
  float ez0 = M[6 * n + q], ez1 = M[7 * n + q], ez2 = M[8 * n + q];
  hT[0] = l2m * ex0 * X[0] + lam * ex1 * X[1] + lam * ex2 * X[2] + l2m * ey0 * Y[0] + lam * ey1 * Y[1] +
          lam * ey2 * Y[2] + l2m * ez0 * Z[0] + lam * ez1 * Z[1] + lam * ez2 * Z[2];
  hT[1] = lam * ex0 * X[0] + l2m * ex1 * X[1] + lam * ex2 * X[2] + lam * ey0 * Y[0] + l2m * ey1 * Y[1] +
          lam * ey2 * Y[2] + lam * ez0 * Z[0] + l2m * ez1 * Z[1] + lam * ez2 * Z[2];
  hT[2] = lam * ex0 * X[0] + lam * ex1 * X[1] + l2m * ex2 * X[2] + lam * ey0 * Y[0] + lam * ey1 * Y[1] +
          l2m * ey2 * Y[2] + lam * ez0 * Z[0] + lam * ez1 * Z[1] + l2m * ez2 * Z[2];
  hT[3] = (ex1 * X[0] + ex0 * X[1] + ey1 * Y[0] + ey0 * Y[1] + ez1 * Z[0] + ez0 * Z[1]) * mu;
  hT[4] = (ex2 * X[0] + ex0 * X[2] + ey2 * Y[0] + ey0 * Y[2] + ez2 * Z[0] + ez0 * Z[2]) * mu;
  hT[5] = (ex2 * X[1] + ex1 * X[2] + ey2 * Y[1] + ey1 * Y[2] + ez2 * Z[1] + ez1 * Z[2]) * mu;
}

// RK4 registers and stage output of the nine fields of volume node q, every load before
// the first store (rk4.cu:20-33)
__device__ __forceinline__ void rk_store9(const FaultArgs& a, long long q, const float* h, float damp) {
  const long long n = a.d.nxyz;
  float r0[9], r1[9];
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    if (a.irk == 0) {
      r0[f] = a.Win[x];
    } else if (a.irk < 3) {
      r1[f] = a.T[x];
      r0[f] = a.W0[x];
    } else {
      r1[f] = a.T[x];
    }
  }
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const long long x = f * n + q;
    float w;
    if (a.irk == 0) {
      a.T[x] = fmaf(a.rkb, h[f], r0[f]);
      w = fmaf(a.rka, h[f], r0[f]);
    } else if (a.irk < 3) {
      a.T[x] = fmaf(a.rkb, h[f], r1[f]);
      w = fmaf(a.rka, h[f], r0[f]);
    } else {
      w = fmaf(a.rkb, h[f], r1[f]);
    }
    a.Wout[x] = w * damp;
  }
}

template <int FX, int FY, int FZ>
__device__ __forceinline__ void fault_band_body(const FaultArgs& a, int bx, int by, int part) {
  const Dims& d = a.d;
  int j = bx * blockDim.x + threadIdx.x;
  int k = by * blockDim.y + threadIdx.y;
  if (j >= d.nj || k >= d.nk) return;
  int q2 = j + k * d.nj;
  if (a.united[q2]) {
    // welded nodes: the RK-weighted outputs run over every node in the reference
    // (rk4.cu:521-569) and are zero there (no trial traction, no split velocity)
    if (a.irk == 0 && part == 6) {
      a.Tn[q2] = 0.0f; a.Ts1[q2] = 0.0f; a.Ts2[q2] = 0.0f;
      a.Vs1[q2] = 0.0f; a.Vs2[q2] = 0.0f; a.hslip[q2] = 0.0f;
    }
    return;
  }
  const long long n = d.nxyz, nyz = d.nyz;
  const int j1 = j + 3, k1 = k + 3, km = d.nk - k, i0 = d.i0;
  const long long pf = j1 + (long long)k1 * d.ny;
  const float* W = a.Win;
  const float* FW = a.FWin;
  const float* M = a.M;
  const float r = a.rDH;
  const bool ry = a.rupy[q2] % 7, rz = a.rupz[q2] % 7;
  float dampyz = 1.0f;
  if (a.dampx) dampyz = fminf(a.dampy[j1], a.dampz[k1]);

  // ---------------- volume nodes of one of the six off-fault layers (parts 0..5)
  if (part < 6) {
    const int l = part < 3 ? part - 3 : part - 2;
    const int i = i0 + l;
    const long long q = idx3(d, i, j1, k1);
    // velocity RHS (fault_dvelo.cu:153-254), traction image across the fault
    int nn = i0 - i;
    float hv[3];
    {
      float v1[3][7], v2[3][7], v3[3][7];
#pragma unroll
      for (int s = 0; s < 7; s++) {
        float t[3];
        trac3(W, M, n, q + (long long)(s - 3) * d.sx, 0, t);
        v1[0][s] = t[0]; v1[1][s] = t[1]; v1[2][s] = t[2];
        trac3(W, M, n, q + (s - 3), 3, t);
        v2[0][s] = t[0]; v2[1][s] = t[1]; v2[2][s] = t[2];
        trac3(W, M, n, q + (long long)(s - 3) * d.py, 6, t);
        v3[0][s] = t[0]; v3[1][s] = t[1]; v3[2][s] = t[2];
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float* v = v1[c];
        v[nn + 3] = a.T1[(c * 7 + 3) * nyz + pf];
        if (nn == 2) v[6] = 2.0f * v[5] - v[4];
        if (nn == 1) { v[5] = 2.0f * v[4] - v[3]; v[6] = 2.0f * v[4] - v[2]; }
        if (nn == -1) { v[0] = 2.0f * v[2] - v[4]; v[1] = 2.0f * v[2] - v[3]; }
        if (nn == -2) v[0] = 2.0f * v[1] - v[2];
        if (a.freenode && km <= 3) {
          v3[c][km + 2] = 0.0f;
          for (int s = km + 3; s < 7; s++) v3[c][s] = -v3[c][2 * (km + 2) - s];
        }
      }
      float rrj = 1.0f / (M[12 * n + q] * M[9 * n + q]);
#pragma unroll
      for (int c = 0; c < 3; c++) hv[c] = (L5(v1[c], 3, FX) * r + L5(v2[c], 3, FY) * r + L5(v3[c], 3, FZ) * r) * rrj;
    }
    // stress RHS (fault_dstrs_{f,b}.cu, volume columns)
    float X[3], Y[3], Z[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* wv = W + c * n;
      float fm = FW[c * 2 * nyz + pf], fp = FW[c * 2 * nyz + nyz + pf];
      float x;
      if (FX == 1) {
        if (l == 3) x = G5(wv, q, d.sx, 1);
        else if (l == 2) x = G3(wv, q, d.sx, 1);
        else if (l == 1) x = wv[q + d.sx] - wv[q];
        else if (l == -1) x = fm - wv[q];
        else if (l == -2) x = -DFD_C24_1 * wv[q] + DFD_C24_2 * wv[q + d.sx] - DFD_C24_3 * fm;
        else x = -DFD_C1 * wv[q - d.sx] - DFD_C2 * wv[q] + DFD_C3 * wv[q + d.sx] - DFD_C4 * wv[q + 2 * d.sx] + DFD_C5 * fm;
      } else {
        if (l == -3) x = G5(wv, q, d.sx, -1);
        else if (l == -2) x = G3(wv, q, d.sx, -1);
        else if (l == -1) x = wv[q] - wv[q - d.sx];
        else if (l == 1) x = wv[q] - fp;
        else if (l == 2) x = DFD_C24_3 * fp - DFD_C24_2 * wv[q - d.sx] + DFD_C24_1 * wv[q];
        else x = -DFD_C5 * fp + DFD_C4 * wv[q - 2 * d.sx] - DFD_C3 * wv[q - d.sx] + DFD_C2 * wv[q] + DFD_C1 * wv[q + d.sx];
      }
      X[c] = x * r;
      Y[c] = G5(wv, q, 1, FY) * r;
    }
    if (a.freenode && km == 1) {
      const float* mx = a.mVx2Vz + (j1 + (long long)i * d.ny) * 9;
      const float* my = a.mVy2Vz + (j1 + (long long)i * d.ny) * 9;
#pragma unroll
      for (int c = 0; c < 3; c++)
        Z[c] = mx[3 * c] * X[0] + mx[3 * c + 1] * X[1] + mx[3 * c + 2] * X[2] + my[3 * c] * Y[0] + my[3 * c + 1] * Y[1] +
               my[3 * c + 2] * Y[2];
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float* wv = W + c * n;
        float zz;
        if (a.freenode && km == 2) zz = G2(wv, q, d.py, FZ);
        else if (a.freenode && km == 3) zz = G3(wv, q, d.py, FZ);
        else zz = G5(wv, q, d.py, FZ);
        Z[c] = zz * r;
      }
    }
    float hT[6];
    hooke(M, n, q, X, Y, Z, hT);
    float damp = a.dampx ? fminf(a.dampx[i], dampyz) : 1.0f;
    const float h9[9] = {hv[0], hv[1], hv[2], hT[0], hT[1], hT[2], hT[3], hT[4], hT[5]};
    rk_store9(a, q, h9, damp);
  }

  // ---------------- split nodes (part 6)
  if (part != 6) return;
  float hF[9][2];
  // velocity RHS on both sides (fault_dvelo.cu:260-385)
#pragma unroll
  for (int m = 0; m < 2; m++) {
    float rrj = 1.0f / (a.rhof[m * nyz + pf] * M[9 * n + idx3(d, i0, j1, k1)]);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* T = a.T1 + c * 7 * nyz + pf;
      float dx = m == 0 ? r * (DFD_A0M * T[3 * nyz] - DFD_A1 * T[2 * nyz] - DFD_A2 * T[1 * nyz] - DFD_A3 * T[0])
                        : r * (DFD_A0P * T[3 * nyz] + DFD_A1 * T[4 * nyz] + DFD_A2 * T[5 * nyz] + DFD_A3 * T[6 * nyz]);
      const float* t2 = FW + (3 + c) * 2 * nyz + m * nyz;
      float dy = (ry ? G2(t2, pf, 1, FY) : G5(t2, pf, 1, FY)) * r;
      float v3[7];
      const float* t3 = FW + (6 + c) * 2 * nyz + m * nyz;
#pragma unroll
      for (int s = 0; s < 7; s++) v3[s] = t3[pf + (long long)(s - 3) * d.ny];
      float dz;
      if (a.freenode && km <= 3) {
        v3[km + 2] = 0.0f;
        for (int s = km + 3; s < 7; s++) v3[s] = -v3[2 * (km + 2) - s];
        dz = L5(v3, 3, FZ) * r;
      } else {
        dz = (rz ? L2(v3, 3, FZ) : L5(v3, 3, FZ)) * r;
      }
      hF[c][m] = (dx + dy + dz) * rrj;
    }
  }
  // split-node velocity gradients (fault_dstrs_{f,b}.cu:175-872)
  {
    float DxV[2][3], DyV[2][3], DzV[2][3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* fv = FW + c * 2 * nyz;
      const float* wv = W + c * n;
#pragma unroll
      for (int m = 0; m < 2; m++) DyV[m][c] = (ry ? G2(fv + m * nyz, pf, 1, FY) : G5(fv + m * nyz, pf, 1, FY)) * r;
      if (FX == 1) DxV[1][c] = (wv[idx3(d, i0 + 1, j1, k1)] - fv[nyz + pf]) * r;
      else DxV[0][c] = (fv[pf] - wv[idx3(d, i0 - 1, j1, k1)]) * r;
    }
    if (a.freenode && km == 1) {
      float o1[3], o2[3], o3[3];
      if (FX == 1) {
        tfmv(a.tabf, TF_P2M1, d.ny, j1, DxV[1], o1);
        tfmv(a.tabf, TF_P2M2, d.ny, j1, DyV[1], o2);
        tfmv(a.tabf, TF_P2M3, d.ny, j1, DyV[0], o3);
#pragma unroll
        for (int c = 0; c < 3; c++) DxV[0][c] = o1[c] + o2[c] - o3[c];
      } else {
        tfmv(a.tabf, TF_M2P1, d.ny, j1, DxV[0], o1);
        tfmv(a.tabf, TF_M2P2, d.ny, j1, DyV[0], o2);
        tfmv(a.tabf, TF_M2P3, d.ny, j1, DyV[1], o3);
#pragma unroll
        for (int c = 0; c < 3; c++) DxV[1][c] = o1[c] + o2[c] - o3[c];
      }
      tfmv(a.tabf, TF_VX2VZ1, d.ny, j1, DxV[0], o1);
      tfmv(a.tabf, TF_VY2VZ1, d.ny, j1, DyV[0], o2);
#pragma unroll
      for (int c = 0; c < 3; c++) DzV[0][c] = o1[c] + o2[c];
      tfmv(a.tabf, TF_VX2VZ2, d.ny, j1, DxV[1], o1);
      tfmv(a.tabf, TF_VY2VZ2, d.ny, j1, DyV[1], o2);
#pragma unroll
      for (int c = 0; c < 3; c++) DzV[1][c] = o1[c] + o2[c];
    } else {
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int m = 0; m < 2; m++) {
          const float* fv = FW + c * 2 * nyz + m * nyz;
          float zz;
          if (a.freenode && km == 2) zz = G2(fv, pf, d.ny, FZ);
          else if (a.freenode && km == 3) zz = G3(fv, pf, d.ny, FZ);
          else zz = rz ? G2(fv, pf, d.ny, FZ) : G5(fv, pf, d.ny, FZ);
          DzV[m][c] = zz * r;
        }
      float dt[3] = {0.0f, 0.0f, 0.0f};
      if (a.faultgrid[q2]) {
#pragma unroll
        for (int c = 0; c < 3; c++) dt[c] = a.hT1[c * nyz + pf];
      }
      float o1[3], o2[3], o3[3];
      tmv(a.tab, T_T1VXM, nyz, pf, dt, o1);
      tmv(a.tab, T_VYVXM, nyz, pf, DyV[0], o2);
      tmv(a.tab, T_VZVXM, nyz, pf, DzV[0], o3);
#pragma unroll
      for (int c = 0; c < 3; c++) DxV[0][c] = o1[c] - o2[c] - o3[c];
      tmv(a.tab, T_T1VXP, nyz, pf, dt, o1);
      tmv(a.tab, T_VYVXP, nyz, pf, DyV[1], o2);
      tmv(a.tab, T_VZVXP, nyz, pf, DzV[1], o3);
#pragma unroll
      for (int c = 0; c < 3; c++) DxV[1][c] = o1[c] - o2[c] - o3[c];
    }
    // split-node traction rates (fault_dstrs_f.cu:876-1006)
#pragma unroll
    for (int m = 0; m < 2; m++)
#pragma unroll
      for (int g = 0; g < 2; g++) {
        int t0 = (m == 0 ? T_D21_1 : T_D21_2) + 3 * g;
        float o1[3], o2[3], o3[3];
        tmv(a.tab, t0, nyz, pf, DxV[m], o1);
        tmv(a.tab, t0 + 1, nyz, pf, DyV[m], o2);
        tmv(a.tab, t0 + 2, nyz, pf, DzV[m], o3);
#pragma unroll
        for (int c = 0; c < 3; c++) hF[3 + 3 * g + c][m] = o1[c] + o2[c] + o3[c];
      }
  }
  // split-node RK4 + viscosity (rk4.cu:656-727), then the RK-weighted on-fault outputs
  // (rk4.cu:521-569) and the fault plane of the stage output (transform.cu via
  // main.cu:504).  Every load comes before the first store: the compiler cannot prove the
  // buffers distinct, and a load behind a store would wait a memory round trip each.
  float r0[9][2], r1[9][2];
#pragma unroll
  for (int f = 0; f < 9; f++)
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const long long x = f * 2 * nyz + m * nyz + pf;
      if (a.irk == 0) {
        r0[f][m] = FW[x];
      } else if (a.irk < 3) {
        r0[f][m] = a.Fm[x];
        r1[f][m] = a.Ft[x];
      } else {
        r1[f][m] = a.Ft[x];
      }
    }
  float s1[3], s2[3];
#pragma unroll
  for (int c = 0; c < 3; c++) { s1[c] = a.vecs1[c * nyz + pf]; s2[c] = a.vecs2[c * nyz + pf]; }
  const float tts1 = a.tTs1[q2], tts2 = a.tTs2[q2], ttn = a.tTn[q2];
  float ts1 = 0.0f, ts2 = 0.0f, tn = 0.0f;
  if (a.irk != 0) { ts1 = a.Ts1[q2]; ts2 = a.Ts2[q2]; tn = a.Tn[q2]; }
  const float vis = a.viscosity * a.DT;
  float wv[9][2];
#pragma unroll
  for (int f = 0; f < 9; f++)
#pragma unroll
    for (int m = 0; m < 2; m++) {
      const long long x = f * 2 * nyz + m * nyz + pf;
      const float h = hF[f][m];
      float w;
      if (a.irk == 0) {
        a.Fm[x] = r0[f][m];
        a.Ft[x] = fmaf(a.rkb, h, r0[f][m]);
        w = fmaf(a.rka, h, r0[f][m]);
      } else if (a.irk < 3) {
        a.Ft[x] = fmaf(a.rkb, h, r1[f][m]);
        w = fmaf(a.rka, h, r0[f][m]);
      } else {
        w = fmaf(a.rkb, h, r1[f][m]);
      }
      if (f >= 3) w += vis * h;
      a.FWout[x] = w;
      wv[f][m] = w;
    }
  {
    float dV[3];
#pragma unroll
    for (int c = 0; c < 3; c++) dV[c] = wv[c][1] - wv[c][0];
    float vs1 = dV[0] * s1[0] + dV[1] * s1[1] + dV[2] * s1[2];
    float vs2 = dV[0] * s2[0] + dV[1] * s2[1] + dV[2] * s2[2];
    a.hslip[q2] = sqrtf(vs2 * vs2 + vs1 * vs1);
    a.Vs1[q2] = vs1;
    a.Vs2[q2] = vs2;
    float rkb1 = a.rkb / a.DT;
    if (a.irk == 0) {
      a.Ts1[q2] = rkb1 * tts1; a.Ts2[q2] = rkb1 * tts2; a.Tn[q2] = rkb1 * ttn;
    } else {
      a.Ts1[q2] = ts1 + rkb1 * tts1; a.Ts2[q2] = ts2 + rkb1 * tts2; a.Tn[q2] = tn + rkb1 * ttn;
    }
  }
  float damp0 = a.dampx ? fminf(a.dampx[i0], dampyz) : 1.0f;
  fault_to_volume_r(a, wv, a.Wout, j1, k1, damp0);
}

template <int FY, int FZ>
__global__ void __launch_bounds__(128) fault_node_kernel(const __grid_constant__ FaultArgs a) {
  __shared__ __align__(16) float snet[4 * NET_PIECES];
  fault_node_body<FY, FZ>(a, blockIdx.x, snet);
}
// grid z: the part (six off-fault layers, then the split nodes), so that the seven
// independent pieces of a fault column run in parallel.  At most 128 registers (four
// blocks per SM): this latency-bound kernel gains more from the resident warps than it
// loses to the few spilled values (measured: 3, 4, 5, 6 blocks per SM).
template <int FX, int FY, int FZ>
__global__ void __launch_bounds__(128, 4) fault_band_kernel(const __grid_constant__ FaultArgs a) {
  fault_band_body<FX, FY, FZ>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Batched launches over the scenarios of an ensemble: scenario s owns the blocks
// [start[s], start[s+1]) of a 1-D grid, laid out as its own (32, 4)-block grid over (NY, NZ).
template <int FY, int FZ>
__global__ void __launch_bounds__(128) fault_node_batch(const FaultArgs* __restrict__ tab, const int* __restrict__ start,
                                                        int n) {
  __shared__ __align__(16) float snet[4 * NET_PIECES];
  __shared__ __align__(16) unsigned char raw[sizeof(FaultArgs)];
  FaultArgs* sa = reinterpret_cast<FaultArgs*>(raw);
  int loc;
  const int sc = scenario_of(start, n, blockIdx.x, &loc);
  stage_args(sa, tab + sc);
  __syncthreads();
  fault_node_body<FY, FZ>(*sa, loc, snet);
}
template <int FX, int FY, int FZ>
__global__ void __launch_bounds__(128, 4) fault_band_batch(const FaultArgs* __restrict__ tab, const int* __restrict__ start,
                                                        int n) {
  __shared__ __align__(16) unsigned char raw[sizeof(FaultArgs)];
  FaultArgs* sa = reinterpret_cast<FaultArgs*>(raw);
  int loc;
  const int sc = scenario_of(start, n, blockIdx.x, &loc);
  stage_args(sa, tab + sc);
  __syncthreads();
  const FaultArgs& a = *sa;
  const int gx = (a.d.nj + 31) / 32, gxy = gx * ((a.d.nk + 3) / 4);
  // the scenario's blocks: seven parts of its (32, 4)-block grid
  fault_band_body<FX, FY, FZ>(a, (loc % gxy) % gx, (loc % gxy) / gx, loc / gxy);
}

// Thermal pressurisation (thermpress.cu:22-236), once per step before the stages.  Each
// fault node carries a column of n points normal to the fault with temperature T and pore
// pressure P; nsub explicit sub-steps of
//   dT = alpha_th T'' + omega(x),  dP = alpha_hy P'' + Lambda dT,
// with mirrored ends, the frictional work tau V = -friction (Tn + P0) V spread as a Gaussian
// of half-width h = 20 mm, column width sqrt(100 alpha_max), spacing width / (n - 1) and
// sub-step 0.1 dh^2 / alpha_max, so nsub grows as (n - 1)^2.  The second differences and the
// Gaussian are evaluated in double as the reference's double literals make them; stored
// values are FP32.  Columns are node-major ([q][i]); point 0 of T and P is also written to
// two (NZ, NY) planes, which the friction law and the outputs read.

// per-node scalars of the scheme (thermpress.cu:150-175), as the reference rounds them
struct TpNode {
  float rate, Tau_n, fr, ahy, dh, dh2, dt;
  int nsub;
  double fden;
};
__device__ __forceinline__ TpNode tp_node(const TpArgs& a, int q) {
  const float rho_c = 2.7e6f, h = 20e-3f, alpha_th = 1.0e-6f;
  TpNode t;
  const float vs1 = a.Vs1[q], vs2 = a.Vs2[q];
  t.rate = sqrtf(vs1 * vs1 + vs2 * vs2);
  t.Tau_n = a.Tn[q];
  t.fr = a.friction[q];
  t.ahy = a.hy[q];
  const float amax = fmaxf(alpha_th, t.ahy);
  const float w = (float)sqrt(4.0 * (double)amax * 25.0);
  t.dh = (float)((double)w / (double)(a.n - 1));
  t.dh2 = t.dh * t.dh;
  const float dt0 = (float)(0.1 * (double)t.dh2 / (double)amax);
  t.nsub = (int)(a.DT / dt0) + 1;
  t.dt = (float)((double)a.DT / (double)t.nsub);
  t.fden = (double)(rho_c * h) * 2.506628274631000;
  return t;
}

// one point: new T and P from the old values of the point (c) and its plus (r) and minus
// (l) neighbours; g = exp(-x^2 / 2h^2) in double, fac = tau V / (rho_c h sqrt(2 pi))
__device__ __forceinline__ void tp_point(const TpNode& t, double g, double fac, float Tc, float Tr, float Tl, float Pc,
                                         float Pr, float Pl, float* To, float* Po) {
  const float Lamb = 0.1e6f, alpha_th = 1.0e-6f;
  const float omega = (float)(g * fac);
  const float dT = (float)((double)alpha_th * ((double)Tr - 2.0 * (double)Tc + (double)Tl) / (double)t.dh2 +
                           (double)omega);
  const float dP = (float)((double)t.ahy * ((double)Pr - 2.0 * (double)Pc + (double)Pl) / (double)t.dh2 +
                           (double)(Lamb * dT));
  *To = fmaf(t.dt, dT, Tc);
  *Po = fmaf(t.dt, dP, Pc);
}

__device__ __forceinline__ double tp_gauss(const TpNode& t, int i) {
  const float h = 20e-3f, h2 = h * h;
  const float x = (float)i * t.dh;
  const float x2 = x * x;
  return exp(-0.5 * (double)x2 / (double)h2);
}

// One warp per node for n <= 32 K: lane l holds points l + 32 m (m < K) in registers, so a
// column is read and written once per step (coalesced: the points of a column are
// contiguous) and every sub-step runs in registers, the neighbours exchanged by shuffles.
template <int K>
__global__ void __launch_bounds__(256) thermpress_warp_kernel(const TpArgs a) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int q = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);  // uniform in the warp
  if (q >= a.nf || a.united[q]) return;
  const TpNode t = tp_node(a, q);
  const int n = a.n;
  float* Tq = a.T + (long long)q * n;
  float* Pq = a.P + (long long)q * n;
  float T[K], P[K];
  double g[K];
#pragma unroll
  for (int m = 0; m < K; m++) {
    const int i = lane + 32 * m;
    T[m] = i < n ? Tq[i] : 0.0f;
    P[m] = i < n ? Pq[i] : 0.0f;
    g[m] = tp_gauss(t, i);
  }
  for (int sub = 0; sub < t.nsub; sub++) {
    const float P0 = __shfl_sync(FULL, P[0], 0);
    const float tau = -t.fr * (t.Tau_n + P0);
    const double fac = (double)(tau * t.rate) / t.fden;
    float Tn[K], Pn[K];
#pragma unroll
    for (int m = 0; m < K; m++) {
      const int i = lane + 32 * m;
      // plus neighbour: lane + 1 of the same m, lane 0 of m + 1 for lane 31
      float Tr = __shfl_down_sync(FULL, T[m], 1), Pr = __shfl_down_sync(FULL, P[m], 1);
      const float Tr2 = __shfl_sync(FULL, m + 1 < K ? T[m + 1 < K ? m + 1 : m] : 0.0f, 0);
      const float Pr2 = __shfl_sync(FULL, m + 1 < K ? P[m + 1 < K ? m + 1 : m] : 0.0f, 0);
      // minus neighbour: lane - 1 of the same m, lane 31 of m - 1 for lane 0
      float Tl = __shfl_up_sync(FULL, T[m], 1), Pl = __shfl_up_sync(FULL, P[m], 1);
      const float Tl2 = __shfl_sync(FULL, m > 0 ? T[m > 0 ? m - 1 : 0] : 0.0f, 31);
      const float Pl2 = __shfl_sync(FULL, m > 0 ? P[m > 0 ? m - 1 : 0] : 0.0f, 31);
      if (lane == 31) { Tr = Tr2; Pr = Pr2; }
      if (lane == 0) { Tl = Tl2; Pl = Pl2; }
      // the ends mirror their one neighbour (thermpress.cu:201-207)
      if (i == 0) { Tl = Tr; Pl = Pr; }
      if (i == n - 1) { Tr = Tl; Pr = Pl; }
      tp_point(t, g[m], fac, T[m], Tr, Tl, P[m], Pr, Pl, &Tn[m], &Pn[m]);
    }
#pragma unroll
    for (int m = 0; m < K; m++)
      if (lane + 32 * m < n) { T[m] = Tn[m]; P[m] = Pn[m]; }
  }
#pragma unroll
  for (int m = 0; m < K; m++) {
    const int i = lane + 32 * m;
    if (i < n) { Tq[i] = T[m]; Pq[i] = P[m]; }
  }
  if (lane == 0) { a.T0[q] = T[0]; a.P0[q] = P[0]; }
}

// Longer columns: one thread per node walking its column in place each sub-step, the old
// value of the point below kept in a register.
__global__ void __launch_bounds__(128) thermpress_column_kernel(const TpArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.nf || a.united[q]) return;
  const TpNode t = tp_node(a, q);
  const int n = a.n;
  float* T = a.T + (long long)q * n;
  float* P = a.P + (long long)q * n;
  for (int sub = 0; sub < t.nsub; sub++) {
    const float tau = -t.fr * (t.Tau_n + P[0]);
    const double fac = (double)(tau * t.rate) / t.fden;
    float Tb = 0.0f, Pb = 0.0f;  // old values of point i - 1
    float Tc = T[0], Pc = P[0];  // old values of point i
    for (int i = 0; i < n; i++) {
      float Ta = 0.0f, Pa = 0.0f;  // old values of point i + 1
      if (i + 1 < n) { Ta = T[i + 1]; Pa = P[i + 1]; }
      const float Tr = i == n - 1 ? Tb : Ta, Pr = i == n - 1 ? Pb : Pa;
      const float Tl = i == 0 ? Ta : Tb, Pl = i == 0 ? Pa : Pb;
      tp_point(t, tp_gauss(t, i), fac, Tc, Tr, Tl, Pc, Pr, Pl, &T[i], &P[i]);
      Tb = Tc; Pb = Pc;
      Tc = Ta; Pc = Pa;
    }
  }
  a.T0[q] = T[0];
  a.P0[q] = P[0];
}

void launch_thermpress(const TpArgs& a, cudaStream_t s) {
  const int K = (a.n + 31) / 32;
  const unsigned wblocks = (unsigned)(((long long)a.nf * 32 + 255) / 256);
  if (K <= 1) thermpress_warp_kernel<1><<<wblocks, 256, 0, s>>>(a);
  else if (K <= 2) thermpress_warp_kernel<2><<<wblocks, 256, 0, s>>>(a);
  else if (K <= 4) thermpress_warp_kernel<4><<<wblocks, 256, 0, s>>>(a);
  else if (K <= 8) thermpress_warp_kernel<8><<<wblocks, 256, 0, s>>>(a);
  else if (K <= 16) thermpress_warp_kernel<16><<<wblocks, 256, 0, s>>>(a);
  else thermpress_column_kernel<<<(a.nf + 127) / 128, 128, 0, s>>>(a);
}

// Rupture sensor (rup_sensor.cu:8-95), once per step before the stages.  On the fault
// grid shrunk by 3 nodes (1-based indices), with p = Ts1 and, for non-united nodes,
//   Dy = 0.25 (2 p - p[j+1] - p[j-1]),  Dz = 0.25 (2 p - p[k+1] - p[k-1])  (zero elsewhere),
//   sensor = 0.5 ((Dy - Dy[j+1])^2 + (Dy - Dy[j-1])^2)
//          + 0.5 ((Dz - Dy[k+1])^2 + (Dz - Dy[k-1])^2),  divided by p^2 + 1e-16, + 1e-16,
// zero on united nodes; the z term takes Dy at the z neighbours, as the reference does.
// The reference's two kernels (differences, then magnitude) become one: each thread
// evaluates the five differences it needs.  Nodes outside the shrunk grid keep their zero.
struct SensorGrid {
  const SensorArgs& a;
  __device__ bool inside(int j, int k) const {
    return j + 1 >= a.fg[0] + 3 && j + 1 <= a.fg[1] - 3 && k + 1 >= a.fg[2] + 3 && k + 1 <= a.fg[3] - 3 &&
           (!a.slab || (j >= 2 && j < a.nj - 2));
  }
  // second difference of Ts1 along stride s at node (j, k), zero where the reference never
  // writes it
  __device__ float diff(int j, int k, int s) const {
    const int q = j + a.nj * k;
    if (!inside(j, k) || a.united[q]) return 0.0f;
    const float* p = a.Ts1;
    return (float)(0.25 * (-p[q + s] + 2.0 * p[q] - p[q - s]));
  }
};

__global__ void __launch_bounds__(128) rup_sensor_kernel(const SensorArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, k = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= a.nj || k >= a.nk) return;
  const SensorGrid g{a};
  if (!g.inside(j, k)) return;
  const int q = j + a.nj * k, nj = a.nj;
  const float dy = g.diff(j, k, 1), dz = g.diff(j, k, nj);
  float D1 = dy - g.diff(j + 1, k, 1);
  float D2 = dy - g.diff(j - 1, k, 1);
  float mag = (float)(0.5 * (D1 * D1 + D2 * D2));
  D1 = dz - g.diff(j, k + 1, 1);
  D2 = dz - g.diff(j, k - 1, 1);
  mag = (float)(mag + 0.5 * (D1 * D1 + D2 * D2));
  const float p0 = a.Ts1[q] * a.Ts1[q];
  a.out[q] = a.united[q] ? 0.0f : (float)(mag / (p0 + 1e-16) + 1e-16);
}

void launch_rup_sensor(const SensorArgs& a, cudaStream_t s) {
  dim3 block(32, 4, 1);
  dim3 grid((a.nj + 31) / 32, (a.nk + 3) / 4, 1);
  rup_sensor_kernel<<<grid, block, 0, s>>>(a);
}

void launch_fault_node(const FaultArgs& a, cudaStream_t s) {
  dim3 block(128, 1, 1);
  dim3 grid(node_blocks(a.NY, a.NZ, a.freenode, a.jg0, a.d.nj), 1, 1);
  int code = (a.FY > 0) * 2 + (a.FZ > 0);
  switch (code) {
    case 0: fault_node_kernel<-1, -1><<<grid, block, 0, s>>>(a); break;
    case 1: fault_node_kernel<-1, 1><<<grid, block, 0, s>>>(a); break;
    case 2: fault_node_kernel<1, -1><<<grid, block, 0, s>>>(a); break;
    default: fault_node_kernel<1, 1><<<grid, block, 0, s>>>(a); break;
  }
}

void launch_fault_band(const FaultArgs& a, cudaStream_t s) {
  dim3 block(32, 4, 1);
  dim3 grid((a.d.nj + 31) / 32, (a.d.nk + 3) / 4, 7);
  int code = (a.FX > 0) * 4 + (a.FY > 0) * 2 + (a.FZ > 0);
  switch (code) {
    case 0: fault_band_kernel<-1, -1, -1><<<grid, block, 0, s>>>(a); break;
    case 1: fault_band_kernel<-1, -1, 1><<<grid, block, 0, s>>>(a); break;
    case 2: fault_band_kernel<-1, 1, -1><<<grid, block, 0, s>>>(a); break;
    case 3: fault_band_kernel<-1, 1, 1><<<grid, block, 0, s>>>(a); break;
    case 4: fault_band_kernel<1, -1, -1><<<grid, block, 0, s>>>(a); break;
    case 5: fault_band_kernel<1, -1, 1><<<grid, block, 0, s>>>(a); break;
    case 6: fault_band_kernel<1, 1, -1><<<grid, block, 0, s>>>(a); break;
    default: fault_band_kernel<1, 1, 1><<<grid, block, 0, s>>>(a); break;
  }
}

// tab, start: device arrays of n scenarios (start has n + 1 entries, start[n] = blocks);
// FX, FY, FZ are the ensemble's (every scenario is at the same step and stage)
void launch_fault_node_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FY, int FZ,
                             cudaStream_t s) {
  dim3 block(128, 1, 1);
  int code = (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: fault_node_batch<-1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 1: fault_node_batch<-1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 2: fault_node_batch<1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    default: fault_node_batch<1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
  }
}
void launch_fault_band_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FX, int FY, int FZ,
                             cudaStream_t s) {
  dim3 block(32, 4, 1);
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: fault_band_batch<-1, -1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 1: fault_band_batch<-1, -1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 2: fault_band_batch<-1, 1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 3: fault_band_batch<-1, 1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 4: fault_band_batch<1, -1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 5: fault_band_batch<1, -1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
    case 6: fault_band_batch<1, 1, -1><<<blocks, block, 0, s>>>(tab, start, n); break;
    default: fault_band_batch<1, 1, 1><<<blocks, block, 0, s>>>(tab, start, n); break;
  }
}

}  // namespace dfd
