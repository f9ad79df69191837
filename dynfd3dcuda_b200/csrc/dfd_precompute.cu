// FP64 precompute of the split-node coefficient tables and the free-surface velocity
// transforms on the GPU (reference fault_coef.cu:26-1312 and :1320-1486, which compute
// them in the working precision).  One thread per padded fault node (j, k) or per
// surface node (i, j); results are rounded to FP32 planes once.
#include "dfd_internal.cuh"

namespace dfd {

typedef double D3[3][3];

__device__ inline void dinv3(const D3 a, D3 r) {
  double c00 = a[1][1] * a[2][2] - a[2][1] * a[1][2], c01 = a[2][1] * a[0][2] - a[0][1] * a[2][2];
  double c02 = a[0][1] * a[1][2] - a[0][2] * a[1][1], c10 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
  double c11 = a[0][0] * a[2][2] - a[2][0] * a[0][2], c12 = a[1][0] * a[0][2] - a[0][0] * a[1][2];
  double c20 = a[1][0] * a[2][1] - a[1][1] * a[2][0], c21 = a[2][0] * a[0][1] - a[0][0] * a[2][1];
  double c22 = a[0][0] * a[1][1] - a[0][1] * a[1][0];
  double det = 1.0 / (c00 * a[0][0] + c01 * a[1][0] + c02 * a[2][0]);
  r[0][0] = c00 * det; r[0][1] = c01 * det; r[0][2] = c02 * det;
  r[1][0] = c10 * det; r[1][1] = c11 * det; r[1][2] = c12 * det;
  r[2][0] = c20 * det; r[2][1] = c21 * det; r[2][2] = c22 * det;
}
__device__ inline void dmul3(const D3 a, const D3 b, D3 c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) c[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
}
__device__ inline void dcross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
// traction-gradient coupling D_ab[p][q] = s*(lam ea[p] eb[q] + mu ea[q] eb[p] + delta_pq mu ea.eb)
// (the expanded matrices of fault_coef.cu:362-581 and :1411-1440)
__device__ inline void dmat(const double* ea, const double* eb, double lam, double mu, double s, D3 D) {
  double dot = ea[0] * eb[0] + ea[1] * eb[1] + ea[2] * eb[2];
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) D[p][q] = s * (lam * ea[p] * eb[q] + mu * ea[q] * eb[p] + (p == q ? mu * dot : 0.0));
}
__device__ inline void put(float* tab, int t, long long nyz, long long f, const D3 m) {
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) tab[(long long)(t * 9 + 3 * r + c) * nyz + f] = (float)m[r][c];
}

__global__ void fault_coef_kernel(Dims d, const float* __restrict__ M, float* tab, float* tabf, float* vecn,
                                  float* vecs1, float* vecs2, float* rhof) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int k = blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= d.ny || k >= d.nz) return;
  const long long n = d.nxyz, nyz = d.nyz;
  long long q = idx3(d, d.i0, j, k), f = j + (long long)k * d.ny;
  double e[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) e[r][c] = M[(3 * r + c) * n + q];
  double jac = M[9 * n + q];
  D3 inv;
  dinv3(e, inv);
  double xxi[3] = {inv[0][0], inv[1][0], inv[2][0]};
  double xet[3] = {inv[0][1], inv[1][1], inv[2][1]};
  double xzt[3] = {inv[0][2], inv[1][2], inv[2][2]};
  // base vectors (fault_coef.cu:206-248)
  double s1[3], nv[3], s2[3];
  double ns = sqrt(xet[0] * xet[0] + xet[1] * xet[1] + xet[2] * xet[2]);
  double nn = sqrt(e[0][0] * e[0][0] + e[0][1] * e[0][1] + e[0][2] * e[0][2]);
  for (int c = 0; c < 3; c++) { s1[c] = xet[c] / ns; nv[c] = e[0][c] / nn; }
  dcross(nv, s1, s2);
  for (int c = 0; c < 3; c++) {
    vecn[c * nyz + f] = (float)nv[c];
    vecs1[c * nyz + f] = (float)s1[c];
    vecs2[c * nyz + f] = (float)s2[c];
  }
  double lamf[2], muf[2];
  for (int m = 0; m < 2; m++) {
    long long qm = q + (m == 0 ? -d.sx : d.sx);
    rhof[m * nyz + f] = M[12 * n + qm];
    lamf[m] = M[10 * n + qm];
    muf[m] = M[11 * n + qm];
  }
  D3 Dm[2][3][3];
  for (int m = 0; m < 2; m++)
    for (int aa = 0; aa < 3; aa++)
      for (int bb = 0; bb < 3; bb++) dmat(e[aa], e[bb], lamf[m], muf[m], jac, Dm[m][aa][bb]);
  for (int m = 0; m < 2; m++)
    for (int g = 0; g < 2; g++)
      for (int bb = 0; bb < 3; bb++) put(tab, (m ? T_D21_2 : T_D21_1) + 3 * g + bb, nyz, f, Dm[m][1 + g][bb]);
  // B_b = Q D_1b + A2 D_2b + A3 D_3b (fault_coef.cu:158-196, 628-672)
  D3 Q, A2, A3;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) Q[r][c] = e[0][c];
  double a2[3][3] = {{xet[1], -xet[0], 0.0}, {xet[2], 0.0, -xet[0]}, {0.0, xet[2], -xet[1]}};
  double a3[3][3] = {{xzt[1], -xzt[0], 0.0}, {xzt[2], 0.0, -xzt[0]}, {0.0, xzt[2], -xzt[1]}};
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) { A2[r][c] = a2[r][c]; A3[r][c] = a3[r][c]; }
  (void)xxi;
  D3 B[2][3];
  for (int m = 0; m < 2; m++)
    for (int bb = 0; bb < 3; bb++) {
      D3 t1, t2, t3;
      dmul3(Q, Dm[m][0][bb], t1); dmul3(A2, Dm[m][1][bb], t2); dmul3(A3, Dm[m][2][bb], t3);
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) B[m][bb][r][c] = t1[r][c] + t2[r][c] + t3[r][c];
    }
  D3 t, iD;
  // T1-rate maps (the final definitions of fault_coef.cu:823-865)
  for (int m = 0; m < 2; m++) {
    dinv3(Dm[m][0][0], iD);
    put(tab, m ? T_T1VXP : T_T1VXM, nyz, f, iD);
    dmul3(iD, Dm[m][0][1], t); put(tab, m ? T_VYVXP : T_VYVXM, nyz, f, t);
    dmul3(iD, Dm[m][0][2], t); put(tab, m ? T_VZVXP : T_VZVXM, nyz, f, t);
  }
  // continuity maps (fault_coef.cu:868-968)
  dinv3(B[1][0], iD);
  dmul3(iD, B[0][0], t); put(tab, T_M2P1, nyz, f, t);
  dmul3(iD, B[0][1], t); put(tab, T_M2P2, nyz, f, t);
  dmul3(iD, B[0][2], t); put(tab, T_M2P3, nyz, f, t);
  dmul3(iD, B[1][1], t); put(tab, T_M2P4, nyz, f, t);
  dmul3(iD, B[1][2], t); put(tab, T_M2P5, nyz, f, t);
  dinv3(B[0][0], iD);
  dmul3(iD, B[1][0], t); put(tab, T_P2M1, nyz, f, t);
  dmul3(iD, B[1][1], t); put(tab, T_P2M2, nyz, f, t);
  dmul3(iD, B[1][2], t); put(tab, T_P2M3, nyz, f, t);
  dmul3(iD, B[0][1], t); put(tab, T_P2M4, nyz, f, t);
  dmul3(iD, B[0][2], t); put(tab, T_P2M5, nyz, f, t);
  // free-surface row (fault_coef.cu:1046-1240)
  if (k == d.nz - 4) {
    D3 iA, mB, mC, vx[2], vy[2];
    for (int m = 0; m < 2; m++) {
      dinv3(Dm[m][2][2], iA);
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) { mB[r][c] = -Dm[m][2][0][r][c]; mC[r][c] = -Dm[m][2][1][r][c]; }
      dmul3(iA, mB, vx[m]); dmul3(iA, mC, vy[m]);
    }
    put(tabf, TF_VX2VZ1, d.ny, j, vx[0]); put(tabf, TF_VY2VZ1, d.ny, j, vy[0]);
    put(tabf, TF_VX2VZ2, d.ny, j, vx[1]); put(tabf, TF_VY2VZ2, d.ny, j, vy[1]);
    double v1[3] = {e[0][0], e[0][1], e[0][2]};
    double v1n = sqrt(v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2]);
    double v3[3];
    dcross(v1, xet, v3);
    double h[3];
    for (int aa = 0; aa < 3; aa++) h[aa] = (v3[0] * e[aa][0] + v3[1] * e[aa][1] + v3[2] * e[aa][2]) / v1n;
    double muc = M[11 * n + q];
    D3 Df[2][3];
    for (int m = 0; m < 2; m++)
      for (int bb = 0; bb < 3; bb++)
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) Df[m][bb][r][c] = Dm[m][0][bb][r][c] + muc * h[bb] * v3[r] * v1[c];
    D3 Vx1, Vy1, Vx2, Vy2, tmp;
    dmul3(Df[0][2], vx[0], tmp);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vx1[r][c] = Df[0][0][r][c] + tmp[r][c];
    dmul3(Df[0][2], vy[0], tmp);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vy1[r][c] = Df[0][1][r][c] + tmp[r][c];
    dmul3(Df[1][2], vx[1], tmp);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vx2[r][c] = Df[1][0][r][c] + tmp[r][c];
    dmul3(Df[1][2], vy[1], tmp);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vy2[r][c] = Df[1][1][r][c] + tmp[r][c];
    D3 iv;
    dinv3(Vx1, iv);
    dmul3(iv, Vx2, t); put(tabf, TF_P2M1, d.ny, j, t);
    dmul3(iv, Vy2, t); put(tabf, TF_P2M2, d.ny, j, t);
    dmul3(iv, Vy1, t); put(tabf, TF_P2M3, d.ny, j, t);
    dinv3(Vx2, iv);
    dmul3(iv, Vx1, t); put(tabf, TF_M2P1, d.ny, j, t);
    dmul3(iv, Vy1, t); put(tabf, TF_M2P2, d.ny, j, t);
    dmul3(iv, Vy2, t); put(tabf, TF_M2P3, d.ny, j, t);
  }
}

// Dz V = A^-1 (B Dx V + C Dy V) on the top row with the PML 1/beta factors
// (fault_coef.cu:1320-1486).  Output layout (nx, ny, 9).
__global__ void wave_free_kernel(Dims d, const float* __restrict__ M, const float* __restrict__ Bx,
                                 const float* __restrict__ By, const float* __restrict__ Bz, float* mx, float* my) {
  int j = blockIdx.x * blockDim.x + threadIdx.x + 3;
  int i = blockIdx.y * blockDim.y + threadIdx.y + 3;
  if (j >= d.ny - 3 || i >= d.nx - 3) return;
  int k = d.nz - 4;
  const long long n = d.nxyz;
  long long q = idx3(d, i, j, k);
  double rb1 = 1.0 / (double)Bx[i - 3], rb2 = 1.0 / (double)By[j - 3], rb3 = 1.0 / (double)Bz[k - 3];
  double e[3][3];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) e[r][c] = M[(3 * r + c) * n + q];
  double lam = M[10 * n + q], mu = M[11 * n + q];
  D3 A, Bm, C, iA, AB, AC;
  dmat(e[2], e[2], lam, mu, rb3, A);
  dmat(e[2], e[0], lam, mu, -rb1, Bm);
  dmat(e[2], e[1], lam, mu, -rb2, C);
  dinv3(A, iA);
  dmul3(iA, Bm, AB);
  dmul3(iA, C, AC);
  long long o = (j + (long long)i * d.ny) * 9;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) { mx[o + 3 * r + c] = (float)AB[r][c]; my[o + 3 * r + c] = (float)AC[r][c]; }
}

void launch_fault_coef(const Dims& d, const float* M, float* tab, float* tabf, float* vecn, float* vecs1,
                       float* vecs2, float* rhof, cudaStream_t s) {
  dim3 block(32, 4);
  dim3 grid((d.ny + 31) / 32, (d.nz + 3) / 4);
  fault_coef_kernel<<<grid, block, 0, s>>>(d, M, tab, tabf, vecn, vecs1, vecs2, rhof);
}
void launch_wave_free(const Dims& d, const float* M, const float* Bx, const float* By, const float* Bz, float* mx,
                      float* my, cudaStream_t s) {
  dim3 block(32, 4);
  dim3 grid((d.ny - 6 + 31) / 32, (d.nx - 6 + 3) / 4);
  wave_free_kernel<<<grid, block, 0, s>>>(d, M, Bx, By, Bz, mx, my);
}

}  // namespace dfd
