// ORACLE -- test infrastructure only.
//
// CPU restatement of the single-rank curved-grid finite-difference
// dynamic-rupture time step of wenqiang-geophys/dynfd3dcuda, written from the
// reference's algorithm (not its code).  It is templated on the arithmetic type:
// double is the FP64 checker the CUDA path is compared against; float is the
// OpenMP CPU baseline that bench.py times.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it; the product never does.
//
// The organisation deliberately mirrors the reference's unfused kernel sequence
// (one function per reference kernel, each citing the reference file:line it
// restates) so that it checks the fused CUDA design independently.
//
// Layout (reference, common.h:99-101, wave.cu:101): a volume field is
// (nx, nz, ny) with y fastest, pos = j + k*ny + i*ny*nz, 3 ghost nodes per side.
// Split-node arrays (alloc.cu:96) are [field][side][nz][ny].
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
// Flat parameter block passed from Python (tests parse params.json themselves).
// Fields follow the reference Params struct (common.h:49-84) plus the compile-time
// switches of the reference Makefile (Makefile:57-161) as runtime flags.
typedef struct {
  int NX, NY, NZ;
  int NT;
  double TMAX, DT, DH;
  int INPORT_GRID_TYPE, INPORT_STRESS_TYPE, Friction_type;
  int PML_N;
  double PML_velocity, PML_bmax, PML_fc;
  int DAMP_N;
  double mu_s, mu_d, mu_0, Dc, C0;
  double f0, V0, Vini, fw, L;
  double smooth_load_T, viscosity;
  int Fault_grid[4];
  int Asp_grid[4];
  double bi_vp1, bi_vs1, bi_rho1, bi_vp2, bi_vs2, bi_rho2;
  int free_surface, use_pml, use_cerjan, normal_refine;
  int TP_n;  // points across the fault of the thermal-pressurisation columns (Friction_type 3)
} orc_params;
}

namespace orc {

// DRP / MacCormack coefficients (macdrp.h:23-40) and the 2-/3-point one-sided
// operators (macdrp.h:101-130).
static const double C1 = 0.29164704779069994;
static const double C2 = 0.66674514216519998;
static const double C3 = 1.2501177132452999;
static const double C4 = 0.33341180882999999;
static const double C5 = 0.041686285540599999;
static const double A0P = -1.250039237746600;  // a_0pF == a_0pB
static const double A0M = 1.250039237746600;   // a_0mF == a_0mB
static const double A1 = 1.541764761036000;
static const double A2 = -0.333411808829999;
static const double A3 = 0.0416862855405999;
static const double C24_1 = 7.0 / 6.0, C24_2 = 4.0 / 3.0, C24_3 = 1.0 / 6.0;
static const double PI_ = 3.141592653589793238463;

// The reference's vector norm (device.cu:84-89): squares summed in real_t, then sqrtf,
// so its FP64 build too rounds every norm3 to single precision.
static inline double ref_norm3(double a, double b, double c) {
  double s = a * a + b * b + c * c;
  return (double)sqrtf((float)s);
}

template <typename R> static inline R opF(const R* v, long p, long s) {
  return R(-C1 * v[p - s] - C2 * v[p] + C3 * v[p + s] - C4 * v[p + 2 * s] + C5 * v[p + 3 * s]);
}
template <typename R> static inline R opB(const R* v, long p, long s) {
  return R(-C5 * v[p - 3 * s] + C4 * v[p - 2 * s] - C3 * v[p - s] + C2 * v[p] + C1 * v[p + s]);
}
// 5-point one-sided DRP derivative in direction `fl` (macdrp.h:60-75)
template <typename R> static inline R op5(const R* v, long p, long s, int fl) {
  return fl == 1 ? opF(v, p, s) : opB(v, p, s);
}
template <typename R> static inline R op2(const R* v, long p, long s, int fl) {
  return fl == 1 ? R(v[p + s] - v[p]) : R(v[p] - v[p - s]);
}
template <typename R> static inline R op3F(const R* v, long p, long s) {
  return R(-C24_1 * v[p] + C24_2 * v[p + s] - C24_3 * v[p + 2 * s]);
}
template <typename R> static inline R op3B(const R* v, long p, long s) {
  return R(C24_3 * v[p - 2 * s] - C24_2 * v[p - s] + C24_1 * v[p]);
}
template <typename R> static inline R op3(const R* v, long p, long s, int fl) {
  return fl == 1 ? op3F(v, p, s) : op3B(v, p, s);
}

typedef double M3[3][3];
static void inv3(const M3 a, M3 r) {  // device.cu:56-82 (cofactor inverse)
  double c00 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double c01 = a[2][1] * a[0][2] - a[0][1] * a[2][2];
  double c02 = a[0][1] * a[1][2] - a[0][2] * a[1][1];
  double c10 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
  double c11 = a[0][0] * a[2][2] - a[2][0] * a[0][2];
  double c12 = a[1][0] * a[0][2] - a[0][0] * a[1][2];
  double c20 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
  double c21 = a[2][0] * a[0][1] - a[0][0] * a[2][1];
  double c22 = a[0][0] * a[1][1] - a[0][1] * a[1][0];
  double det = 1.0 / (c00 * a[0][0] + c01 * a[1][0] + c02 * a[2][0]);
  r[0][0] = c00 * det; r[0][1] = c01 * det; r[0][2] = c02 * det;
  r[1][0] = c10 * det; r[1][1] = c11 * det; r[1][2] = c12 * det;
  r[2][0] = c20 * det; r[2][1] = c21 * det; r[2][2] = c22 * det;
}
static void mul3(const M3 a, const M3 b, M3 c) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += a[i][k] * b[k][j];
      c[i][j] = s;
    }
}
static void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Time-smoothed loading G(t) (device.cu:134-143) and the nucleation taper
// F(r) (device.cu:125-132).
static double Gt(double t, double T) {
  if (t < T) {
    double t1 = t - T, t2 = t - 2.0 * T;
    return std::exp(t1 * t1 / t / t2);
  }
  return 1.0;
}
static double Fr(double r, double R) { return r < R ? std::exp(r * r / (r * r - R * R)) : 0.0; }

// RK4 stage weights, computed in the reference's single-precision way
// (rk4.cu:188-198): the weight is rounded to float and multiplied by DT in float.
static void rk_weights(int irk, float DT, float* rka, float* rkb) {
  float a, b;
  if (irk == 0) { a = 0.5f; b = (float)(1.0 / 6.0); }
  else if (irk == 1) { a = 0.5f; b = (float)(1.0 / 3.0); }
  else if (irk == 2) { a = 1.0f; b = (float)(1.0 / 3.0); }
  else { a = 1e10f; b = (float)(1.0 / 6.0); }
  *rka = a * DT;
  *rkb = b * DT;
}

// Forward/backward operator cycle (main.cu:86-94)
static const int FD_FLAGS[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, -1, 1},
                                   {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};

template <typename R> struct Sim {
  orc_params p;
  int ni, nj, nk, nx, ny, nz, i0, N;
  long nxyz, nyz;
  R DT, DH, rDH;
  bool freenode;
  // volume
  std::vector<R> W, hW, mW, tW;     // 9 * nxyz each
  std::vector<R> M;                 // 13 * nxyz (xix..ztz, jac, lam, mu, rho)
  std::vector<double> Cd;           // 3 * nxyz coordinates (double)
  std::vector<R> matVx2Vz, matVy2Vz;  // 9 * nx * ny
  // PML
  std::vector<R> Ax, Bx, Dx, Ay, By, Dy, Az, Bz, Dz;
  int isx1, isx2, isy1, isy2, isz1, isz2;
  std::vector<R> aux[6][4];  // [face][W,h,m,t]
  // Cerjan
  std::vector<R> damp;
  // fault
  std::vector<R> FW, FhW, FmW, FtW;  // 9 * 2 * nyz
  std::vector<R> T11, T12, T13, mT11, mT12, mT13, hT11, hT12, hT13;  // 7 * nyz
  std::map<std::string, std::vector<R>> fc;  // fault coefficient tables
  std::vector<R> Tn, Ts1, Ts2, tTn, tTs1, tTs2, str_init_x, str_init_y, str_init_z;
  std::vector<R> T0x, T0y, T0z, dT0x, dT0y, dT0z, str_peak, mu_d, Dc, C0, a, b, L, Vw;
  std::vector<R> hslip, slip, tslip, mslip, Vs1, Vs2, State, mState, hState, tState;
  std::vector<R> init_t0, friction;
  // thermal pressurisation: columns of TP_n points, plane i at [i * nf] (alloc.cu:94-118)
  std::vector<R> TP_T, TP_P, TP_hy;
  std::vector<R> rup_sensor, rup_Dy, rup_Dz;  // rupture sensor (rup_sensor.cu)
  std::vector<int> init_t0_flag, rup_index_y, rup_index_z, united, faultgrid, flag_rup;
  // bookkeeping for the learned-guess study: Newton iterations of the last RS trial
  long newton_iters = 0;

  R* Wf(std::vector<R>& v, int f) { return v.data() + (long)f * nxyz; }
  R* Mf(int f) { return M.data() + (long)f * nxyz; }
  long P3(int i, int j, int k) const { return j + (long)k * ny + (long)i * nyz; }

  // ---------------------------------------------------------------- setup --
  void alloc() {
    ni = p.NX; nj = p.NY; nk = p.NZ;
    nx = ni + 6; ny = nj + 6; nz = nk + 6;
    nxyz = (long)nx * ny * nz; nyz = (long)ny * nz;
    i0 = nx / 2;
    N = p.PML_N;
    DT = (R)p.DT; DH = (R)p.DH; rDH = (R)(1.0 / p.DH);
    freenode = p.free_surface != 0;
    W.assign(9 * nxyz, 0); hW.assign(9 * nxyz, 0); mW.assign(9 * nxyz, 0); tW.assign(9 * nxyz, 0);
    M.assign(13 * nxyz, 0); Cd.assign(3 * nxyz, 0);
    matVx2Vz.assign(9L * nx * ny, 0); matVy2Vz.assign(9L * nx * ny, 0);
    long nf2 = 9 * 2 * nyz;
    FW.assign(nf2, 0); FhW.assign(nf2, 0); FmW.assign(nf2, 0); FtW.assign(nf2, 0);
    for (auto* v : {&T11, &T12, &T13, &mT11, &mT12, &mT13, &hT11, &hT12, &hT13}) v->assign(7 * nyz, 0);
    long nf = (long)nj * nk;
    for (auto* v : {&Tn, &Ts1, &Ts2, &tTn, &tTs1, &tTs2, &str_init_x, &str_init_y, &str_init_z, &T0x, &T0y,
                    &T0z, &dT0x, &dT0y, &dT0z, &str_peak, &mu_d, &Dc, &C0, &a, &b, &L, &Vw, &hslip, &slip,
                    &tslip, &mslip, &Vs1, &Vs2, &State, &mState, &hState, &tState, &init_t0, &friction})
      v->assign(nf, 0);
    for (auto* v : {&init_t0_flag, &rup_index_y, &rup_index_z, &united, &faultgrid, &flag_rup}) v->assign(nf, 0);
    const int ntp = std::max(p.TP_n, 1);
    TP_T.assign(ntp * nf, 0); TP_P.assign(ntp * nf, 0); TP_hy.assign(nf, 0);
    rup_sensor.assign(nf, 0); rup_Dy.assign(nf, 0); rup_Dz.assign(nf, 0);
  }

  // PML damping profiles (init_pml.cu:18-133): d ~ x^2, alpha ~ (1-x), beta ~ 1+(bmax-1)x^2,
  // and D is stored divided by B.
  void pml_init() {
    isx1 = isx2 = isy1 = isy2 = isz1 = p.use_pml ? 1 : 0;
    isz2 = (p.use_pml && !freenode) ? 1 : 0;
    auto prof = [&](int n, int lo, int hi, std::vector<R>& A, std::vector<R>& B, std::vector<R>& D) {
      A.assign(n, 0); B.assign(n, 1); D.assign(n, 0);
      std::vector<double> Lx(n, -1.0);
      double DHd = p.DH;
      if (lo) for (int i = 0; i < N; i++) Lx[i] = (N - 1 - i) * DHd;
      if (hi) for (int i = 0; i < N; i++) Lx[n - N + i] = i * DHd;
      double Rpp = std::pow(10.0, -((std::log10((double)N) - 1.0) / std::log10(2.0) + 3.0));
      double amax = PI_ * p.PML_fc;
      double L0 = DHd * (N - 1);
      double dmax = -p.PML_velocity / (2.0 * L0) * std::log(Rpp) * (2.0 + 1.0);
      for (int i = 0; i < n; i++) {
        double x = Lx[i];
        double av = x < 0 ? 0.0 : amax * (1.0 - std::pow(x / L0, 1.0));
        double bv = x < 0 ? 1.0 : 1.0 + (p.PML_bmax - 1.0) * std::pow(x / L0, 2.0);
        double dv = x < 0 ? 0.0 : dmax * std::pow(x / L0, 2.0);
        A[i] = (R)av; B[i] = (R)bv; D[i] = (R)(dv / bv);
      }
    };
    prof(ni, isx1, isx2, Ax, Bx, Dx);
    prof(nj, isy1, isy2, Ay, By, Dy);
    prof(nk, isz1, isz2, Az, Bz, Dz);
    long sz[6] = {(long)N * nj * nk, (long)N * nj * nk, (long)N * nk * ni,
                  (long)N * nk * ni, (long)N * ni * nj, (long)N * ni * nj};
    int on[6] = {isx1, isx2, isy1, isy2, isz1, isz2};
    for (int f = 0; f < 6; f++)
      for (int r = 0; r < 4; r++) aux[f][r].assign(on[f] ? 9 * sz[f] : 0, 0);
  }

  // Grid construction (coord.cu:153-328): x-line with normal refinement near the
  // fault (coord.cu:173-209), fault surface (x,y,z)(j,k) extruded along x.
  void construct_coord(const float* fxyz) {
    std::vector<double> xline(ni + 6, 0.0);
    int ic = p.NX / 2 + 3;
    xline[ic] = 0;
    const int w1 = 10, w2 = 55;
    for (int i = ic + 1; i < ni + 6; i++) {
      int dist = std::abs(i - ic);
      double c = dist < w1 ? 0.0 : (dist < w2 ? 1.0 - std::cos(PI_ * (i - (ic + w1)) / (double)(w2 - w1)) : 2.0);
      c = 0.5 + 0.25 * c;
      xline[i] = xline[i - 1] + p.DH * c;
    }
    for (int i = ic - 1; i >= 0; i--) {
      int dist = std::abs(i - ic);
      double c = dist < w1 ? 0.0 : (dist < w2 ? 1.0 - std::cos(PI_ * (i - (ic - w1)) / (double)(w2 - w1)) : 2.0);
      c = 0.5 + 0.25 * c;
      xline[i] = xline[i + 1] - p.DH * c;
    }
    double* X = Cd.data(); double* Y = X + nxyz; double* Z = Y + nxyz;
    double x0 = -(p.NX / 2) * p.DH, y0 = -(p.NY / 2) * p.DH, z0 = (1 - p.NZ) * p.DH;
#pragma omp parallel for schedule(static)
    for (int i = 3; i < nx - 3; i++)
      for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++) {
          int gi = i - 3, gj = j - 3, gk = k - 3;
          double x = gi * p.DH + x0, y = gj * p.DH + y0, z = gk * p.DH + z0;
          if (p.normal_refine) x = xline[i];
          if (p.INPORT_GRID_TYPE == 1 && fxyz) {
            long q = (j - 3) + (long)(k - 3) * nj;
            double fx = fxyz[q], fy = fxyz[(long)nj * nk + q], fz = fxyz[2L * nj * nk + q];
            x = p.normal_refine ? fx + xline[i] : fx + gi * p.DH + x0;
            y = fy; z = fz;
          }
          long q = P3(i, j, k);
          X[q] = x; Y[q] = y; Z[q] = z;
        }
    // ghost extrapolation 2*c - d (metric.cu:248-313)
    for (int l = 0; l < 3; l++) {
      double* A = Cd.data() + l * nxyz;
      int i1 = 3, i2 = nx - 4, j1 = 3, j2 = ny - 4, k1 = 3, k2 = nz - 4;
      for (int n = 1; n <= 3; n++)
        for (int k = 0; k < nz; k++)
          for (int j = 0; j < ny; j++) {
            A[P3(i1 - n, j, k)] = 2.0 * A[P3(i1, j, k)] - A[P3(i1 + n, j, k)];
            A[P3(i2 + n, j, k)] = 2.0 * A[P3(i2, j, k)] - A[P3(i2 - n, j, k)];
          }
      for (int i = 0; i < nx; i++)
        for (int k = 0; k < nz; k++)
          for (int n = 1; n <= 3; n++) {
            A[P3(i, j1 - n, k)] = 2.0 * A[P3(i, j1, k)] - A[P3(i, j1 + n, k)];
            A[P3(i, j2 + n, k)] = 2.0 * A[P3(i, j2, k)] - A[P3(i, j2 - n, k)];
          }
      for (int i = 0; i < nx; i++)
        for (int n = 1; n <= 3; n++)
          for (int j = 0; j < ny; j++) {
            A[P3(i, j, k1 - n)] = 2.0 * A[P3(i, j, k1)] - A[P3(i, j, k1 + n)];
            A[P3(i, j, k2 + n)] = 2.0 * A[P3(i, j, k2)] - A[P3(i, j, k2 - n)];
          }
    }
  }

  // Second-order central metric and bimaterial media (metric.cu:15-171), 1-D layered
  // media override (media.cu:63-138), then mirror ghost fill (metric.cu:173-246).
  void cal_metric(int nlayer, const float* layers) {
    const double* X = Cd.data(); const double* Y = X + nxyz; const double* Z = Y + nxyz;
    double r = 1.0 / p.DH;
#pragma omp parallel for schedule(static)
    for (int i = 3; i < nx - 3; i++)
      for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++) {
          long q = P3(i, j, k);
          double v1[3] = {0.5 * r * (X[q + nyz] - X[q - nyz]), 0.5 * r * (Y[q + nyz] - Y[q - nyz]),
                          0.5 * r * (Z[q + nyz] - Z[q - nyz])};
          double v2[3] = {0.5 * r * (X[q + 1] - X[q - 1]), 0.5 * r * (Y[q + 1] - Y[q - 1]),
                          0.5 * r * (Z[q + 1] - Z[q - 1])};
          double v3[3] = {0.5 * r * (X[q + ny] - X[q - ny]), 0.5 * r * (Y[q + ny] - Y[q - ny]),
                          0.5 * r * (Z[q + ny] - Z[q - ny])};
          double g[3];
          cross3(v1, v2, g);
          double jac = g[0] * v3[0] + g[1] * v3[1] + g[2] * v3[2];
          double rj = 1.0 / jac;
          double e1[3], e2[3], e3[3];
          cross3(v2, v3, e1); cross3(v3, v1, e2); cross3(v1, v2, e3);
          for (int c = 0; c < 3; c++) {
            Mf(c)[q] = (R)(e1[c] * rj);
            Mf(3 + c)[q] = (R)(e2[c] * rj);
            Mf(6 + c)[q] = (R)(e3[c] * rj);
          }
          Mf(9)[q] = (R)jac;
          int gi = i;  // the reference compares the padded index with NX/2 (metric.cu:140-142)
          double rho, vp, vs;
          if (gi < p.NX / 2) { rho = p.bi_rho1; vp = p.bi_vp1; vs = p.bi_vs1; }
          else { rho = p.bi_rho2; vp = p.bi_vp2; vs = p.bi_vs2; }
          if (nlayer > 0) {
            double depth = -Z[q];
            int l0 = nlayer - 1;
            for (int l = nlayer - 1; l >= 0; l--)
              if (depth > layers[4 * l + 0]) { l0 = l; break; }
            rho = layers[4 * l0 + 1]; vp = layers[4 * l0 + 2]; vs = layers[4 * l0 + 3];
          }
          Mf(10)[q] = (R)(rho * (vp * vp - 2 * vs * vs));
          Mf(11)[q] = (R)(rho * vs * vs);
          Mf(12)[q] = (R)rho;
        }
    for (int l = 0; l < 13; l++) {
      R* A = Mf(l);
      int i1 = 3, i2 = nx - 4, j1 = 3, j2 = ny - 4, k1 = 3, k2 = nz - 4;
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int n = 1; n <= 3; n++) {
            A[P3(i1 - n, j, k)] = A[P3(i1 + n, j, k)];
            A[P3(i2 + n, j, k)] = A[P3(i2 - n, j, k)];
          }
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nx; i++)
          for (int n = 1; n <= 3; n++) {
            A[P3(i, j1 - n, k)] = A[P3(i, j1 + n, k)];
            A[P3(i, j2 + n, k)] = A[P3(i, j2 - n, k)];
          }
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
          for (int n = 1; n <= 3; n++) {
            A[P3(i, j, k1 - n)] = A[P3(i, j, k1 + n)];
            A[P3(i, j, k2 + n)] = A[P3(i, j, k2 - n)];
          }
    }
  }

  // Per-node split-node coefficient tables (fault_coef.cu:26-1302), in double.
  // D_ab = jac * (lam e_a e_b^T-ish contraction): D_ab[p][q] = lam*ea[p]*eb[q] +
  // mu*ea[q]*eb[p] + delta_pq*mu*(ea.eb) with e_1,e_2,e_3 the xi/eta/zeta metric rows.
  static void Dmat(const double* ea, const double* eb, double lam, double mu, double jac, M3 D) {
    double dot = ea[0] * eb[0] + ea[1] * eb[1] + ea[2] * eb[2];
    for (int pp = 0; pp < 3; pp++)
      for (int qq = 0; qq < 3; qq++)
        D[pp][qq] = jac * (lam * ea[pp] * eb[qq] + mu * ea[qq] * eb[pp] + (pp == qq ? mu * dot : 0.0));
  }
  void put9(const char* name, long idx, const M3 m) {
    std::vector<R>& v = fc[name];
    for (int a_ = 0; a_ < 3; a_++)
      for (int b_ = 0; b_ < 3; b_++) v[idx * 9 + a_ * 3 + b_] = (R)m[a_][b_];
  }
  void init_fault_coef() {
    const char* full[] = {"D21_1", "D22_1", "D23_1", "D31_1", "D32_1", "D33_1", "D21_2", "D22_2", "D23_2",
                          "D31_2", "D32_2", "D33_2", "D11_1", "D12_1", "D13_1", "D11_2", "D12_2", "D13_2",
                          "matMin2Plus1", "matMin2Plus2", "matMin2Plus3", "matMin2Plus4", "matMin2Plus5",
                          "matPlus2Min1", "matPlus2Min2", "matPlus2Min3", "matPlus2Min4", "matPlus2Min5",
                          "matT1toVxm", "matVytoVxm", "matVztoVxm", "matT1toVxp", "matVytoVxp", "matVztoVxp"};
    for (auto n : full) fc[n].assign(9 * nyz, 0);
    const char* lines[] = {"matVx2Vz1", "matVy2Vz1", "matVx2Vz2", "matVy2Vz2", "matPlus2Min1f", "matPlus2Min2f",
                           "matPlus2Min3f", "matMin2Plus1f", "matMin2Plus2f", "matMin2Plus3f"};
    for (auto n : lines) fc[n].assign(9L * ny, 0);
    fc["vec_n"].assign(3 * nyz, 0); fc["vec_s1"].assign(3 * nyz, 0); fc["vec_s2"].assign(3 * nyz, 0);
    fc["rho_f"].assign(2 * nyz, 0); fc["lam_f"].assign(2 * nyz, 0); fc["mu_f"].assign(2 * nyz, 0);
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++) {
        long q = P3(i0, j, k);
        long f = j + (long)k * ny;
        double e[3][3];
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) e[r][c] = Mf(3 * r + c)[q];
        double jac = Mf(9)[q];
        M3 inv;
        inv3(e, inv);  // columns: x_xi.. (fault_coef.cu:136-156)
        double xet[3] = {inv[0][1], inv[1][1], inv[2][1]};
        double xzt[3] = {inv[0][2], inv[1][2], inv[2][2]};
        // base vectors n = xi_grad/|.|, s1 = x_eta/|.|, s2 = n x s1 (fault_coef.cu:206-248)
        double s1[3], nn[3], s2[3];
        double ns1 = ref_norm3(xet[0], xet[1], xet[2]);
        for (int c = 0; c < 3; c++) s1[c] = xet[c] / ns1;
        double nnn = ref_norm3(e[0][0], e[0][1], e[0][2]);
        for (int c = 0; c < 3; c++) nn[c] = e[0][c] / nnn;
        cross3(nn, s1, s2);
        for (int c = 0; c < 3; c++) {
          fc["vec_n"][3 * f + c] = (R)nn[c];
          fc["vec_s1"][3 * f + c] = (R)s1[c];
          fc["vec_s2"][3 * f + c] = (R)s2[c];
        }
        double lamf[2], muf[2];
        for (int m = 0; m < 2; m++) {
          long qm = q + (m == 0 ? -nyz : nyz);
          fc["rho_f"][f + m * nyz] = Mf(12)[qm];
          fc["lam_f"][f + m * nyz] = Mf(10)[qm];
          fc["mu_f"][f + m * nyz] = Mf(11)[qm];
          lamf[m] = (double)Mf(10)[qm];
          muf[m] = (double)Mf(11)[qm];
        }
        M3 D[2][3][3];
        for (int m = 0; m < 2; m++)
          for (int aa = 0; aa < 3; aa++)
            for (int bb = 0; bb < 3; bb++) Dmat(e[aa], e[bb], lamf[m], muf[m], jac, D[m][aa][bb]);
        const char* dn[2][3][3] = {{{"D11_1", "D12_1", "D13_1"}, {"D21_1", "D22_1", "D23_1"}, {"D31_1", "D32_1", "D33_1"}},
                                   {{"D11_2", "D12_2", "D13_2"}, {"D21_2", "D22_2", "D23_2"}, {"D31_2", "D32_2", "D33_2"}}};
        for (int m = 0; m < 2; m++)
          for (int aa = 0; aa < 3; aa++)
            for (int bb = 0; bb < 3; bb++) put9(dn[m][aa][bb], f, D[m][aa][bb]);
        // B_b = Q D_1b + A2 D_2b + A3 D_3b with Q rows = xi-gradient and A2/A3 built from
        // the eta/zeta tangents (fault_coef.cu:158-196, 628-672)
        M3 Q, A2m, A3m, B0;
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) Q[r][c] = e[0][c];
        double xxi[3] = {inv[0][0], inv[1][0], inv[2][0]};
        M3 A1m = {{-xxi[1], xxi[0], 0.0}, {-xxi[2], 0.0, xxi[0]}, {0.0, -xxi[2], xxi[1]}};
        double A2v[3][3] = {{xet[1], -xet[0], 0.0}, {xet[2], 0.0, -xet[0]}, {0.0, xet[2], -xet[1]}};
        double A3v[3][3] = {{xzt[1], -xzt[0], 0.0}, {xzt[2], 0.0, -xzt[0]}, {0.0, xzt[2], -xzt[1]}};
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) { A2m[r][c] = A2v[r][c]; A3m[r][c] = A3v[r][c]; B0[r][c] = Q[r][c] + A1m[r][c]; }
        (void)B0;
        M3 Bm[2][3];
        for (int m = 0; m < 2; m++)
          for (int bb = 0; bb < 3; bb++) {
            M3 t1, t2, t3;
            mul3(Q, D[m][0][bb], t1); mul3(A2m, D[m][1][bb], t2); mul3(A3m, D[m][2][bb], t3);
            for (int r = 0; r < 3; r++)
              for (int c = 0; c < 3; c++) Bm[m][bb][r][c] = t1[r][c] + t2[r][c] + t3[r][c];
          }
        M3 t, u;
        // final (overwriting) definitions of the T1 -> DxV maps (fault_coef.cu:823-865)
        for (int m = 0; m < 2; m++) {
          M3 iD;
          inv3(D[m][0][0], iD);
          put9(m == 0 ? "matT1toVxm" : "matT1toVxp", f, iD);
          mul3(iD, D[m][0][1], t); put9(m == 0 ? "matVytoVxm" : "matVytoVxp", f, t);
          mul3(iD, D[m][0][2], t); put9(m == 0 ? "matVztoVxm" : "matVztoVxp", f, t);
        }
        // continuity maps (fault_coef.cu:868-968)
        M3 iB;
        inv3(Bm[1][0], iB);
        mul3(iB, Bm[0][0], t); put9("matMin2Plus1", f, t);
        mul3(iB, Bm[0][1], t); put9("matMin2Plus2", f, t);
        mul3(iB, Bm[0][2], t); put9("matMin2Plus3", f, t);
        mul3(iB, Bm[1][1], t); put9("matMin2Plus4", f, t);
        mul3(iB, Bm[1][2], t); put9("matMin2Plus5", f, t);
        inv3(Bm[0][0], iB);
        mul3(iB, Bm[1][0], t); put9("matPlus2Min1", f, t);
        mul3(iB, Bm[1][1], t); put9("matPlus2Min2", f, t);
        mul3(iB, Bm[1][2], t); put9("matPlus2Min3", f, t);
        mul3(iB, Bm[0][1], t); put9("matPlus2Min4", f, t);
        mul3(iB, Bm[0][2], t); put9("matPlus2Min5", f, t);
        (void)u;
        // free-surface row (fault_coef.cu:1046-1240), stored per j
        if (k == nz - 4) {
          M3 iA, mB, mC, vx[2], vy[2];
          for (int m = 0; m < 2; m++) {
            inv3(D[m][2][2], iA);
            for (int r = 0; r < 3; r++)
              for (int c = 0; c < 3; c++) { mB[r][c] = -D[m][2][0][r][c]; mC[r][c] = -D[m][2][1][r][c]; }
            mul3(iA, mB, vx[m]); mul3(iA, mC, vy[m]);
          }
          put9("matVx2Vz1", j, vx[0]); put9("matVy2Vz1", j, vy[0]);
          put9("matVx2Vz2", j, vx[1]); put9("matVy2Vz2", j, vy[1]);
          double v1[3] = {e[0][0], e[0][1], e[0][2]};
          double v1n = ref_norm3(v1[0], v1[1], v1[2]);
          double v3[3];
          cross3(v1, xet, v3);
          double h[3];
          for (int aa = 0; aa < 3; aa++) h[aa] = (v3[0] * e[aa][0] + v3[1] * e[aa][1] + v3[2] * e[aa][2]) / v1n;
          double muc = Mf(11)[q];
          M3 Df[2][3];  // D_1b + mu*h_b * v3 v1^T
          for (int m = 0; m < 2; m++)
            for (int bb = 0; bb < 3; bb++)
              for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) Df[m][bb][r][c] = D[m][0][bb][r][c] + muc * h[bb] * v3[r] * v1[c];
          M3 Vx1, Vy1, Vx2, Vy2, tmp;
          mul3(Df[0][2], vx[0], tmp);
          for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vx1[r][c] = Df[0][0][r][c] + tmp[r][c];
          mul3(Df[0][2], vy[0], tmp);
          for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vy1[r][c] = Df[0][1][r][c] + tmp[r][c];
          mul3(Df[1][2], vx[1], tmp);
          for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vx2[r][c] = Df[1][0][r][c] + tmp[r][c];
          mul3(Df[1][2], vy[1], tmp);
          for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) Vy2[r][c] = Df[1][1][r][c] + tmp[r][c];
          M3 iv;
          inv3(Vx1, iv);
          mul3(iv, Vx2, t); put9("matPlus2Min1f", j, t);
          mul3(iv, Vy2, t); put9("matPlus2Min2f", j, t);
          mul3(iv, Vy1, t); put9("matPlus2Min3f", j, t);
          inv3(Vx2, iv);
          mul3(iv, Vx1, t); put9("matMin2Plus1f", j, t);
          mul3(iv, Vy1, t); put9("matMin2Plus2f", j, t);
          mul3(iv, Vy2, t); put9("matMin2Plus3f", j, t);
        }
      }
  }

  // Free-surface velocity-gradient transform Dz V = A^-1 (B Dx V + C Dy V) at the top
  // row, with the PML 1/beta factors (fault_coef.cu:1320-1486).
  void init_wave_free() {
    if (!freenode) return;
    int k = nz - 4;
    for (int i = 3; i < nx - 3; i++)
      for (int j = 3; j < ny - 3; j++) {
        long q = P3(i, j, k);
        double rb1 = 1.0 / Bx[i - 3], rb2 = 1.0 / By[j - 3], rb3 = 1.0 / Bz[k - 3];
        double e[3][3];
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) e[r][c] = Mf(3 * r + c)[q];
        double lam = Mf(10)[q], mu = Mf(11)[q];
        M3 A, B, C, iA, AB, AC;
        Dmat(e[2], e[2], lam, mu, rb3, A);
        Dmat(e[2], e[0], lam, mu, -rb1, B);
        Dmat(e[2], e[1], lam, mu, -rb2, C);
        inv3(A, iA);
        mul3(iA, B, AB); mul3(iA, C, AC);
        long o = (j + (long)i * ny) * 9;
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) { matVx2Vz[o + 3 * r + c] = (R)AB[r][c]; matVy2Vz[o + 3 * r + c] = (R)AC[r][c]; }
      }
  }

  // Fault masks and background state (init.cu:160-849), followed by the file-loaded
  // stress and friction fields (init.cu:904-1022).  stress: 15 planes of nj*nk in the
  // order Tx,Ty,Tz,dTx,dTy,dTz,mu_s,mu_d,Dc,C0,a,b,L,Vw,State.
  void init_fault(const float* stress) {
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q = j + (long)k * nj;
        int gj1 = j + 1, gk1 = k + 1;
        rup_index_y[q] = (gj1 <= p.Fault_grid[0] + 3 || gj1 >= p.Fault_grid[1] - 3) ? 0 : 1;
        rup_index_z[q] = (gk1 <= p.Fault_grid[2] + 3 || gk1 >= p.Fault_grid[3] - 3) ? 0 : 1;
        bool inner = gj1 > 30 && gj1 < p.NY - 30 && gk1 > 30 && (freenode || gk1 < p.NZ - 30);
        united[q] = inner ? 0 : 1;
        faultgrid[q] = (gj1 >= p.Fault_grid[0] + 3 && gj1 <= p.Fault_grid[1] - 3 && gk1 >= p.Fault_grid[2] + 3 &&
                        gk1 <= p.Fault_grid[3] - 3) ? 1 : 0;
        // rate-and-state runs test a-b before the friction fields are loaded; on the
        // zero-filled allocation this always yields 0 (init.cu:833-844)
        if (p.Friction_type >= 1 && p.Friction_type <= 3) faultgrid[q] = 0;
        str_peak[q] = (gj1 >= p.Fault_grid[0] && gj1 <= p.Fault_grid[1] && gk1 >= p.Fault_grid[2] &&
                       gk1 <= p.Fault_grid[3]) ? (R)p.mu_s : (R)10000.;
        init_t0[q] = (R)-9999.9;
        Tn[q] = (R)-120.0e6;
        Ts1[q] = (R)(-120.0e6 * p.mu_0);
        Ts2[q] = 0;
        if (gj1 >= p.Asp_grid[0] && gj1 <= p.Asp_grid[1] && gk1 >= p.Asp_grid[2] && gk1 <= p.Asp_grid[3])
          Ts1[q] = (R)((p.mu_s + (p.mu_s - p.mu_d) * 0.001) * -120.0e6);
        long fq = 3 * ((j + 3) + (long)(k + 3) * ny);
        for (int c = 0; c < 3; c++) {
          double vsi = Tn[q] * fc["vec_n"][fq + c] + Ts1[q] * fc["vec_s1"][fq + c] + Ts2[q] * fc["vec_s2"][fq + c];
          (c == 0 ? str_init_x : c == 1 ? str_init_y : str_init_z)[q] = (R)vsi;
        }
      }
    if (p.INPORT_STRESS_TYPE == 1 && stress) {
      long nf = (long)nj * nk;
      std::vector<R>* dst[5] = {&T0x, &T0y, &T0z, &dT0x, &dT0y};
      for (int c = 0; c < 5; c++)
        for (long q = 0; q < nf; q++) (*dst[c])[q] = stress[c * nf + q];
      for (long q = 0; q < nf; q++) dT0z[q] = stress[5 * nf + q];
      if (p.Friction_type == 0) {
        for (long q = 0; q < nf; q++) {
          str_peak[q] = stress[6 * nf + q]; mu_d[q] = stress[7 * nf + q];
          Dc[q] = stress[8 * nf + q]; C0[q] = stress[9 * nf + q];
        }
      } else {
        for (long q = 0; q < nf; q++) {
          a[q] = stress[10 * nf + q]; b[q] = stress[11 * nf + q]; L[q] = stress[12 * nf + q];
          Vw[q] = stress[13 * nf + q]; State[q] = stress[14 * nf + q];
        }
      }
      // local frame of the loaded traction (init.cu:859-902)
      for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++) {
          long q = j + (long)k * nj, fq = 3 * ((j + 3) + (long)(k + 3) * ny);
          auto dotv = [&](const char* nm) {
            const std::vector<R>& v = fc[nm];
            return (R)(T0x[q] * v[fq] + T0y[q] * v[fq + 1] + T0z[q] * v[fq + 2]);
          };
          Tn[q] = dotv("vec_n"); Ts1[q] = dotv("vec_s1"); Ts2[q] = dotv("vec_s2");
        }
    }
  }

  // Cerjan sponge table (cerjan.cu:31-164): exp(-(alpha*(ND-d))^2), min over faces,
  // the x faces assign, the y/z faces take the minimum; no top face with a free surface.
  void init_cerjan() {
    damp.assign(nxyz, (R)1);
    if (!p.use_cerjan) return;
    int ND = p.DAMP_N;
    float alpha = (float)(std::sqrt(-std::log((double)0.92f)) / ND);
    auto dv = [&](int d) { return (R)std::exp(-std::pow((double)(alpha * (ND - d)), 2.0)); };
    int a1 = 3, a2x = nx - 3, a2y = ny - 3, a2z = nz - 3;
    for (int d = 0; d < ND; d++)
      for (int j = a1; j < a2y; j++)
        for (int k = a1; k < a2z; k++) { damp[P3(a1 + d, j, k)] = dv(d); damp[P3(a2x - d - 1, j, k)] = dv(d); }
    std::vector<R> tmp = damp;
    for (int d = 0; d < ND; d++)
      for (int i = a1; i < a2x; i++)
        for (int k = a1; k < a2z; k++) {
          long q1 = P3(i, a1 + d, k), q2 = P3(i, a2y - d - 1, k);
          damp[q1] = std::min(dv(d), tmp[q1]);
          damp[q2] = std::min(dv(d), tmp[q2]);
        }
    tmp = damp;
    for (int d = 0; d < ND; d++)
      for (int i = a1; i < a2x; i++)
        for (int j = a1; j < a2y; j++) {
          long q1 = P3(i, j, a1 + d);
          damp[q1] = std::min(dv(d), tmp[q1]);
          if (!freenode) { long q2 = P3(i, j, a2z - d - 1); damp[q2] = std::min(dv(d), tmp[q2]); }
        }
  }

  // ------------------------------------------------------------- volume RHS --
  // Velocity-stress right-hand side at every interior node (wave.cu:8-494).
  // Returns the nine unscaled directional contributions for the PML faces too.
  void deriv_axis(long q, long s, int fl, const double* e, double lam, double mu, double rrho, double* D,
                  double* dv) {
    const R* V[9];
    for (int f = 0; f < 9; f++) V[f] = Wf(W, f);
    double d[9];
    for (int f = 0; f < 9; f++) d[f] = (double)op5(V[f], q, s, fl) * (double)rDH;
    // d: Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz
    if (dv) { dv[0] = d[0]; dv[1] = d[1]; dv[2] = d[2]; }
    double lam2mu = lam + 2.0 * mu;
    D[0] = (d[3] * e[0] + d[6] * e[1] + d[7] * e[2]) * rrho;
    D[1] = (d[6] * e[0] + d[4] * e[1] + d[8] * e[2]) * rrho;
    D[2] = (d[7] * e[0] + d[8] * e[1] + d[5] * e[2]) * rrho;
    D[3] = d[0] * e[0] * lam2mu + d[1] * e[1] * lam + d[2] * e[2] * lam;
    D[4] = d[0] * e[0] * lam + d[1] * e[1] * lam2mu + d[2] * e[2] * lam;
    D[5] = d[0] * e[0] * lam + d[1] * e[1] * lam + d[2] * e[2] * lam2mu;
    D[6] = (d[0] * e[1] + d[1] * e[0]) * mu;
    D[7] = (d[0] * e[2] + d[2] * e[0]) * mu;
    D[8] = (d[1] * e[2] + d[2] * e[1]) * mu;
  }
  void wave_deriv(int FX, int FY, int FZ) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; i++)
      for (int k = 0; k < nk; k++)
        for (int j = 0; j < nj; j++) {
          long q = P3(i + 3, j + 3, k + 3);
          double lam = Mf(10)[q], mu = Mf(11)[q], rrho = 1.0 / (double)Mf(12)[q];
          double lam2mu = lam + 2.0 * mu;
          double ex[3] = {Mf(0)[q], Mf(1)[q], Mf(2)[q]}, ey[3] = {Mf(3)[q], Mf(4)[q], Mf(5)[q]},
                 ez[3] = {Mf(6)[q], Mf(7)[q], Mf(8)[q]};
          double Dx_[9], Dy_[9], Dz_[9], dxv[3], dyv[3];
          deriv_axis(q, nyz, FX, ex, lam, mu, rrho, Dx_, dxv);
          deriv_axis(q, 1, FY, ey, lam, mu, rrho, Dy_, dyv);
          deriv_axis(q, ny, FZ, ez, lam, mu, rrho, Dz_, nullptr);
          if (freenode && k >= nk - 3) {
            // velocity z-derivatives at the top rows (wave.cu:205-245)
            double dz[3];
            if (k == nk - 1) {
              const R* mx = &matVx2Vz[(j + 3 + (long)(i + 3) * ny) * 9];
              const R* my = &matVy2Vz[(j + 3 + (long)(i + 3) * ny) * 9];
              for (int r = 0; r < 3; r++)
                dz[r] = (mx[3 * r] * dxv[0] + mx[3 * r + 1] * dxv[1] + mx[3 * r + 2] * dxv[2]) +
                        (my[3 * r] * dyv[0] + my[3 * r + 1] * dyv[1] + my[3 * r + 2] * dyv[2]);
            } else {
              for (int r = 0; r < 3; r++)
                dz[r] = (double)(k == nk - 2 ? op2(Wf(W, r), q, ny, FZ) : op3(Wf(W, r), q, ny, FZ)) * (double)rDH;
            }
            Dz_[3] = dz[0] * ez[0] * lam2mu + dz[1] * ez[1] * lam + dz[2] * ez[2] * lam;
            Dz_[4] = dz[0] * ez[0] * lam + dz[1] * ez[1] * lam2mu + dz[2] * ez[2] * lam;
            Dz_[5] = dz[0] * ez[0] * lam + dz[1] * ez[1] * lam + dz[2] * ez[2] * lam2mu;
            Dz_[6] = (dz[0] * ez[1] + dz[1] * ez[0]) * mu;
            Dz_[7] = (dz[0] * ez[2] + dz[2] * ez[0]) * mu;
            Dz_[8] = (dz[1] * ez[2] + dz[2] * ez[1]) * mu;
          }
          double rb1 = 1.0 / (double)Bx[i], rb2 = 1.0 / (double)By[j], rb3 = 1.0 / (double)Bz[k];
          for (int f = 0; f < 9; f++) Wf(hW, f)[q] = (R)(Dx_[f] * rb1 + Dy_[f] * rb2 + Dz_[f] * rb3);
          if (freenode && k >= nk - 3) {
            // traction image for the momentum equation at the top three rows (wave.cu:398-487)
            int ik = nk - 1 - k;
            double rrhojac = rrho / (double)Mf(9)[q];
            double v1[3][7], v2[3][7], v3[3][7];
            for (int l = 0; l < 7; l++) {
              long qx = P3(i + 3 + l - 3, j + 3, k + 3), qy = P3(i + 3, j + 3 + l - 3, k + 3),
                   qz = P3(i + 3, j + 3, k + 3 + l - 3);
              trac(qx, 0, v1[0][l], v1[1][l], v1[2][l]);
              trac(qy, 3, v2[0][l], v2[1][l], v2[2][l]);
              trac(qz, 6, v3[0][l], v3[1][l], v3[2][l]);
            }
            for (int c = 0; c < 3; c++) {
              v3[c][ik + 3] = 0.0;
              for (int l = 0; l < 3 - ik; l++) v3[c][6 - l] = -v3[c][l + 2 * ik];
            }
            for (int c = 0; c < 3; c++) {
              double dx = op5(v1[c], 3, 1, FX) * (double)rDH, dy = op5(v2[c], 3, 1, FY) * (double)rDH,
                     dz = op5(v3[c], 3, 1, FZ) * (double)rDH;
              Wf(hW, c)[q] = (R)((dx * rb1 + dy * rb2 + dz * rb3) * rrhojac);
            }
          }
        }
  }
  // traction vector jac * e_axis . sigma at node q, axis metric offset mo (0, 3, 6)
  void trac(long q, int mo, double& t1, double& t2, double& t3) {
    double e0 = Mf(mo)[q], e1 = Mf(mo + 1)[q], e2 = Mf(mo + 2)[q], jac = Mf(9)[q];
    double txx = Wf(W, 3)[q], tyy = Wf(W, 4)[q], tzz = Wf(W, 5)[q], txy = Wf(W, 6)[q], txz = Wf(W, 7)[q],
           tyz = Wf(W, 8)[q];
    t1 = (e0 * txx + e1 * txy + e2 * txz) * jac;
    t2 = (e0 * txy + e1 * tyy + e2 * tyz) * jac;
    t3 = (e0 * txz + e1 * tyz + e2 * tzz) * jac;
  }

  // ADE CFS-PML on one face slab (pmlx.cu:8-214, pmly.cu:8-213, pmlz.cu:8-180):
  // hW -= aux/beta; aux_h = -(alpha+d)*aux + d*Deriv (+ free-surface Dz term on x/y).
  void abs_deriv(int face, int Flag) {
    int axis = face / 2;
    bool hi = face % 2;
    int pni = axis == 0 ? N : ni, pnj = axis == 1 ? N : nj, pnk = axis == 2 ? N : nk;
    int idx0 = hi ? (axis == 0 ? ni - N : axis == 1 ? nj - N : nk - N) : 0;
    std::vector<R>& aW = aux[face][0];
    std::vector<R>& ah = aux[face][1];
    long st = (long)pni * pnj * pnk;
    const std::vector<R>& Av = axis == 0 ? Ax : axis == 1 ? Ay : Az;
    const std::vector<R>& Bv = axis == 0 ? Bx : axis == 1 ? By : Bz;
    const std::vector<R>& Dv = axis == 0 ? Dx : axis == 1 ? Dy : Dz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < pni; i++)
      for (int k = 0; k < pnk; k++)
        for (int j = 0; j < pnj; j++) {
          int gi = i + (axis == 0 ? idx0 : 0), gj = j + (axis == 1 ? idx0 : 0), gk = k + (axis == 2 ? idx0 : 0);
          long q = P3(gi + 3, gj + 3, gk + 3);
          long s = axis == 0 ? nyz : axis == 1 ? 1 : ny;
          int mo = 3 * axis;
          double e[3] = {Mf(mo)[q], Mf(mo + 1)[q], Mf(mo + 2)[q]};
          double lam = Mf(10)[q], mu = Mf(11)[q], rrho = 1.0 / (double)Mf(12)[q];
          double lam2mu = lam + 2.0 * mu;
          double Dr[9], dv[3];
          deriv_axis(q, s, Flag, e, lam, mu, rrho, Dr, dv);
          int g = axis == 0 ? gi : axis == 1 ? gj : gk;
          double b1 = Bv[g], d1 = Dv[g], ad1 = -((double)Av[g] + d1), rb1 = 1.0 / b1;
          long qa = j + (long)k * pnj + (long)i * pnj * pnk;
          for (int f = 0; f < 9; f++) {
            Wf(hW, f)[q] += (R)(-(double)aW[f * st + qa] * rb1);
            ah[f * st + qa] = (R)(ad1 * aW[f * st + qa] + d1 * Dr[f]);
          }
          if (axis < 2 && freenode && gk == nk - 1) {
            const R* mm = &(axis == 0 ? matVx2Vz : matVy2Vz)[(gj + 3 + (long)(gi + 3) * ny) * 9];
            double dz[3];
            for (int r = 0; r < 3; r++) dz[r] = mm[3 * r] * dv[0] + mm[3 * r + 1] * dv[1] + mm[3 * r + 2] * dv[2];
            double ez[3] = {Mf(6)[q], Mf(7)[q], Mf(8)[q]};
            double c = d1 * b1;
            double add[6] = {c * (lam2mu * ez[0] * dz[0] + lam * ez[1] * dz[1] + lam * ez[2] * dz[2]),
                             c * (lam * ez[0] * dz[0] + lam2mu * ez[1] * dz[1] + lam * ez[2] * dz[2]),
                             c * (lam * ez[0] * dz[0] + lam * ez[1] * dz[1] + lam2mu * ez[2] * dz[2]),
                             c * mu * (ez[1] * dz[0] + ez[0] * dz[1]), c * mu * (ez[2] * dz[0] + ez[0] * dz[2]),
                             c * mu * (ez[2] * dz[1] + ez[1] * dz[2])};
            for (int f = 3; f < 9; f++) ah[f * st + qa] = (R)((double)ah[f * st + qa] + add[f - 3]);
          }
        }
  }

  // Classic RK4 register update (rk4.cu:20-33), applied to the volume and every PML
  // auxiliary array (rk4.cu:154-257).
  static void rk_update(R* Wv, R* mWv, const R* h, R* tWv, long n, int irk, float rka, float rkb) {
#pragma omp parallel for schedule(static)
    for (long x = 0; x < n; x++) {
      if (irk == 0) { mWv[x] = Wv[x]; tWv[x] = (R)(rkb * h[x] + mWv[x]); }
      else if (irk == 1 || irk == 2) tWv[x] = (R)(tWv[x] + rkb * h[x]);
      if (irk == 3) Wv[x] = (R)(rkb * h[x] + tWv[x]);
      else Wv[x] = (R)(rka * h[x] + mWv[x]);
    }
  }
  void wave_rk(int irk) {
    float rka, rkb;
    rk_weights(irk, (float)p.DT, &rka, &rkb);
    rk_update(W.data(), mW.data(), hW.data(), tW.data(), 9 * nxyz, irk, rka, rkb);
    for (int f = 0; f < 6; f++)
      if (!aux[f][0].empty())
        rk_update(aux[f][0].data(), aux[f][2].data(), aux[f][1].data(), aux[f][3].data(), aux[f][0].size(), irk,
                  rka, rkb);
  }
  // W *= damp over the interior (cerjan.cu:166-410)
  void apply_cerjan() {
    if (!p.use_cerjan) return;
#pragma omp parallel for schedule(static)
    for (int i = 3; i < nx - 3; i++)
      for (int k = 3; k < nz - 3; k++)
        for (int j = 3; j < ny - 3; j++) {
          long q = P3(i, j, k);
          for (int f = 0; f < 9; f++) Wf(W, f)[q] *= damp[q];
        }
  }

  // ------------------------------------------------------------- fault side --
  R* FWf(std::vector<R>& v, int f) { return v.data() + (long)f * 2 * nyz; }
  double vecn(const char* nm, long f, int c) { return fc[nm][3 * f + c]; }

  // dpsi/dt (aging or slip law with flash weakening) and RK4 of state and slip
  // (rk4.cu:791-938).  Slip-weakening runs never write hState (zero).
  void state_rk(int irk) {
    float rka, rkb;
    rk_weights(irk, (float)p.DT, &rka, &rkb);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q = j + (long)k * nj;
        if (united[q]) continue;
        long f = (j + 3) + (long)(k + 3) * ny;
        double dV[3];
        for (int c = 0; c < 3; c++) dV[c] = (double)FWf(FW, c)[f + nyz] - (double)FWf(FW, c)[f];
        double vs1 = 0, vs2 = 0;
        for (int c = 0; c < 3; c++) { vs1 += dV[c] * vecn("vec_s1", f, c); vs2 += dV[c] * vecn("vec_s2", f, c); }
        hslip[q] = (R)std::sqrt(vs2 * vs2 + vs1 * vs1);
        double V = std::max((double)hslip[q], 1e-30);
        double st = State[q];
        double ra = a[q], rb = b[q], rvw = Vw[q];
        double f0 = p.f0, V0 = p.V0, rl = L[q];
        if (p.Friction_type == 1) {
          hState[q] = (R)(rb * V0 / rl * (std::exp((f0 - st) / rb) - V / V0));
        } else if (p.Friction_type == 2 || p.Friction_type == 3) {
          double flv = f0 - (rb - ra) * std::log(V / V0);
          double fss = p.fw + (flv - p.fw) / std::pow(1. + std::pow(V / rvw, 8), 0.125);
          double psiss = ra * (std::log(std::sinh(fss / ra)) + std::log(2. * (V0 / V)));
          hState[q] = (R)(-V / rl * (st - psiss));
        }
        if (irk == 0) {
          mState[q] = State[q]; tState[q] = (R)(mState[q] + rkb * hState[q]);
          mslip[q] = slip[q]; tslip[q] = (R)(mslip[q] + rkb * hslip[q]);
        } else if (irk == 1 || irk == 2) {
          tState[q] = (R)(tState[q] + rkb * hState[q]);
          tslip[q] = (R)(tslip[q] + rkb * hslip[q]);
        }
        if (irk == 3) {
          State[q] = (R)(tState[q] + rkb * hState[q]);
          slip[q] = (R)(tslip[q] + rkb * hslip[q]);
        } else {
          State[q] = (R)(mState[q] + rka * hState[q]);
          slip[q] = (R)(mslip[q] + rka * hslip[q]);
        }
      }
  }

  // Shared front half of both trial kernels (trial_slipweakening.cu:130-312,
  // trial_ratestate.cu:167-378): traction T1 on the six off-fault layers, the
  // split-node DyT2/DzT3 and the momentum residuals R[m] of the two half cells.
  struct TrialPre {
    double Mrho[2], Rx[2], Ry[2], Rz[2], jac_last, rho_last;
  };
  void trial_front(int j, int k, int FY, int FZ, TrialPre& t) {
    int j1 = j + 3, k1 = k + 3, km = nk - k;
    long q2 = j + (long)k * nj;
    long pf = j1 + (long)k1 * ny;
    double DHd = DH, DH2 = DHd * DHd;
    for (int m = 0; m < 2; m++) {
      double jac = 0, rho = fc["rho_f"][pf + m * nyz];
      for (int l = 1; l <= 3; l++) {
        long q = P3(i0 + (2 * m - 1) * l, j1, k1);
        double t1, t2, t3;
        trac(q, 0, t1, t2, t3);
        jac = Mf(9)[q];  // the last value (i0 -/+ 3) feeds Mrho (quirk of the reference)
        int lay = 3 + (2 * m - 1) * l;
        T11[lay * nyz + pf] = (R)t1; T12[lay * nyz + pf] = (R)t2; T13[lay * nyz + pf] = (R)t3;
      }
      const R* t2x[3] = {FWf(FW, 3) + m * nyz, FWf(FW, 4) + m * nyz, FWf(FW, 5) + m * nyz};
      double DyT[3], DzT[3];
      for (int c = 0; c < 3; c++)
        DyT[c] = (double)(rup_index_y[q2] % 7 ? op2(t2x[c], pf, 1, FY) : op5(t2x[c], pf, 1, FY)) * (double)rDH;
      double v3[3][7];
      for (int l = -3; l <= 3; l++)
        for (int c = 0; c < 3; c++) v3[c][l + 3] = FWf(FW, 6 + c)[pf + (long)l * ny + m * nyz];
      if (freenode && km <= 3)
        for (int c = 0; c < 3; c++) {
          v3[c][km + 2] = 0.0;
          for (int l = km + 3; l < 7; l++) v3[c][l] = -v3[c][2 * (km + 2) - l];
        }
      for (int c = 0; c < 3; c++)
        DzT[c] = (rup_index_z[q2] % 7 ? op2(v3[c], 3, 1, FZ) : op5(v3[c], 3, 1, FZ)) * (double)rDH;
      std::vector<R>* T1c[3] = {&T11, &T12, &T13};
      double Rv[3];
      for (int c = 0; c < 3; c++) {
        const std::vector<R>& T = *T1c[c];
        double r_ = m == 0 ? A1 * T[2 * nyz + pf] + A2 * T[1 * nyz + pf] + A3 * T[0 * nyz + pf]
                           : A1 * T[4 * nyz + pf] + A2 * T[5 * nyz + pf] + A3 * T[6 * nyz + pf];
        Rv[c] = 0.5 * ((2 * m - 1) * r_ + (DyT[c] + DzT[c]) * DHd) * DH2;
      }
      t.Rx[m] = Rv[0]; t.Ry[m] = Rv[1]; t.Rz[m] = Rv[2];
      t.Mrho[m] = 0.5 * jac * rho * DHd * DH2;
      t.jac_last = jac; t.rho_last = rho;
    }
  }
  double stage_time(int it, int irk) {
    return irk == 0 ? it * p.DT : (irk == 3 ? (it + 1) * p.DT : (it + 0.5) * p.DT);
  }
  // common back half: store T1, its rate, outputs (trial_slipweakening.cu:629-709)
  void trial_back(int it, int irk, long q2, long pf, const double* Tau, double Tn_out, double jacvec,
                  const double* T1new, bool from_tau, double Vcheck) {
    long p1 = pf + 3 * nyz;
    double nv[3];
    if (from_tau) {
      T11[p1] = (R)((Tau[0] - str_init_x[q2]) * jacvec);
      T12[p1] = (R)((Tau[1] - str_init_y[q2]) * jacvec);
      T13[p1] = (R)((Tau[2] - str_init_z[q2]) * jacvec);
    } else {
      T11[p1] = (R)T1new[0]; T12[p1] = (R)T1new[1]; T13[p1] = (R)T1new[2];
    }
    nv[0] = ((double)T11[p1] - mT11[p1]) / p.DT;
    nv[1] = ((double)T12[p1] - mT12[p1]) / p.DT;
    nv[2] = ((double)T13[p1] - mT13[p1]) / p.DT;
    if (irk == 3) { hT11[pf] = (R)nv[0]; hT12[pf] = (R)nv[1]; hT13[pf] = (R)nv[2]; }
    double vis = p.viscosity * p.DT;
    T11[p1] = (R)(T11[p1] + vis * nv[0]); T12[p1] = (R)(T12[p1] + vis * nv[1]); T13[p1] = (R)(T13[p1] + vis * nv[2]);
    double ts1 = 0, ts2 = 0;
    for (int c = 0; c < 3; c++) { ts1 += Tau[c] * vecn("vec_s1", pf, c); ts2 += Tau[c] * vecn("vec_s2", pf, c); }
    tTs1[q2] = (R)ts1; tTs2[q2] = (R)ts2; tTn[q2] = (R)Tn_out;
    if (!init_t0_flag[q2] && Vcheck > 1e-3) {
      init_t0[q2] = (R)(it * p.DT); init_t0_flag[q2] = 1; flag_rup[q2] = 1;
    }
  }

  // Slip-weakening trial traction and friction (trial_slipweakening.cu:23-741).
  void trial_sw(int it, int irk, int FX, int FY, int FZ) {
    (void)FX;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        long pf = (j + 3) + (long)(k + 3) * ny, p1 = pf + 3 * nyz;
        if (irk == 0) { mT11[p1] = T11[p1]; mT12[p1] = T12[p1]; mT13[p1] = T13[p1]; }
        TrialPre t;
        trial_front(j, k, FY, FZ, t);
        double tt = stage_time(it, irk);
        if (p.INPORT_STRESS_TYPE == 1) {
          double G = Gt(tt, p.smooth_load_T);
          str_init_x[q2] = (R)(T0x[q2] + G * dT0x[q2]);
          str_init_y[q2] = (R)(T0y[q2] + G * dT0y[q2]);
          str_init_z[q2] = (R)(T0z[q2] + G * dT0z[q2]);
        }
        double dV[3];
        for (int c = 0; c < 3; c++) dV[c] = (double)FWf(FmW, c)[pf + nyz] - (double)FWf(FmW, c)[pf];
        double den = p.DH * p.DH * (t.Mrho[0] * A0P - A0M * t.Mrho[1]);
        double Rm[3][2] = {{t.Rx[0], t.Rx[1]}, {t.Ry[0], t.Ry[1]}, {t.Rz[0], t.Rz[1]}};
        double Trial[3];
        for (int c = 0; c < 3; c++)
          Trial[c] = -(t.Mrho[0] * t.Mrho[1] * dV[c] / p.DT + t.Mrho[0] * Rm[c][1] - t.Mrho[1] * Rm[c][0]) / den * 2.0;
        long qm = P3(i0, j + 3, k + 3);
        double nv[3] = {Mf(0)[qm], Mf(1)[qm], Mf(2)[qm]};
        double n0 = ref_norm3(nv[0], nv[1], nv[2]);
        double jacvec = (double)Mf(9)[qm] * n0;
        for (int c = 0; c < 3; c++) nv[c] /= n0;
        double si[3] = {str_init_x[q2], str_init_y[q2], str_init_z[q2]};
        double TL[3], Ts[3];
        for (int c = 0; c < 3; c++) TL[c] = Trial[c] / jacvec + si[c];
        double Trn = TL[0] * nv[0] + TL[1] * nv[1] + TL[2] * nv[2];
        for (int c = 0; c < 3; c++) Ts[c] = TL[c] - nv[c] * Trn;
        double Ts0 = ref_norm3(Ts[0], Ts[1], Ts[2]);
        bool change = false;
        double Tau_n, Tau_s;
        if (Trn >= 0.0) { Tau_n = 0.0; change = true; } else Tau_n = Trn;
        double mus = str_peak[q2], sl = slip[q2], dc = Dc[q2], mud = p.mu_d;
        double fr = sl <= dc ? mus - (mus - mud) * sl / dc : mud;
        double Tau_c = -fr * Tau_n + (double)C0[q2];
        if (Ts0 >= Tau_c) { Tau_s = Tau_c; flag_rup[q2] = 1; change = true; }
        else { Tau_s = Ts0; flag_rup[q2] = 0; }
        double Tau[3];
        if (change) {
          if (std::fabs(Ts0) < 1e-1) for (int c = 0; c < 3; c++) Tau[c] = Tau_n * nv[c];
          else for (int c = 0; c < 3; c++) Tau[c] = Tau_n * nv[c] + (Tau_s / Ts0) * Ts[c];
        } else for (int c = 0; c < 3; c++) Tau[c] = TL[c];
        trial_back(it, irk, q2, pf, Tau, Tau_n, jacvec, Trial, change, hslip[q2]);
      }
  }

  // Newton on x = asinh(V e^{psi/a} / 2V0) (trial_ratestate.cu:20-57): bounded at 100
  // iterations, relative step tolerance 1e-12, V0 fixed at 1e-6.
  static double newton(double x, double psi, double ra, double Vhat, double coef, int* iters) {
    const double V0 = 1e-6;
    int it = 0;
    double xn = x;
    while (it < 100) {
      double e = 2.0 * std::exp(-psi / ra) * V0;
      double fv = e * std::sinh(x) + coef * x - Vhat;
      double df = e * std::cosh(x) + coef;
      double d = -fv / (df + 1e-100);
      xn = x + d;
      double err = std::fabs(d) / (std::fabs(x) + 1e-100);
      x = xn; it++;
      if (err < 1e-12) break;
    }
    *iters = it;
    return xn;
  }

  // Rate-and-state trial traction with the Newton solve (trial_ratestate.cu:59-893).
  void trial_rs(int it, int irk, int FX, int FY, int FZ) {
    (void)FX;
    long iters = 0;
#pragma omp parallel for schedule(static) reduction(+ : iters)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        long pf = (j + 3) + (long)(k + 3) * ny, p1 = pf + 3 * nyz;
        if (irk == 0) { mT11[p1] = T11[p1]; mT12[p1] = T12[p1]; mT13[p1] = T13[p1]; }
        double s1[3], s2[3], nv[3];
        for (int c = 0; c < 3; c++) { s1[c] = vecn("vec_s1", pf, c); s2[c] = vecn("vec_s2", pf, c); }
        long qm = P3(i0, j + 3, k + 3);
        for (int c = 0; c < 3; c++) nv[c] = Mf(c)[qm];
        double n0 = ref_norm3(nv[0], nv[1], nv[2]);
        double jacvec = (double)Mf(9)[qm] * n0;
        for (int c = 0; c < 3; c++) nv[c] /= n0;
        TrialPre t;
        trial_front(j, k, FY, FZ, t);
        double Rr[3][2];
        for (int m = 0; m < 2; m++) {
          double rx = t.Rx[m], ry = t.Ry[m], rz = t.Rz[m];
          Rr[0][m] = nv[0] * rx + nv[1] * ry + nv[2] * rz;
          Rr[1][m] = s1[0] * rx + s1[1] * ry + s1[2] * rz;
          Rr[2][m] = s2[0] * rx + s2[1] * ry + s2[2] * rz;
        }
        // hard-coded nucleation default, replaced by the file fields (trial_ratestate.cu:383-422)
        int gj = j, gk = k;
        double y1 = gj - p.NY / 2;
        double z1 = freenode ? (double)((p.NZ - 1 - gk) - (int)(7.5e3 / p.DH)) : (double)(gk - p.NZ / 2);
        double r = std::sqrt(y1 * y1 + z1 * z1) * p.DH;
        double tt = stage_time(it, irk);
        double G = Gt(tt, p.smooth_load_T);
        double Fv = Fr(r, 3.0e3);
        str_init_x[q2] = (R)-120e6;
        str_init_y[q2] = (R)(-25e6 * Fv * G + -75e6);
        str_init_z[q2] = 0;
        if (p.INPORT_STRESS_TYPE == 1) {
          str_init_x[q2] = (R)(T0x[q2] + G * dT0x[q2]);
          str_init_y[q2] = (R)(T0y[q2] + G * dT0y[q2]);
          str_init_z[q2] = (R)(T0z[q2] + G * dT0z[q2]);
        }
        double T0[3] = {str_init_x[q2], str_init_y[q2], str_init_z[q2]};
        double T0l[3] = {nv[0] * T0[0] + nv[1] * T0[1] + nv[2] * T0[2], s1[0] * T0[0] + s1[1] * T0[1] + s1[2] * T0[2],
                         s2[0] * T0[0] + s2[1] * T0[1] + s2[2] * T0[2]};
        double dV[3];
        for (int c = 0; c < 3; c++) dV[c] = (double)FWf(FmW, c)[pf + nyz] - (double)FWf(FmW, c)[pf];
        double dt1 = p.DT;
        double Rl[3] = {nv[0] * dV[0] + nv[1] * dV[1] + nv[2] * dV[2], s1[0] * dV[0] + s1[1] * dV[1] + s1[2] * dV[2],
                        s2[0] * dV[0] + s2[1] * dV[1] + s2[2] * dV[2]};
        Rl[1] -= p.Vini;
        double M0 = t.Mrho[0], M1 = t.Mrho[1], DH2 = p.DH * p.DH;
        double den = DH2 * (M0 * A0P - A0M * M1) * jacvec;
        double Tl[3];
        for (int c = 0; c < 3; c++) Tl[c] = T0l[c] - 2.0 * (M0 * M1 * Rl[c] / dt1 + M0 * Rr[c][1] - M1 * Rr[c][0]) / den;
        double cc = -(A0P - A0M) * dt1 * jacvec / (t.jac_last * t.rho_last * p.DH);
        double Tau_n = Tl[0] >= -1e-1 ? -1e-1 : Tl[0];
        double Vt[3] = {cc * Tl[0], cc * Tl[1], cc * Tl[2]};
        // thermal pressurisation: the pore pressure at the fault makes the normal stress of
        // the friction law effective (trial_ratestate.cu:636-643)
        R Pf = 0;
        if (p.Friction_type == 3) { Pf = TP_P[q2]; Tau_n += Pf; }
        double ra = a[q2], st = State[q2];
        double coef = cc * ra * std::fabs(Tau_n);
        double Vtn = std::sqrt(Vt[1] * Vt[1] + Vt[2] * Vt[2]);
        double Ttn = std::sqrt(Tl[1] * Tl[1] + Tl[2] * Tl[2]);
        double Rn = std::sqrt(Rl[1] * Rl[1] + Rl[2] * Rl[2]);
        double x = std::asinh(std::exp(st / ra) * Rn / (2.0 * 1e-6));
        int nit = 0;
        double xn = newton(x, st, ra, Vtn, coef, &nit);
        iters += nit;
        double V = 2.0 * 1e-6 * std::exp(-st / ra) * std::sinh(xn);
        double T = ra * xn * std::fabs(Tau_n);
        friction[q2] = (R)(ra * xn);
        Ttn = std::max(Ttn, 1e-8);
        double Ts1_ = Tl[1] / Ttn * T, Ts2_ = Tl[2] / Ttn * T;
        float Vf = (float)V;  // stored in single precision in the reference
        Vf = std::max(Vf, 1e-30f);
        if (p.Friction_type == 3) Tau_n -= Pf;
        double Tau[3];
        for (int c = 0; c < 3; c++) Tau[c] = Tau_n * nv[c] + Ts1_ * s1[c] + Ts2_ * s2[c];
        Tau[0] = str_init_x[q2];  // the normal-traction perturbation is forced to zero (:797)
        double tn = Tau[0] * nv[0] + Tau[1] * nv[1] + Tau[2] * nv[2];
        trial_back(it, irk, q2, pf, Tau, tn, jacvec, nullptr, true, Vf);
      }
    newton_iters = iters;
  }

  // Split-node averages into the volume at the fault plane (transform.cu:224-403).
  void fault2wave() {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        long pf = (j + 3) + (long)(k + 3) * ny, qm = P3(i0, j + 3, k + 3);
        M3 met, im;  // columns: xi, eta, zeta gradients
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) met[r][c] = Mf(3 * c + r)[qm];
        double rj = 1.0 / (double)Mf(9)[qm];
        M3 tr;
        tr[0][0] = T11[pf + 3 * nyz]; tr[1][0] = T12[pf + 3 * nyz]; tr[2][0] = T13[pf + 3 * nyz];
        for (int c = 0; c < 3; c++) {
          tr[c][1] = ((double)FWf(FW, 3 + c)[pf] + FWf(FW, 3 + c)[pf + nyz]) * 0.5;
          tr[c][2] = ((double)FWf(FW, 6 + c)[pf] + FWf(FW, 6 + c)[pf + nyz]) * 0.5;
        }
        inv3(met, im);
        M3 sg;
        mul3(tr, im, sg);
        for (int c = 0; c < 3; c++) Wf(W, c)[qm] = (R)(((double)FWf(FW, c)[pf] + FWf(FW, c)[pf + nyz]) * 0.5);
        Wf(W, 3)[qm] = (R)(sg[0][0] * rj);
        Wf(W, 4)[qm] = (R)(sg[1][1] * rj);
        Wf(W, 5)[qm] = (R)(sg[2][2] * rj);
        Wf(W, 6)[qm] = (R)((sg[0][1] * rj + sg[1][0] * rj) * 0.5);
        Wf(W, 7)[qm] = (R)((sg[0][2] * rj + sg[2][0] * rj) * 0.5);
        Wf(W, 8)[qm] = (R)((sg[1][2] * rj + sg[2][1] * rj) * 0.5);
      }
  }

  // Velocity RHS on the six off-fault layers and on both split-node sides
  // (fault_dvelo.cu:17-389), traction-image variant.
  void fault_dvelo(int FX, int FY, int FZ) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        int j1 = j + 3, k1 = k + 3, km = nk - k;
        long pf = j1 + (long)k1 * ny;
        for (int i = i0 - 3; i <= i0 + 3; i++) {
          int n = i0 - i;
          if (n == 0) continue;
          double v1[3][7], v2[3][7], v3[3][7];
          for (int l = -3; l <= 3; l++) {
            trac(P3(i + l, j1, k1), 0, v1[0][l + 3], v1[1][l + 3], v1[2][l + 3]);
            trac(P3(i, j1 + l, k1), 3, v2[0][l + 3], v2[1][l + 3], v2[2][l + 3]);
            trac(P3(i, j1, k1 + l), 6, v3[0][l + 3], v3[1][l + 3], v3[2][l + 3]);
          }
          v1[0][n + 3] = T11[pf + 3 * nyz]; v1[1][n + 3] = T12[pf + 3 * nyz]; v1[2][n + 3] = T13[pf + 3 * nyz];
          for (int c = 0; c < 3; c++) {
            double* v = v1[c];
            if (n == 2) v[6] = 2.0 * v[5] - v[4];
            if (n == 1) { v[5] = 2.0 * v[4] - v[3]; v[6] = 2.0 * v[4] - v[2]; }
            if (n == -1) { v[0] = 2.0 * v[2] - v[4]; v[1] = 2.0 * v[2] - v[3]; }
            if (n == -2) v[0] = 2.0 * v[1] - v[2];
          }
          if (freenode && km <= 3)
            for (int c = 0; c < 3; c++) {
              v3[c][km + 2] = 0.0;
              for (int l = km + 3; l < 7; l++) v3[c][l] = -v3[c][2 * (km + 2) - l];
            }
          long q = P3(i, j1, k1);
          double rrj = 1.0 / ((double)Mf(12)[q] * (double)Mf(9)[q]);
          for (int c = 0; c < 3; c++) {
            double dx = op5(v1[c], 3, 1, FX) * (double)rDH, dy = op5(v2[c], 3, 1, FY) * (double)rDH,
                   dz = op5(v3[c], 3, 1, FZ) * (double)rDH;
            Wf(hW, c)[q] = (R)((dx + dy + dz) * rrj);
          }
        }
        for (int mm = 0; mm < 2; mm++) {
          double dx[3], dy[3], dz[3];
          std::vector<R>* T1c[3] = {&T11, &T12, &T13};
          for (int c = 0; c < 3; c++) {
            const std::vector<R>& T = *T1c[c];
            if (mm == 0)
              dx[c] = (double)rDH * (A0M * T[pf + 3 * nyz] - A1 * T[pf + 2 * nyz] - A2 * T[pf + 1 * nyz] - A3 * T[pf]);
            else
              dx[c] = (double)rDH * (A0P * T[pf + 3 * nyz] + A1 * T[pf + 4 * nyz] + A2 * T[pf + 5 * nyz] + A3 * T[pf + 6 * nyz]);
          }
          double v2[3][7], v3[3][7];
          for (int l = -3; l <= 3; l++)
            for (int c = 0; c < 3; c++) {
              v2[c][l + 3] = FWf(FW, 3 + c)[pf + l + mm * nyz];
              v3[c][l + 3] = FWf(FW, 6 + c)[pf + (long)l * ny + mm * nyz];
            }
          if (freenode && km <= 3) {
            for (int c = 0; c < 3; c++) {
              v3[c][km + 2] = 0.0;
              for (int l = km + 3; l < 7; l++) v3[c][l] = -v3[c][2 * (km + 2) - l];
              dz[c] = op5(v3[c], 3, 1, FZ) * (double)rDH;
            }
          } else {
            for (int c = 0; c < 3; c++)
              dz[c] = (rup_index_z[q2] % 7 ? op2(v3[c], 3, 1, FZ) : op5(v3[c], 3, 1, FZ)) * (double)rDH;
          }
          for (int c = 0; c < 3; c++)
            dy[c] = (rup_index_y[q2] % 7 ? op2(v2[c], 3, 1, FY) : op5(v2[c], 3, 1, FY)) * (double)rDH;
          double rrj = 1.0 / ((double)fc["rho_f"][pf + mm * nyz] * (double)Mf(9)[P3(i0, j1, k1)]);
          for (int c = 0; c < 3; c++) FWf(FhW, c)[pf + mm * nyz] = (R)((dx[c] + dy[c] + dz[c]) * rrj);
        }
      }
  }

  void mv(const char* nm, long idx, const double* v, double* out) {
    const R* m = &fc[nm][idx * 9];
    for (int r = 0; r < 3; r++) out[r] = m[3 * r] * v[0] + m[3 * r + 1] * v[1] + m[3 * r + 2] * v[2];
  }
  // Stress RHS near the fault: one-sided DxV on the eight columns, split-node DxV from
  // the T1-rate / continuity matrices, split-node hT2/hT3 and the volume hT on the six
  // off-fault columns (fault_dstrs_f.cu:17-1254 for FX=+1, fault_dstrs_b.cu:17-1249 for FX=-1).
  void fault_dstrs(int FX, int FY, int FZ) {
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        int j1 = j + 3, k1 = k + 3, km = nk - k;
        long pf = j1 + (long)k1 * ny;
        double DxV[8][3], DyV[8][3], DzV[8][3];
        const R* wv[3] = {Wf(W, 0), Wf(W, 1), Wf(W, 2)};
        const R* fv[3] = {FWf(FW, 0), FWf(FW, 1), FWf(FW, 2)};
        auto w = [&](int c, int i) { return (double)wv[c][P3(i, j1, k1)]; };
        auto fs = [&](int c, int m) { return (double)fv[c][pf + m * nyz]; };
        double r = rDH;
        for (int c = 0; c < 3; c++) {
          if (FX == 1) {
            DxV[7][c] = (double)opF(wv[c], P3(i0 + 3, j1, k1), nyz) * r;
            DxV[6][c] = (double)op3F(wv[c], P3(i0 + 2, j1, k1), nyz) * r;
            DxV[5][c] = (w(c, i0 + 2) - w(c, i0 + 1)) * r;
            DxV[4][c] = (w(c, i0 + 1) - fs(c, 1)) * r;
            DxV[2][c] = (fs(c, 0) - w(c, i0 - 1)) * r;
            DxV[1][c] = (-C24_1 * w(c, i0 - 2) + C24_2 * w(c, i0 - 1) - C24_3 * fs(c, 0)) * r;
            DxV[0][c] = (-C1 * w(c, i0 - 4) - C2 * w(c, i0 - 3) + C3 * w(c, i0 - 2) - C4 * w(c, i0 - 1) + C5 * fs(c, 0)) * r;
          } else {
            DxV[0][c] = (double)opB(wv[c], P3(i0 - 3, j1, k1), nyz) * r;
            DxV[1][c] = (double)op3B(wv[c], P3(i0 - 2, j1, k1), nyz) * r;
            DxV[2][c] = (w(c, i0 - 1) - w(c, i0 - 2)) * r;
            DxV[3][c] = (fs(c, 0) - w(c, i0 - 1)) * r;
            DxV[5][c] = (w(c, i0 + 1) - fs(c, 1)) * r;
            DxV[6][c] = (C24_3 * fs(c, 1) - C24_2 * w(c, i0 + 1) + C24_1 * w(c, i0 + 2)) * r;
            DxV[7][c] = (-C5 * fs(c, 1) + C4 * w(c, i0 + 1) - C3 * w(c, i0 + 2) + C2 * w(c, i0 + 3) + C1 * w(c, i0 + 4)) * r;
          }
          for (int m = 0; m < 2; m++) {
            long pm = pf + m * nyz;
            DyV[3 + m][c] = (double)(rup_index_y[q2] % 7 ? op2(fv[c], pm, 1, FY) : op5(fv[c], pm, 1, FY)) * r;
          }
        }
        long f9 = pf;
        if (freenode && km == 1) {
          double o1[3], o2[3], o3[3];
          if (FX == 1) {
            mv("matPlus2Min1f", j1, DxV[4], o1); mv("matPlus2Min2f", j1, DyV[4], o2); mv("matPlus2Min3f", j1, DyV[3], o3);
            for (int c = 0; c < 3; c++) DxV[3][c] = o1[c] + o2[c] - o3[c];
          } else {
            mv("matMin2Plus1f", j1, DxV[3], o1); mv("matMin2Plus2f", j1, DyV[3], o2); mv("matMin2Plus3f", j1, DyV[4], o3);
            for (int c = 0; c < 3; c++) DxV[4][c] = o1[c] + o2[c] - o3[c];
          }
          mv("matVx2Vz1", j1, DxV[3], o1); mv("matVy2Vz1", j1, DyV[3], o2);
          for (int c = 0; c < 3; c++) DzV[3][c] = o1[c] + o2[c];
          mv("matVx2Vz2", j1, DxV[4], o1); mv("matVy2Vz2", j1, DyV[4], o2);
          for (int c = 0; c < 3; c++) DzV[4][c] = o1[c] + o2[c];
        } else {
          for (int c = 0; c < 3; c++)
            for (int m = 0; m < 2; m++) {
              long pm = pf + m * nyz;
              double d;
              if (freenode && km == 2) d = op2(fv[c], pm, ny, FZ);
              else if (freenode && km == 3) d = op3(fv[c], pm, ny, FZ);
              else d = rup_index_z[q2] % 7 ? op2(fv[c], pm, ny, FZ) : op5(fv[c], pm, ny, FZ);
              DzV[3 + m][c] = d * r;
            }
          double dt[3] = {0, 0, 0};
          if (faultgrid[q2]) { dt[0] = hT11[pf]; dt[1] = hT12[pf]; dt[2] = hT13[pf]; }
          double o1[3], o2[3], o3[3];
          mv("matT1toVxm", f9, dt, o1); mv("matVytoVxm", f9, DyV[3], o2); mv("matVztoVxm", f9, DzV[3], o3);
          for (int c = 0; c < 3; c++) DxV[3][c] = o1[c] - o2[c] - o3[c];
          mv("matT1toVxp", f9, dt, o1); mv("matVytoVxp", f9, DyV[4], o2); mv("matVztoVxp", f9, DzV[4], o3);
          for (int c = 0; c < 3; c++) DxV[4][c] = o1[c] - o2[c] - o3[c];
        }
        // split-node traction rates (fault_dstrs_f.cu:876-1006)
        const char* Dn[2][2][3] = {{{"D21_1", "D22_1", "D23_1"}, {"D31_1", "D32_1", "D33_1"}},
                                   {{"D21_2", "D22_2", "D23_2"}, {"D31_2", "D32_2", "D33_2"}}};
        for (int m = 0; m < 2; m++)
          for (int g = 0; g < 2; g++) {
            double o1[3], o2[3], o3[3];
            mv(Dn[m][g][0], f9, DxV[3 + m], o1); mv(Dn[m][g][1], f9, DyV[3 + m], o2); mv(Dn[m][g][2], f9, DzV[3 + m], o3);
            for (int c = 0; c < 3; c++) FWf(FhW, 3 + 3 * g + c)[pf + m * nyz] = (R)(o1[c] + o2[c] + o3[c]);
          }
        // volume stress RHS on the off-fault columns (fault_dstrs_f.cu:1156-1250)
        for (int n = 0; n < 8; n++) {
          int l = n < 4 ? n - 3 : n - 4;
          if (l == 0) continue;
          int i = i0 + l;
          long q = P3(i, j1, k1);
          for (int c = 0; c < 3; c++) DyV[n][c] = (double)op5(wv[c], q, 1, FY) * r;
          if (freenode && km == 1) {
            const R* mx = &matVx2Vz[(j1 + (long)i * ny) * 9];
            const R* my = &matVy2Vz[(j1 + (long)i * ny) * 9];
            for (int c = 0; c < 3; c++)
              DzV[n][c] = mx[3 * c] * DxV[n][0] + mx[3 * c + 1] * DxV[n][1] + mx[3 * c + 2] * DxV[n][2] +
                          my[3 * c] * DyV[n][0] + my[3 * c + 1] * DyV[n][1] + my[3 * c + 2] * DyV[n][2];
          } else {
            for (int c = 0; c < 3; c++) {
              double d;
              if (freenode && km == 2) d = op2(wv[c], q, ny, FZ);
              else if (freenode && km == 3) d = op3(wv[c], q, ny, FZ);
              else d = op5(wv[c], q, ny, FZ);
              DzV[n][c] = d * r;
            }
          }
          double lam = Mf(10)[q], mu = Mf(11)[q], l2m = lam + 2.0 * mu;
          double ex[3] = {Mf(0)[q], Mf(1)[q], Mf(2)[q]}, ey[3] = {Mf(3)[q], Mf(4)[q], Mf(5)[q]},
                 ez[3] = {Mf(6)[q], Mf(7)[q], Mf(8)[q]};
          double* X = DxV[n]; double* Y = DyV[n]; double* Z = DzV[n];
          Wf(hW, 3)[q] = (R)(l2m * ex[0] * X[0] + lam * ex[1] * X[1] + lam * ex[2] * X[2] + l2m * ey[0] * Y[0] +
                             lam * ey[1] * Y[1] + lam * ey[2] * Y[2] + l2m * ez[0] * Z[0] + lam * ez[1] * Z[1] +
                             lam * ez[2] * Z[2]);
          Wf(hW, 4)[q] = (R)(lam * ex[0] * X[0] + l2m * ex[1] * X[1] + lam * ex[2] * X[2] + lam * ey[0] * Y[0] +
                             l2m * ey[1] * Y[1] + lam * ey[2] * Y[2] + lam * ez[0] * Z[0] + l2m * ez[1] * Z[1] +
                             lam * ez[2] * Z[2]);
          Wf(hW, 5)[q] = (R)(lam * ex[0] * X[0] + lam * ex[1] * X[1] + l2m * ex[2] * X[2] + lam * ey[0] * Y[0] +
                             lam * ey[1] * Y[1] + l2m * ey[2] * Y[2] + lam * ez[0] * Z[0] + lam * ez[1] * Z[1] +
                             l2m * ez[2] * Z[2]);
          Wf(hW, 6)[q] = (R)((ex[1] * X[0] + ex[0] * X[1] + ey[1] * Y[0] + ey[0] * Y[1] + ez[1] * Z[0] + ez[0] * Z[1]) * mu);
          Wf(hW, 7)[q] = (R)((ex[2] * X[0] + ex[0] * X[2] + ey[2] * Y[0] + ey[0] * Y[2] + ez[2] * Z[0] + ez[0] * Z[2]) * mu);
          Wf(hW, 8)[q] = (R)((ex[2] * X[1] + ex[1] * X[2] + ey[2] * Y[1] + ey[1] * Y[2] + ez[2] * Z[1] + ez[1] * Z[2]) * mu);
        }
      }
  }

  // Split-node RK4 (+ viscosity) and the RK-weighted on-fault outputs
  // (rk4.cu:466-789, fault_rk launches both at rk4.cu:940-956).
  void fault_rk(int irk) {
    float rka, rkb;
    rk_weights(irk, (float)p.DT, &rka, &rkb);
    double vis = p.viscosity * p.DT;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj;
        if (united[q2]) continue;
        for (int m = 0; m < 2; m++) {
          long x = (j + 3) + (long)(k + 3) * ny + m * nyz;
          for (int f = 0; f < 9; f++) {
            R* Wv = FWf(FW, f); R* mWv = FWf(FmW, f); R* h = FWf(FhW, f); R* tWv = FWf(FtW, f);
            if (irk == 0) { mWv[x] = Wv[x]; tWv[x] = (R)(rkb * h[x] + mWv[x]); }
            else if (irk == 1 || irk == 2) tWv[x] = (R)(tWv[x] + rkb * h[x]);
            if (irk == 3) Wv[x] = (R)(rkb * h[x] + tWv[x]);
            else Wv[x] = (R)(rka * h[x] + mWv[x]);
            if (f >= 3) Wv[x] = (R)(Wv[x] + vis * h[x]);
          }
        }
      }
    float rkb1 = rkb / (float)p.DT;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q2 = j + (long)k * nj, f = (j + 3) + (long)(k + 3) * ny;
        double dV[3];
        for (int c = 0; c < 3; c++) dV[c] = (double)FWf(FW, c)[f + nyz] - (double)FWf(FW, c)[f];
        double vs1 = 0, vs2 = 0;
        for (int c = 0; c < 3; c++) { vs1 += dV[c] * vecn("vec_s1", f, c); vs2 += dV[c] * vecn("vec_s2", f, c); }
        hslip[q2] = (R)std::sqrt(vs2 * vs2 + vs1 * vs1);
        Vs1[q2] = (R)vs1; Vs2[q2] = (R)vs2;
        if (irk == 0) {
          Ts1[q2] = (R)(rkb1 * tTs1[q2]); Ts2[q2] = (R)(rkb1 * tTs2[q2]); Tn[q2] = (R)(rkb1 * tTn[q2]);
        } else {
          Ts1[q2] = (R)(Ts1[q2] + rkb1 * tTs1[q2]); Ts2[q2] = (R)(Ts2[q2] + rkb1 * tTs2[q2]);
          Tn[q2] = (R)(Tn[q2] + rkb1 * tTn[q2]);
        }
      }
  }

  // Thermal pressurisation (thermpress.cu:22-236), once per step before the stages
  // (main.cu:444-447).  Per non-united node: nt_sub explicit sub-steps of 1-D diffusion of
  // temperature T and pore pressure P over TP_n points normal to the fault (mirror ends),
  // heated by the frictional work tau*V spread as a Gaussian of half-width h:
  //   dT = alpha_th T'' + omega(x),  dP = alpha_hy P'' + Lambda dT,
  // tau = -friction (Tn + P[0]); column width sqrt(100 alpha_max), sub-step 0.1 dh^2/alpha_max.
  // Types as the reference's: real_t locals, the double literals promote the second
  // differences and the Gaussian to double.
  void thermpress() {
    const R Lamb = (R)0.1e6, rho_c = (R)2.7e6, h = (R)20e-3, alpha_th = (R)1.0e-6;
    const R h2 = h * h;
    const double SQRT2PI = 2.506628274631000;
    const long nf = (long)nj * nk;
    const int n = p.TP_n;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < nf; q++) {
      if (united[q]) continue;
      R rate = std::sqrt(Vs1[q] * Vs1[q] + Vs2[q] * Vs2[q]);
      R Tau_n = Tn[q], fr = friction[q], ahy = TP_hy[q];
      R amax = std::max(alpha_th, ahy);
      R w = (R)std::sqrt(4.0 * amax * 25.0);
      R dh = (R)(w / (double)(n - 1));
      R dh2 = dh * dh;
      R dt = (R)(0.1 * dh2 / amax);
      int nsub = (int)((R)p.DT / dt) + 1;
      dt = (R)((R)p.DT / (double)nsub);
      std::vector<R> dT(n), dP(n);
      for (int sub = 0; sub < nsub; sub++) {
        R tau = -fr * (Tau_n + TP_P[q]);
        R tauV = tau * rate;
        for (int i = 0; i < n; i++) {
          R x = i * dh;
          R x2 = x * x;
          R omega = (R)(std::exp(-0.5 * x2 / h2) * (tauV / (rho_c * h * SQRT2PI)));
          long c = q + i * nf;
          long pl = i == n - 1 ? c - nf : c + nf;  // the ends mirror their one neighbour
          long mi = i == 0 ? c + nf : c - nf;
          dT[i] = (R)(alpha_th * (TP_T[pl] - 2.0 * TP_T[c] + TP_T[mi]) / dh2 + omega);
          dP[i] = (R)(ahy * (TP_P[pl] - 2.0 * TP_P[c] + TP_P[mi]) / dh2 + Lamb * dT[i]);
        }
        for (int i = 0; i < n; i++) {
          TP_T[q + i * nf] += dt * dT[i];
          TP_P[q + i * nf] += dt * dP[i];
        }
      }
    }
  }

  // Rupture sensor (rup_sensor.cu:8-95), once per step before the stages: on the fault
  // grid shrunk by 3 nodes (1-based global indices), second differences of Ts1 along y and
  // z for the non-united nodes, then
  //   sensor = (0.5 (D1^2 + D2^2)_y + 0.5 (D1^2 + D2^2)_z) / (Ts1^2 + 1e-16) + 1e-16,
  // zero on united nodes.  The z term differences Dz at the node with Dy (not Dz) at its z
  // neighbours, as the reference's second kernel does.  Untouched entries keep their zero.
  void rup_sensor_step() {
    const int* fg = p.Fault_grid;
    auto inside = [&](int j, int k) {
      return j + 1 >= fg[0] + 3 && j + 1 <= fg[1] - 3 && k + 1 >= fg[2] + 3 && k + 1 <= fg[3] - 3;
    };
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q = j + (long)nj * k;
        if (!inside(j, k) || united[q]) continue;
        const R* t = Ts1.data();
        rup_Dy[q] = (R)(0.25 * (-t[q + 1] + 2.0 * t[q] - t[q - 1]));
        rup_Dz[q] = (R)(0.25 * (-t[q + nj] + 2.0 * t[q] - t[q - nj]));
      }
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        long q = j + (long)nj * k;
        if (!inside(j, k)) continue;
        R D1 = rup_Dy[q] - rup_Dy[q + 1];
        R D2 = rup_Dy[q] - rup_Dy[q - 1];
        R mag = (R)(0.5 * (D1 * D1 + D2 * D2));
        D1 = rup_Dz[q] - rup_Dy[q + nj];
        D2 = rup_Dz[q] - rup_Dy[q - nj];
        mag = (R)(mag + 0.5 * (D1 * D1 + D2 * D2));
        R p0 = Ts1[q] * Ts1[q];
        rup_sensor[q] = (R)(mag / (p0 + 1e-16) + 1e-16);
        if (united[q]) rup_sensor[q] = 0;
      }
  }

  // One time step: four RK stages with the reference's launch order (main.cu:420-535).
  void step(int it) {
    int FX = FD_FLAGS[it % 8][0], FY = FD_FLAGS[it % 8][1], FZ = FD_FLAGS[it % 8][2];
    rup_sensor_step();
    if (p.Friction_type == 3) thermpress();
    for (int irk = 0; irk < 4; irk++) {
      state_rk(irk);
      if (p.Friction_type == 0) trial_sw(it, irk, FX, FY, FZ);
      else trial_rs(it, irk, FX, FY, FZ);
      fault2wave();
      wave_deriv(FX, FY, FZ);
      if (isx1) abs_deriv(0, FX);
      if (isx2) abs_deriv(1, FX);
      if (isy1) abs_deriv(2, FY);
      if (isy2) abs_deriv(3, FY);
      if (isz1) abs_deriv(4, FZ);
      if (isz2) abs_deriv(5, FZ);
      fault_dvelo(FX, FY, FZ);
      fault_dstrs(FX, FY, FZ);
      wave_rk(irk);
      fault_rk(irk);
      fault2wave();
      apply_cerjan();
      FX = -FX; FY = -FY; FZ = -FZ;
    }
  }
  // One part of stage irk of step it, the stage split as the product's dfd_stage_part
  // splits it: 0 = (stage 0: rupture sensor, thermal pressurisation) state_rk, trial,
  // fault2wave; 1 = wave_deriv, abs_deriv of the PML faces; 2 = fault_dvelo, fault_dstrs,
  // wave_rk, fault_rk, fault2wave, apply_cerjan.  Parts 0, 1, 2 of stages 0..3 are step().
  void stage_part(int it, int irk, int part) {
    const int sg = (irk % 2) ? -1 : 1;
    const int FX = FD_FLAGS[it % 8][0] * sg, FY = FD_FLAGS[it % 8][1] * sg, FZ = FD_FLAGS[it % 8][2] * sg;
    if (part == 0) {
      if (irk == 0) {
        rup_sensor_step();
        if (p.Friction_type == 3) thermpress();
      }
      state_rk(irk);
      if (p.Friction_type == 0) trial_sw(it, irk, FX, FY, FZ);
      else trial_rs(it, irk, FX, FY, FZ);
      fault2wave();
    } else if (part == 1) {
      wave_deriv(FX, FY, FZ);
      if (isx1) abs_deriv(0, FX);
      if (isx2) abs_deriv(1, FX);
      if (isy1) abs_deriv(2, FY);
      if (isy2) abs_deriv(3, FY);
      if (isz1) abs_deriv(4, FZ);
      if (isz2) abs_deriv(5, FZ);
    } else {
      fault_dvelo(FX, FY, FZ);
      fault_dstrs(FX, FY, FZ);
      wave_rk(irk);
      fault_rk(irk);
      fault2wave();
      apply_cerjan();
    }
  }
  // Volume-only stage sequence (no rupture kernels) used by the pure-stencil checks.
  void step_volume(int it) {
    int FX = FD_FLAGS[it % 8][0], FY = FD_FLAGS[it % 8][1], FZ = FD_FLAGS[it % 8][2];
    for (int irk = 0; irk < 4; irk++) {
      wave_deriv(FX, FY, FZ);
      if (isx1) abs_deriv(0, FX);
      if (isx2) abs_deriv(1, FX);
      if (isy1) abs_deriv(2, FY);
      if (isy2) abs_deriv(3, FY);
      if (isz1) abs_deriv(4, FZ);
      if (isz2) abs_deriv(5, FZ);
      wave_rk(irk);
      apply_cerjan();
      FX = -FX; FY = -FY; FZ = -FZ;
    }
  }

  void setup(const orc_params* pp, const float* fxyz, const float* stress, int nlayer, const float* layers) {
    p = *pp;
    alloc();
    pml_init();
    construct_coord(fxyz);
    cal_metric(nlayer, layers);
    init_fault_coef();
    init_fault(stress);
    init_wave_free();
    init_cerjan();
  }

  // named-array lookup for the C ABI
  bool lookup(const std::string& nm, const R** ptr, long* n, const int** iptr) {
    *iptr = nullptr;
    std::map<std::string, std::vector<R>*> t = {
        {"W", &W}, {"hW", &hW}, {"mW", &mW}, {"tW", &tW}, {"M", &M}, {"FW", &FW}, {"FhW", &FhW}, {"FmW", &FmW},
        {"FtW", &FtW}, {"T11", &T11}, {"T12", &T12}, {"T13", &T13}, {"hT11", &hT11}, {"hT12", &hT12},
        {"hT13", &hT13}, {"mT11", &mT11}, {"Tn", &Tn}, {"Ts1", &Ts1}, {"Ts2", &Ts2}, {"tTn", &tTn},
        {"tTs1", &tTs1}, {"tTs2", &tTs2}, {"str_init_x", &str_init_x}, {"str_init_y", &str_init_y},
        {"str_init_z", &str_init_z}, {"slip", &slip}, {"hslip", &hslip}, {"Vs1", &Vs1}, {"Vs2", &Vs2},
        {"State", &State}, {"init_t0", &init_t0}, {"friction", &friction}, {"str_peak", &str_peak},
        {"TP_T", &TP_T}, {"TP_P", &TP_P}, {"TP_hy", &TP_hy}, {"rup_sensor", &rup_sensor},
        {"matVx2Vz", &matVx2Vz}, {"matVy2Vz", &matVy2Vz}, {"damp", &damp}, {"Bx", &Bx}, {"By", &By},
        {"Bz", &Bz}, {"Dx", &Dx}, {"Dy", &Dy}, {"Dz", &Dz}, {"Ax", &Ax}, {"Ay", &Ay}, {"Az", &Az},
        {"aux_x1", &aux[0][0]}, {"aux_x2", &aux[1][0]}, {"aux_y1", &aux[2][0]}, {"aux_y2", &aux[3][0]},
        {"aux_z1", &aux[4][0]}, {"aux_z2", &aux[5][0]}};
    auto itv = t.find(nm);
    if (itv != t.end()) { *ptr = itv->second->data(); *n = itv->second->size(); return true; }
    auto itf = fc.find(nm);
    if (itf != fc.end()) { *ptr = itf->second.data(); *n = itf->second.size(); return true; }
    std::map<std::string, std::vector<int>*> ti = {{"united", &united}, {"faultgrid", &faultgrid},
                                                   {"rup_index_y", &rup_index_y}, {"rup_index_z", &rup_index_z},
                                                   {"init_t0_flag", &init_t0_flag}, {"flag_rup", &flag_rup}};
    auto iti = ti.find(nm);
    if (iti != ti.end()) { *iptr = iti->second->data(); *n = iti->second->size(); return true; }
    return false;
  }
};

}  // namespace orc

// ------------------------------------------------------------------- C ABI --
struct orc_handle {
  int dp;
  orc::Sim<double>* d;
  orc::Sim<float>* f;
};

extern "C" {
void* orc_create(const orc_params* p, int double_precision, const float* fxyz, const float* stress, int nlayer,
                 const float* layers) {
  orc_handle* h = new orc_handle();
  h->dp = double_precision;
  h->d = nullptr; h->f = nullptr;
  if (double_precision) { h->d = new orc::Sim<double>(); h->d->setup(p, fxyz, stress, nlayer, layers); }
  else { h->f = new orc::Sim<float>(); h->f->setup(p, fxyz, stress, nlayer, layers); }
  return h;
}
void orc_destroy(void* hv) {
  orc_handle* h = (orc_handle*)hv;
  delete h->d; delete h->f; delete h;
}
int orc_step(void* hv, int it) {
  orc_handle* h = (orc_handle*)hv;
  if (h->dp) h->d->step(it); else h->f->step(it);
  return 0;
}
int orc_stage_part(void* hv, int it, int irk, int part) {
  orc_handle* h = (orc_handle*)hv;
  if (irk < 0 || irk > 3 || part < 0 || part > 2) return 1;
  if (h->dp) h->d->stage_part(it, irk, part); else h->f->stage_part(it, irk, part);
  return 0;
}
int orc_step_volume(void* hv, int it) {
  orc_handle* h = (orc_handle*)hv;
  if (h->dp) h->d->step_volume(it); else h->f->step_volume(it);
  return 0;
}
long orc_newton_iters(void* hv) {
  orc_handle* h = (orc_handle*)hv;
  return h->dp ? h->d->newton_iters : h->f->newton_iters;
}
// Copy a named array into out (float64).  Returns the element count, or -1.
long orc_get(void* hv, const char* name, double* out) {
  orc_handle* h = (orc_handle*)hv;
  long n = 0;
  const int* ip = nullptr;
  if (h->dp) {
    const double* p = nullptr;
    if (!h->d->lookup(name, &p, &n, &ip)) return -1;
    if (out) for (long x = 0; x < n; x++) out[x] = ip ? ip[x] : p[x];
  } else {
    const float* p = nullptr;
    if (!h->f->lookup(name, &p, &n, &ip)) return -1;
    if (out) for (long x = 0; x < n; x++) out[x] = ip ? ip[x] : p[x];
  }
  return n;
}
// Overwrite a named floating array from float64 input (same element count).
long orc_set(void* hv, const char* name, const double* in) {
  orc_handle* h = (orc_handle*)hv;
  long n = 0;
  const int* ip = nullptr;
  if (h->dp) {
    const double* p = nullptr;
    if (!h->d->lookup(name, &p, &n, &ip) || ip) return -1;
    double* q = const_cast<double*>(p);
    for (long x = 0; x < n; x++) q[x] = in[x];
  } else {
    const float* p = nullptr;
    if (!h->f->lookup(name, &p, &n, &ip) || ip) return -1;
    float* q = const_cast<float*>(p);
    for (long x = 0; x < n; x++) q[x] = (float)in[x];
  }
  return n;
}
int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
}
