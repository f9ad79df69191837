// FP64 grid / metric / media construction on the GPU.
//
// The reference builds 3-D coordinate arrays on the host (construct_coord,
// coord.cu:153-328), extrapolates their ghost layers (extend_crew_array, metric.cu:248-313),
// computes a second-order central metric and the media on the host (cal_metric
// metric.cu:15-171, init_media1d media.cu:63-138) and mirrors the ghost layers
// (extend_Symm_array metric.cu:173-246).  Its grid is separable -- x = xline(i) + fx(j,k),
// y = fy(j,k), z = fz(j,k) -- and the linear ghost extrapolation keeps that form, so here
// the coordinates are never stored: the host extends the 1-D line and the 2-D surface,
// and one FP64 kernel evaluates metric and media per node, a second fills the ghosts by
// mirroring, and a third computes the CFL spacing (dist_point2plane_h, mathFuncs.cu:73-97).
#include "dfd_internal.cuh"

namespace dfd {


__device__ inline void coord(const GridArgs& g, int i, int j, int k, double* c) {
  long long f = j + (long long)k * g.d.ny;
  c[0] = g.xl[i] + g.fx[f];
  c[1] = g.fy[f];
  c[2] = g.fz[f];
}

__global__ void metric_kernel(GridArgs g, float* M) {
  const Dims& d = g.d;
  int j = blockIdx.x * blockDim.x + threadIdx.x + 3;
  int k = blockIdx.y * blockDim.y + threadIdx.y + 3;
  int i = blockIdx.z * blockDim.z + threadIdx.z + 3;
  if (j >= d.ny - 3 || k >= d.nz - 3 || i >= d.nx - 3) return;
  double xp[3], xm[3], yp[3], ym[3], zp[3], zm[3], c0[3];
  coord(g, i + 1, j, k, xp); coord(g, i - 1, j, k, xm);
  coord(g, i, j + 1, k, yp); coord(g, i, j - 1, k, ym);
  coord(g, i, j, k + 1, zp); coord(g, i, j, k - 1, zm);
  coord(g, i, j, k, c0);
  double v1[3], v2[3], v3[3];
  for (int c = 0; c < 3; c++) {
    v1[c] = 0.5 * g.rDH * (xp[c] - xm[c]);
    v2[c] = 0.5 * g.rDH * (yp[c] - ym[c]);
    v3[c] = 0.5 * g.rDH * (zp[c] - zm[c]);
  }
  double e1[3], e2[3], e3[3];
  e3[0] = v1[1] * v2[2] - v1[2] * v2[1]; e3[1] = v1[2] * v2[0] - v1[0] * v2[2]; e3[2] = v1[0] * v2[1] - v1[1] * v2[0];
  e1[0] = v2[1] * v3[2] - v2[2] * v3[1]; e1[1] = v2[2] * v3[0] - v2[0] * v3[2]; e1[2] = v2[0] * v3[1] - v2[1] * v3[0];
  e2[0] = v3[1] * v1[2] - v3[2] * v1[1]; e2[1] = v3[2] * v1[0] - v3[0] * v1[2]; e2[2] = v3[0] * v1[1] - v3[1] * v1[0];
  double jac = e3[0] * v3[0] + e3[1] * v3[1] + e3[2] * v3[2];
  double rj = 1.0 / jac;
  long long n = d.nxyz, q = idx3(d, i, j, k);
  for (int c = 0; c < 3; c++) {
    M[c * n + q] = (float)(e1[c] * rj);
    M[(3 + c) * n + q] = (float)(e2[c] * rj);
    M[(6 + c) * n + q] = (float)(e3[c] * rj);
  }
  M[9 * n + q] = (float)jac;
  double lam, mu, rho;
  if (g.nlayer > 0) {
    double depth = -c0[2];
    int l0 = g.nlayer - 1;
    for (int l = g.nlayer - 1; l >= 0; l--)
      if (depth > (double)g.layers[4 * l]) { l0 = l; break; }
    double r = g.layers[4 * l0 + 1], vp = g.layers[4 * l0 + 2], vs = g.layers[4 * l0 + 3];
    lam = r * (vp * vp - 2 * vs * vs); mu = r * vs * vs; rho = r;
  } else if (i < g.NXhalf) {
    lam = g.lam1; mu = g.mu1; rho = g.rho1;
  } else {
    lam = g.lam2; mu = g.mu2; rho = g.rho2;
  }
  M[10 * n + q] = (float)lam;
  M[11 * n + q] = (float)mu;
  M[12 * n + q] = (float)rho;
}

// ghost value = value at the mirrored node in every ghost axis (the composition of the
// three sequential mirror passes of metric.cu:173-246)
__device__ inline int mirror(int i, int n) { return i < 3 ? 6 - i : (i > n - 4 ? 2 * (n - 4) - i : i); }
__global__ void ghost_mirror_kernel(Dims d, float* M, int nfield) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int k = blockIdx.y * blockDim.y + threadIdx.y;
  int i = blockIdx.z * blockDim.z + threadIdx.z;
  if (j >= d.ny || k >= d.nz || i >= d.nx) return;
  int mi = mirror(i, d.nx), mj = mirror(j, d.ny), mk = mirror(k, d.nz);
  if (mi == i && mj == j && mk == k) return;
  long long q = idx3(d, i, j, k), s = idx3(d, mi, mj, mk);
  for (int f = 0; f < nfield; f++) M[f * d.nxyz + q] = M[f * d.nxyz + s];
}

// minimum node-to-face distance of every interior node (cal_range_steph, coord.cu:330-391)
// and maximum P velocity, reduced per (j, k) column over i
__device__ inline double dist_plane(const double* x0, const double* x1, const double* x2, const double* x3) {
  double a[3] = {x2[0] - x1[0], x2[1] - x1[1], x2[2] - x1[2]};
  double b[3] = {x3[0] - x1[0], x3[1] - x1[1], x3[2] - x1[2]};
  double p[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
  double dd = p[0] * x1[0] + p[1] * x1[1] + p[2] * x1[2];
  double px = p[0] * x0[0] + p[1] * x0[1] + p[2] * x0[2];
  return fabs(px - dd) / sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
}
__global__ void cfl_kernel(GridArgs g, const float* M, float* hmin, float* vpmax) {
  const Dims& d = g.d;
  int j = blockIdx.x * blockDim.x + threadIdx.x + 3;
  int k = blockIdx.y * blockDim.y + threadIdx.y + 3;
  if (j >= d.ny - 3 || k >= d.nz - 3) return;
  double hm = 1e38, vm = 0;
  for (int i = 3; i < d.nx - 3; i++) {
    double x0[3], x1[3], x2[3], x3[3];
    coord(g, i, j, k, x0);
    for (int ii = -1; ii <= 1; ii += 2)
      for (int jj = -1; jj <= 1; jj += 2)
        for (int kk = -1; kk <= 1; kk += 2) {
          coord(g, i + ii, j, k, x1);
          coord(g, i, j + jj, k, x2);
          coord(g, i, j, k + kk, x3);
          hm = fmin(hm, dist_plane(x0, x1, x2, x3));
        }
    long long q = idx3(d, i, j, k);
    double lam = M[10 * d.nxyz + q], mu = M[11 * d.nxyz + q], rho = M[12 * d.nxyz + q];
    vm = fmax(vm, sqrt((lam + 2 * mu) / rho));
  }
  long long f = (j - 3) + (long long)(k - 3) * (d.ny - 6);
  hmin[f] = (float)hm;
  vpmax[f] = (float)vm;
}

// Separable factors of the same discrete metric for the tiled interior kernel.  With
// v1 = (a, 0, 0) (a = d xline / d xi), v2 = (p, q, r) and v3 = (s, t, w) the derivatives
// along eta and zeta of the fault surface (fx, fy, fz), the inverse metric of
// metric_kernel is
//   xi = (1, (r s - p w) / D, (p t - q s) / D) / a,  et = (0, w, -t) / D,
//   zt = (0, -r, q) / D,  D = q w - r t,
// so it splits into six (j, k) planes U V ety etz zty ztz and the 1-D line 1/a(i); the
// media are (j, k) planes for the two sides of the bimaterial split (equal otherwise).
// Planes are stored (12, nz, py) with the volume row offset, so that the tiled kernel's
// TMA boxes use the volume coordinates.
__global__ void plane_metric_kernel(GridArgs g, float* pl, float* rxa) {
  const Dims& d = g.d;
  int j = blockIdx.x * blockDim.x + threadIdx.x + 3;
  int k = blockIdx.y * blockDim.y + threadIdx.y + 3;
  if (blockIdx.x == 0 && blockIdx.y == 0) {
    for (int i = 3 + threadIdx.x + threadIdx.y * blockDim.x; i < d.nx - 3; i += blockDim.x * blockDim.y)
      rxa[i] = (float)(1.0 / (0.5 * g.rDH * (g.xl[i + 1] - g.xl[i - 1])));
  }
  if (j >= d.ny - 3 || k >= d.nz - 3) return;
  auto at = [&](int jj, int kk, int c) {
    long long f = jj + (long long)kk * d.ny;
    return c == 0 ? g.fx[f] : c == 1 ? g.fy[f] : g.fz[f];
  };
  double v2[3], v3[3];
  for (int c = 0; c < 3; c++) {
    v2[c] = 0.5 * g.rDH * (at(j + 1, k, c) - at(j - 1, k, c));
    v3[c] = 0.5 * g.rDH * (at(j, k + 1, c) - at(j, k - 1, c));
  }
  double pp = v2[0], q = v2[1], r = v2[2], sv = v3[0], t = v3[1], w = v3[2];
  double D = q * w - r * t;
  const long long np = (long long)d.py * d.nz, o = (j + d.oy) + (long long)k * d.py;
  pl[0 * np + o] = (float)((r * sv - pp * w) / D);
  pl[1 * np + o] = (float)((pp * t - q * sv) / D);
  pl[2 * np + o] = (float)(w / D);
  pl[3 * np + o] = (float)(-t / D);
  pl[4 * np + o] = (float)(-r / D);
  pl[5 * np + o] = (float)(q / D);
  double m[2][3];
  if (g.nlayer > 0) {
    double depth = -at(j, k, 2);
    int l0 = g.nlayer - 1;
    for (int l = g.nlayer - 1; l >= 0; l--)
      if (depth > (double)g.layers[4 * l]) { l0 = l; break; }
    double rh = g.layers[4 * l0 + 1], vp = g.layers[4 * l0 + 2], vs = g.layers[4 * l0 + 3];
    m[0][0] = m[1][0] = rh * (vp * vp - 2 * vs * vs);
    m[0][1] = m[1][1] = rh * vs * vs;
    m[0][2] = m[1][2] = rh;
  } else {
    m[0][0] = g.lam1; m[0][1] = g.mu1; m[0][2] = g.rho1;
    m[1][0] = g.lam2; m[1][1] = g.mu2; m[1][2] = g.rho2;
  }
  for (int sd = 0; sd < 2; sd++)
    for (int c = 0; c < 3; c++) pl[(6 + 3 * sd + c) * np + o] = (float)m[sd][c];
}

void launch_plane_metric(const GridArgs& g, float* pl, float* rxa, cudaStream_t s) {
  dim3 b(32, 4);
  dim3 gr((g.d.ny - 6 + 31) / 32, (g.d.nz - 6 + 3) / 4);
  plane_metric_kernel<<<gr, b, 0, s>>>(g, pl, rxa);
}

void launch_metric(const GridArgs& g, float* M, cudaStream_t s) {
  dim3 b(32, 4, 2);
  dim3 gr((g.d.ny - 6 + 31) / 32, (g.d.nz - 6 + 3) / 4, (g.d.nx - 6 + 1) / 2);
  metric_kernel<<<gr, b, 0, s>>>(g, M);
  dim3 gg((g.d.ny + 31) / 32, (g.d.nz + 3) / 4, (g.d.nx + 1) / 2);
  ghost_mirror_kernel<<<gg, b, 0, s>>>(g.d, M, 13);
}
void launch_cfl(const GridArgs& g, const float* M, float* hmin, float* vpmax, cudaStream_t s) {
  dim3 b(32, 4);
  dim3 gr((g.d.ny - 6 + 31) / 32, (g.d.nz - 6 + 3) / 4);
  cfl_kernel<<<gr, b, 0, s>>>(g, M, hmin, vpmax);
}

}  // namespace dfd
