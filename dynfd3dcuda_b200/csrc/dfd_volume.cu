// Fused volume stage: one pass per RK stage computes the velocity-stress right-hand
// side with the 5-point one-sided DRP operators and curvilinear metric terms
// (reference wave.cu:8-494), the free-surface rows and traction image (wave.cu:205-487),
// the ADE PML auxiliary equations of all six faces (pmlx.cu:8-214, pmly.cu, pmlz.cu),
// the classic RK4 register update (rk4.cu:20-33,154-257) and the Cerjan sponge
// (cerjan.cu:166-200).  The right-hand side never reaches HBM: each stage reads the
// stencil input (9 fields), the 12 metric/media fields and its RK registers, and writes
// its output and accumulator -- 39/57/57/39 floats per node for stages 0..3.
//
// Nodes of the seven x-layers around the fault whose (j,k) is not "united" are left
// to the band kernel (dfd_fault.cu), exactly the nodes whose right-hand side the
// reference overwrites in fault_dvelo / fault_dstrs.
#include <cstring>

#include "dfd_stencil.cuh"

namespace dfd {

template <int F>
__device__ __forceinline__ float d5(const float* __restrict__ v, long long q, long long s) {
  if (F == 1)
    return -DFD_C1 * __ldg(v + q - s) - DFD_C2 * __ldg(v + q) + DFD_C3 * __ldg(v + q + s) -
           DFD_C4 * __ldg(v + q + 2 * s) + DFD_C5 * __ldg(v + q + 3 * s);
  else
    return -DFD_C5 * __ldg(v + q - 3 * s) + DFD_C4 * __ldg(v + q - 2 * s) - DFD_C3 * __ldg(v + q - s) +
           DFD_C2 * __ldg(v + q) + DFD_C1 * __ldg(v + q + s);
}
template <int F>
__device__ __forceinline__ float d5a(const float* v, int c) {  // on a 7-point register line, centre c
  if (F == 1) return -DFD_C1 * v[c - 1] - DFD_C2 * v[c] + DFD_C3 * v[c + 1] - DFD_C4 * v[c + 2] + DFD_C5 * v[c + 3];
  else return -DFD_C5 * v[c - 3] + DFD_C4 * v[c - 2] - DFD_C3 * v[c - 1] + DFD_C2 * v[c] + DFD_C1 * v[c + 1];
}

// traction vector jac * e_axis . sigma at node q
__device__ __forceinline__ void traction(const float* __restrict__ W, const float* __restrict__ M, long long n,
                                         long long q, int mo, float& t1, float& t2, float& t3) {
  float e0 = __ldg(M + mo * n + q), e1 = __ldg(M + (mo + 1) * n + q), e2 = __ldg(M + (mo + 2) * n + q);
  float jac = __ldg(M + 9 * n + q);
  float txx = __ldg(W + 3 * n + q), tyy = __ldg(W + 4 * n + q), tzz = __ldg(W + 5 * n + q);
  float txy = __ldg(W + 6 * n + q), txz = __ldg(W + 7 * n + q), tyz = __ldg(W + 8 * n + q);
  t1 = (e0 * txx + e1 * txy + e2 * txz) * jac;
  t2 = (e0 * txy + e1 * tyy + e2 * tyz) * jac;
  t3 = (e0 * txz + e1 * tyz + e2 * tzz) * jac;
}

// General node update: every boundary treatment (PML faces, free-surface rows and
// traction image, sponge).  Used for the shell of the domain outside the interior box;
// TOP = false leaves out the free-surface terms (nodes below the top three rows).
template <int FX, int FY, int FZ, bool TOP, int IRK>
__device__ __forceinline__ void volume_point_general(const VolArgs& a, int i, int j, int k) {
  const Dims& d = a.d;
  int i1 = i + 3, j1 = j + 3, k1 = k + 3;
  if (a.united && i1 >= d.i0 - 3 && i1 <= d.i0 + 3 && !a.united[j + k * d.nj]) return;  // band node
  const long long n = d.nxyz;
  const long long q = idx3(d, i1, j1, k1);
  const float* __restrict__ W = a.Win;
  const float* __restrict__ M = a.M;

  float lam = __ldg(M + 10 * n + q), mu = __ldg(M + 11 * n + q);
  float rrho = 1.0f / __ldg(M + 12 * n + q);
  float rb1 = __ldg(a.rBx + i), rb2 = __ldg(a.rBy + j), rb3 = __ldg(a.rBz + k);
  float h[9], p[9], dv[9], D[9];
#pragma unroll
  for (int f = 0; f < 9; f++) p[f] = 0.0f;
  float dxv[3], dyv[3];
  // free-surface rows (only in the TOP variant; the other boxes lie below them)
  const bool fs = TOP && a.freenode && k >= d.nk - 3;
  const bool top = fs && k == d.nk - 1;
  const bool px1 = a.aux[0] && i < d.N, px2 = a.aux[1] && i >= d.ni - d.N;
  const bool py1 = a.aux[2] && j < d.N, py2 = a.aux[3] && j >= d.nj - d.N;
  const bool pz1 = a.aux[4] && k < d.N, pz2 = a.aux[5] && k >= d.nk - d.N;
  float ez0 = __ldg(M + 6 * n + q), ez1 = __ldg(M + 7 * n + q), ez2 = __ldg(M + 8 * n + q);

  // ---- x ----
#pragma unroll
  for (int f = 0; f < 9; f++) dv[f] = d5<FX>(W + f * n, q, d.sx) * a.rDH;
  dxv[0] = dv[0]; dxv[1] = dv[1]; dxv[2] = dv[2];
  axis_terms(dv, __ldg(M + q), __ldg(M + n + q), __ldg(M + 2 * n + q), lam, mu, rrho, D);
#pragma unroll
  for (int f = 0; f < 9; f++) h[f] = D[f] * rb1;
  if (px1 || px2) {
    float dz[3];
    if (top) {
      const float* m = a.mVx2Vz + (j1 + (long long)i1 * d.ny) * 9;
#pragma unroll
      for (int r = 0; r < 3; r++) dz[r] = m[3 * r] * dxv[0] + m[3 * r + 1] * dxv[1] + m[3 * r + 2] * dxv[2];
    }
    const int fc = px1 ? 0 : 1;
    const long long st = pml_fstride(d, fc), qa = pml_index(d, fc, i, j, k);
    pml_face<IRK>(a, fc, qa, st, rb1, __ldg(a.Bx + i), __ldg(a.Dpx + i), __ldg(a.Apx + i), D,
             top ? dz : nullptr, ez0, ez1, ez2, lam, mu, p);
  }
  // ---- y ----
#pragma unroll
  for (int f = 0; f < 9; f++) dv[f] = d5<FY>(W + f * n, q, 1) * a.rDH;
  dyv[0] = dv[0]; dyv[1] = dv[1]; dyv[2] = dv[2];
  axis_terms(dv, __ldg(M + 3 * n + q), __ldg(M + 4 * n + q), __ldg(M + 5 * n + q), lam, mu, rrho, D);
#pragma unroll
  for (int f = 0; f < 9; f++) h[f] += D[f] * rb2;
  if (py1 || py2) {
    float dz[3];
    if (top) {
      const float* m = a.mVy2Vz + (j1 + (long long)i1 * d.ny) * 9;
#pragma unroll
      for (int r = 0; r < 3; r++) dz[r] = m[3 * r] * dyv[0] + m[3 * r + 1] * dyv[1] + m[3 * r + 2] * dyv[2];
    }
    const int fc = py1 ? 2 : 3;
    const long long st = pml_fstride(d, fc), qa = pml_index(d, fc, i, j, k);
    pml_face<IRK>(a, fc, qa, st, rb2, __ldg(a.By + j), __ldg(a.Dpy + j), __ldg(a.Apy + j), D,
             top ? dz : nullptr, ez0, ez1, ez2, lam, mu, p);
  }
  // ---- z ----
#pragma unroll
  for (int f = 0; f < 9; f++) dv[f] = d5<FZ>(W + f * n, q, d.py) * a.rDH;
  float Dz_plain[9];
  axis_terms(dv, ez0, ez1, ez2, lam, mu, rrho, Dz_plain);
#pragma unroll
  for (int f = 0; f < 9; f++) D[f] = Dz_plain[f];
  if (fs) {
    // velocity z-derivatives on the top rows (wave.cu:205-245)
    float dz[3];
    if (k == d.nk - 1) {
      const float* mx = a.mVx2Vz + (j1 + (long long)i1 * d.ny) * 9;
      const float* my = a.mVy2Vz + (j1 + (long long)i1 * d.ny) * 9;
#pragma unroll
      for (int r = 0; r < 3; r++)
        dz[r] = (mx[3 * r] * dxv[0] + mx[3 * r + 1] * dxv[1] + mx[3 * r + 2] * dxv[2]) +
                (my[3 * r] * dyv[0] + my[3 * r + 1] * dyv[1] + my[3 * r + 2] * dyv[2]);
    } else if (k == d.nk - 2) {
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float* v = W + r * n;
        dz[r] = (FZ == 1 ? (__ldg(v + q + d.py) - __ldg(v + q)) : (__ldg(v + q) - __ldg(v + q - d.py))) * a.rDH;
      }
    } else {
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const float* v = W + r * n;
        dz[r] = (FZ == 1 ? (-DFD_C24_1 * __ldg(v + q) + DFD_C24_2 * __ldg(v + q + d.py) - DFD_C24_3 * __ldg(v + q + 2 * d.py))
                         : (DFD_C24_3 * __ldg(v + q - 2 * d.py) - DFD_C24_2 * __ldg(v + q - d.py) + DFD_C24_1 * __ldg(v + q))) *
                a.rDH;
      }
    }
    float dd[9];
    dd[0] = dz[0]; dd[1] = dz[1]; dd[2] = dz[2];
    dd[3] = dv[3]; dd[4] = dv[4]; dd[5] = dv[5]; dd[6] = dv[6]; dd[7] = dv[7]; dd[8] = dv[8];
    float Dm[9];
    axis_terms(dd, ez0, ez1, ez2, lam, mu, rrho, Dm);
#pragma unroll
    for (int f = 3; f < 9; f++) D[f] = Dm[f];
  }
#pragma unroll
  for (int f = 0; f < 9; f++) h[f] += D[f] * rb3;
  if (pz1 || pz2) {
    const int fc = pz1 ? 4 : 5;
    const long long st = pml_fstride(d, fc), qa = pml_index(d, fc, i, j, k);
    pml_face<IRK>(a, fc, qa, st, rb3, __ldg(a.Bz + k), __ldg(a.Dpz + k), __ldg(a.Apz + k), Dz_plain, nullptr,
             ez0, ez1, ez2, lam, mu, p);
  }
  // ---- traction image for the momentum equation on the top three rows (wave.cu:398-487)
  if (fs) {
    int ik = d.nk - 1 - k;
    float rrhojac = rrho / __ldg(M + 9 * n + q);
    float v1[3][7], v2[3][7], v3[3][7];
#pragma unroll
    for (int l = 0; l < 7; l++) {
      traction(W, M, n, q + (l - 3) * d.sx, 0, v1[0][l], v1[1][l], v1[2][l]);
      traction(W, M, n, q + (l - 3), 3, v2[0][l], v2[1][l], v2[2][l]);
      traction(W, M, n, q + (long long)(l - 3) * d.py, 6, v3[0][l], v3[1][l], v3[2][l]);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      v3[c][ik + 3] = 0.0f;
      for (int l = 0; l < 3 - ik; l++) v3[c][6 - l] = -v3[c][l + 2 * ik];
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float tx = d5a<FX>(v1[c], 3) * a.rDH, ty = d5a<FY>(v2[c], 3) * a.rDH, tz = d5a<FZ>(v3[c], 3) * a.rDH;
      h[c] = (tx * rb1 + ty * rb2 + tz * rb3) * rrhojac;
    }
  }
  // ---- RK4 registers and Cerjan sponge
  float damp = 1.0f;
  if (a.dampx) damp = fminf(fminf(__ldg(a.dampx + i1), __ldg(a.dampy + j1)), __ldg(a.dampz + k1));
  rk_store<IRK>(a, q, h, p, damp);
}


// Shell kernels: the general update on up to eight boxes (PML slabs, free-surface rows)
// that surround the interior box; one 1-D grid of 128-thread blocks is split over the
// boxes below the free-surface rows and a second over the rows themselves.  At most 170
// registers, three blocks per SM: the PML path needs about 160; the traction image of the
// free-surface rows would take about 230, but the third resident block is worth more than
// the few values it spills (measured against two and four blocks per SM).  A box at least 32 nodes wide in y and 4 in z is tiled (32 y, 4 z) per block; a
// thinner box (the y slabs of the PML, the free-surface rows) is flattened over (y, z)
// with y fastest, so that no thread idles and the y-face PML state (y fastest over N
// nodes, then z) is read contiguously.
constexpr int SHELL_THREADS = 128;

// block blk of the shell grid of one scenario: of the boxes below the free-surface rows
// (TOP = false, blk counted from box 0) or of the free-surface boxes (TOP, blk counted
// from box ntop); IRK: the stage (compiled per stage for the free-surface rows), or -1
template <int FX, int FY, int FZ, bool TOP, int IRK>
__device__ __forceinline__ void volume_shell_body(const VolArgs& a, const Boxes& bx, int blk) {
  int b = TOP ? bx.ntop : 0;
  const int bend = TOP ? bx.n : bx.ntop;
  if (TOP) blk += bx.start[bx.ntop];
  while (b + 1 < bend && blk >= bx.start[b + 1]) b++;
  int loc = blk - bx.start[b];
  int ni = bx.hi[b][0] - bx.lo[b][0], nj = bx.hi[b][1] - bx.lo[b][1], nk = bx.hi[b][2] - bx.lo[b][2];
  int i, j, k;
  if (bx.thin[b]) {
    int gyz = (nj * nk + SHELL_THREADS - 1) / SHELL_THREADS;
    int t = (loc % gyz) * SHELL_THREADS + threadIdx.x;
    i = loc / gyz;
    j = t % nj;
    k = t / nj;
    if (k >= nk) return;
  } else {
    int gj = (nj + 31) / 32, gk = (nk + 3) / 4;
    int bj = loc % gj, bk = (loc / gj) % gk, bi = loc / (gj * gk);
    j = bj * 32 + (threadIdx.x & 31);
    k = bk * 4 + (threadIdx.x >> 5);
    i = bi;
    if (i >= ni || j >= nj || k >= nk) return;
  }
  volume_point_general<FX, FY, FZ, TOP, IRK>(a, bx.lo[b][0] + i, bx.lo[b][1] + j, bx.lo[b][2] + k);
}
template <int FX, int FY, int FZ, bool TOP, int IRK>
__global__ void __launch_bounds__(SHELL_THREADS, 3)
    volume_shell_kernel(const __grid_constant__ VolArgs a, const __grid_constant__ Boxes bx) {
  volume_shell_body<FX, FY, FZ, TOP, IRK>(a, bx, blockIdx.x);
}
// all scenarios of an ensemble in one launch: scenario s owns blocks [start[s], start[s+1])
template <int FX, int FY, int FZ, bool TOP, int IRK>
__global__ void __launch_bounds__(SHELL_THREADS, 3)
    volume_shell_batch(const VolArgs* __restrict__ tab, const Boxes* __restrict__ boxes,
                       const int* __restrict__ start, int n) {
  __shared__ __align__(16) unsigned char raw_a[sizeof(VolArgs)];
  __shared__ __align__(16) unsigned char raw_b[sizeof(Boxes)];
  VolArgs* sa = reinterpret_cast<VolArgs*>(raw_a);
  Boxes* sb = reinterpret_cast<Boxes*>(raw_b);
  int loc;
  const int sc = scenario_of(start, n, blockIdx.x, &loc);
  stage_args(sa, tab + sc);
  stage_args(sb, boxes + sc);
  __syncthreads();
  volume_shell_body<FX, FY, FZ, TOP, IRK>(*sa, *sb, loc);
}

// Interior kernel: no PML (beta = 1, no auxiliary state), no free-surface rows.  Each
// derivative is scattered into the nine right-hand sides as soon as it is formed, which
// keeps the register count low enough for three resident blocks per SM; each thread
// walks a chunk of x so that the x-stencil halo is reused from L1.
template <int FX, int FY, int FZ>
__device__ __forceinline__ void interior_point(const VolArgs& a, long long q, float damp) {
  const long long n = a.d.nxyz;
  const float* __restrict__ W = a.Win;
  const float* __restrict__ M = a.M;
  const float r = a.rDH;
  float lam = __ldg(M + 10 * n + q), mu = __ldg(M + 11 * n + q);
  float rrho = 1.0f / __ldg(M + 12 * n + q);
  float l2m = lam + 2.0f * mu;
  float h0 = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f, h4 = 0.f, h5 = 0.f, h6 = 0.f, h7 = 0.f, h8 = 0.f;
#define DFD_AXIS(F, S, MO)                                                                         \
  {                                                                                                \
    float e0 = __ldg(M + (MO) * n + q), e1 = __ldg(M + ((MO) + 1) * n + q), e2 = __ldg(M + ((MO) + 2) * n + q); \
    float dv;                                                                                      \
    dv = d5<F>(W, q, S) * r;                                                                       \
    h3 += dv * e0 * l2m; h4 += dv * e0 * lam; h5 += dv * e0 * lam; h6 += dv * e1 * mu; h7 += dv * e2 * mu; \
    dv = d5<F>(W + n, q, S) * r;                                                                   \
    h3 += dv * e1 * lam; h4 += dv * e1 * l2m; h5 += dv * e1 * lam; h6 += dv * e0 * mu; h8 += dv * e2 * mu; \
    dv = d5<F>(W + 2 * n, q, S) * r;                                                               \
    h3 += dv * e2 * lam; h4 += dv * e2 * lam; h5 += dv * e2 * l2m; h7 += dv * e0 * mu; h8 += dv * e1 * mu; \
    float er0 = e0 * rrho, er1 = e1 * rrho, er2 = e2 * rrho;                                       \
    dv = d5<F>(W + 3 * n, q, S) * r; h0 += dv * er0;                                               \
    dv = d5<F>(W + 4 * n, q, S) * r; h1 += dv * er1;                                               \
    dv = d5<F>(W + 5 * n, q, S) * r; h2 += dv * er2;                                               \
    dv = d5<F>(W + 6 * n, q, S) * r; h0 += dv * er1; h1 += dv * er0;                               \
    dv = d5<F>(W + 7 * n, q, S) * r; h0 += dv * er2; h2 += dv * er0;                               \
    dv = d5<F>(W + 8 * n, q, S) * r; h1 += dv * er2; h2 += dv * er1;                               \
  }
  DFD_AXIS(FX, a.d.sx, 0)
  DFD_AXIS(FY, 1, 3)
  DFD_AXIS(FZ, a.d.py, 6)
#undef DFD_AXIS
  const float hv[9] = {h0, h1, h2, h3, h4, h5, h6, h7, h8};
  rk_store<-1>(a, q, hv, nullptr, damp);
}

template <int FX, int FY, int FZ>
__global__ void __launch_bounds__(256, 3) volume_interior_kernel(VolArgs a, int3 lo, int3 hi, int chunk) {
  const Dims& d = a.d;
  int j = lo.y + blockIdx.x * blockDim.x + threadIdx.x;
  int k = lo.z + blockIdx.y * blockDim.y + threadIdx.y;
  if (j >= hi.y || k >= hi.z) return;
  int ib = lo.x + blockIdx.z * chunk, ie = min(ib + chunk, hi.x);
  bool band = a.united && !a.united[j + k * d.nj];
  float dyz = 1.0f;
  if (a.dampx) dyz = fminf(__ldg(a.dampy + j + 3), __ldg(a.dampz + k + 3));
  long long q = idx3(d, ib + 3, j + 3, k + 3);
  for (int i = ib; i < ie; i++, q += d.sx) {
    if (band && i + 3 >= d.i0 - 3 && i + 3 <= d.i0 + 3) continue;
    float damp = a.dampx ? fminf(__ldg(a.dampx + i + 3), dyz) : 1.0f;
    interior_point<FX, FY, FZ>(a, q, damp);
  }
}

// Volume work of one stage: which box the tiled (or plain) interior kernel takes, the
// units of the tiled PML kernel and the boxes of the general kernel.
VolPlan plan_volume(const VolArgs& a, const TileCtx* tc) {
  const Dims& d = a.d;
  VolPlan pl;
  pl.tiled = pl.plain = false;
  pl.nodes = 0;
  pl.pgrid = 0;
  memset(&pl.ps, 0, sizeof pl.ps);
  Boxes& bx = pl.bx;
  bx.n = bx.ntop = 0;
  auto add = [&](int i0, int i1, int j0, int j1, int k0, int k1) {
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) return;
    bx.lo[bx.n][0] = i0; bx.lo[bx.n][1] = j0; bx.lo[bx.n][2] = k0;
    bx.hi[bx.n][0] = i1; bx.hi[bx.n][1] = j1; bx.hi[bx.n][2] = k1;
    bx.n++;
  };
  // interior box: outside every PML slab, below the free-surface rows
  int nx0 = a.aux[0] ? d.N : 0, nx1 = a.aux[1] ? d.N : 0;
  int ny0 = a.aux[2] ? d.N : 0, ny1 = a.aux[3] ? d.N : 0;
  int nz0 = a.aux[4] ? d.N : 0, nz1 = a.aux[5] ? d.N : (a.freenode ? 3 : 0);
  int3 lo = make_int3(nx0, ny0, nz0), hi = make_int3(d.ni - nx1, d.nj - ny1, d.nk - nz1);
  const int ktop = a.freenode ? d.nk - 3 : d.nk;
  bool done = false;
  if (tc && tc->ok) {
    // the interior kernel takes the box between the slabs (its y start a multiple of 16,
    // where the PML kernel's y1 strips end; its y end a multiple of 4, where the y2
    // strips start); the PML kernel every other node below the free-surface rows
    int ya = a.aux[2] ? (d.N + STRIP - 1) / STRIP * STRIP : 0;
    int yb = a.aux[3] ? (d.nj - d.N) / 4 * 4 : d.nj;
    if (a.aux[3] && yb > ya) {
      // A column of the interior kernel's 32-wide tiles and a column of the PML kernel's
      // 16-wide strips cost about the same (half the nodes at about twice the cost per
      // node), and a partial column costs nearly a full one.  Of the y ends up to 28
      // columns earlier, take the one with the fewest columns of both (ties: the latest):
      // with NY = 600 and PML 20 that is 576 (17 whole tiles, two strips), not 580 (an
      // 18th tile 4 columns wide, the same two strips).
      auto cols = [&](int y) { return (y - ya + TILE_J - 1) / TILE_J + (d.nj - y + STRIP - 1) / STRIP; };
      int best = yb;
      for (int y = yb - 4; y >= yb - 28 && y > ya; y -= 4)
        if (cols(y) < cols(best)) best = y;
      yb = best;
    }
    int za = a.aux[4] ? d.N : 0;
    int zb = a.aux[5] ? d.nk - d.N : ktop;
    if (yb <= ya) ya = yb = 0;     // no interior column: strips over every column
    // whole 8-row tiles in z: the rows left over go to the PML kernel's z tiles (whose
    // second tile row over a 12-row slab has room for them), not to a nearly empty row of
    // interior tiles
    const int zr = (zb - za) % TILE_K;
    if (zb - za >= TILE_K && zr) {
      if (a.aux[4]) za += zr;
      else zb -= zr;
    }
    // ... unless they then cost the z1 slab a row of z tiles of its own: a row of the PML
    // kernel's tiles costs about two of the interior kernel's, so with PML 20 and 297 rows
    // (25 rows: a fourth z-tile row holding one) the slab keeps its 20 rows in three tile
    // rows and the interior box ends in a partial tile row
    if (a.aux[4] && zb - za >= TILE_K) {
      auto rows = [&](int z) { return 2 * ((z + TILE_K - 1) / TILE_K) + (zb - z + TILE_K - 1) / TILE_K; };
      int best = za;
      for (int z = d.N; z < za; z++)
        if (rows(z) < rows(best)) best = z;
      za = best;
    }
    if (zb <= za || zb - za < TILE_K) za = zb = ktop;  // no interior row: z tiles over every row
    int grid = 0;
    TileSched ps = pml_plan(a, ya, yb, za, zb, ktop, tc->nsm, &grid);
    const int3 rlo = make_int3(lo.x, ya, za), rhi = make_int3(hi.x, yb, zb);
    const bool inner = rhi.x > rlo.x && rhi.y > rlo.y && rhi.z > rlo.z;
    if (ps.nunits >= 0 && (!inner || tile_feasible(tc, a, rlo, rhi))) {
      done = true;
      pl.ps = ps;
      pl.pgrid = grid;
      if (inner) {
        pl.tiled = true;
        pl.lo = rlo;
        pl.hi = rhi;
      }
      add(0, d.ni, 0, d.nj, ktop, d.nk);  // the free-surface rows
    }
  }
  if (!done) {
    // the plain interior kernel on the interior box, the general kernel on the slabs
    // around it, then on the free-surface rows
    const bool some = hi.x > lo.x && hi.y > lo.y && hi.z > lo.z;
    if (some) {
      pl.plain = true;
      pl.lo = lo;
      pl.hi = hi;
    } else {
      lo = hi = make_int3(0, 0, 0);
    }
    add(0, lo.x, 0, d.nj, 0, ktop);
    add(hi.x, d.ni, 0, d.nj, 0, ktop);
    add(lo.x, hi.x, 0, lo.y, 0, ktop);
    add(lo.x, hi.x, hi.y, d.nj, 0, ktop);
    add(lo.x, hi.x, lo.y, hi.y, 0, lo.z);
    add(lo.x, hi.x, lo.y, hi.y, hi.z, ktop);
    bx.ntop = bx.n;
    add(0, d.ni, 0, d.nj, ktop, d.nk);
  }
  if (pl.tiled || pl.plain) pl.nodes = (long long)(pl.hi.x - pl.lo.x) * (pl.hi.y - pl.lo.y) * (pl.hi.z - pl.lo.z);
  int tot = 0;
  for (int b = 0; b < bx.n; b++) {
    bx.start[b] = tot;
    int ni = bx.hi[b][0] - bx.lo[b][0], nj = bx.hi[b][1] - bx.lo[b][1], nk = bx.hi[b][2] - bx.lo[b][2];
    bx.thin[b] = nj < 32 || nk < 4;
    tot += bx.thin[b] ? ((nj * nk + SHELL_THREADS - 1) / SHELL_THREADS) * ni : ((nj + 31) / 32) * ((nk + 3) / 4) * ni;
  }
  bx.start[bx.n] = tot;
  pl.shell_blocks = tot;
  return pl;
}

template <int FX, int FY, int FZ>
static long long launch_flags(const VolArgs& a, cudaStream_t s, cudaStream_t s_shell, const TileCtx* tc, int bin,
                              cudaEvent_t* kb, cudaEvent_t* ke, VolPlan* out, cudaEvent_t* fork) {
  const VolPlan pl = plan_volume(a, tc);
  if (out) *out = pl;
  if (kb) cudaEventRecord(*kb, s);
  if (pl.tiled) {
    launch_tile(tc, a, FX, FY, FZ, bin, pl.lo, pl.hi, s);
  } else if (pl.plain) {
    const int chunk = 8;
    dim3 block(32, 8, 1);
    dim3 grid((pl.hi.y - pl.lo.y + 31) / 32, (pl.hi.z - pl.lo.z + 7) / 8, (pl.hi.x - pl.lo.x + chunk - 1) / chunk);
    volume_interior_kernel<FX, FY, FZ><<<grid, block, 0, s>>>(a, pl.lo, pl.hi, chunk);
  }
  if (ke) cudaEventRecord(*ke, s);
  // directly behind the interior kernel unless timing events separate them
  if (pl.ps.nunits > 0) launch_pml(tc, a, FX, FY, FZ, bin, pl.ps, pl.pgrid, pl.tiled && !ke, s);
  if (fork && s_shell != s) {
    // the general kernel on s_shell once the tiled kernels are done
    cudaEventRecord(*fork, s);
    cudaStreamWaitEvent(s_shell, *fork, 0);
  }
  const int below = pl.bx.start[pl.bx.ntop], above = pl.bx.start[pl.bx.n] - below;
  if (below > 0) volume_shell_kernel<FX, FY, FZ, false, -1><<<below, SHELL_THREADS, 0, s_shell>>>(a, pl.bx);
  if (above > 0) {
#define DFD_L(K) volume_shell_kernel<FX, FY, FZ, true, K><<<above, SHELL_THREADS, 0, s_shell>>>(a, pl.bx)
    DFD_BY_STAGE(a.irk, DFD_L);
#undef DFD_L
  }
  return pl.nodes;
}

template <int FX, int FY, int FZ>
static void shell_batch_t(const VolArgs* tab, const Boxes* boxes, const int* start, int n, int blocks, bool top,
                          int irk, cudaStream_t s) {
  if (top) {
#define DFD_L(K) volume_shell_batch<FX, FY, FZ, true, K><<<blocks, SHELL_THREADS, 0, s>>>(tab, boxes, start, n)
    DFD_BY_STAGE(irk, DFD_L);
#undef DFD_L
  } else {
    volume_shell_batch<FX, FY, FZ, false, -1><<<blocks, SHELL_THREADS, 0, s>>>(tab, boxes, start, n);
  }
}
void launch_shell_batch(const VolArgs* tab, const Boxes* boxes, const int* start, int n, int blocks, int FX, int FY,
                        int FZ, bool top, int irk, cudaStream_t s) {
  if (blocks <= 0) return;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: shell_batch_t<-1, -1, -1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 1: shell_batch_t<-1, -1, 1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 2: shell_batch_t<-1, 1, -1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 3: shell_batch_t<-1, 1, 1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 4: shell_batch_t<1, -1, -1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 5: shell_batch_t<1, -1, 1>(tab, boxes, start, n, blocks, top, irk, s); break;
    case 6: shell_batch_t<1, 1, -1>(tab, boxes, start, n, blocks, top, irk, s); break;
    default: shell_batch_t<1, 1, 1>(tab, boxes, start, n, blocks, top, irk, s); break;
  }
}

// Launches the volume kernels of one stage; kb/ke (optional) are recorded on s right
// before and after the interior (tiled) kernel; with fork (and s_shell != s) the general
// kernel runs on s_shell after the tiled kernels, else on s_shell right away.  Returns the
// nodes of the box the interior kernel covers.
long long launch_volume_stage(const VolArgs& a, int FX, int FY, int FZ, cudaStream_t s, cudaStream_t s_shell,
                              const TileCtx* tc, int bin, cudaEvent_t* kb, cudaEvent_t* ke, VolPlan* out,
                              cudaEvent_t* fork) {
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: return launch_flags<-1, -1, -1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 1: return launch_flags<-1, -1, 1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 2: return launch_flags<-1, 1, -1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 3: return launch_flags<-1, 1, 1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 4: return launch_flags<1, -1, -1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 5: return launch_flags<1, -1, 1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    case 6: return launch_flags<1, 1, -1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
    default: return launch_flags<1, 1, 1>(a, s, s_shell, tc, bin, kb, ke, out, fork);
  }
}

}  // namespace dfd
