// Volume stage staged through shared memory by TMA (interior box, and optionally the PML
// slabs too).
//
// The box is cut into tiles of 32 (y) x 8 (z) nodes; a CTA owns one tile column and
// marches along x over a chunk of planes.  Per plane it needs
//   - the stencil input (9 fields) of the planes x-1..x+3 (forward x operator) or
//     x-3..x+1 (backward), with a y/z halo on the current plane: one 4-D TMA box
//     (40 y, 12 z, 1 x, 9 fields) per plane, held in a ring of NS plane slots;
//   - the pointwise streams of the node: 12 metric/media fields, and the RK registers
//     W0 (stages 1, 2) and T (stages 1..3): TMA boxes (32, 8, 1, n) in a ring of NP slots.
// A dedicated warp issues the copies ahead of the eight computing warps (full/empty
// mbarrier pairs per slot, no block-wide barrier in the loop), so HBM traffic stays in
// flight while the stencils are evaluated from shared memory with immediate offsets.
// Nodes inside a PML slab take the general path (per-axis 1/beta and the ADE auxiliary
// state, read and written in global memory); the others the lean interior path.  Outputs
// (Wout, T) are written straight from registers.
//
// The kernel is persistent: one CTA per SM takes units (tile column x chunk) from a global
// counter, and its copy stream runs across unit boundaries, so the next unit's planes
// arrive while the current one finishes.
//
// The right-hand side follows the reference's wave.cu:8-204, pmlx.cu / pmly.cu / pmlz.cu
// and rk4.cu:20-33, as the general kernel in dfd_volume.cu does.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "dfd_stencil.cuh"

namespace dfd {

namespace {
constexpr int TJ = 32, TK = 8, NTHR = TJ * TK;
constexpr int HW = TJ + 8;           // halo box width (y): 4 nodes each side (16-byte aligned)
constexpr int HH = TK + 4;           // halo box height (z): 1 + 3 rows, side set by the z operator
constexpr int HBOX = HW * HH;        // floats per field of a halo box
constexpr int HSLOT = 9 * HBOX;      // floats per stencil plane slot
constexpr int PB = TJ * TK;          // floats per field of a pointwise box
constexpr int PSLOT = 18 * PB;       // RK registers W0 9 + T 9
constexpr int QSLOT = 12 * PB;       // metric / media planes of a unit: U V ety etz zty ztz, 2 x (lam mu rho)
constexpr int NS = 8, NP = 3, NQ = 2;  // ring depths (stencil planes, RK registers, unit planes)
constexpr size_t SMEM_BYTES = (size_t)(NS * HSLOT + NP * PSLOT + NQ * QSLOT) * 4 + 2 * (NS + NP + NQ) * 8 + NQ * 4;
constexpr long long WAIT_LIMIT = 1LL << 22;  // polls of one mbarrier before giving up
static_assert(SMEM_BYTES <= 232448, "tile ring exceeds the shared memory of one CTA");
static_assert((HSLOT * 4) % 128 == 0 && (PSLOT * 4) % 128 == 0 && (QSLOT * 4) % 128 == 0 && (PB * 4) % 128 == 0,
              "slot alignment");
}  // namespace

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the completion of phase `parity`; false if it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
  for (long long n = 0; n < WAIT_LIMIT; n++)
    if (mbar_try(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_load4(float* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(b))
      : "memory");
}

__device__ __forceinline__ void tma_load3(float* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(b))
      : "memory");
}

// one-sided 5-point operators on values (v0..v4 = the five stencil points in order)
template <int F>
__device__ __forceinline__ float d5v(float v0, float v1, float v2, float v3, float v4) {
  if (F == 1) return -DFD_C1 * v0 - DFD_C2 * v1 + DFD_C3 * v2 - DFD_C4 * v3 + DFD_C5 * v4;
  else return -DFD_C5 * v0 + DFD_C4 * v1 - DFD_C3 * v2 + DFD_C2 * v3 + DFD_C1 * v4;
}
// on a shared-memory line through p with stride S (forward: p-S..p+3S, backward: p-3S..p+S)
template <int F, int S>
__device__ __forceinline__ float d5s(const float* p) {
  if (F == 1) return d5v<1>(p[-S], p[0], p[S], p[2 * S], p[3 * S]);
  else return d5v<-1>(p[-3 * S], p[-2 * S], p[-S], p[0], p[S]);
}


constexpr int NCW = 2 * NTHR / 32;  // computing warps: two per 32-node row of the tile
constexpr int NTOT = NCW * 32 + 32;  // plus one copy-issuing warp

// slot / phase-parity cursor over a ring of N mbarrier-guarded slots
struct Ring {
  int slot = 0, phase = 0;
  template <int N>
  __device__ __forceinline__ void next() {
    if (++slot == N) { slot = 0; phase ^= 1; }
  }
};

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

// RK4 register update of fields F0..F1-1 of node q with right-hand side hv, then the
// sponge factor (rk4.cu:20-33, cerjan.cu:166-200): step-start values from the stencil
// input at stage 0, the RK registers from the pointwise slot P at stages 1..3.
template <int F0, int F1>
__device__ __forceinline__ void rk_tile_store(const VolArgs& a, long long n, long long q, const float* cur,
                                              const float* P, const float* hv, float damp) {
#pragma unroll
  for (int f = F0; f < F1; f++) {
    const long long x = f * n + q;
    float w;
    if (a.irk == 0) {
      const float w0 = cur[f * HBOX];
      a.T[x] = fmaf(a.rkb, hv[f], w0);
      w = fmaf(a.rka, hv[f], w0);
    } else if (a.irk < 3) {
      a.T[x] = fmaf(a.rkb, hv[f], P[(9 + f) * PB]);
      w = fmaf(a.rka, hv[f], P[f * PB]);
    } else {
      w = fmaf(a.rkb, hv[f], P[(9 + f) * PB]);
    }
    a.Wout[x] = w * damp;
  }
}

// Metric and media of a node of the tiled box: x row (xi), y row (eta), z row (zeta) and
// the elastic constants (the separable factors of dfd_setup.cu's plane_metric_kernel; the
// x components of eta and zeta are exactly zero there and in the stored metric).
struct NodeMetric {
  float ex0, ex1, ex2, ey1, ey2, ez1, ez2, lam, mu, rrho;
};

// Right-hand side of a node inside at least one PML slab: every axis with its 1/beta and
// the ADE auxiliary update of the faces the node lies in (reference wave.cu:8-204 with
// pmlx.cu / pmly.cu / pmlz.cu).  xv[m] are the five x-stencil planes, cur the plane x.
template <int FX, int FY, int FZ>
__device__ __forceinline__ void tile_pml_point(const VolArgs& a, const float* const* xv, const float* cur,
                                               const NodeMetric& g, int i, int j, int k, float* hv) {
  const Dims& d = a.d;
  const float r = a.rDH;
  const float rb1 = __ldg(a.rBx + i), rb2 = __ldg(a.rBy + j), rb3 = __ldg(a.rBz + k);
  // the x-face ADE state first, so that its latency overlaps the stencil evaluation
  const bool px1 = a.aux[0] && i < d.N, px2 = a.aux[1] && i >= d.ni - d.N;
  const long long stx = (long long)d.N * d.nj * d.nk;
  const long long qax = j + (long long)k * d.nj + (long long)(px1 ? i : i - (d.ni - d.N)) * d.nj * d.nk;
  PmlState psx;
  if (px1 || px2) pml_load(a, px1 ? 0 : 1, qax, stx, psx);
  float p[9], D[9], dv[9];
#pragma unroll
  for (int f = 0; f < 9; f++) p[f] = 0.0f;
  // x
#pragma unroll
  for (int f = 0; f < 9; f++) {
    const int o = f * HBOX;
    dv[f] = d5v<FX>(xv[0][o], xv[1][o], xv[2][o], xv[3][o], xv[4][o]) * r;
  }
  axis_terms(dv, g.ex0, g.ex1, g.ex2, g.lam, g.mu, g.rrho, D);
#pragma unroll
  for (int f = 0; f < 9; f++) hv[f] = D[f] * rb1;
  if (px1 || px2)
    pml_update(a, px1 ? 0 : 1, qax, stx, rb1, __ldg(a.Bx + i), __ldg(a.Dpx + i), __ldg(a.Apx + i), D, nullptr, 0.f,
               0.f, 0.f, g.lam, g.mu, psx, p);
  // y
#pragma unroll
  for (int f = 0; f < 9; f++) dv[f] = d5s<FY, 1>(cur + f * HBOX) * r;
  axis_terms(dv, 0.0f, g.ey1, g.ey2, g.lam, g.mu, g.rrho, D);
#pragma unroll
  for (int f = 0; f < 9; f++) hv[f] += D[f] * rb2;
  const bool py1 = a.aux[2] && j < d.N, py2 = a.aux[3] && j >= d.nj - d.N;
  if (py1 || py2) {
    long long st = (long long)d.N * d.nk * d.ni;
    int ja = py1 ? j : j - (d.nj - d.N);
    long long qa = ja + (long long)k * d.N + (long long)i * d.N * d.nk;
    pml_face(a, py1 ? 2 : 3, qa, st, rb2, __ldg(a.By + j), __ldg(a.Dpy + j), __ldg(a.Apy + j), D, nullptr, 0.f,
             0.f, 0.f, g.lam, g.mu, p);
  }
  // z
#pragma unroll
  for (int f = 0; f < 9; f++) dv[f] = d5s<FZ, HW>(cur + f * HBOX) * r;
  axis_terms(dv, 0.0f, g.ez1, g.ez2, g.lam, g.mu, g.rrho, D);
#pragma unroll
  for (int f = 0; f < 9; f++) hv[f] += D[f] * rb3;
  const bool pz1 = a.aux[4] && k < d.N, pz2 = a.aux[5] && k >= d.nk - d.N;
  if (pz1 || pz2) {
    long long st = (long long)d.N * d.ni * d.nj;
    int ka = pz1 ? k : k - (d.nk - d.N);
    long long qa = j + (long long)ka * d.nj + (long long)i * d.nj * d.N;
    pml_face(a, pz1 ? 4 : 5, qa, st, rb3, __ldg(a.Bz + k), __ldg(a.Dpz + k), __ldg(a.Apz + k), D, nullptr, 0.f,
             0.f, 0.f, g.lam, g.mu, p);
  }
#pragma unroll
  for (int f = 0; f < 9; f++) hv[f] += p[f];
}

// Warp NCW issues the copies; warps 0..NCW-1 compute one node each per plane.  Each ring
// slot has a "full" barrier (completed by the copy's transaction bytes) and an "empty"
// barrier (one arrival per computing warp once it has finished reading the slot).  Three
// rings: stencil planes (NS), RK registers of the step (NP; none at stage 0, whose
// step-start values are the stencil input), metric/media planes of the unit (NQ).  At
// most 96 registers: the 17 warps are spread over the SM's four 16 K-register partitions,
// five warps on one of them.
// first scenario of a batched launch whose units include the global unit u
__device__ __forceinline__ int tile_scenario(const TileScen* tab, int n, int u) {
  int lo = 0, hi = n;  // tab[lo].unit0 <= u < tab[hi].unit0
  while (hi - lo > 1) {
    int m = (lo + hi) / 2;
    if (tab[m].unit0 <= u) lo = m; else hi = m;
  }
  return lo;
}

// BATCH: the units of the nscen scenarios of tab (an ensemble) in one launch; the
// parameters mp0, a0, sc0 then describe scenario 0 and give the stage's common values.
template <int FX, int FY, int FZ, bool PMLP, bool BATCH>
__global__ void __maxnreg__(96)
    volume_tile_kernel(const __grid_constant__ TileMaps mp0, const __grid_constant__ VolArgs a0,
                       const __grid_constant__ TileSched sc0, const TileScen* __restrict__ tab, int nscen,
                       int nunits, int* err, int* sched) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  float* win = reinterpret_cast<float*>(smraw);
  float* pw = win + NS * HSLOT;
  float* qs = pw + NP * PSLOT;
  uint64_t* full_w = reinterpret_cast<uint64_t*>(qs + NQ * QSLOT);
  uint64_t* empty_w = full_w + NS;
  uint64_t* full_p = empty_w + NS;
  uint64_t* empty_p = full_p + NP;
  uint64_t* full_q = empty_p + NP;
  uint64_t* empty_q = full_q + NQ;
  int* qunit = reinterpret_cast<int*>(empty_q + NQ);  // unit of each plane slot (-1: no more)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int XLO = FX == 1 ? -1 : -3;  // first stencil plane relative to x
  constexpr int RZ = FZ == 1 ? 1 : 3;     // row of the tile's first z node inside the halo box
  const int irk = a0.irk;
  const bool needW0 = irk == 1 || irk == 2, needT = irk >= 1, usep = needW0 || needT;
  const int G = gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; s++) { mbar_init(full_w + s, 1); mbar_init(empty_w + s, NCW); }
    for (int s = 0; s < NP; s++) { mbar_init(full_p + s, 1); mbar_init(empty_p + s, NCW); }
    for (int s = 0; s < NQ; s++) { mbar_init(full_q + s, 1); mbar_init(empty_q + s, NCW); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_async_shared();
  }
  __syncthreads();

  if (warp == NCW) {
    // ---------------- copy-issuing warp (one lane)
    if (lane != 0) return;
    const unsigned ptx = ((needW0 ? 9 : 0) + (needT ? 9 : 0)) * PB * 4;
    Ring wr, pr, qr;
    int wcount = 0, pcount = 0, qcount = 0;
    bool ok = true;
    // units are taken from a global counter, so that CTAs that start late (their SM busy
    // with a concurrent kernel) simply take fewer
    while (ok) {
      const int u = atomicAdd(sched, 1);
      if (qcount >= NQ && !(ok = mbar_wait(empty_q + qr.slot, qr.phase ^ 1))) break;
      if (u >= nunits) {
        qunit[qr.slot] = -1;  // tell the computing warps that there is no further unit
        mbar_arrive(full_q + qr.slot);
        break;
      }
      const int scn = BATCH ? tile_scenario(tab, nscen, u) : 0;
      const TileMaps& mp = BATCH ? tab[scn].mp : mp0;
      const VolArgs& a = BATCH ? tab[scn].a : a0;
      const TileSched& sc = BATCH ? tab[scn].sc : sc0;
      const Dims& d = a.d;
      const int lu = BATCH ? u - tab[scn].unit0 : u;
      const int ntile = sc.ntj * sc.ntk;
      const int tc = lu / ntile, ru = lu % ntile;
      const int ib = sc.lo_x + tc * sc.ci, ie = min(ib + sc.ci, sc.hi_x);
      const int j0 = sc.lo_y + (ru % sc.ntj) * TJ, k0 = sc.lo_z + (ru / sc.ntj) * TK;
      const int cw0 = j0 + 3 + d.oy - 4, cw1 = k0 + 3 - RZ, cp0 = j0 + 3 + d.oy, cp1 = k0 + 3;
      const int nst = ie - ib;
      // metric / media planes of the unit, with the unit's index
      qunit[qr.slot] = u;
      mbar_expect_tx(full_q + qr.slot, QSLOT * 4);
      tma_load3(qs + qr.slot * QSLOT, &mp.plane, cp0, cp1, 0, full_q + qr.slot);
      qr.next<NQ>();
      qcount++;
      for (int m = 0; m < nst + 4 && ok; m++) {
        // stencil plane m of the unit (first needed by step m - 4)
        if (wcount >= NS && !(ok = mbar_wait(empty_w + wr.slot, wr.phase ^ 1))) break;
        mbar_expect_tx(full_w + wr.slot, HSLOT * 4);
        tma_load4(win + wr.slot * HSLOT, &mp.win, cw0, cw1, ib + XLO + m + 3, 0, full_w + wr.slot);
        wr.next<NS>();
        wcount++;
        if (m < 4 || !usep) continue;
        // RK registers of step m - 4
        if (pcount >= NP && !(ok = mbar_wait(empty_p + pr.slot, pr.phase ^ 1))) break;
        uint64_t* b = full_p + pr.slot;
        float* dst = pw + pr.slot * PSLOT;
        const int cp2 = ib + (m - 4) + 3;
        mbar_expect_tx(b, ptx);
        if (needW0) tma_load4(dst, &mp.w0, cp0, cp1, cp2, 0, b);
        if (needT) tma_load4(dst + 9 * PB, &mp.t, cp0, cp1, cp2, 0, b);
        pr.next<NP>();
        pcount++;
      }
    }
    if (!ok) {
      // a slot was not released in time: flag it and let the copies in flight land
      atomicExch(err, 1);
      for (int c = max(0, wcount - NS); c < wcount; c++) mbar_wait(full_w + c % NS, (c / NS) & 1);
      for (int c = max(0, pcount - NP); c < pcount; c++) mbar_wait(full_p + c % NP, (c / NP) & 1);
      for (int c = max(0, qcount - NQ); c < qcount; c++) mbar_wait(full_q + c % NQ, (c / NQ) & 1);
    }
    // the last CTA to stop taking units resets the counter for the next launch
    __threadfence();
    if (atomicAdd(sched + 1, 1) == G - 1) {
      atomicExch(sched, 0);
      atomicExch(sched + 1, 0);
    }
    return;
  }

  // ---------------- computing warps: warps w and w + NCW/2 share the row of nodes
  // (y = lane, z = w): the first computes the momentum equation (velocity fields), the
  // second the constitutive law (stress fields)
  const int role = warp >= NCW / 2 ? 1 : 0;
  const int ty = warp - role * (NCW / 2);
  const int hc = (ty + RZ) * HW + lane + 4;  // node inside a halo field box
  const int pc = ty * TJ + lane;             // node inside a pointwise field box
  Ring wr, pr, qr;  // next stencil plane to wait for; RK-register slot of the step; unit planes
  int sb = 0;       // slot of the step's first stencil plane
  for (;;) {
    if (!__all_sync(0xffffffffu, mbar_wait(full_q + qr.slot, qr.phase))) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    const int u = qunit[qr.slot];
    if (u < 0) break;
    const int scn = BATCH ? tile_scenario(tab, nscen, u) : 0;
    const VolArgs& a = BATCH ? tab[scn].a : a0;
    const TileSched& sc = BATCH ? tab[scn].sc : sc0;
    const Dims& d = a.d;
    const long long n = d.nxyz;
    const float r = a.rDH;
    const int lu = BATCH ? u - tab[scn].unit0 : u;
    const int ntile = sc.ntj * sc.ntk;
    const int tc = lu / ntile, ru = lu % ntile;
    const int ib = sc.lo_x + tc * sc.ci, ie = min(ib + sc.ci, sc.hi_x);
    const int j = sc.lo_y + (ru % sc.ntj) * TJ + lane, k = sc.lo_z + (ru / sc.ntj) * TK + ty;
    const bool active = j < sc.hi_y && k < sc.hi_z;
    const bool band = active && a.united && !a.united[j + k * d.nj];
    const bool pml_yz = (a.aux[2] && j < d.N) || (a.aux[3] && j >= d.nj - d.N) || (a.aux[4] && k < d.N) ||
                        (a.aux[5] && k >= d.nk - d.N);
    float dyz = 1.0f;
    if (active && a.dampx) dyz = fminf(__ldg(a.dampy + j + 3), __ldg(a.dampz + k + 3));
    const long long qyz = idx3(d, 0, j + 3, k + 3);
    const int nst = ie - ib;
    const float* Q = qs + qr.slot * QSLOT + pc;
    const float mU = Q[0], mV = Q[PB], ety = Q[2 * PB], etz = Q[3 * PB], zty = Q[4 * PB], ztz = Q[5 * PB];
    for (int s = 0; s < nst; s++) {
      bool ok = true;
      for (int c = s == 0 ? 5 : 1; c > 0; c--) {
        ok = ok && mbar_wait(full_w + wr.slot, wr.phase);
        wr.next<NS>();
      }
      if (usep) ok = ok && mbar_wait(full_p + pr.slot, pr.phase);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(err, 1);
        return;
      }
      const int i = ib + s;
      const float* P = pw + pr.slot * PSLOT + pc;
      if (active && !(band && i + 3 >= d.i0 - 3 && i + 3 <= d.i0 + 3)) {
        const int s1 = sb + 1 == NS ? 0 : sb + 1;
        const int s2 = s1 + 1 == NS ? 0 : s1 + 1;
        const int s3 = s2 + 1 == NS ? 0 : s2 + 1;
        const int s4 = s3 + 1 == NS ? 0 : s3 + 1;
        const float* xs0 = win + sb * HSLOT + hc;
        const float* xs1 = win + s1 * HSLOT + hc;
        const float* xs2 = win + s2 * HSLOT + hc;
        const float* xs3 = win + s3 * HSLOT + hc;
        const float* xs4 = win + s4 * HSLOT + hc;
        const float* cur = FX == 1 ? xs1 : xs3;  // plane x itself
        // metric (xi row from the 1-D factor) and media of the side of the bimaterial split
        NodeMetric g;
        const float rA = __ldg(a.rxa + i + 3);
        g.ex0 = rA; g.ex1 = mU * rA; g.ex2 = mV * rA;
        g.ey1 = ety; g.ey2 = etz; g.ez1 = zty; g.ez2 = ztz;
        const int side = i + 3 < a.nxhalf ? 6 : 9;
        g.lam = Q[side * PB]; g.mu = Q[(side + 1) * PB]; g.rrho = 1.0f / Q[(side + 2) * PB];
        const bool pml = PMLP && (pml_yz || (a.aux[0] && i < d.N) || (a.aux[1] && i >= d.ni - d.N));
        const float damp = a.dampx ? fminf(__ldg(a.dampx + i + 3), dyz) : 1.0f;
        const long long q = qyz + (long long)(i + 3) * d.sx;
        float hv[9];
        if (pml) {
          // a node in a PML slab is taken whole by the velocity warp of the pair
          if (PMLP && role == 0) {
            const float* xv[5] = {xs0, xs1, xs2, xs3, xs4};
            tile_pml_point<FX, FY, FZ>(a, xv, cur, g, i, j, k, hv);
            rk_tile_store<0, 9>(a, n, q, cur, P, hv, damp);
          }
        } else {
          const float lam = g.lam, mu = g.mu, rrho = g.rrho;
          const float l2m = lam + 2.0f * mu;
#define DFD_DERX(f) d5v<FX>(xs0[(f) * HBOX], xs1[(f) * HBOX], xs2[(f) * HBOX], xs3[(f) * HBOX], xs4[(f) * HBOX])
#define DFD_DERY(f) d5s<FY, 1>(cur + (f) * HBOX)
#define DFD_DERZ(f) d5s<FZ, HW>(cur + (f) * HBOX)
          // the x row has three components; the y and z rows have no x component, so the
          // terms with it (exact zeros) and the derivative of Txx along y and z drop out
          if (role == 0) {
            // momentum: velocity rates from the six stress derivatives per axis
            float h0 = 0.f, h1 = 0.f, h2 = 0.f;
            {
              const float er0 = g.ex0 * rrho, er1 = g.ex1 * rrho, er2 = g.ex2 * rrho;
              float dv;
              dv = DFD_DERX(3) * r; h0 += dv * er0;
              dv = DFD_DERX(4) * r; h1 += dv * er1;
              dv = DFD_DERX(5) * r; h2 += dv * er2;
              dv = DFD_DERX(6) * r; h0 += dv * er1; h1 += dv * er0;
              dv = DFD_DERX(7) * r; h0 += dv * er2; h2 += dv * er0;
              dv = DFD_DERX(8) * r; h1 += dv * er2; h2 += dv * er1;
            }
#define DFD_VAXIS0(DER, E1, E2)                                                                     \
  {                                                                                                 \
    const float er1 = (E1) * rrho, er2 = (E2) * rrho;                                               \
    float dv;                                                                                       \
    dv = DER(4) * r; h1 += dv * er1;                                                                \
    dv = DER(5) * r; h2 += dv * er2;                                                                \
    dv = DER(6) * r; h0 += dv * er1;                                                                \
    dv = DER(7) * r; h0 += dv * er2;                                                                \
    dv = DER(8) * r; h1 += dv * er2; h2 += dv * er1;                                                \
  }
            DFD_VAXIS0(DFD_DERY, g.ey1, g.ey2)
            DFD_VAXIS0(DFD_DERZ, g.ez1, g.ez2)
#undef DFD_VAXIS0
            hv[0] = h0; hv[1] = h1; hv[2] = h2;
            rk_tile_store<0, 3>(a, n, q, cur, P, hv, damp);
          } else {
            // constitutive law: stress rates from the three velocity derivatives per axis
            float h3 = 0.f, h4 = 0.f, h5 = 0.f, h6 = 0.f, h7 = 0.f, h8 = 0.f;
            {
              const float e0 = g.ex0, e1 = g.ex1, e2 = g.ex2;
              float dv;
              dv = DFD_DERX(0) * r;
              h3 += dv * e0 * l2m; h4 += dv * e0 * lam; h5 += dv * e0 * lam; h6 += dv * e1 * mu; h7 += dv * e2 * mu;
              dv = DFD_DERX(1) * r;
              h3 += dv * e1 * lam; h4 += dv * e1 * l2m; h5 += dv * e1 * lam; h6 += dv * e0 * mu; h8 += dv * e2 * mu;
              dv = DFD_DERX(2) * r;
              h3 += dv * e2 * lam; h4 += dv * e2 * lam; h5 += dv * e2 * l2m; h7 += dv * e0 * mu; h8 += dv * e1 * mu;
            }
#define DFD_SAXIS0(DER, E1, E2)                                                                     \
  {                                                                                                 \
    const float e1 = (E1), e2 = (E2);                                                               \
    float dv;                                                                                       \
    dv = DER(0) * r; h6 += dv * e1 * mu; h7 += dv * e2 * mu;                                        \
    dv = DER(1) * r;                                                                                \
    h3 += dv * e1 * lam; h4 += dv * e1 * l2m; h5 += dv * e1 * lam; h8 += dv * e2 * mu;              \
    dv = DER(2) * r;                                                                                \
    h3 += dv * e2 * lam; h4 += dv * e2 * lam; h5 += dv * e2 * l2m; h8 += dv * e1 * mu;              \
  }
            DFD_SAXIS0(DFD_DERY, g.ey1, g.ey2)
            DFD_SAXIS0(DFD_DERZ, g.ez1, g.ez2)
#undef DFD_SAXIS0
            hv[3] = h3; hv[4] = h4; hv[5] = h5; hv[6] = h6; hv[7] = h7; hv[8] = h8;
            rk_tile_store<3, 9>(a, n, q, cur, P, hv, damp);
          }
#undef DFD_DERX
#undef DFD_DERY
#undef DFD_DERZ
        }
      }
      // release the slots this warp has finished with
      __syncwarp();
      if (lane == 0) {
        if (s + 1 < nst) {
          mbar_arrive(empty_w + sb);
        } else {
          for (int m = 0, sl = sb; m < 5; m++, sl = sl + 1 == NS ? 0 : sl + 1) mbar_arrive(empty_w + sl);
          mbar_arrive(empty_q + qr.slot);
        }
        if (usep) mbar_arrive(empty_p + pr.slot);
      }
      if (usep) pr.next<NP>();
      sb += s + 1 < nst ? 1 : 5;
      if (sb >= NS) sb -= NS;
    }
    qr.next<NQ>();
  }
}

// ---------------- host side

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 4-D map over nf fields of the volume layout (py, nz, nx, nf) with box (bw, bh, 1, bf)
static bool make_map(CUtensorMap* m, const Dims& d, const float* base, int nf, int bw, int bh, int bf) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)d.py, (cuuint64_t)d.nz, (cuuint64_t)d.nx, (cuuint64_t)nf};
  cuuint64_t strides[3] = {(cuuint64_t)d.py * 4, (cuuint64_t)d.sx * 4, (cuuint64_t)d.nxyz * 4};
  cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, (cuuint32_t)bf};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int FX, int FY, int FZ>
static bool set_smem() {
  auto one = [](const void* f) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES) == cudaSuccess;
  };
  return one((const void*)volume_tile_kernel<FX, FY, FZ, false, false>) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, true, false>) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, false, true>) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, true, true>);
}

// 3-D map over the 12 metric / media planes (py, nz, 12) with box (32, 8, 12)
static bool make_plane_map(CUtensorMap* m, const Dims& d, const float* base) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)d.py, (cuuint64_t)d.nz, 12};
  cuuint64_t strides[2] = {(cuuint64_t)d.py * 4, (cuuint64_t)d.py * d.nz * 4};
  cuuint32_t box[3] = {(cuuint32_t)TJ, (cuuint32_t)TK, 12};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tile_setup(TileCtx* tc, const Dims& d, float* const W[4], const float* planes, int* err, int* sched,
                int device) {
  tc->ok = false;
  tc->err = err;
  tc->sched = sched;
  if (cudaDeviceGetAttribute(&tc->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return false;
  // the tile's halo box must start on a 16-byte boundary: (first interior row node) % 4 == 0
  bool ok = true;
  for (int b = 0; b < 4 && ok; b++) {
    ok = make_map(&tc->halo[b], d, W[b], 9, HW, HH, 9);
    ok = ok && make_map(&tc->centre[b], d, W[b], 9, TJ, TK, 9);
  }
  ok = ok && make_plane_map(&tc->plane, d, planes);
  ok = ok && set_smem<-1, -1, -1>() && set_smem<-1, -1, 1>() && set_smem<-1, 1, -1>() && set_smem<-1, 1, 1>();
  ok = ok && set_smem<1, -1, -1>() && set_smem<1, -1, 1>() && set_smem<1, 1, -1>() && set_smem<1, 1, 1>();
  tc->ok = ok;
  cudaGetLastError();  // a failed attribute call leaves no sticky error; clear it
  return ok;
}

// Chunking of the x range: minimise the busiest CTA's plane loads, ceil(units / grid) x
// (planes per chunk + 4 halo planes).
TileSched tile_plan(int3 lo, int3 hi, int nsm, int* grid) {
  TileSched s;
  s.lo_x = lo.x; s.lo_y = lo.y; s.lo_z = lo.z; s.hi_x = hi.x; s.hi_y = hi.y; s.hi_z = hi.z;
  s.ntj = (hi.y - lo.y + TJ - 1) / TJ;
  s.ntk = (hi.z - lo.z + TK - 1) / TK;
  int nx = hi.x - lo.x, ntile = s.ntj * s.ntk;
  long long best = -1;
  for (int nch = 1; nch <= 64 && nch <= nx; nch++) {
    int ci = (nx + nch - 1) / nch;
    int nchr = (nx + ci - 1) / ci;
    long long units = (long long)ntile * nchr;
    long long g = std::min<long long>(units, nsm);
    long long cost = (units + g - 1) / g * (ci + 4);
    if (best < 0 || cost < best) { best = cost; s.ci = ci; s.nunits = (int)units; *grid = (int)g; }
  }
  return s;
}

template <int FX, int FY, int FZ>
static void launch_t(const TileCtx& tc, const VolArgs& a, int bin, int3 lo, int3 hi, bool pmlp, cudaStream_t s) {
  TileMaps mp;
  mp.win = tc.halo[bin];
  mp.w0 = tc.centre[0];
  mp.t = tc.centre[3];
  mp.plane = tc.plane;
  int grid = 0;
  TileSched sc = tile_plan(lo, hi, tc.nsm, &grid);
  if (pmlp)
    volume_tile_kernel<FX, FY, FZ, true, false>
        <<<grid, NTOT, SMEM_BYTES, s>>>(mp, a, sc, nullptr, 1, sc.nunits, tc.err, tc.sched);
  else
    volume_tile_kernel<FX, FY, FZ, false, false>
        <<<grid, NTOT, SMEM_BYTES, s>>>(mp, a, sc, nullptr, 1, sc.nunits, tc.err, tc.sched);
}

// true when the tiled kernel took the interior box
bool tile_feasible(const TileCtx* tc, const VolArgs& a, int3 lo, int3 hi) {
  if (!tc || !tc->ok) return false;
  return (lo.y + 3 + a.d.oy) % 4 == 0 && lo.z >= 0 && hi.x > lo.x && hi.y > lo.y && hi.z > lo.z;
}

template <int FX, int FY, int FZ>
static void launch_tb(const TileScen& f, const TileScen* tab, int n, int nunits, int grid, bool pmlp, int* err,
                      int* sched, cudaStream_t s) {
  if (pmlp)
    volume_tile_kernel<FX, FY, FZ, true, true>
        <<<grid, NTOT, SMEM_BYTES, s>>>(f.mp, f.a, f.sc, tab, n, nunits, err, sched);
  else
    volume_tile_kernel<FX, FY, FZ, false, true>
        <<<grid, NTOT, SMEM_BYTES, s>>>(f.mp, f.a, f.sc, tab, n, nunits, err, sched);
}
// every scenario of an ensemble in one persistent launch (units numbered across them)
void launch_tile_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int FX, int FY,
                       int FZ, bool pmlp, int* err, int* sched, cudaStream_t s) {
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_tb<-1, -1, -1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 1: launch_tb<-1, -1, 1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 2: launch_tb<-1, 1, -1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 3: launch_tb<-1, 1, 1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 4: launch_tb<1, -1, -1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 5: launch_tb<1, -1, 1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    case 6: launch_tb<1, 1, -1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
    default: launch_tb<1, 1, 1>(first, tab, n, nunits, grid, pmlp, err, sched, s); break;
  }
}

bool launch_tile(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, int3 lo, int3 hi, bool pmlp,
                 cudaStream_t s) {
  if (!tile_feasible(tc, a, lo, hi)) return false;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_t<-1, -1, -1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 1: launch_t<-1, -1, 1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 2: launch_t<-1, 1, -1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 3: launch_t<-1, 1, 1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 4: launch_t<1, -1, -1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 5: launch_t<1, -1, 1>(*tc, a, bin, lo, hi, pmlp, s); break;
    case 6: launch_t<1, 1, -1>(*tc, a, bin, lo, hi, pmlp, s); break;
    default: launch_t<1, 1, 1>(*tc, a, bin, lo, hi, pmlp, s); break;
  }
  return true;
}

}  // namespace dfd
