// Device helpers of the TMA-staged volume kernels (dfd_tile.cu: interior box,
// dfd_pml.cu: PML slabs): tile geometry, mbarrier and bulk-copy primitives, the
// one-sided operators on shared-memory lines, the per-node metric and the RK4 store.
//
// A tile is 32 (y) x 8 (z) nodes; a CTA owns one tile column and marches along x.  Every
// tile starts on a 16-byte boundary in y (the volume rows start one element early, so
// node j = 0 sits at a 16-byte boundary), as TMA requires for the innermost coordinate.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "dfd_stencil.cuh"

namespace dfd {

namespace {
constexpr int TJ = TILE_J, TK = TILE_K, NTHR = TJ * TK;
constexpr int HW = TJ + 8;           // halo box width (y): 4 nodes each side (16-byte aligned)
constexpr int HH = TK + 4;           // halo box height (z): 1 + 3 rows, side set by the z operator
constexpr int HBOX = HW * HH;        // floats per field of a halo box
constexpr int HSLOT = 9 * HBOX;      // floats per stencil plane slot
constexpr int PB = TJ * TK;          // floats per field of a pointwise box
constexpr int QSLOT = 12 * PB;       // metric / media planes of a unit: U V ety etz zty ztz, 2 x (lam mu rho)
constexpr int NCW = 2 * NTHR / 32;   // computing warps: two per 32-node row of the tile
constexpr int NTOT = NCW * 32 + 32;  // plus one copy-issuing warp
constexpr long long WAIT_LIMIT = 1LL << 22;  // polls of one mbarrier before giving up
constexpr long long DRILL_LIMIT = 1LL << 12; // the same in the test drill of the bounded waits
static_assert((HSLOT * 4) % 128 == 0 && (QSLOT * 4) % 128 == 0 && (PB * 4) % 128 == 0, "slot alignment");
static_assert(sizeof(TileUnit) % 16 == 0 && offsetof(TileScen, u) % 16 == 0, "bulk copy of the scenario values");
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
__device__ __forceinline__ bool mbar_wait_n(uint64_t* b, unsigned parity, long long limit) {
  for (long long n = 0; n < limit; n++)
    if (mbar_try(b, parity)) return true;
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) { return mbar_wait_n(b, parity, WAIT_LIMIT); }
__device__ __forceinline__ void tma_load4(float* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                          uint64_t* b) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(b))
      : "memory");
}

// plain bulk copy (no tensor map) of bytes (a multiple of 16, both addresses 16-byte
// aligned) from global to shared memory, completing on mbarrier b
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
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
// input at stage 0, from the pointwise slot P at stages 1 and 2; at stage 2 the slot's
// second box holds the stage-1 input, from which, with y0 and the stage input, the
// accumulator is formed (rk_sum, rk_acc); at stage 3 the slot holds the accumulator
// alone, first.  IRK: the
// stage (the kernels are compiled per stage).
template <int F0, int F1, int IRK, int HB = HBOX, int PBB = PB>
__device__ __forceinline__ void rk_tile_store(const VolArgs& a, long long n, long long q, const float* cur,
                                              const float* P, const float* hv, float damp) {
  const float rd = IRK == 2 ? rk_rd(damp) : 1.0f;
#pragma unroll
  for (int f = F0; f < F1; f++) {
    const long long x = f * n + q;
    float w;
    if (IRK == 0) {
      w = fmaf(a.rka, hv[f], cur[f * HB]);
    } else if (IRK == 1) {
      w = fmaf(a.rka, hv[f], P[f * PBB]);
    } else if (IRK == 2) {
      const float y0 = P[f * PBB];
      a.T[x] = rk_acc(y0, rk_sum(y0, P[(9 + f) * PBB], cur[f * HB], rd), a.rkb, hv[f]);
      w = fmaf(a.rka, hv[f], y0);
    } else {
      w = fmaf(a.rkb, hv[f], P[f * PBB]);
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


// Lean right-hand side of a node outside every PML slab and below the free-surface rows
// (rB = 1, no ADE state): momentum (velocity rates, hv[0..2]) and constitutive law (stress
// rates, hv[3..8]) from the one-sided derivatives on the shared-memory stencil planes
// (xs0..xs4 the five x planes, cur the node's plane, PW the row pitch of the stencil box).
// The x row of the metric has three
// components; the y and z rows have no x component, so the terms with it (exact zeros)
// and the derivative of Txx along y and z drop out.  Reference wave.cu:8-204.
// HB: floats per field of the stencil box.
#define DFD_DERX(f) d5v<FX>(xs0[(f) * HB], xs1[(f) * HB], xs2[(f) * HB], xs3[(f) * HB], xs4[(f) * HB])
#define DFD_DERY(f) d5s<FY, 1>(cur + (f) * HB)
#define DFD_DERZ(f) d5s<FZ, PW>(cur + (f) * HB)
template <int FX, int FY, int FZ, int PW = HW, int HB = HBOX>
__device__ __forceinline__ void lean_velocity(const float* xs0, const float* xs1, const float* xs2, const float* xs3,
                                              const float* xs4, const float* cur, const NodeMetric& g, float r,
                                              float* hv) {
  const float rrho = g.rrho;
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
}
template <int FX, int FY, int FZ, int PW = HW, int HB = HBOX>
__device__ __forceinline__ void lean_stress(const float* xs0, const float* xs1, const float* xs2, const float* xs3,
                                            const float* xs4, const float* cur, const NodeMetric& g, float r,
                                            float* hv) {
  const float lam = g.lam, mu = g.mu;
  const float l2m = lam + 2.0f * mu;
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
}
#undef DFD_DERX
#undef DFD_DERY
#undef DFD_DERZ

// first scenario of a batched launch whose units include the global unit u
__device__ __forceinline__ int tile_scenario(const TileScen* tab, int n, int u) {
  int lo = 0, hi = n;  // tab[lo].unit0 <= u < tab[hi].unit0
  while (hi - lo > 1) {
    int m = (lo + hi) / 2;
    if (tab[m].u.unit0 <= u) lo = m; else hi = m;
  }
  return lo;
}

}  // namespace dfd
