// Interior box of the volume stage, staged through shared memory by TMA.
//
// The box is cut into tiles of 32 (y) x 8 (z) nodes (or 32 x 4, TileShape); a CTA owns
// one tile column and marches along x over a chunk of planes.  Per plane it needs
//   - the stencil input (9 fields) of the planes x-1..x+3 (forward x operator) or
//     x-3..x+1 (backward), with a y/z halo on the current plane: one 4-D TMA box
//     (40 y, 12 z, 1 x, 9 fields) per plane, held in a ring of NS plane slots;
//   - the pointwise streams of the node: 12 metric/media fields, and the RK registers
//     W0 (stages 1, 2), the stage-1 input (stage 2) and T (stage 3): TMA boxes (32, 8, 1, n)
//     in a ring of NP slots.
// A dedicated warp issues the copies ahead of the sixteen (eight) computing warps (full/empty
// mbarrier pairs per slot, no block-wide barrier in the loop), so HBM traffic stays in
// flight while the stencils are evaluated from shared memory with immediate offsets.
// No node of the box lies in a PML slab or the free-surface rows (dfd_pml.cu and the
// general kernel take those).  Outputs (Wout, and T at stage 2) are written straight from
// registers.
//
// The kernel is persistent: one CTA per SM (two with 4-row tiles) takes units (tile column x chunk) from a global
// counter, and its copy stream runs across unit boundaries, so the next unit's planes
// arrive while the current one finishes.
//
// The right-hand side follows the reference's wave.cu:8-204 and rk4.cu:20-33, as the
// general kernel in dfd_volume.cu does.
#include <algorithm>
#include <cstring>

#include "dfd_tma.cuh"

namespace dfd {

namespace {
// Shape of the interior kernel's tiles: 32 (y) x TR (z) nodes.  TR = 8: 16 computing warps
// and one CTA per SM; TR = 4: 8 computing warps, shallower stencil ring and two CTAs per
// SM (each within half of the SM's 228 KB of shared memory, 1 KB of it reserved per CTA).
// An RK slot holds W0 and the stage-1 input (stage 2), W0 (stage 1) or T alone (stage 3).
template <int TR>
struct TileShape {
  static constexpr int HH = TR + 4, HB = HW * HH, HSLOT = 9 * HB, PB = TJ * TR, QSLOT = 12 * PB;
  static constexpr int PSLOT = 18 * PB;
  static constexpr int NCW = 2 * TR, NTOT = NCW * 32 + 32;
  static constexpr int NS = TR == 8 ? 8 : 6, NP = 3, NQ = 2;  // stencil planes, RK slots, unit planes
  static constexpr int CTAS = TR == 8 ? 1 : 2;
  static constexpr size_t SMEM =
      (size_t)(NS * HSLOT + NP * PSLOT + NQ * QSLOT) * 4 + NQ * sizeof(TileUnit) + 2 * (NS + NP + NQ) * 8 + NQ * 4;
  static_assert(TR == 8 || TR == 4, "tiles of 8 or 4 rows");
  static_assert(SMEM <= 232448 && CTAS * (SMEM + 1024) <= 233472, "tile ring exceeds the shared memory");
  static_assert((PSLOT * 4) % 128 == 0 && (HSLOT * 4) % 128 == 0 && (QSLOT * 4) % 128 == 0, "slot alignment");
};
}  // namespace

int tile_ctas_per_sm(int tr) { return tr == 4 ? TileShape<4>::CTAS : TileShape<8>::CTAS; }

// Warp NCW issues the copies; warps 0..NCW-1 compute one node each per plane (NCW = 2 TR).  Each ring
// slot has a "full" barrier (completed by the copy's transaction bytes) and an "empty"
// barrier (one arrival per computing warp once it has finished reading the slot).  Three
// rings: stencil planes (NS), RK registers of the step (NP; none at stage 0, whose
// step-start values are the stencil input), metric/media planes of the unit (NQ).  At
// most 96 registers: with 8-row tiles the 17 warps are spread over the SM's four 16 K-register
// partitions, five warps on one of them; with 4-row tiles two CTAs of 9 warps share them.

// IRK: the RK stage (a0.irk), a compile-time constant so that each stage's code and
// register allocation carry only its own RK registers.  BATCH: the units of the nscen
// scenarios of tab (an ensemble) in one launch; the parameters mp0, a0, sc0 then
// describe scenario 0 and give the stage's common values.  TR: rows of a tile (TileShape).
template <int FX, int FY, int FZ, int IRK, bool BATCH, int TR>
__global__ void __maxnreg__(96)
    volume_tile_kernel(const __grid_constant__ TileMaps mp0, const __grid_constant__ VolArgs a0,
                       const __grid_constant__ TileSched sc0, const TileScen* __restrict__ tab, int nscen,
                       int nunits, int* err, int* sched) {
  using SH = TileShape<TR>;
  constexpr int TK = TR, HSLOT = SH::HSLOT, PSLOT = SH::PSLOT, QSLOT = SH::QSLOT, PB = SH::PB, NCW = SH::NCW;
  constexpr int NS = SH::NS, NP = SH::NP, NQ = SH::NQ;
  extern __shared__ __align__(1024) unsigned char smraw[];
  float* win = reinterpret_cast<float*>(smraw);
  float* pw = win + NS * HSLOT;
  float* qs = pw + NP * PSLOT;
  TileUnit* uarg = reinterpret_cast<TileUnit*>(qs + NQ * QSLOT);  // scenario values per unit slot (BATCH)
  uint64_t* full_w = reinterpret_cast<uint64_t*>(uarg + NQ);
  uint64_t* empty_w = full_w + NS;
  uint64_t* full_p = empty_w + NS;
  uint64_t* empty_p = full_p + NP;
  uint64_t* full_q = empty_p + NP;
  uint64_t* empty_q = full_q + NQ;
  int* qunit = reinterpret_cast<int*>(empty_q + NQ);  // unit of each plane slot (-1: no more)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int XLO = FX == 1 ? -1 : -3;  // first stencil plane relative to x
  constexpr int RZ = FZ == 1 ? 1 : 3;     // row of the tile's first z node inside the halo box
  constexpr int irk = IRK;
  // pointwise boxes: y0 at stages 1 and 2, a second box at stages 2 (the stage-1 input)
  // and 3 (the accumulator); stage 0 takes everything from the stencil planes
  constexpr bool needW0 = irk == 1 || irk == 2, needT = irk >= 2, usep = needW0 || needT;
  const int G = gridDim.x;
  // the PML kernel that follows on the stream touches other nodes only: it may take the
  // SMs that this persistent grid's CTAs leave as they finish
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");

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
    // with a concurrent kernel) simply take fewer.  In the test drill of the bounded waits
    // this warp takes no unit and issues nothing: no copy is ever in flight, and the
    // computing warps' first wait runs out.
    while (ok && !sc0.drill) {
      const int u = atomicAdd(sched, 1);
      if (qcount >= NQ && !(ok = mbar_wait(empty_q + qr.slot, qr.phase ^ 1))) break;
      if (u >= nunits) {
        qunit[qr.slot] = -1;  // tell the computing warps that there is no further unit
        mbar_arrive(full_q + qr.slot);
        break;
      }
      const int scn = BATCH ? tile_scenario(tab, nscen, u) : 0;
      const TileMaps& mp = BATCH ? tab[scn].mp : mp0;
      const VolArgs& a = BATCH ? tab[scn].u.a : a0;
      const TileSched& sc = BATCH ? tab[scn].u.sc : sc0;
      const Dims& d = a.d;
      const int lu = BATCH ? u - tab[scn].u.unit0 : u;
      const int ntile = sc.ntj * sc.ntk;
      const int tc = lu / ntile, ru = lu % ntile;
      const int ib = sc.lo_x + tc * sc.ci, ie = min(ib + sc.ci, sc.hi_x);
      const int j0 = sc.lo_y + (ru % sc.ntj) * TJ, k0 = sc.lo_z + (ru / sc.ntj) * TK;
      const int cw0 = j0 + 3 + d.oy - 4, cw1 = k0 + 3 - RZ, cp0 = j0 + 3 + d.oy, cp1 = k0 + 3;
      const int nst = ie - ib;
      // metric / media planes of the unit, with the unit's index
      qunit[qr.slot] = u;
      if (BATCH) {
        // with the scenario's values for the computing warps
        mbar_expect_tx(full_q + qr.slot, QSLOT * 4 + (unsigned)sizeof(TileUnit));
        bulk_load(uarg + qr.slot, &tab[scn].u, (unsigned)sizeof(TileUnit), full_q + qr.slot);
      } else {
        mbar_expect_tx(full_q + qr.slot, QSLOT * 4);
      }
      tma_load3(qs + qr.slot * QSLOT, &mp.plane_i, cp0, cp1, 0, full_q + qr.slot);
      qr.next<NQ>();
      qcount++;
      for (int m = 0; m < nst + 4 && ok; m++) {
        // stencil plane m of the unit (first needed by step m - 4)
        if (wcount >= NS && !(ok = mbar_wait(empty_w + wr.slot, wr.phase ^ 1))) break;
        mbar_expect_tx(full_w + wr.slot, HSLOT * 4);
        tma_load4(win + wr.slot * HSLOT, &mp.win_i, cw0, cw1, ib + XLO + m + 3, 0, full_w + wr.slot);
        wr.next<NS>();
        wcount++;
        if (m < 4 || !usep) continue;
        // RK registers of step m - 4
        if (pcount >= NP && !(ok = mbar_wait(empty_p + pr.slot, pr.phase ^ 1))) break;
        uint64_t* b = full_p + pr.slot;
        float* dst = pw + pr.slot * PSLOT;
        const int cp2 = ib + (m - 4) + 3;
        mbar_expect_tx(b, ptx);
        if (needW0) tma_load4(dst, &mp.w0_i, cp0, cp1, cp2, 0, b);
        if (needT) tma_load4(dst + (needW0 ? 9 : 0) * PB, &mp.t_i, cp0, cp1, cp2, 0, b);
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
    if (!__all_sync(0xffffffffu, mbar_wait_n(full_q + qr.slot, qr.phase, sc0.drill ? DRILL_LIMIT : WAIT_LIMIT))) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    const int u = qunit[qr.slot];
    if (u < 0) break;
    const TileUnit& ua = uarg[qr.slot];
    const VolArgs& a = BATCH ? ua.a : a0;
    const TileSched& sc = BATCH ? ua.sc : sc0;
    const Dims& d = a.d;
    const long long n = d.nxyz;
    const int lu = BATCH ? u - ua.unit0 : u;
    const int ntile = sc.ntj * sc.ntk;
    const int tc = lu / ntile, ru = lu % ntile;
    const int ib = sc.lo_x + tc * sc.ci, ie = min(ib + sc.ci, sc.hi_x);
    const int j = sc.lo_y + (ru % sc.ntj) * TJ + lane, k = sc.lo_z + (ru / sc.ntj) * TK + ty;
    const bool active = j < sc.hi_y && k < sc.hi_z;
    const bool band = active && a.united && !a.united[j + k * d.nj];
    float dyz = 1.0f;
    if (active && a.dampx) dyz = fminf(__ldg(a.dampy + j + 3), __ldg(a.dampz + k + 3));
    const long long qyz = idx3(d, 0, j + 3, k + 3);
    const int nst = ie - ib;
    const float* Q = qs + qr.slot * QSLOT + pc;
    const float mU = Q[0], mV = Q[PB], ety = Q[2 * PB], etz = Q[3 * PB], zty = Q[4 * PB], ztz = Q[5 * PB];
    // per-plane 1-D factors, loaded one plane ahead so that their latency overlaps a plane
    float rA_next = __ldg(a.rxa + ib + 3);
    float dx_next = a.dampx ? __ldg(a.dampx + ib + 3) : 1.0f;
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
      const float rA = rA_next, dx = dx_next;
      if (s + 1 < nst) {
        rA_next = __ldg(a.rxa + i + 4);
        if (a.dampx) dx_next = __ldg(a.dampx + i + 4);
      }
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
        g.ex0 = rA; g.ex1 = mU * rA; g.ex2 = mV * rA;
        g.ey1 = ety; g.ey2 = etz; g.ez1 = zty; g.ez2 = ztz;
        const int side = i + 3 < a.nxhalf ? 6 : 9;
        g.lam = Q[side * PB]; g.mu = Q[(side + 1) * PB]; g.rrho = 1.0f / Q[(side + 2) * PB];
        const float damp = a.dampx ? fminf(dx, dyz) : 1.0f;
        const long long q = qyz + (long long)(i + 3) * d.sx;
        float hv[9];
        if (role == 0) {
          lean_velocity<FX, FY, FZ, HW, SH::HB>(xs0, xs1, xs2, xs3, xs4, cur, g, a.rDH, hv);
          rk_tile_store<0, 3, IRK, SH::HB, PB>(a, n, q, cur, P, hv, damp);
        } else {
          lean_stress<FX, FY, FZ, HW, SH::HB>(xs0, xs1, xs2, xs3, xs4, cur, g, a.rDH, hv);
          rk_tile_store<3, 9, IRK, SH::HB, PB>(a, n, q, cur, P, hv, damp);
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

template <int FX, int FY, int FZ, int IRK>
static bool set_smem_k() {
  auto one = [](const void* f, size_t bytes) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
  };
  return one((const void*)volume_tile_kernel<FX, FY, FZ, IRK, false, 8>, TileShape<8>::SMEM) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, IRK, true, 8>, TileShape<8>::SMEM) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, IRK, false, 4>, TileShape<4>::SMEM) &&
         one((const void*)volume_tile_kernel<FX, FY, FZ, IRK, true, 4>, TileShape<4>::SMEM);
}
template <int FX, int FY, int FZ>
static bool set_smem() {
  return set_smem_k<FX, FY, FZ, 0>() && set_smem_k<FX, FY, FZ, 1>() && set_smem_k<FX, FY, FZ, 2>() &&
         set_smem_k<FX, FY, FZ, 3>();
}

// 3-D map over the 12 metric / media planes (py, nz, 12) with box (bw, bh, 12)
static bool make_plane_map(CUtensorMap* m, const Dims& d, const float* base, int bw, int bh) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)d.py, (cuuint64_t)d.nz, 12};
  cuuint64_t strides[2] = {(cuuint64_t)d.py * 4, (cuuint64_t)d.py * d.nz * 4};
  cuuint32_t box[3] = {(cuuint32_t)bw, (cuuint32_t)bh, 12};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// 4-D map over the 27-field PML state of face f (columns, rows, planes, fields; the
// layouts of pml_index) with box (bw, bh, 1, 9)
static bool make_aux_map(CUtensorMap* m, const Dims& d, int f, const float* base, int bw, int bh) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t w = f < 2 ? d.py : f < 4 ? d.wy : d.py;
  cuuint64_t rows = f < 2 ? d.nz : f < 4 ? d.nz : d.N;
  cuuint64_t planes = f < 2 ? d.N : d.ni;
  cuuint64_t dims[4] = {w, rows, planes, 27};
  cuuint64_t strides[3] = {w * 4, w * rows * 4, (cuuint64_t)pml_fstride(d, f) * 4};
  cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, 9};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

bool tile_setup(TileCtx* tc, const Dims& d, float* const W[4], const float* planes, float* const aux[6], int* err,
                int* sched, int device) {
  tc->ok = false;
  tc->err = err;
  tc->sched = sched;
  if (cudaDeviceGetAttribute(&tc->nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return false;
  bool ok = true;
  for (int b = 0; b < 4 && ok; b++) {
    ok = make_map(&tc->halo[b], d, W[b], 9, HW, HH, 9);
    ok = ok && make_map(&tc->centre[b], d, W[b], 9, TJ, TK, 9);
    // 32 x 4 tiles of the interior kernel: halo box 40 x 8
    ok = ok && make_map(&tc->halo4[b], d, W[b], 9, HW, TileShape<4>::HH, 9);
    ok = ok && make_map(&tc->centre4[b], d, W[b], 9, TJ, 4, 9);
    // strip tiles of the PML kernel: 16 x 16 nodes, halo box 24 x 20
    ok = ok && make_map(&tc->halo_s[b], d, W[b], 9, STRIP + 8, STRIP + 4, 9);
    ok = ok && make_map(&tc->centre_s[b], d, W[b], 9, STRIP, STRIP, 9);
  }
  ok = ok && make_plane_map(&tc->plane, d, planes, TJ, TK);
  ok = ok && make_plane_map(&tc->plane4, d, planes, TJ, 4);
  ok = ok && make_plane_map(&tc->plane_s, d, planes, STRIP, STRIP);
  for (int f = 0; f < 6 && ok; f++) {
    memset(&tc->aux[f], 0, sizeof(CUtensorMap));
    if (aux[f]) ok = make_aux_map(&tc->aux[f], d, f, aux[f], TJ, TK);
  }
  for (int f = 2; f < 4 && ok; f++) {
    memset(&tc->auxy_s[f - 2], 0, sizeof(CUtensorMap));
    if (aux[f]) ok = make_aux_map(&tc->auxy_s[f - 2], d, f, aux[f], STRIP, STRIP);
  }
  ok = ok && set_smem<-1, -1, -1>() && set_smem<-1, -1, 1>() && set_smem<-1, 1, -1>() && set_smem<-1, 1, 1>();
  ok = ok && set_smem<1, -1, -1>() && set_smem<1, -1, 1>() && set_smem<1, 1, -1>() && set_smem<1, 1, 1>();
  ok = ok && pml_setup();
  tc->ok = ok;
  cudaGetLastError();  // a failed attribute call leaves no sticky error; clear it
  return ok;
}

// Chunking of the x range: minimise the busiest CTA's plane loads, ceil(units / grid) x
// (planes per chunk + 4 halo planes).
TileSched tile_plan(int3 lo, int3 hi, int slots, int* grid, int tr) {
  TileSched s;
  memset(&s, 0, sizeof s);
  s.lo_x = lo.x; s.lo_y = lo.y; s.lo_z = lo.z; s.hi_x = hi.x; s.hi_y = hi.y; s.hi_z = hi.z;
  s.ntj = (hi.y - lo.y + TJ - 1) / TJ;
  s.ntk = (hi.z - lo.z + tr - 1) / tr;
  const int nsm = slots;
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

// maps of stage irk with stencil input buffer bin; the second pointwise box reads, at
// stage 2, the stage-1 input (the buffer the stage overwrites) and otherwise the accumulator
TileMaps tile_maps(const TileCtx& tc, int bin, int irk, int tr) {
  TileMaps mp;
  memset(&mp, 0, sizeof mp);
  const int p2 = irk == 2 ? stage_out(2) : 3;
  mp.win = tc.halo[bin];
  mp.w0 = tc.centre[0];
  mp.t = tc.centre[p2];
  mp.plane = tc.plane;
  for (int f = 0; f < 6; f++) mp.aux[f] = tc.aux[f];
  mp.win_s = tc.halo_s[bin];
  mp.w0_s = tc.centre_s[0];
  mp.t_s = tc.centre_s[p2];
  mp.plane_s = tc.plane_s;
  mp.auxy_s[0] = tc.auxy_s[0];
  mp.auxy_s[1] = tc.auxy_s[1];
  const bool four = tr == 4;
  mp.win_i = four ? tc.halo4[bin] : mp.win;
  mp.w0_i = four ? tc.centre4[0] : mp.w0;
  mp.t_i = four ? tc.centre4[p2] : mp.t;
  mp.plane_i = four ? tc.plane4 : mp.plane;
  return mp;
}

template <int FX, int FY, int FZ, int TR>
static void launch_tr(const TileCtx& tc, const VolArgs& a, int bin, int3 lo, int3 hi, cudaStream_t s) {
  using SH = TileShape<TR>;
  const TileMaps mp = tile_maps(tc, bin, a.irk, TR);
  int grid = 0;
  TileSched sc = tile_plan(lo, hi, tc.nsm * SH::CTAS, &grid, TR);
  sc.drill = tc.drill;
#define DFD_L(K)                                                                                             \
  volume_tile_kernel<FX, FY, FZ, K, false, TR><<<grid, SH::NTOT, SH::SMEM, s>>>(mp, a, sc, nullptr, 1, sc.nunits, \
                                                                               tc.err, tc.sched)
  DFD_BY_STAGE(a.irk, DFD_L);
#undef DFD_L
}
template <int FX, int FY, int FZ>
static void launch_t(const TileCtx& tc, const VolArgs& a, int bin, int3 lo, int3 hi, cudaStream_t s) {
  if (tc.tr == 4) launch_tr<FX, FY, FZ, 4>(tc, a, bin, lo, hi, s);
  else launch_tr<FX, FY, FZ, 8>(tc, a, bin, lo, hi, s);
}

// true when the tiled kernel can take the box lo..hi
bool tile_feasible(const TileCtx* tc, const VolArgs& a, int3 lo, int3 hi) {
  if (!tc || !tc->ok) return false;
  return (lo.y + 3 + a.d.oy) % 4 == 0 && lo.z >= 0 && hi.x > lo.x && hi.y > lo.y && hi.z > lo.z;
}

template <int FX, int FY, int FZ, int TR>
static void launch_tbr(const TileScen& f, const TileScen* tab, int n, int nunits, int grid, int* err, int* sched,
                       cudaStream_t s) {
  using SH = TileShape<TR>;
#define DFD_L(K)                                                                                                \
  volume_tile_kernel<FX, FY, FZ, K, true, TR><<<grid * SH::CTAS, SH::NTOT, SH::SMEM, s>>>(f.mp, f.u.a, f.u.sc, tab, n, \
                                                                                         nunits, err, sched)
  DFD_BY_STAGE(f.u.a.irk, DFD_L);
#undef DFD_L
}
template <int FX, int FY, int FZ>
static void launch_tb(const TileScen& f, const TileScen* tab, int n, int nunits, int grid, int tr, int* err,
                      int* sched, cudaStream_t s) {
  if (tr == 4) launch_tbr<FX, FY, FZ, 4>(f, tab, n, nunits, grid, err, sched, s);
  else launch_tbr<FX, FY, FZ, 8>(f, tab, n, nunits, grid, err, sched, s);
}
// every scenario of an ensemble in one persistent launch (units numbered across them);
// grid: SMs (each takes tile_ctas_per_sm(tr) CTAs); tr: the scenarios' tile rows
void launch_tile_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int tr, int FX,
                       int FY, int FZ, int* err, int* sched, cudaStream_t s) {
  if (nunits <= 0) return;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_tb<-1, -1, -1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 1: launch_tb<-1, -1, 1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 2: launch_tb<-1, 1, -1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 3: launch_tb<-1, 1, 1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 4: launch_tb<1, -1, -1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 5: launch_tb<1, -1, 1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    case 6: launch_tb<1, 1, -1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
    default: launch_tb<1, 1, 1>(first, tab, n, nunits, grid, tr, err, sched, s); break;
  }
}

bool launch_tile(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, int3 lo, int3 hi,
                 cudaStream_t s) {
  if (!tile_feasible(tc, a, lo, hi)) return false;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_t<-1, -1, -1>(*tc, a, bin, lo, hi, s); break;
    case 1: launch_t<-1, -1, 1>(*tc, a, bin, lo, hi, s); break;
    case 2: launch_t<-1, 1, -1>(*tc, a, bin, lo, hi, s); break;
    case 3: launch_t<-1, 1, 1>(*tc, a, bin, lo, hi, s); break;
    case 4: launch_t<1, -1, -1>(*tc, a, bin, lo, hi, s); break;
    case 5: launch_t<1, -1, 1>(*tc, a, bin, lo, hi, s); break;
    case 6: launch_t<1, 1, -1>(*tc, a, bin, lo, hi, s); break;
    default: launch_t<1, 1, 1>(*tc, a, bin, lo, hi, s); break;
  }
  return true;
}

}  // namespace dfd
