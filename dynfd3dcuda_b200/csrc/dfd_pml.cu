// Nodes of the volume stage below the free-surface rows that the interior kernel does
// not take, staged through shared memory by TMA: the PML slabs of all six faces and the
// nodes that fill their tiles (the interior kernel takes whole tiles only).
//
// Units (dfd_internal.cuh, TileSched): every 32 x 8 tile of the two x slabs, one unit
// per tile and slab; then, in chunks of x planes between the slabs, the 16 x 16 strip
// tiles of the y slabs (a y slab is 12 to 20 nodes wide: a 32-wide tile would leave most
// lanes without a PML node) and the 32 x 8 tiles of the z slabs.  Each unit stages, per
// plane, the stencil input with its halo, the RK registers and the ADE state of one PML
// face (its "own" face: x for the x slabs, y for the strips, z for the z tiles); a node
// that also lies in another face (edges and corners of the slabs) reads that face's
// state from global memory.  One computing warp per row of nodes
// integrates all nine fields and their PML state.
//
// Right-hand side with the ADE CFS-PML as in the reference's wave.cu:8-204 and
// pmlx.cu:8-214 / pmly.cu / pmlz.cu, the RK4 registers as rk4.cu:20-33 and 154-257.
#include <algorithm>
#include <cstring>

#include "dfd_tma.cuh"

namespace dfd {

namespace {
constexpr int PCW = TK;                 // computing warps: one per row of the tile, all nine fields
constexpr int PTOT = PCW * 32 + 32;     // plus one copy-issuing warp
}  // namespace

// Ring shapes of stage IRK.  A pointwise slot holds, in this order, W0 (stages 1, 2), the
// second box (stage 2: the stage-1 input; stage 3: the accumulator) and the ADE blocks of
// the unit's own face that the stage reads (the current value, then y0 or the accumulator,
// then y1: aux_block): 9, 27, 45 and 27 fields at stages 0..3.  The shared memory that
// the smaller slots leave goes to more slots: the stencil ring (5 planes in use) then runs
// 4, 3, 1 and 3 planes ahead.
template <int IRK>
struct PmlRing {
  static constexpr bool W0 = IRK == 1 || IRK == 2, T = IRK >= 2;
  static constexpr int NAUX = IRK == 0 ? 9 : IRK == 2 ? 27 : 18;  // ADE fields staged per plane
  static constexpr int TOFF = W0 ? 9 : 0;                          // second box in the slot
  static constexpr int AOFF = 9 * ((W0 ? 1 : 0) + (T ? 1 : 0));    // ADE blocks in the slot
  static constexpr int PF = AOFF + NAUX;                           // fields per slot
  static constexpr int PSLOT = PF * PB;
  static constexpr int MS = IRK == 0 ? 9 : IRK == 2 ? 6 : 8;      // stencil planes
  static constexpr int MP = IRK == 0 ? 4 : 2;                      // pointwise planes
  static constexpr int MQ = 2;                                     // unit-plane sets
  static constexpr size_t SMEM =
      (size_t)(MS * HSLOT + MP * PSLOT + MQ * QSLOT) * 4 + MQ * sizeof(TileUnit) + 2 * (MS + MP + MQ) * 8 + MQ * 4;
  static_assert(SMEM <= 232448, "PML ring exceeds the shared memory of one CTA");
  static_assert((PSLOT * 4) % 128 == 0, "slot alignment");
};

// tile origin, x range, own face (-1: none), node bounds (j < jhi, k < khi) and shape
// (strip: 16 x 16, else 32 x 8) of local unit lu
struct PmlUnit {
  int j0, k0, ib, ie, face, jhi, khi;
  bool strip;
};
__device__ __forceinline__ PmlUnit pml_unit(const TileSched& sc, const VolArgs& a, int lu) {
  const Dims& d = a.d;
  PmlUnit r;
  r.strip = false;
  const int ntile = sc.ntj * sc.ntk;
  if ((sc.nx1 > 0 && lu < ntile) || (sc.nx2 > 0 && lu < ntile + (sc.nx1 > 0 ? ntile : 0))) {
    // a tile of an x slab
    const bool second = !(sc.nx1 > 0 && lu < ntile);
    if (second && sc.nx1 > 0) lu -= ntile;
    r.j0 = (lu % sc.ntj) * TJ;
    r.k0 = (lu / sc.ntj) * TK;
    r.ib = second ? d.ni - sc.nx2 : 0;
    r.ie = second ? d.ni : sc.nx1;
    r.face = second ? 1 : 0;
    r.jhi = d.nj;
    r.khi = sc.ktop;
    return r;
  }
  if (sc.nx1 > 0) lu -= ntile;
  if (sc.nx2 > 0) lu -= ntile;
  const int c = lu / sc.nedge;
  int e = lu % sc.nedge;
  r.ib = sc.nx1 + c * sc.ci;
  r.ie = min(r.ib + sc.ci, d.ni - sc.nx2);
  const int ns = sc.ny1 + sc.ny2;
  if (e < ns * sc.nrs) {
    // a strip tile of a y slab
    const int st = e % ns;
    r.strip = true;
    r.j0 = st < sc.ny1 ? st * STRIP : sc.yb + (st - sc.ny1) * STRIP;
    r.k0 = (e / ns) * STRIP;
    r.jhi = d.nj;
    r.khi = sc.ktop;
    r.face = (a.aux[2] && r.j0 < d.N) ? 2 : (a.aux[3] && r.j0 + STRIP > d.nj - d.N) ? 3 : -1;
    return r;
  }
  // a tile of a z slab
  e -= ns * sc.nrs;
  const int zt = e % sc.ntz, zr = e / sc.ntz;
  r.j0 = sc.ya + zt * TJ;
  r.jhi = sc.yb;
  if (zr < sc.nz1) {
    r.k0 = zr * TK;
    r.khi = sc.za;
  } else {
    r.k0 = sc.zb + (zr - sc.nz1) * TK;
    r.khi = sc.ktop;
  }
  r.face = (a.aux[4] && r.k0 < d.N) ? 4 : (a.aux[5] && r.k0 + TK > d.nk - d.N) ? 5 : -1;
  return r;
}

// Block of the ADE state staged in slot n (0..2) of a pointwise slot at stage irk: the
// current value, then y0 (stages 1, 2) or the accumulator (stage 3), then y1 (stage 2).
__host__ __device__ constexpr int aux_block(int irk, int n) {
  return n == 0 ? aux_cur(irk) : n == 1 ? (irk == 3 ? 2 : 0) : 1;
}

// ADE update of face `face` for fields F0..F0+2 at this node (pml_update of
// dfd_stencil.cuh, restricted to three fields): adds -aux/beta to the rates p and advances
// the state with the RK4 blocks of aux_cur.  The state comes from shared memory (A, the
// staged own face, in the order of aux_block) or from global memory; every load precedes
// the stores, which may alias them as far as the compiler knows.
template <int F0, int AX, int IRK>
__device__ __forceinline__ void role_face(const VolArgs& a, int face, bool staged, const float* A, int i, int j,
                                          int k, float rb, float dd, float al, const float* D, float* p) {
  const Dims& d = a.d;
  // face is 2 AX or 2 AX + 1: the layout branch of pml_index is known here
  const long long fs = pml_fstride(d, 2 * AX);
  long long qa;
  if (AX == 0) {
    const int ia = face == 0 ? i : i - (d.ni - d.N);
    qa = (long long)(j + 3 + d.oy) + (long long)(k + 3) * d.py + (long long)ia * d.sx;
  } else if (AX == 1) {
    const int c = j + 3 + d.oy - (face == 2 ? 0 : d.yb3);
    qa = (long long)c + (long long)(k + 3) * d.wy + (long long)i * d.wy * d.nz;
  } else {
    const int kz = face == 4 ? k : k - (d.nk - d.N);
    qa = (long long)(j + 3 + d.oy) + (long long)kz * d.py + (long long)i * d.py * d.N;
  }
  float* base = a.aux[face];
  constexpr int irk = IRK;
  const long long b9 = 9 * fs;
  const float ad = -(al + dd);
  float w[3], s2[3], y1[3];  // current value; y0 or the accumulator; y1
#pragma unroll
  for (int m = 0; m < 3; m++) {
    const int f = F0 + m;
    if (staged) {
      w[m] = A[f * PB];
      if (irk >= 1) s2[m] = A[(9 + f) * PB];
      if (irk == 2) y1[m] = A[(18 + f) * PB];
    } else {
      const float* x = base + f * fs + qa;
      if (irk == 0) {
        w[m] = x[0];
      } else if (irk == 1) {
        w[m] = x[b9];
        s2[m] = x[0];
      } else if (irk == 2) {
        w[m] = x[2 * b9];
        s2[m] = x[0];
        y1[m] = x[b9];
      } else {
        w[m] = x[b9];
        s2[m] = x[2 * b9];
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 3; m++) {
    float* x = base + (F0 + m) * fs + qa;
    p[m] += -w[m] * rb;
    const float h = ad * w[m] + dd * D[m];
    if (irk == 0) {
      x[b9] = fmaf(a.rka, h, w[m]);
    } else if (irk == 1) {
      x[2 * b9] = fmaf(a.rka, h, s2[m]);
    } else if (irk == 2) {
      x[2 * b9] = rk_acc(s2[m], rk_sum(s2[m], y1[m], w[m], 1.0f), a.rkb, h);
      x[b9] = fmaf(a.rka, h, s2[m]);
    } else {
      x[0] = fmaf(a.rkb, h, s2[m]);
    }
  }
}

// axis contribution (axis_terms of dfd_stencil.cuh) to fields F0..F0+2 from the
// derivatives dv[] along one axis (metric row e0 e1 e2; X0: the row has an x component --
// the y and z rows of the separable metric have none).  F0 = 0: dv = d(Txx Tyy Tzz Txy Txz
// Tyz); F0 = 3 (normal stresses) or 6 (shear stresses): dv = d(Vx Vy Vz).
template <int F0, bool X0>
__device__ __forceinline__ void role_terms(const float* dv, float e0, float e1, float e2, float lam, float mu,
                                           float rr, float* D) {
  if (F0 == 0) {
    if (X0) {
      D[0] = (dv[0] * e0 + dv[3] * e1 + dv[4] * e2) * rr;
      D[1] = (dv[3] * e0 + dv[1] * e1 + dv[5] * e2) * rr;
      D[2] = (dv[4] * e0 + dv[5] * e1 + dv[2] * e2) * rr;
    } else {
      D[0] = (dv[3] * e1 + dv[4] * e2) * rr;
      D[1] = (dv[1] * e1 + dv[5] * e2) * rr;
      D[2] = (dv[5] * e1 + dv[2] * e2) * rr;
    }
  } else if (F0 == 3) {
    const float l2m = lam + 2.0f * mu;
    if (X0) {
      D[0] = dv[0] * e0 * l2m + dv[1] * e1 * lam + dv[2] * e2 * lam;
      D[1] = dv[0] * e0 * lam + dv[1] * e1 * l2m + dv[2] * e2 * lam;
      D[2] = dv[0] * e0 * lam + dv[1] * e1 * lam + dv[2] * e2 * l2m;
    } else {
      D[0] = dv[1] * e1 * lam + dv[2] * e2 * lam;
      D[1] = dv[1] * e1 * l2m + dv[2] * e2 * lam;
      D[2] = dv[1] * e1 * lam + dv[2] * e2 * l2m;
    }
  } else {
    if (X0) {
      D[0] = (dv[0] * e1 + dv[1] * e0) * mu;
      D[1] = (dv[0] * e2 + dv[2] * e0) * mu;
      D[2] = (dv[1] * e2 + dv[2] * e1) * mu;
    } else {
      D[0] = (dv[0] * e1) * mu;
      D[1] = (dv[0] * e2) * mu;
      D[2] = (dv[1] * e2 + dv[2] * e1) * mu;
    }
  }
}

// One node, all nine fields: the three axes with their 1/beta, the ADE state of the faces
// the node lies in (fx, fy, fz; -1: none; own: the staged face, read from A), the RK4
// store.  PW: row pitch of the stencil box (40 for 32 x 8 tiles, 24 for strips).  g: separable metric (xi = (1, U, V)/a(x), eta = (0, ety, etz), zeta = (0, zty,
// ztz)) and media.
// one-sided 5-point operator along a shared-memory line with a runtime stride
template <int F>
__device__ __forceinline__ float d5r(const float* p, int S) {
  if (F == 1) return d5v<1>(p[-S], p[0], p[S], p[2 * S], p[3 * S]);
  else return d5v<-1>(p[-3 * S], p[-2 * S], p[-S], p[0], p[S]);
}

// the y and z PML factors of a node (1/beta, d, alpha): fixed over a unit, loaded once per
// unit so that no global load waits inside the plane loop
struct YZFactors {
  float rby, ddy, aly, rbz, ddz, alz;
};

template <int FX, int FY, int FZ, int IRK>
__device__ __forceinline__ void pml_node(const VolArgs& a, int PW, const float* x0, const float* x1, const float* x2,
                                         const float* x3, const float* x4, const float* cur, const NodeMetric& g,
                                         int i, int j, int k, int fx, int fy, int fz, int own, const float* A,
                                         long long q, const float* P, float damp, float rbx, float ddx, float alx,
                                         const YZFactors& yz) {
  const float r = a.rDH;
  float hv[9], D[9], dv[9];
  // x
  {
#pragma unroll
    for (int f = 0; f < 9; f++) {
      const int o = f * HBOX;
      dv[f] = d5v<FX>(x0[o], x1[o], x2[o], x3[o], x4[o]) * r;
    }
    role_terms<0, true>(dv + 3, g.ex0, g.ex1, g.ex2, g.lam, g.mu, g.rrho, D);
    role_terms<3, true>(dv, g.ex0, g.ex1, g.ex2, g.lam, g.mu, g.rrho, D + 3);
    role_terms<6, true>(dv, g.ex0, g.ex1, g.ex2, g.lam, g.mu, g.rrho, D + 6);
    const float rb = rbx;
#pragma unroll
    for (int f = 0; f < 9; f++) hv[f] = D[f] * rb;
    if (fx >= 0) {
      const bool st = fx == own;
      const float dd = ddx, al = alx;
      role_face<0, 0, IRK>(a, fx, st, A, i, j, k, rb, dd, al, D, hv + 0);
      role_face<3, 0, IRK>(a, fx, st, A, i, j, k, rb, dd, al, D + 3, hv + 3);
      role_face<6, 0, IRK>(a, fx, st, A, i, j, k, rb, dd, al, D + 6, hv + 6);
    }
  }
  // y
  {
#pragma unroll
    for (int f = 0; f < 9; f++) dv[f] = d5s<FY, 1>(cur + f * HBOX) * r;
    role_terms<0, false>(dv + 3, 0.0f, g.ey1, g.ey2, g.lam, g.mu, g.rrho, D);
    role_terms<3, false>(dv, 0.0f, g.ey1, g.ey2, g.lam, g.mu, g.rrho, D + 3);
    role_terms<6, false>(dv, 0.0f, g.ey1, g.ey2, g.lam, g.mu, g.rrho, D + 6);
    const float rb = yz.rby;
#pragma unroll
    for (int f = 0; f < 9; f++) hv[f] += D[f] * rb;
    if (fy >= 0) {
      const bool st = fy == own;
      const float dd = yz.ddy, al = yz.aly;
      role_face<0, 1, IRK>(a, fy, st, A, i, j, k, rb, dd, al, D, hv + 0);
      role_face<3, 1, IRK>(a, fy, st, A, i, j, k, rb, dd, al, D + 3, hv + 3);
      role_face<6, 1, IRK>(a, fy, st, A, i, j, k, rb, dd, al, D + 6, hv + 6);
    }
  }
  // z
  {
#pragma unroll
    for (int f = 0; f < 9; f++) dv[f] = d5r<FZ>(cur + f * HBOX, PW) * r;
    role_terms<0, false>(dv + 3, 0.0f, g.ez1, g.ez2, g.lam, g.mu, g.rrho, D);
    role_terms<3, false>(dv, 0.0f, g.ez1, g.ez2, g.lam, g.mu, g.rrho, D + 3);
    role_terms<6, false>(dv, 0.0f, g.ez1, g.ez2, g.lam, g.mu, g.rrho, D + 6);
    const float rb = yz.rbz;
#pragma unroll
    for (int f = 0; f < 9; f++) hv[f] += D[f] * rb;
    if (fz >= 0) {
      const bool st = fz == own;
      const float dd = yz.ddz, al = yz.alz;
      role_face<0, 2, IRK>(a, fz, st, A, i, j, k, rb, dd, al, D, hv + 0);
      role_face<3, 2, IRK>(a, fz, st, A, i, j, k, rb, dd, al, D + 3, hv + 3);
      role_face<6, 2, IRK>(a, fz, st, A, i, j, k, rb, dd, al, D + 6, hv + 6);
    }
  }
  rk_tile_store<0, 9, IRK>(a, a.d.nxyz, q, cur, P, hv, damp);
}

// Warp PCW issues the copies; warps 0..PCW-1 compute, one per row of nodes, all nine
// fields (the lean interior path for a warp whose nodes lie in no PML slab).  The nine warps
// allow 168 registers a thread (three warps on one of the SM's four 16 K-register
// partitions), what the ADE path needs without spilling.  Rings as in the interior
// kernel, with shallower rings (PmlRing): a pointwise slot also holds the own face's ADE
// state.
// IRK: the RK stage, compiled per stage as in the interior kernel.  BATCH: the units of
// the nscen scenarios of tab in one launch; mp0, a0, sc0 describe scenario 0 and give the
// stage's common values.
template <int FX, int FY, int FZ, int IRK, bool BATCH>
__global__ void __maxnreg__(168)
    volume_pml_kernel(const __grid_constant__ TileMaps mp0, const __grid_constant__ VolArgs a0,
                      const __grid_constant__ TileSched sc0, const TileScen* __restrict__ tab, int nscen, int nunits,
                      int* err, int* sched) {
  using RG = PmlRing<IRK>;
  constexpr int MS = RG::MS, MP = RG::MP, MQ = RG::MQ, PSLOT = RG::PSLOT;
  extern __shared__ __align__(1024) unsigned char smraw[];
  float* win = reinterpret_cast<float*>(smraw);
  float* pw = win + MS * HSLOT;
  float* qs = pw + MP * PSLOT;
  TileUnit* uarg = reinterpret_cast<TileUnit*>(qs + MQ * QSLOT);
  uint64_t* full_w = reinterpret_cast<uint64_t*>(uarg + MQ);
  uint64_t* empty_w = full_w + MS;
  uint64_t* full_p = empty_w + MS;
  uint64_t* empty_p = full_p + MP;
  uint64_t* full_q = empty_p + MP;
  uint64_t* empty_q = full_q + MQ;
  int* qunit = reinterpret_cast<int*>(empty_q + MQ);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int XLO = FX == 1 ? -1 : -3;
  constexpr int RZ = FZ == 1 ? 1 : 3;
  constexpr int irk = IRK;
  // pointwise boxes as in the interior kernel: y0 at stages 1 and 2, the second box (the
  // stage-1 input, the accumulator) at stages 2 and 3
  constexpr bool needW0 = RG::W0, needT = RG::T;
  constexpr int naux = RG::NAUX;
  const int G = gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < MS; s++) { mbar_init(full_w + s, 1); mbar_init(empty_w + s, PCW); }
    for (int s = 0; s < MP; s++) { mbar_init(full_p + s, 1); mbar_init(empty_p + s, PCW); }
    for (int s = 0; s < MQ; s++) { mbar_init(full_q + s, 1); mbar_init(empty_q + s, PCW); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_async_shared();
  }
  __syncthreads();

  if (warp == PCW) {
    // ---------------- copy-issuing warp (one lane)
    if (lane != 0) return;
    Ring wr, pr, qr;
    int wcount = 0, pcount = 0, qcount = 0;
    bool ok = true;
    while (ok) {
      const int u = atomicAdd(sched, 1);
      if (qcount >= MQ && !(ok = mbar_wait(empty_q + qr.slot, qr.phase ^ 1))) break;
      if (u >= nunits) {
        qunit[qr.slot] = -1;
        mbar_arrive(full_q + qr.slot);
        break;
      }
      const int scn = BATCH ? tile_scenario(tab, nscen, u) : 0;
      const TileMaps& mp = BATCH ? tab[scn].mp : mp0;
      const VolArgs& a = BATCH ? tab[scn].u.a : a0;
      const TileSched& sc = BATCH ? tab[scn].u.sc : sc0;
      const Dims& d = a.d;
      const PmlUnit pu = pml_unit(sc, a, BATCH ? u - tab[scn].u.unit0 : u);
      const int cw0 = pu.j0 + 3 + d.oy - 4, cw1 = pu.k0 + 3 - RZ, cp0 = pu.j0 + 3 + d.oy, cp1 = pu.k0 + 3;
      const int nst = pu.ie - pu.ib;
      const int na = pu.face >= 0 ? naux : 0;
      const bool usep = needW0 || needT || na > 0;
      const unsigned ptx = ((needW0 ? 9 : 0) + (needT ? 9 : 0) + na) * PB * 4;
      // own-face state coordinates: column, row, plane offset
      int ac0 = cp0, ac1 = cp1, aoff = 0;
      if (pu.face == 1) aoff = d.ni - d.N;
      if (pu.face == 3) ac0 = cp0 - d.yb3;
      if (pu.face == 4) ac1 = pu.k0;
      if (pu.face == 5) ac1 = pu.k0 - (d.nk - d.N);
      // the unit's maps: 32 x 8 tiles or 16 x 16 strips (same box sizes in floats)
      const CUtensorMap* m_win = pu.strip ? &mp.win_s : &mp.win;
      const CUtensorMap* m_w0 = pu.strip ? &mp.w0_s : &mp.w0;
      const CUtensorMap* m_t = pu.strip ? &mp.t_s : &mp.t;
      const CUtensorMap* m_aux = pu.face < 0 ? nullptr : pu.strip ? &mp.auxy_s[pu.face - 2] : &mp.aux[pu.face];
      qunit[qr.slot] = u;
      if (BATCH) {
        mbar_expect_tx(full_q + qr.slot, QSLOT * 4 + (unsigned)sizeof(TileUnit));
        bulk_load(uarg + qr.slot, &tab[scn].u, (unsigned)sizeof(TileUnit), full_q + qr.slot);
      } else {
        mbar_expect_tx(full_q + qr.slot, QSLOT * 4);
      }
      tma_load3(qs + qr.slot * QSLOT, pu.strip ? &mp.plane_s : &mp.plane, cp0, cp1, 0, full_q + qr.slot);
      qr.next<MQ>();
      qcount++;
      for (int m = 0; m < nst + 4 && ok; m++) {
        if (wcount >= MS && !(ok = mbar_wait(empty_w + wr.slot, wr.phase ^ 1))) break;
        mbar_expect_tx(full_w + wr.slot, HSLOT * 4);
        tma_load4(win + wr.slot * HSLOT, m_win, cw0, cw1, pu.ib + XLO + m + 3, 0, full_w + wr.slot);
        wr.next<MS>();
        wcount++;
        if (m < 4 || !usep) continue;
        if (pcount >= MP && !(ok = mbar_wait(empty_p + pr.slot, pr.phase ^ 1))) break;
        uint64_t* b = full_p + pr.slot;
        float* dst = pw + pr.slot * PSLOT;
        const int i = pu.ib + (m - 4);
        mbar_expect_tx(b, ptx);
        if (needW0) tma_load4(dst, m_w0, cp0, cp1, i + 3, 0, b);
        if (needT) tma_load4(dst + RG::TOFF * PB, m_t, cp0, cp1, i + 3, 0, b);
        for (int nb = 0; nb * 9 < na; nb++)
          tma_load4(dst + (RG::AOFF + 9 * nb) * PB, m_aux, ac0, ac1, i - aoff, 9 * aux_block(irk, nb), b);
        pr.next<MP>();
        pcount++;
      }
    }
    if (!ok) {
      atomicExch(err, 1);
      for (int c = max(0, wcount - MS); c < wcount; c++) mbar_wait(full_w + c % MS, (c / MS) & 1);
      for (int c = max(0, pcount - MP); c < pcount; c++) mbar_wait(full_p + c % MP, (c / MP) & 1);
      for (int c = max(0, qcount - MQ); c < qcount; c++) mbar_wait(full_q + c % MQ, (c / MQ) & 1);
    }
    __threadfence();
    if (atomicAdd(sched + 1, 1) == G - 1) {
      atomicExch(sched, 0);
      atomicExch(sched + 1, 0);
    }
    // launched behind the interior kernel (programmatic serialisation), this grid must not
    // complete before that one: what follows on the stream relies on both
    asm volatile("griddepcontrol.wait;" ::: "memory");
    return;
  }

  // ---------------- computing warps.  32 x 8 tiles: warp = row, lane = column.  16 x 16
  // strips: the two half-warps take rows two apart (their stencil rows then fall on
  // disjoint shared-memory banks), lane & 15 the column.
  const int hl = lane >> 4, jl = lane & 15;
  const int srow = (warp >> 1) * 4 + (warp & 1) + 2 * hl;
  Ring wr, pr, qr;
  int sb = 0;
  for (;;) {
    if (!__all_sync(0xffffffffu, mbar_wait(full_q + qr.slot, qr.phase))) {
      if (lane == 0) atomicExch(err, 1);
      return;
    }
    const int u = qunit[qr.slot];
    if (u < 0) break;
    const TileUnit& ua = uarg[qr.slot];
    const VolArgs& a = BATCH ? ua.a : a0;
    const TileSched& sc = BATCH ? ua.sc : sc0;
    const Dims& d = a.d;
    const PmlUnit pu = pml_unit(sc, a, BATCH ? u - ua.unit0 : u);
    const int row = pu.strip ? srow : warp, col = pu.strip ? jl : lane;
    const int hc = pu.strip ? (row + RZ) * (STRIP + 8) + col + 4 : (row + RZ) * HW + col + 4;
    const int pc = pu.strip ? row * STRIP + col : row * TJ + col;
    const int j = pu.j0 + col, k = pu.k0 + row;
    const bool active = j < pu.jhi && k < pu.khi;
    const bool band = active && a.united && !a.united[j + k * d.nj];
    const int fy = (a.aux[2] && j < d.N) ? 2 : (a.aux[3] && j >= d.nj - d.N) ? 3 : -1;
    const int fz = (a.aux[4] && k < d.N) ? 4 : (a.aux[5] && k >= d.nk - d.N) ? 5 : -1;
    float dyz = 1.0f;
    if (active && a.dampx) dyz = fminf(__ldg(a.dampy + j + 3), __ldg(a.dampz + k + 3));
    YZFactors yz = {1.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f};
    if (active) {
      yz.rby = __ldg(a.rBy + j);
      yz.rbz = __ldg(a.rBz + k);
      if (fy >= 0) { yz.ddy = __ldg(a.Dpy + j); yz.aly = __ldg(a.Apy + j); }
      if (fz >= 0) { yz.ddz = __ldg(a.Dpz + k); yz.alz = __ldg(a.Apz + k); }
    }
    const long long qyz = idx3(d, 0, j + 3, k + 3);
    const int nst = pu.ie - pu.ib;
    const bool usep = needW0 || needT || pu.face >= 0;
    const float* Q = qs + qr.slot * QSLOT + pc;
    // per-plane 1-D factors, loaded one plane ahead so that their latency overlaps a plane
    float nx_rA = __ldg(a.rxa + pu.ib + 3), nx_dx = a.dampx ? __ldg(a.dampx + pu.ib + 3) : 1.0f;
    float nx_rb = __ldg(a.rBx + pu.ib), nx_dd = __ldg(a.Dpx + pu.ib), nx_al = __ldg(a.Apx + pu.ib);
    for (int s = 0; s < nst; s++) {
      bool ok = true;
      for (int c = s == 0 ? 5 : 1; c > 0; c--) {
        ok = ok && mbar_wait(full_w + wr.slot, wr.phase);
        wr.next<MS>();
      }
      if (usep) ok = ok && mbar_wait(full_p + pr.slot, pr.phase);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(err, 1);
        return;
      }
      const int i = pu.ib + s;
      const float* P = pw + pr.slot * PSLOT + pc;
      const float rA = nx_rA, dx = nx_dx, rbx = nx_rb, ddx = nx_dd, alx = nx_al;
      if (s + 1 < nst) {
        nx_rA = __ldg(a.rxa + i + 4);
        if (a.dampx) nx_dx = __ldg(a.dampx + i + 4);
        nx_rb = __ldg(a.rBx + i + 1);
        nx_dd = __ldg(a.Dpx + i + 1);
        nx_al = __ldg(a.Apx + i + 1);
      }
      const bool node = active && !(band && i + 3 >= d.i0 - 3 && i + 3 <= d.i0 + 3);
      const int fx = (a.aux[0] && i < d.N) ? 0 : (a.aux[1] && i >= d.ni - d.N) ? 1 : -1;
      // a warp none of whose nodes lies in a PML slab in this plane takes the lean path
      const bool pml = __any_sync(0xffffffffu, node && (fx >= 0 || fy >= 0 || fz >= 0));
      if (node) {
        const int s1 = sb + 1 == MS ? 0 : sb + 1;
        const int s2 = s1 + 1 == MS ? 0 : s1 + 1;
        const int s3 = s2 + 1 == MS ? 0 : s2 + 1;
        const int s4 = s3 + 1 == MS ? 0 : s3 + 1;
        const float* x0 = win + sb * HSLOT + hc;
        const float* x1 = win + s1 * HSLOT + hc;
        const float* x2 = win + s2 * HSLOT + hc;
        const float* x3 = win + s3 * HSLOT + hc;
        const float* x4 = win + s4 * HSLOT + hc;
        const float* cur = FX == 1 ? x1 : x3;
        NodeMetric g;
        g.ex0 = rA; g.ex1 = Q[0] * rA; g.ex2 = Q[PB] * rA;
        g.ey1 = Q[2 * PB]; g.ey2 = Q[3 * PB]; g.ez1 = Q[4 * PB]; g.ez2 = Q[5 * PB];
        const int side = i + 3 < a.nxhalf ? 6 : 9;
        g.lam = Q[side * PB]; g.mu = Q[(side + 1) * PB]; g.rrho = 1.0f / Q[(side + 2) * PB];
        const float damp = a.dampx ? fminf(dx, dyz) : 1.0f;
        const long long q = qyz + (long long)(i + 3) * d.sx;
        if (pu.strip || pml) {
          // (strips hold y-slab nodes and the few interior columns beside them)
          pml_node<FX, FY, FZ, IRK>(a, pu.strip ? STRIP + 8 : HW, x0, x1, x2, x3, x4, cur, g, i, j, k, fx, fy, fz, pu.face,
                               P + RG::AOFF * PB, q, P, damp, rbx, ddx, alx, yz);
        } else {
          float hv[9];
          lean_velocity<FX, FY, FZ>(x0, x1, x2, x3, x4, cur, g, a.rDH, hv);
          lean_stress<FX, FY, FZ>(x0, x1, x2, x3, x4, cur, g, a.rDH, hv);
          rk_tile_store<0, 9, IRK>(a, d.nxyz, q, cur, P, hv, damp);
        }
      }
      __syncwarp();
      if (lane == 0) {
        if (s + 1 < nst) {
          mbar_arrive(empty_w + sb);
        } else {
          for (int m = 0, sl = sb; m < 5; m++, sl = sl + 1 == MS ? 0 : sl + 1) mbar_arrive(empty_w + sl);
          mbar_arrive(empty_q + qr.slot);
        }
        if (usep) mbar_arrive(empty_p + pr.slot);
      }
      if (usep) pr.next<MP>();
      sb += s + 1 < nst ? 1 : 5;
      if (sb >= MS) sb -= MS;
    }
    qr.next<MQ>();
  }
}

// ---------------- host side

template <int FX, int FY, int FZ, int IRK>
static bool pml_smem_k() {
  auto one = [](const void* f) {
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PmlRing<IRK>::SMEM) ==
           cudaSuccess;
  };
  return one((const void*)volume_pml_kernel<FX, FY, FZ, IRK, false>) &&
         one((const void*)volume_pml_kernel<FX, FY, FZ, IRK, true>);
}
template <int FX, int FY, int FZ>
static bool pml_smem() {
  return pml_smem_k<FX, FY, FZ, 0>() && pml_smem_k<FX, FY, FZ, 1>() && pml_smem_k<FX, FY, FZ, 2>() &&
         pml_smem_k<FX, FY, FZ, 3>();
}

bool pml_setup() {
  return pml_smem<-1, -1, -1>() && pml_smem<-1, -1, 1>() && pml_smem<-1, 1, -1>() && pml_smem<-1, 1, 1>() &&
         pml_smem<1, -1, -1>() && pml_smem<1, -1, 1>() && pml_smem<1, 1, -1>() && pml_smem<1, 1, 1>();
}

// Units around the interior box [nx1, ni - nx2) x [ya, yb) x [za, zb): the x slabs
// whole, then the y strips and z tiles of the middle x range in chunks chosen as in
// tile_plan.  ya is a multiple of 16 (the y1 strips end there), yb a multiple of 4 (the
// y2 strips start there); ya == yb: no interior columns, the strips take every column
// from 0; za == zb: no interior rows, the z tiles take every row from 0.  nunits 0 when
// there is nothing to do, -1 when the x slabs overlap (the general kernel then takes all).
TileSched pml_plan(const VolArgs& a, int ya, int yb, int za, int zb, int ktop, int nsm, int* grid) {
  const Dims& d = a.d;
  TileSched s;
  memset(&s, 0, sizeof s);
  s.ntj = (d.nj + TJ - 1) / TJ;
  s.ntk = (ktop + TK - 1) / TK;
  s.nx1 = a.aux[0] ? d.N : 0;
  s.nx2 = a.aux[1] ? d.N : 0;
  s.ktop = ktop;
  s.ya = ya; s.yb = yb; s.za = za; s.zb = zb;
  *grid = 0;
  if (s.nx1 + s.nx2 > d.ni || ktop <= 0) {
    s.nunits = -1;
    return s;
  }
  s.ny1 = ya / STRIP;
  s.ny2 = (d.nj - yb + STRIP - 1) / STRIP;
  s.nrs = (ktop + STRIP - 1) / STRIP;
  s.ntz = (yb - ya + TJ - 1) / TJ;
  s.nz1 = (za + TK - 1) / TK;
  s.nz2 = (ktop - zb + TK - 1) / TK;
  s.nedge = (s.ny1 + s.ny2) * s.nrs + s.ntz * (s.nz1 + s.nz2);
  const int ntile = s.ntj * s.ntk;
  const int slab = (s.nx1 > 0 ? ntile : 0) + (s.nx2 > 0 ? ntile : 0);
  const int nxm = d.ni - s.nx1 - s.nx2;
  s.ci = std::max(nxm, 1);
  s.nunits = slab;
  if (nxm > 0 && s.nedge > 0) {
    long long best = -1;
    for (int nch = 1; nch <= 64 && nch <= nxm; nch++) {
      int ci = (nxm + nch - 1) / nch;
      int nchr = (nxm + ci - 1) / ci;
      long long units = (long long)s.nedge * nchr + slab;
      long long g = std::min<long long>(units, nsm);
      long long cost = (units + g - 1) / g * (ci + 4);
      if (best < 0 || cost < best) { best = cost; s.ci = ci; s.nunits = (int)units; }
    }
  }
  *grid = std::min(s.nunits, nsm);
  return s;
}

// pdl: launched with programmatic stream serialisation right behind the interior kernel,
// whose CTAs allow it at their start; the two grids update disjoint nodes of the stage.
// The PML kernel takes the second pair of the 4-int counter block sched.
template <int FX, int FY, int FZ, bool BATCH>
static void pml_launch(const TileMaps& mp, const VolArgs& a, const TileSched& sc, const TileScen* tab, int n,
                       int nunits, int grid, int* err, int* sched, bool pdl, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(PTOT);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
#define DFD_L(K)                                   \
  cfg.dynamicSmemBytes = PmlRing<K>::SMEM;         \
  cudaLaunchKernelEx(&cfg, volume_pml_kernel<FX, FY, FZ, K, BATCH>, mp, a, sc, tab, n, nunits, err, sched + 2)
  DFD_BY_STAGE(a.irk, DFD_L);
#undef DFD_L
}

template <int FX, int FY, int FZ>
static void launch_p(const TileCtx& tc, const VolArgs& a, int bin, const TileSched& ps, int grid, bool pdl,
                     cudaStream_t s) {
  const TileMaps mp = tile_maps(tc, bin, a.irk, tc.tr);
  pml_launch<FX, FY, FZ, false>(mp, a, ps, nullptr, 1, ps.nunits, grid, tc.err, tc.sched, pdl, s);
}

void launch_pml(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, const TileSched& ps, int grid,
                bool pdl, cudaStream_t s) {
  if (ps.nunits <= 0 || grid <= 0) return;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_p<-1, -1, -1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 1: launch_p<-1, -1, 1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 2: launch_p<-1, 1, -1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 3: launch_p<-1, 1, 1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 4: launch_p<1, -1, -1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 5: launch_p<1, -1, 1>(*tc, a, bin, ps, grid, pdl, s); break;
    case 6: launch_p<1, 1, -1>(*tc, a, bin, ps, grid, pdl, s); break;
    default: launch_p<1, 1, 1>(*tc, a, bin, ps, grid, pdl, s); break;
  }
}

template <int FX, int FY, int FZ>
static void launch_pb(const TileScen& f, const TileScen* tab, int n, int nunits, int grid, int* err, int* sched,
                      bool pdl, cudaStream_t s) {
  pml_launch<FX, FY, FZ, true>(f.mp, f.u.a, f.u.sc, tab, n, nunits, grid, err, sched, pdl, s);
}
void launch_pml_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int FX, int FY, int FZ,
                      int* err, int* sched, bool pdl, cudaStream_t s) {
  if (nunits <= 0 || grid <= 0) return;
  int code = (FX > 0) * 4 + (FY > 0) * 2 + (FZ > 0);
  switch (code) {
    case 0: launch_pb<-1, -1, -1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 1: launch_pb<-1, -1, 1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 2: launch_pb<-1, 1, -1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 3: launch_pb<-1, 1, 1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 4: launch_pb<1, -1, -1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 5: launch_pb<1, -1, 1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    case 6: launch_pb<1, 1, -1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
    default: launch_pb<1, 1, 1>(first, tab, n, nunits, grid, err, sched, pdl, s); break;
  }
}

}  // namespace dfd
