// Internal definitions shared by the CUDA kernels and the host side of the
// B200 dynamic-rupture time step.
//
// HBM layout (per context, all FP32 unless noted):
//   W[4]      four 9-field volume buffers (nx, nz, py), y fastest, 3 ghost nodes;
//             a step cycles A -> B -> C -> B -> A so that the stencil input of a stage is
//             never written during that stage and no right-hand-side array exists
//   M         13 fields xix xiy xiz etx ety etz ztx zty ztz jac lam mu rho, same layout
//   aux       per PML face, 3 blocks of 9 fields cycled through the RK stages (aux_cur)
//   FW[2]     split-node state ping-pong (9, 2, nz, ny); Fm / Ft RK registers
//   tables    fault coefficient tables as planes [table][element][nz*ny] (coalesced)
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace dfd {

// 5-point one-sided DRP (MacCormack-type) coefficients and the traction-image
// coefficients (reference macdrp.h:23-40), with the 2-/3-point boundary operators
// (macdrp.h:101-130).
#define DFD_C1 0.29164704779069994f
#define DFD_C2 0.66674514216519998f
#define DFD_C3 1.2501177132452999f
#define DFD_C4 0.33341180882999999f
#define DFD_C5 0.041686285540599999f
#define DFD_A0P (-1.250039237746600f)
#define DFD_A0M (1.250039237746600f)
#define DFD_A1 1.541764761036000f
#define DFD_A2 (-0.333411808829999f)
#define DFD_A3 0.0416862855405999f
#define DFD_C24_1 (7.0f / 6.0f)
#define DFD_C24_2 (4.0f / 3.0f)
#define DFD_C24_3 (1.0f / 6.0f)

// fault coefficient table planes (index t of ntab, each 9 elements per node unless noted)
enum Tab {
  T_D21_1 = 0, T_D22_1, T_D23_1, T_D31_1, T_D32_1, T_D33_1,
  T_D21_2, T_D22_2, T_D23_2, T_D31_2, T_D32_2, T_D33_2,
  T_M2P1, T_M2P2, T_M2P3, T_M2P4, T_M2P5,
  T_P2M1, T_P2M2, T_P2M3, T_P2M4, T_P2M5,
  T_T1VXM, T_VYVXM, T_VZVXM, T_T1VXP, T_VYVXP, T_VZVXP,
  NTAB9
};
// free-surface row tables, 9 elements per j
enum TabF { TF_VX2VZ1 = 0, TF_VY2VZ1, TF_VX2VZ2, TF_VY2VZ2, TF_P2M1, TF_P2M2, TF_P2M3, TF_M2P1, TF_M2P2, TF_M2P3, NTABF };

// The volume buffer cycle of a step: stage inputs A B C B, outputs B C B A (buffers 0..2),
// buffer 3 the RK accumulator.
__host__ __device__ constexpr int stage_in(int irk) { return irk == 0 ? 0 : irk == 2 ? 2 : 1; }
__host__ __device__ constexpr int stage_out(int irk) { return irk == 1 ? 2 : irk == 3 ? 0 : 1; }

// Volume fields are stored with a padded row pitch: node (i, j, k) (padded indices, 3 ghost
// nodes per side) of a field sits at element (j + oy) + k*py + i*sx.  The row offset oy = 1
// puts the first interior node of every row (j = 3) on a 16-byte boundary and the pitch
// py >= ny + 1 is a multiple of 8, as tiled TMA loads need.  Fault-plane arrays keep the
// dense (nz, ny) layout.
struct Dims {
  int ni, nj, nk;       // interior sizes NX NY NZ
  int nx, ny, nz;       // padded sizes
  int i0;               // padded x index of the fault plane (nx/2)
  int N;                // PML thickness
  int py, oy;           // volume row pitch and row offset (elements)
  long long sx;         // volume x stride, py * nz
  long long nxyz;       // volume field size, sx * nx
  long long nyz;        // fault-plane size, ny * nz
  int wy;               // row width of the y-face PML state (N + 4 rounded up to 4)
  int yb3;              // first stored column of the y2-face PML state (a multiple of 4)
};

// ADE state of PML face f (x1 x2 y1 y2 z1 z2): 27 fields per face, three blocks of nine
// (0..8, 9..17, 18..26) that hold the step-start value, the stage values and the RK
// accumulator in turn (aux_cur, dfd_stencil.cuh), each field pml_fstride apart.  The layouts keep the volume's row frame, so
// that a 32 x 8 tile of nodes is one TMA box at a 16-byte aligned column:
//   x faces: N planes of (nz rows, py columns), column j + 3 + oy, row k + 3;
//   y faces: ni planes of (nz rows, wy columns), column j + 3 + oy - (0 | yb3), row k + 3;
//   z faces: ni planes of (N rows, py columns), column j + 3 + oy, row k - (0 | nk - N).
__host__ __device__ inline long long pml_fstride(const Dims& d, int f) {
  if (f < 2) return (long long)d.N * d.sx;
  if (f < 4) return (long long)d.ni * d.wy * d.nz;
  return (long long)d.ni * d.py * d.N;
}
__host__ __device__ inline long long pml_index(const Dims& d, int f, int i, int j, int k) {
  if (f < 2) {
    int ia = f == 0 ? i : i - (d.ni - d.N);
    return (long long)(j + 3 + d.oy) + (long long)(k + 3) * d.py + (long long)ia * d.sx;
  }
  if (f < 4) {
    int c = j + 3 + d.oy - (f == 2 ? 0 : d.yb3);
    return (long long)c + (long long)(k + 3) * d.wy + (long long)i * d.wy * d.nz;
  }
  int kz = f == 4 ? k : k - (d.nk - d.N);
  return (long long)(j + 3 + d.oy) + (long long)kz * d.py + (long long)i * d.py * d.N;
}

// Arguments of the fused volume stage kernel.
struct VolArgs {
  Dims d;
  const float* __restrict__ Win;   // stencil input of this stage
  const float* __restrict__ W0;    // step-start state (stages 1, 2)
  float* __restrict__ Wout;        // output of this stage (at stage 2 first read: the stage-1 input)
  float* __restrict__ T;           // RK accumulator (written at stage 2, read at stage 3)
  const float* __restrict__ M;
  const float* __restrict__ rBx;   // 1/beta per axis (PML), 1 outside
  const float* __restrict__ rBy;
  const float* __restrict__ rBz;
  const float* __restrict__ Bx;    // beta per axis
  const float* __restrict__ By;
  const float* __restrict__ Bz;
  const float* __restrict__ Dpx;   // d/beta per axis
  const float* __restrict__ Dpy;
  const float* __restrict__ Dpz;
  const float* __restrict__ Apx;   // alpha per axis
  const float* __restrict__ Apy;
  const float* __restrict__ Apz;
  float* aux[6];                   // PML state per face (x1 x2 y1 y2 z1 z2, 27 fields) or null
  const float* __restrict__ mVx2Vz;  // (nx, ny, 9) free-surface transforms
  const float* __restrict__ mVy2Vz;
  const float* __restrict__ dampx;   // Cerjan 1-D profiles (padded index) or null
  const float* __restrict__ dampy;
  const float* __restrict__ dampz;
  const int* __restrict__ united;    // (NZ, NY) or null when the fault is off
  const float* __restrict__ rxa;     // 1/(d x / d xi) per padded x index (separable metric)
  int nxhalf;                        // bimaterial split: padded x index < nxhalf is side 1
  float rDH, rka, rkb;
  int irk, freenode;
};

// Arguments of the two fault kernels (per-node trial kernel and band kernel).
struct FaultArgs {
  Dims d;
  float* Win;                      // stage input volume (the trial kernel writes W[i0])
  const float* __restrict__ W0;
  float* Wout;
  float* T;
  const float* __restrict__ M;
  const float* __restrict__ mVx2Vz;
  const float* __restrict__ mVy2Vz;
  const float* __restrict__ dampx;
  const float* __restrict__ dampy;
  const float* __restrict__ dampz;
  const float* FWin;               // split nodes, stage input
  float* FWout;                    // split nodes, stage output
  float* Fm;                       // split nodes, step start
  float* Ft;                       // split nodes, RK accumulator
  float* T1;                       // (3, 7, nz, ny) traction layers T11 T12 T13
  float* mT1;                      // (3, nz, ny) T1 at the fault at step start
  float* hT1;                      // (3, nz, ny) T1 rate
  const float* __restrict__ tab;   // NTAB9 * 9 * nyz
  const float* __restrict__ tabf;  // NTABF * 9 * ny
  const float* __restrict__ vecn;  // (3, nz, ny) planes
  const float* __restrict__ vecs1;
  const float* __restrict__ vecs2;
  const float* __restrict__ rhof;  // (2, nz, ny)
  // (NZ, NY) planes
  float *slip, *mslip, *tslip, *hslip, *State, *mState, *tState;
  float *cslip, *cState;           // compensation terms of the step-to-step sums of slip and state
  const float* tpP;                // thermal pressurisation: pore pressure at the fault (plane 0), or null
  float *Vs1, *Vs2, *Tn, *Ts1, *Ts2, *tTn, *tTs1, *tTs2;
  float *sx, *sy, *sz;             // str_init
  const float *T0x, *T0y, *T0z, *dT0x, *dT0y, *dT0z;
  const float *str_peak, *Dc, *C0, *a, *b, *L, *Vw;
  float *init_t0, *friction;
  int *init_t0_flag, *flag_rup;
  const int *united, *faultgrid, *rupy, *rupz;
  // [0] Newton iterations, [1] capped solves, [2] accepted learned guesses, [3] learned
  // guesses that fell back to the plain solve, [4] clock cycles of timed solves, [5] solves
  // timed, [6] largest relative difference of an accepted value from the plain solve (float
  // bits, judge mode), [7] unused
  unsigned long long* newton;
  int prof;                        // time the rate-and-state solve section (clock64)
  int judge;                       // also run the plain solve after a learned one and compare
  double guess_tol;                // residual test of the learned guess: error bound <= guess_tol |x|
  const int* it_dev;               // current step index (device copy, advanced inside graphs)
  const float* guess_net;          // learned-guess MLP weights or null
  float* rec;                      // Newton sample recording buffer (cap x 5) or null
  unsigned* rec_n;                 // samples recorded
  int rec_cap;
  int rec_every;                   // record one solve in rec_every (by node and stage)
  // scalars
  float rDH, DH, DT, rka, rkb, mu_d, viscosity;
  double dDT, smooth_load_T, f0, V0, fw, Vini;
  int it, irk, FX, FY, FZ, freenode, friction_type, inport_stress, NY, NZ, rs_guess;
  int jg0;                         // global column of local column 0 (a slab of a decomposed domain)
};

// The non-united fault nodes, where the fault node kernel works: the rectangle
// 30 < j + 1 < NY - 30, k + 1 > 30 (and k + 1 < NZ - 30 without a free surface)
// (init.cu:806-816).  The kernel numbers its nodes row by row over the rectangle, so that
// every warp but the last holds 32 live nodes.
struct NodeRect {
  int j0, k0, w, h;
  __host__ __device__ long long count() const { return (long long)w * h; }
};
// in the local columns [0, nj) of a slab whose first column is global column jg0 (a domain
// decomposed along y; jg0 = 0, nj = NY for one domain)
__host__ __device__ inline NodeRect node_rect(int NY, int NZ, int freenode, int jg0, int nj) {
  NodeRect r;
  const int jlo = 30 - jg0 > 0 ? 30 - jg0 : 0, jhi = NY - 31 - jg0 < nj ? NY - 31 - jg0 : nj;
  r.j0 = jlo;
  r.k0 = 30;
  r.w = jhi - jlo > 0 ? jhi - jlo : 0;
  const int kh = freenode ? NZ : NZ - 31;
  r.h = kh - 30 > 0 ? kh - 30 : 0;
  return r;
}
// blocks of the fault node kernel (128 threads, one node each; at least one)
inline int node_blocks(int NY, int NZ, int freenode, int jg0, int nj) {
  const long long c = node_rect(NY, NZ, freenode, jg0, nj).count();
  return c > 0 ? (int)((c + 127) / 128) : 1;
}

// Separable grid description for the FP64 metric kernel (dfd_setup.cu).
struct GridArgs {
  Dims d;
  const double* xl;  // (nx) extended x line
  const double* fx;  // (nz, ny) extended fault surface
  const double* fy;
  const double* fz;
  const float* layers;  // (nlayer, 4) depth rho vp vs
  int nlayer;
  int NXhalf;           // NX/2: bimaterial split on the padded index (metric.cu:140-142)
  double rDH;
  double lam1, mu1, rho1, lam2, mu2, rho2;
};

// Tile of the TMA-staged kernels: 32 nodes along y (one warp) by 8 along z; the PML
// kernel's y-slab units use strip tiles of 16 by 16 (half a warp per row).
constexpr int TILE_J = 32, TILE_K = 8, STRIP = 16;

// TMA tensor maps handed to the tiled kernels (dfd_tile.cu, dfd_pml.cu)
struct TileMaps {
  CUtensorMap win;  // stencil input, halo box
  CUtensorMap w0;   // step-start state, pointwise box
  CUtensorMap t;    // second pointwise box: stage 2 the stage-1 input, stage 3 the accumulator
  CUtensorMap plane;  // separable metric / media planes (12, nz, py)
  CUtensorMap aux[6];  // PML state of each face (27 fields), pointwise box of 9 fields
  // the same for the 16 x 16 strip tiles (halo box 24 x 20)
  CUtensorMap win_s, w0_s, t_s, plane_s, auxy_s[2];
  // the interior kernel's: its tiles are 32 x 8 (the maps above) or 32 x 4 (TileCtx::tr)
  CUtensorMap win_i, w0_i, t_i, plane_i;
};
// Per-context state of the tiled kernels: maps of the four volume buffers, of the metric
// and of the PML state (fixed addresses, encoded once), the error flag, the SM count.
struct TileCtx {
  CUtensorMap halo[4];
  CUtensorMap centre[4];
  CUtensorMap plane;
  CUtensorMap aux[6];
  CUtensorMap halo_s[4], centre_s[4], plane_s, auxy_s[2];  // strip tiles
  CUtensorMap halo4[4], centre4[4], plane4;                // 32 x 4 tiles of the interior kernel
  int tr = TILE_K;       // rows of the interior kernel's tiles: 8 (one CTA per SM) or 4 (two)
  int* err = nullptr;
  int* sched = nullptr;  // unit counter and finished-CTA counter (zero between launches)
  int nsm = 0;
  int drill = 0;         // test drill of the bounded waits (TileSched::drill), off by default
  bool ok = false;
};
bool tile_setup(TileCtx* tc, const Dims& d, float* const W[4], const float* planes, float* const aux[6], int* err,
                int* sched, int device);
// every map the tiled kernels read at a stage whose stencil input is buffer `bin`
// (the interior kernel's maps for tiles of tr rows)
TileMaps tile_maps(const TileCtx& tc, int bin, int irk, int tr);
// Units of a tiled kernel: tile columns times chunks of x planes.
//   interior kernel: the 32 x 8 tiles of the box lo..hi (the last ones partial);
//   PML kernel: the nodes below the free-surface rows (k < ktop) outside the interior
//   box [nx1, ni - nx2) x [ya, yb) x [za, zb): every 32 x 8 tile of the two x slabs
//   (frame at j = 0, k = 0), then in chunks of ci planes over [nx1, ni - nx2) the nedge
//   tiles of the edges: the 16 x 16 strip tiles of the y slabs, ny1 strips from j = 0
//   and ny2 from j = yb, each over the nrs strip rows of [0, ktop); the 32 x 8 tiles of
//   the z slabs, ntz tiles from j = ya over the nz1 tile rows from k = 0 (below za) and
//   the nz2 tile rows from k = zb (up to ktop).
struct TileSched {
  int lo_x, lo_y, lo_z, hi_x, hi_y, hi_z;  // tiled box, interior indices, half open
  int ntj, ntk, ci, nunits;               // tiles in y and z, planes per chunk, units
  int nx1, nx2, ktop, nedge;              // PML kernel: x slab widths, top row bound, edge tiles
  int ya, yb, za, zb;                     // PML kernel: the interior box in y and z
  int ny1, ny2, nrs, ntz, nz1, nz2;       // PML kernel: edge tile counts
  int drill;  // interior kernel, test drill: the copy warp issues no copies, so the computing
              // warps' first wait runs out (after DRILL_LIMIT polls) and sets the error flag
};
// Values of one scenario of a batched (ensemble) launch of the tiled kernel that the
// computing warps read; a CTA copies them into shared memory with each unit's planes.
struct alignas(16) TileUnit {
  VolArgs a;
  TileSched sc;
  int unit0;  // first global unit of the scenario
};
// One scenario of a batched launch of the tiled kernel, in device memory.
struct alignas(64) TileScen {
  TileMaps mp;
  TileUnit u;
};
// Boxes of the general (shell) kernels: up to eight, each flattened or tiled.  Boxes
// [0, ntop) lie below the free-surface rows (PML slabs, alignment columns) and go to the
// kernel without the free-surface terms; boxes [ntop, n) hold the free-surface rows.
struct Boxes {
  int n, ntop;
  int lo[8][3], hi[8][3];  // (i, j, k) interior-index bounds, half open
  int thin[8];             // flattened (y, z) mapping
  int start[9];            // first block of each box
};
// Volume work of one stage of one scenario: the box of the tiled (or plain) interior
// kernel, the units of the tiled PML kernel and the general kernel's boxes.
struct VolPlan {
  bool tiled, plain;
  int3 lo, hi;        // interior-kernel box
  TileSched ps;       // PML kernel units (tiled plans; ps.nunits 0: none)
  int pgrid;          // PML kernel CTAs
  Boxes bx;
  int shell_blocks;
  long long nodes;    // nodes of the interior-kernel box
};
VolPlan plan_volume(const VolArgs& a, const TileCtx* tc);
bool tile_feasible(const TileCtx* tc, const VolArgs& a, int3 lo, int3 hi);
// slots: CTAs resident at once (SMs x CTAs per SM); tr: rows of a tile
TileSched tile_plan(int3 lo, int3 hi, int slots, int* grid, int tr = TILE_K);
// CTAs of the interior kernel resident per SM with tiles of tr rows
int tile_ctas_per_sm(int tr);
// units of the PML kernel around the interior box (dfd_pml.cu)
TileSched pml_plan(const VolArgs& a, int ya, int yb, int za, int zb, int ktop, int nsm, int* grid);
bool pml_setup();
// pdl: launch behind the interior kernel on the same stream with programmatic
// serialisation; sched: a 4-int counter block (the interior kernel uses the first pair)
void launch_pml(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, const TileSched& ps, int grid,
                bool pdl, cudaStream_t s);
void launch_pml_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int FX, int FY, int FZ,
                      int* err, int* sched, bool pdl, cudaStream_t s);
// batched launches (dfd_volume.cu, dfd_tile.cu, dfd_fault.cu)
void launch_tile_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int tr, int FX,
                       int FY, int FZ, int* err, int* sched, cudaStream_t s);
// top: the free-surface boxes (start: per-scenario block starts of those), else the others;
// irk: the stage of every scenario's arguments
void launch_shell_batch(const VolArgs* tab, const Boxes* boxes, const int* start, int n, int blocks, int FX, int FY,
                        int FZ, bool top, int irk, cudaStream_t s);
void launch_fault_node_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FY, int FZ,
                             cudaStream_t s);
// thermal pressurisation (Friction_type 3): node-major columns of n points across the
// fault (point i of node q at [q * n + i]), updated once per step before the stages; T0
// and P0 receive point 0 of every column (dfd_fault.cu)
struct TpArgs {
  int nf, n;
  float DT;
  const int* united;
  const float *Vs1, *Vs2, *Tn, *friction, *hy;
  float *T, *P, *T0, *P0;
};
void launch_thermpress(const TpArgs& a, cudaStream_t s);
// rupture sensor (rup_sensor.cu), once per step before the stages: from Ts1 into out
struct SensorArgs {
  int nj, nk, fg[4];
  int slab;  // a slab of a domain decomposed along y: no sensor within two columns of its ends
  const int* united;
  const float* Ts1;
  float* out;
};
void launch_rup_sensor(const SensorArgs& a, cudaStream_t s);
void launch_fault_band_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FX, int FY, int FZ,
                             cudaStream_t s);

// scenario owning block b of a batched launch: start[s] <= b < start[s + 1]
// Copy one scenario's argument struct of an ensemble table into shared memory, all
// threads of the block taking part (a __syncthreads must follow): the batched kernels
// then read their arguments from shared memory instead of global memory.
template <class T>
__device__ __forceinline__ void stage_args(T* dst, const T* src) {
  static_assert(sizeof(T) % 4 == 0, "argument struct size");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  for (int w = t; w < (int)(sizeof(T) / 4); w += nt) d[w] = __ldg(s + w);
}

__device__ __forceinline__ int scenario_of(const int* start, int n, int b, int* local) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    int m = (lo + hi) / 2;
    if (start[m] <= b) lo = m; else hi = m;
  }
  *local = b - start[lo];
  return lo;
}

bool launch_tile(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, int3 lo, int3 hi,
                 cudaStream_t s);

__host__ __device__ inline long long idx3(const Dims& d, int i, int j, int k) {
  return (long long)(j + d.oy) + (long long)k * d.py + (long long)i * d.sx;
}

}  // namespace dfd
