// Internal definitions shared by the CUDA kernels and the host side of the
// B200 dynamic-rupture time step.
//
// HBM layout (per context, all FP32 unless noted):
//   W[4]      four 9-field volume buffers (nx, nz, py), y fastest, 3 ghost nodes;
//             a step cycles A -> B -> C -> B -> A so that the stencil input of a stage is
//             never written during that stage and no right-hand-side array exists
//   M         13 fields xix xiy xiz etx ety etz ztx zty ztz jac lam mu rho, same layout
//   aux       per PML face, 3 buffers (current, step start, RK accumulator) of 9 fields
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
};

// Arguments of the fused volume stage kernel.
struct VolArgs {
  Dims d;
  const float* __restrict__ Win;   // stencil input of this stage
  const float* __restrict__ W0;    // step-start state (stages 1, 2)
  float* __restrict__ Wout;        // output of this stage
  float* __restrict__ T;           // RK accumulator
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
  float* aux[6];                   // current PML state per face (x1 x2 y1 y2 z1 z2) or null
  float* aux0[6];                  // step-start copy
  float* auxT[6];                  // RK accumulator
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
  float *Vs1, *Vs2, *Tn, *Ts1, *Ts2, *tTn, *tTs1, *tTs2;
  float *sx, *sy, *sz;             // str_init
  const float *T0x, *T0y, *T0z, *dT0x, *dT0y, *dT0z;
  const float *str_peak, *Dc, *C0, *a, *b, *L, *Vw;
  float *init_t0, *friction;
  int *init_t0_flag, *flag_rup;
  const int *united, *faultgrid, *rupy, *rupz;
  unsigned long long* newton;      // [0] iterations, [1] capped solves
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
};

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

// TMA tensor maps handed to the tiled interior kernel (dfd_tile.cu)
struct TileMaps {
  CUtensorMap win;  // stencil input, halo box
  CUtensorMap w0;   // step-start state, pointwise box
  CUtensorMap t;    // RK accumulator, pointwise box
  CUtensorMap plane;  // separable metric / media planes (12, nz, py)
};
// Per-context state of the tiled interior kernel: maps of the four volume buffers and of
// the metric (fixed addresses, encoded once), the error flag, the SM count.
struct TileCtx {
  CUtensorMap halo[4];
  CUtensorMap centre[4];
  CUtensorMap plane;
  int* err = nullptr;
  int* sched = nullptr;  // unit counter and finished-CTA counter (zero between launches)
  int nsm = 0;
  int pml = 0;  // 1: the tiles cover every PML slab; 3: the two x slabs only
  bool ok = false;
};
bool tile_setup(TileCtx* tc, const Dims& d, float* const W[4], const float* planes, int* err, int* sched,
                int device);
// Units of the tiled kernel over a box: tile columns (32 y x 8 z) times chunks of x planes.
struct TileSched {
  int lo_x, lo_y, lo_z, hi_x, hi_y, hi_z;  // tiled box, interior indices, half open
  int ntj, ntk, ci, nunits;               // tiles in y and z, planes per chunk, units
};
// One scenario of a batched (ensemble) launch of the tiled kernel, in device memory.
struct alignas(64) TileScen {
  TileMaps mp;
  VolArgs a;
  TileSched sc;
  int unit0;  // first global unit of the scenario
};
// Boxes of the general (shell) kernel: up to eight, each flattened or tiled.
struct Boxes {
  int n;
  int lo[8][3], hi[8][3];  // (i, j, k) interior-index bounds, half open
  int thin[8];             // flattened (y, z) mapping
  int start[9];            // first block of each box
};
// Volume work of one stage of one scenario: the box of the tiled (or plain) interior
// kernel and the general kernel's boxes.
struct VolPlan {
  bool tiled, pmlp, plain;
  int3 lo, hi;        // interior-kernel box
  Boxes bx;
  int shell_blocks;
  long long nodes;    // nodes of the interior-kernel box
};
VolPlan plan_volume(const VolArgs& a, const TileCtx* tc);
bool tile_feasible(const TileCtx* tc, const VolArgs& a, int3 lo, int3 hi);
TileSched tile_plan(int3 lo, int3 hi, int nsm, int* grid);
// batched launches (dfd_volume.cu, dfd_tile.cu, dfd_fault.cu)
void launch_tile_batch(const TileScen& first, const TileScen* tab, int n, int nunits, int grid, int FX, int FY,
                       int FZ, bool pmlp, int* err, int* sched, cudaStream_t s);
void launch_shell_batch(const VolArgs* tab, const Boxes* boxes, const int* start, int n, int blocks, int FX, int FY,
                        int FZ, cudaStream_t s);
void launch_fault_node_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FY, int FZ,
                             cudaStream_t s);
void launch_fault_band_batch(const FaultArgs* tab, const int* start, int n, int blocks, int FX, int FY, int FZ,
                             cudaStream_t s);

// scenario owning block b of a batched launch: start[s] <= b < start[s + 1]
__device__ __forceinline__ int scenario_of(const int* start, int n, int b, int* local) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    int m = (lo + hi) / 2;
    if (start[m] <= b) lo = m; else hi = m;
  }
  *local = b - start[lo];
  return lo;
}

// pmlp: the box contains PML nodes (the kernel variant with the PML path)
bool launch_tile(const TileCtx* tc, const VolArgs& a, int FX, int FY, int FZ, int bin, int3 lo, int3 hi, bool pmlp,
                 cudaStream_t s);

__host__ __device__ inline long long idx3(const Dims& d, int i, int j, int k) {
  return (long long)(j + d.oy) + (long long)k * d.py + (long long)i * d.sx;
}

}  // namespace dfd
