// C ABI of the B200 dynamic-rupture time step: context (device memory owner), setup,
// stage sequencing with a side stream for the fault band, CUDA-graph replay of whole
// steps, state access and NetCDF output.
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dfd_host.h"
#include "dfd_internal.cuh"

namespace dfd {
long long launch_volume_stage(const VolArgs& a, int FX, int FY, int FZ, cudaStream_t s, cudaStream_t s_shell,
                              const TileCtx* tc, int bin, cudaEvent_t* kb, cudaEvent_t* ke, VolPlan* out,
                              cudaEvent_t* fork);
void launch_fault_node(const FaultArgs& a, cudaStream_t s);
void launch_fault_band(const FaultArgs& a, cudaStream_t s);
void launch_fault_coef(const Dims& d, const float* M, float* tab, float* tabf, float* vecn, float* vecs1,
                       float* vecs2, float* rhof, cudaStream_t s);
void launch_wave_free(const Dims& d, const float* M, const float* Bx, const float* By, const float* Bz, float* mx,
                      float* my, cudaStream_t s);
void launch_metric(const GridArgs& g, float* M, cudaStream_t s);
void launch_plane_metric(const GridArgs& g, float* pl, float* rxa, cudaStream_t s);
void launch_cfl(const GridArgs& g, const float* M, float* hmin, float* vpmax, cudaStream_t s);

__global__ void set_it_kernel(int* it, int v) { *it = v; }
__global__ void inc_it_kernel(int* it) { *it += 1; }
__global__ void nonfinite_kernel(const float* a, long long n, int* flag) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  for (; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!isfinite(a[i])) *flag = 1;
}
// (nx, nz, ny) field -> (a, b) slice gathers of Vx, Vy, Vz (get_wave_slice_*, io_wave_*.cu)
__global__ void slice_kernel(Dims d, const float* W, int axis, int index, float* out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int na = axis == 0 ? d.nk : d.ni, nb = axis == 1 ? d.nk : d.nj;
  if (t >= na * nb) return;
  int a = t / nb, b = t % nb, i, j, k;
  if (axis == 0) { i = index; k = a; j = b; }
  else if (axis == 1) { j = index; i = a; k = b; }
  else { k = index; i = a; j = b; }
  long long q = idx3(d, i + 3, j + 3, k + 3);
  for (int c = 0; c < 3; c++) out[(long long)c * na * nb + t] = W[c * d.nxyz + q];
}

// Halo message of a slab (domain decomposed along y): three columns starting at padded
// column jp of nvf volume fields (layout (f, x, z, y), pitched rows) and of nff fault
// planes (layout (f, z, y)), in the order ((f, x, z), column) then ((f, z), column).
// unpack = 0 gathers them into buf, unpack = 1 scatters buf into them.
__global__ void halo_kernel(Dims d, float* vol, int nvf, float* fw, int nff, int jp, float* buf, int unpack) {
  const long long nv = (long long)nvf * d.nx * d.nz * 3, nt = nv + (long long)nff * d.nz * 3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nt; t += (long long)gridDim.x * blockDim.x) {
    float* p;
    if (t < nv) {
      const int c = (int)(t % 3);
      const long long r = t / 3;  // (f, x, z)
      const int k = (int)(r % d.nz), i = (int)((r / d.nz) % d.nx), f = (int)(r / ((long long)d.nz * d.nx));
      p = vol + f * d.nxyz + (jp + c + d.oy) + (long long)k * d.py + (long long)i * d.sx;
    } else {
      const long long u = t - nv;
      const int c = (int)(u % 3);
      const long long r = u / 3;  // (f, z)
      const int k = (int)(r % d.nz), f = (int)(r / d.nz);
      p = fw + f * d.nyz + (jp + c) + (long long)k * d.ny;
    }
    if (unpack) *p = buf[t];
    else buf[t] = *p;
  }
}
}  // namespace dfd

using namespace dfd;

// fault 2-D planes held in one allocation
// (the eight per-step output planes come first so one copy fetches them)
enum Plane {
  P_VS1, P_VS2, P_TN, P_TS1, P_TS2, P_SLIP, P_STATE, P_T0,
  P_MSLIP, P_TSLIP, P_HSLIP, P_MSTATE, P_TSTATE, P_TTN, P_TTS1,
  P_TTS2, P_SX, P_SY, P_SZ, P_T0X, P_T0Y, P_T0Z, P_DT0X, P_DT0Y, P_DT0Z, P_PEAK, P_DC, P_C0, P_A, P_B, P_L, P_VW,
  P_FRIC, P_CSLIP, P_CSTATE,  // the two compensation terms of slip and state
  P_TPT0, P_TPP0,              // thermal pressurisation: T and P at the fault
  P_RUPS,                      // rupture sensor
  NPLANE
};
enum IPlane { I_T0FLAG, I_FLAGRUP, I_UNITED, I_FAULTGRID, I_RUPY, I_RUPZ, NIPLANE };

// Asynchronous output (dfd_output_write): the record is copied on the stepping stream
// into one of two device staging sets (a snapshot the next step cannot change), the
// staging set goes to pinned host memory on a side stream, and a writer thread puts the
// finished record into the NetCDF files while the GPU keeps stepping.  Record layout in
// floats: the seven per-step fault planes, init_t0, the two rupture-index planes (int32),
// then the three wave slices (3 components each).
struct OutState {
  size_t nf = 0, bytes = 0;
  size_t slice_off[3] = {0, 0, 0}, slice_n[3] = {0, 0, 0};
  float* dev[2] = {nullptr, nullptr};
  float* host[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};  // the slot's copy to the host has finished
  cudaEvent_t snap = nullptr;                // the snapshot on the stepping stream is done
  cudaStream_t s = nullptr;
  std::thread writer;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<int, int>> q;  // (record index, slot) waiting for the writer
  bool busy[2] = {false, false};      // the slot holds a record not yet written
  bool stop = false;
  int err = 0;
  int next = 0;
};

struct dfd_ctx {
  dfd_params p;
  Dims d;
  int device = 0;
  cudaStream_t s0 = nullptr, s1 = nullptr, s2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
  std::vector<void*> allocs;
  float* W[4] = {};
  float* M = nullptr;
  float* mplane = nullptr;          // separable metric / media planes (12, nz, py)
  float* rxa = nullptr;             // 1/(d x / d xi) per padded x index
  float *rB[3] = {}, *B[3] = {}, *Dp[3] = {}, *Ap[3] = {};
  float* aux[6] = {};
  float *mVx2Vz = nullptr, *mVy2Vz = nullptr;
  float* damp[3] = {};
  float *FW[2] = {}, *Fm = nullptr, *Ft = nullptr, *T1 = nullptr, *mT1 = nullptr, *hT1 = nullptr;
  float *tab = nullptr, *tabf = nullptr, *vecn = nullptr, *vecs1 = nullptr, *vecs2 = nullptr, *rhof = nullptr;
  float* pl = nullptr;
  int* ipl = nullptr;
  // thermal pressurisation (Friction_type 3): node-major columns of TP_n points per fault
  // node and the diffusivity
  float *tp_T = nullptr, *tp_P = nullptr, *tp_hy = nullptr;
  std::vector<float> tp_hy_h;
  unsigned long long* newton = nullptr;
  int* it_dev = nullptr;
  int* flag_dev = nullptr;
  float* guess_net = nullptr;
  float* rec = nullptr;             // Newton sample recording buffer (rec_cap x 5)
  unsigned* rec_n = nullptr;
  int rec_cap = 0;
  int rec_every = 1;
  int rs_prof = 0, rs_judge = 0;   // solve-section timing and judge mode (measurement aids)
  TileCtx tile;                    // tiled interior kernel (TMA maps)
  int* tile_err = nullptr;
  int* tile_sched = nullptr;         // tiled kernel's unit counters
  bool use_tile = true;
  // volume shell and fault band on s0 after the interior kernel (default), or on two
  // further streams beside it (DFD_STREAMS=3)
  bool serial = true;
  long long interior_nodes = 0;   // nodes the interior kernel updates per stage
  long long n_band_columns = 0;   // non-united (j, k) fault columns
  std::vector<int> united_h;      // (NZ, NY) host copy of the united plane
  int inodes_box[6] = {0, 0, 0, 0, 0, 0};  // box of the cached interior node count
  long long inodes_cached = -1;
  float interior_ms = 0;          // interior kernel time of the last dfd_run_timed
  float node_ms = 0;              // fault node kernel time of the last dfd_run_timed
  // host-side inputs
  std::vector<float> fxyz, planes, layers;
  std::vector<double> xl, fx, fy, fz;
  bool ready = false;
  int next_stage = 0;
  int next_part = 0;  // dfd_stage_part: the next part (0..2) of stage next_stage
  std::string err;
  int sticky = DFD_OK;
  cudaGraphExec_t graph[8] = {};
  // output
  NcWriter ncf, ncw[3];
  int vf[24] = {}, vw[3][3] = {};
  bool out_open = false;
  OutState* out = nullptr;
  // dfd_fetch_outputs: two device staging copies of the outputs and a side stream that
  // takes them to the host while the next steps run
  float* fetch_stage[2] = {nullptr, nullptr};
  cudaEvent_t fetch_snap = nullptr, fetch_done[2] = {nullptr, nullptr};
  cudaStream_t s_fetch = nullptr;
  int fetch_k = 0;
  bool fetch_used[2] = {false, false};
};

// a step or a stage issued only in part (dfd_stage, dfd_stage_part)
static inline bool mid_step(const dfd_ctx* c) { return c->next_stage != 0 || c->next_part != 0; }

static int fail(dfd_ctx* c, int code, const std::string& m) {
  if (c) { c->err = m; if (code == DFD_ERR_CUDA) c->sticky = code; }
  return code;
}
static int cuda_check(dfd_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return DFD_OK;
  return fail(c, DFD_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                                     \
  do {                                                               \
    int _r = cuda_check(ctx, (call), #call);                         \
    if (_r) return _r;                                               \
  } while (0)

// Host-to-device copies and clears go through the context's stepping stream s0 and are
// complete when the call returns.  A plain cudaMemcpy from pageable host memory (and a
// plain cudaMemset) runs on the legacy default stream, may still be in flight when it
// returns, and is not ordered with the non-blocking context streams: a kernel launched on
// s0 right after it could read the buffer before the copy lands.
static cudaError_t h2d(dfd_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->s0);
  return e == cudaSuccess ? cudaStreamSynchronize(ctx->s0) : e;
}

template <typename T>
static int dalloc(dfd_ctx* ctx, T** p, size_t n) {
  void* v = nullptr;
  cudaError_t e = cudaMalloc(&v, n * sizeof(T) + 16);
  if (e != cudaSuccess) return cuda_check(ctx, e, "cudaMalloc");
  ctx->allocs.push_back(v);
  e = cudaMemsetAsync(v, 0, n * sizeof(T) + 16, ctx->s0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->s0);
  if (e != cudaSuccess) return cuda_check(ctx, e, "cudaMemset");
  *p = (T*)v;
  return DFD_OK;
}

extern "C" {

const char* dfd_error_string(int s) {
  switch (s) {
    case DFD_OK: return "ok";
    case DFD_ERR_PARAM: return "bad or unsupported parameter";
    case DFD_ERR_CUDA: return "CUDA error";
    case DFD_ERR_IO: return "file missing or malformed";
    case DFD_ERR_STATE: return "call out of order";
    case DFD_ERR_CFL: return "DT above the stability limit";
    case DFD_ERR_NONFINITE: return "non-finite fault state";
    case DFD_ERR_NEWTON: return "Newton solve hit its iteration cap";
  }
  return "unknown status";
}
const char* dfd_last_error(const dfd_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

int dfd_params_size(void) { return (int)sizeof(dfd_params); }

int dfd_params_default(dfd_params* p) {
  if (!p) return DFD_ERR_PARAM;
  params_default(p);
  return DFD_OK;
}

int dfd_params_load_json(const char* path, dfd_params* p) {
  if (!path || !p) return DFD_ERR_PARAM;
  FILE* f = fopen(path, "rb");
  if (!f) return DFD_ERR_IO;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  fclose(f);
  params_default(p);
  return params_from_json(text.c_str(), p, nullptr);
}

int dfd_create(const dfd_params* p, int device, dfd_ctx** out) {
  if (!p || !out) return DFD_ERR_PARAM;
  *out = nullptr;
  std::string e;
  dfd_params q = *p;
  finalize_params(&q);
  int r = check_params(&q, &e);
  if (r) { fprintf(stderr, "dfd_create: %s\n", e.c_str()); return r; }
  dfd_ctx* ctx = new dfd_ctx();
  ctx->p = q;
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return DFD_ERR_CUDA; }
  Dims& d = ctx->d;
  // a slab of a domain decomposed along y holds NY / slabs_y columns (1: the whole domain)
  d.ni = q.NX; d.nj = q.NY / q.slabs_y; d.nk = q.NZ;
  d.nx = q.NX + 6; d.ny = d.nj + 6; d.nz = q.NZ + 6;
  d.i0 = d.nx / 2;
  d.N = q.PML_N;
  // row offset 1: the first interior node (after 3 ghost nodes) of every row on a 16-byte
  // boundary; pitch a multiple of 8 elements
  d.oy = 1;
  d.py = (d.ny + d.oy + 7) / 8 * 8;
  d.sx = (long long)d.py * d.nz;
  d.nxyz = d.sx * d.nx;
  d.nyz = (long long)d.ny * d.nz;
  // y-face PML state rows: the N nodes with the columns before them up to a 16-byte
  // boundary; the y2 face starts at the boundary at or before its first node
  d.wy = (d.N + 4 + 3) / 4 * 4;
  d.yb3 = (d.nj - d.N + 3 + d.oy) / 4 * 4;
  auto done = [&](int rc) { if (rc) { dfd_destroy(ctx); return rc; } return 0; };
  if (done(cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->s0, cudaStreamNonBlocking), "stream"))) return DFD_ERR_CUDA;
  if (done(cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->s1, cudaStreamNonBlocking), "stream"))) return DFD_ERR_CUDA;
  if (done(cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->s2, cudaStreamNonBlocking), "stream"))) return DFD_ERR_CUDA;
  cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&ctx->ev_join2, cudaEventDisableTiming);
  int rc = 0;
  for (int b = 0; b < 4 && !rc; b++) rc = dalloc(ctx, &ctx->W[b], 9 * d.nxyz);
  if (!rc) rc = dalloc(ctx, &ctx->M, 13 * d.nxyz);
  if (!rc) rc = dalloc(ctx, &ctx->mplane, 12LL * d.py * d.nz);
  if (!rc) rc = dalloc(ctx, &ctx->rxa, d.nx);
  int len[3] = {d.ni, d.nj, d.nk};
  for (int a = 0; a < 3 && !rc; a++) {
    rc = dalloc(ctx, &ctx->rB[a], len[a]);
    if (!rc) rc = dalloc(ctx, &ctx->B[a], len[a]);
    if (!rc) rc = dalloc(ctx, &ctx->Dp[a], len[a]);
    if (!rc) rc = dalloc(ctx, &ctx->Ap[a], len[a]);
  }
  if (!rc && q.use_pml) {
    // 27 fields per face: three blocks of nine cycled through the RK stages
    for (int f = 0; f < 6 && !rc; f++) {
      if (f == 5 && q.free_surface) continue;
      // the y faces only on the slabs at the domain's y ends
      if ((f == 2 && q.slab_y > 0) || (f == 3 && q.slab_y < q.slabs_y - 1)) continue;
      const long long fs = pml_fstride(d, f);
      rc = dalloc(ctx, &ctx->aux[f], 27 * fs);
    }
  }
  if (!rc) rc = dalloc(ctx, &ctx->mVx2Vz, 9LL * d.nx * d.ny);
  if (!rc) rc = dalloc(ctx, &ctx->mVy2Vz, 9LL * d.nx * d.ny);
  if (!rc && q.use_cerjan) {
    rc = dalloc(ctx, &ctx->damp[0], d.nx);
    if (!rc) rc = dalloc(ctx, &ctx->damp[1], d.ny);
    if (!rc) rc = dalloc(ctx, &ctx->damp[2], d.nz);
  }
  if (!rc && q.rupture) {
    for (int b = 0; b < 2 && !rc; b++) rc = dalloc(ctx, &ctx->FW[b], 18 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->Fm, 18 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->Ft, 18 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->T1, 21 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->mT1, 3 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->hT1, 3 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->tab, (long long)NTAB9 * 9 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->tabf, (long long)NTABF * 9 * d.ny);
    if (!rc) rc = dalloc(ctx, &ctx->vecn, 3 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->vecs1, 3 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->vecs2, 3 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->rhof, 2 * d.nyz);
    if (!rc) rc = dalloc(ctx, &ctx->pl, (long long)NPLANE * d.nj * d.nk);
    if (!rc) rc = dalloc(ctx, &ctx->ipl, (long long)NIPLANE * d.nj * d.nk);
    if (q.Friction_type == 3) {
      if (!rc) rc = dalloc(ctx, &ctx->tp_T, (long long)q.TP_n * d.nj * d.nk);
      if (!rc) rc = dalloc(ctx, &ctx->tp_P, (long long)q.TP_n * d.nj * d.nk);
      if (!rc) rc = dalloc(ctx, &ctx->tp_hy, (long long)d.nj * d.nk);
    }
  }
  if (!rc) rc = dalloc(ctx, &ctx->newton, 8);
  if (!rc) rc = dalloc(ctx, &ctx->it_dev, 1);
  if (!rc) rc = dalloc(ctx, &ctx->flag_dev, 1);
  if (!rc) rc = dalloc(ctx, &ctx->guess_net, DFD_MLP_PARAMS);
  if (!rc) rc = dalloc(ctx, &ctx->rec_n, 1);
  if (!rc) rc = dalloc(ctx, &ctx->tile_err, 1);
  if (!rc) rc = dalloc(ctx, &ctx->tile_sched, 4);  // unit and finished-CTA counters: interior, PML
  if (rc) { dfd_destroy(ctx); return rc; }
  // volume kernels: DFD_TILE=0 plain interior kernel + general kernel on the PML slabs
  // and free-surface rows; otherwise (default) the TMA-staged interior and PML kernels
  // + the general kernel on the free-surface rows
  const char* tv = getenv("DFD_TILE");
  const int mode = tv && tv[0] == '0' ? 0 : 1;
  float* auxb[6];
  for (int f = 0; f < 6; f++) auxb[f] = ctx->aux[f];
  ctx->use_tile =
      mode > 0 && tile_setup(&ctx->tile, d, ctx->W, ctx->mplane, auxb, ctx->tile_err, ctx->tile_sched, device);
  const char* sv = getenv("DFD_STREAMS");
  ctx->serial = !(sv && sv[0] == '3');
  *out = ctx;
  return DFD_OK;
}

int dfd_destroy(dfd_ctx* ctx) {
  if (!ctx) return DFD_OK;
  cudaSetDevice(ctx->device);
  dfd_output_close(ctx);
  for (auto& g : ctx->graph)
    if (g) cudaGraphExecDestroy(g);
  if (ctx->s0) cudaStreamSynchronize(ctx->s0);
  if (ctx->s1) cudaStreamSynchronize(ctx->s1);
  if (ctx->s2) cudaStreamSynchronize(ctx->s2);
  for (void* v : ctx->allocs) cudaFree(v);
  if (ctx->rec) cudaFree(ctx->rec);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->ev_join2) cudaEventDestroy(ctx->ev_join2);
  if (ctx->s_fetch) {
    cudaStreamSynchronize(ctx->s_fetch);
    for (int b = 0; b < 2; b++) {
      cudaFree(ctx->fetch_stage[b]);
      cudaEventDestroy(ctx->fetch_done[b]);
    }
    cudaEventDestroy(ctx->fetch_snap);
    cudaStreamDestroy(ctx->s_fetch);
  }
  if (ctx->s0) cudaStreamDestroy(ctx->s0);
  if (ctx->s1) cudaStreamDestroy(ctx->s1);
  if (ctx->s2) cudaStreamDestroy(ctx->s2);
  delete ctx;
  return DFD_OK;
}

int dfd_dims(const dfd_ctx* ctx, int* nx, int* ny, int* nz) {
  if (!ctx) return DFD_ERR_PARAM;
  if (nx) *nx = ctx->d.nx;
  if (ny) *ny = ctx->d.ny;
  if (nz) *nz = ctx->d.nz;
  return DFD_OK;
}

int dfd_load_fault_geometry(dfd_ctx* ctx, const float* fxyz) {
  if (!ctx || !fxyz) return DFD_ERR_PARAM;
  size_t n = 3ull * ctx->p.NY * ctx->p.NZ;
  ctx->fxyz.assign(fxyz, fxyz + n);
  ctx->ready = false;
  return DFD_OK;
}
int dfd_load_media1d(dfd_ctx* ctx, int n, const float* layers) {
  if (!ctx || n < 0 || (n > 0 && !layers)) return DFD_ERR_PARAM;
  ctx->layers.assign(layers, layers + 4 * (size_t)n);
  ctx->ready = false;
  return DFD_OK;
}
int dfd_load_fault_init(dfd_ctx* ctx, const float* planes) {
  if (!ctx || !planes) return DFD_ERR_PARAM;
  size_t n = 15ull * ctx->p.NY * ctx->p.NZ;
  ctx->planes.assign(planes, planes + n);
  ctx->ready = false;
  return DFD_OK;
}

int dfd_load_tp_hy(dfd_ctx* ctx, const float* tp_hy) {
  if (!ctx || !tp_hy) return DFD_ERR_PARAM;
  if (ctx->p.Friction_type != 3) return fail(ctx, DFD_ERR_STATE, "TP_hy is read for Friction_type 3 only");
  ctx->tp_hy_h.assign(tp_hy, tp_hy + (size_t)ctx->p.NY * ctx->p.NZ);
  ctx->ready = false;
  return DFD_OK;
}

int dfd_precompute(dfd_ctx* ctx) {
  if (!ctx) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  cudaSetDevice(ctx->device);
  const dfd_params& p = ctx->p;
  const Dims& d = ctx->d;
  cudaStream_t s = ctx->s0;
  if (p.INPORT_GRID_TYPE == 1 && ctx->fxyz.empty())
    return fail(ctx, DFD_ERR_STATE, "INPORT_GRID_TYPE=1 needs dfd_load_fault_geometry");
  if (p.rupture && p.INPORT_STRESS_TYPE != 1)
    return fail(ctx, DFD_ERR_PARAM, "rupture runs need INPORT_STRESS_TYPE=1 and dfd_load_fault_init");
  if (p.rupture && ctx->planes.empty()) return fail(ctx, DFD_ERR_STATE, "missing dfd_load_fault_init");
  // ---- grid, metric, media (FP64 on the GPU)
  x_line(&p, ctx->xl);
  surface(&p, ctx->fxyz.empty() ? nullptr : ctx->fxyz.data(), ctx->fx, ctx->fy, ctx->fz);
  if (p.slabs_y > 1) {
    // this slab's columns of the domain's extended surface, its ghost columns included:
    // the neighbours' coordinates inside the domain, the extrapolated ones at its ends
    const int nyg = p.NY + 6, j0 = p.slab_y * d.nj;
    for (auto* v : {&ctx->fx, &ctx->fy, &ctx->fz}) {
      std::vector<double> loc((size_t)d.ny * d.nz);
      for (int k = 0; k < d.nz; k++)
        for (int j = 0; j < d.ny; j++) loc[j + (size_t)k * d.ny] = (*v)[j0 + j + (size_t)k * nyg];
      v->swap(loc);
    }
  }
  double *dxl, *dfx, *dfy, *dfz;
  float* dlay = nullptr;
  CK(cudaMalloc(&dxl, sizeof(double) * ctx->xl.size()));
  CK(cudaMalloc(&dfx, sizeof(double) * ctx->fx.size()));
  CK(cudaMalloc(&dfy, sizeof(double) * ctx->fy.size()));
  CK(cudaMalloc(&dfz, sizeof(double) * ctx->fz.size()));
  CK(h2d(ctx, dxl, ctx->xl.data(), sizeof(double) * ctx->xl.size()));
  CK(h2d(ctx, dfx, ctx->fx.data(), sizeof(double) * ctx->fx.size()));
  CK(h2d(ctx, dfy, ctx->fy.data(), sizeof(double) * ctx->fy.size()));
  CK(h2d(ctx, dfz, ctx->fz.data(), sizeof(double) * ctx->fz.size()));
  if (!ctx->layers.empty()) {
    CK(cudaMalloc(&dlay, sizeof(float) * ctx->layers.size()));
    CK(h2d(ctx, dlay, ctx->layers.data(), sizeof(float) * ctx->layers.size()));
  }
  GridArgs g;
  g.d = d; g.xl = dxl; g.fx = dfx; g.fy = dfy; g.fz = dfz; g.layers = dlay;
  g.nlayer = (int)(ctx->layers.size() / 4);
  g.NXhalf = p.NX / 2;
  g.rDH = 1.0 / p.DH;
  g.lam1 = p.bi_rho1 * (p.bi_vp1 * p.bi_vp1 - 2 * p.bi_vs1 * p.bi_vs1);
  g.mu1 = p.bi_rho1 * p.bi_vs1 * p.bi_vs1;
  g.rho1 = p.bi_rho1;
  g.lam2 = p.bi_rho2 * (p.bi_vp2 * p.bi_vp2 - 2 * p.bi_vs2 * p.bi_vs2);
  g.mu2 = p.bi_rho2 * p.bi_vs2 * p.bi_vs2;
  g.rho2 = p.bi_rho2;
  launch_metric(g, ctx->M, s);
  launch_plane_metric(g, ctx->mplane, ctx->rxa, s);
  CK(cudaGetLastError());
  // CFL check (main.cu:323-345)
  size_t ncol = (size_t)d.nj * d.nk;
  float *dh, *dv;
  CK(cudaMalloc(&dh, sizeof(float) * ncol));
  CK(cudaMalloc(&dv, sizeof(float) * ncol));
  launch_cfl(g, ctx->M, dh, dv, s);
  CK(cudaGetLastError());
  std::vector<float> hh(ncol), hv(ncol);
  CK(cudaMemcpyAsync(hh.data(), dh, sizeof(float) * ncol, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hv.data(), dv, sizeof(float) * ncol, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  cudaFree(dh); cudaFree(dv); cudaFree(dxl); cudaFree(dfx); cudaFree(dfy); cudaFree(dfz);
  if (dlay) cudaFree(dlay);
  float hmin = 1e38f, vpmax = 0.0f;
  for (size_t i = 0; i < ncol; i++) { hmin = fminf(hmin, hh[i]); vpmax = fmaxf(vpmax, hv[i]); }
  float dtmax = 1.3f * hmin / vpmax;
  if (!(p.DT < dtmax)) {
    char m[160];
    snprintf(m, sizeof m, "DT = %g >= dtmax = %g (hmin %g m, vpmax %g m/s)", p.DT, dtmax, hmin, vpmax);
    return fail(ctx, DFD_ERR_CFL, m);
  }
  // ---- PML 1-D profiles
  bool fs = p.free_surface != 0;
  int len[3] = {d.ni, d.nj, d.nk};
  const bool ylo = p.slab_y == 0, yhi = p.slab_y == p.slabs_y - 1;  // the slab holds a y end
  for (int a = 0; a < 3; a++) {
    std::vector<float> A, B, D, rb;
    bool lo = p.use_pml && !(a == 1 && !ylo), hi = p.use_pml && !(a == 2 && fs) && !(a == 1 && !yhi);
    pml_profile(&p, len[a], lo, hi, A, B, D);
    rb.resize(B.size());
    for (size_t i = 0; i < B.size(); i++) rb[i] = 1.0f / B[i];
    CK(h2d(ctx, ctx->Ap[a], A.data(), sizeof(float) * A.size()));
    CK(h2d(ctx, ctx->B[a], B.data(), sizeof(float) * B.size()));
    CK(h2d(ctx, ctx->Dp[a], D.data(), sizeof(float) * D.size()));
    CK(h2d(ctx, ctx->rB[a], rb.data(), sizeof(float) * rb.size()));
  }
  if (p.use_cerjan) {
    int np[3] = {d.nx, d.ny, d.nz};
    for (int a = 0; a < 3; a++) {
      std::vector<float> prof;
      cerjan_profile(&p, np[a], !(a == 1 && !ylo), !(a == 2 && fs) && !(a == 1 && !yhi), prof);
      CK(h2d(ctx, ctx->damp[a], prof.data(), sizeof(float) * prof.size()));
    }
  }
  if (fs) launch_wave_free(d, ctx->M, ctx->B[0], ctx->B[1], ctx->B[2], ctx->mVx2Vz, ctx->mVy2Vz, s);
  // ---- fault tables and initial state
  size_t nf = (size_t)d.nj * d.nk;
  if (p.rupture) {
    launch_fault_coef(d, ctx->M, ctx->tab, ctx->tabf, ctx->vecn, ctx->vecs1, ctx->vecs2, ctx->rhof, s);
    CK(cudaGetLastError());
    std::vector<float> vn(3 * d.nyz), v1(3 * d.nyz), v2(3 * d.nyz);
    CK(cudaMemcpyAsync(vn.data(), ctx->vecn, sizeof(float) * vn.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(v1.data(), ctx->vecs1, sizeof(float) * v1.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(v2.data(), ctx->vecs2, sizeof(float) * v2.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    FaultHost h;
    fault_init(&p, ctx->planes.data(), vn.data(), v1.data(), v2.data(), h);
    CK(cudaMemsetAsync(ctx->pl, 0, sizeof(float) * NPLANE * nf, s));
    CK(cudaMemsetAsync(ctx->ipl, 0, sizeof(int) * NIPLANE * nf, s));
    struct { int plane; std::vector<float>* v; } up[] = {
        {P_SX, &h.sx}, {P_SY, &h.sy}, {P_SZ, &h.sz}, {P_T0X, &h.T0x}, {P_T0Y, &h.T0y}, {P_T0Z, &h.T0z},
        {P_DT0X, &h.dT0x}, {P_DT0Y, &h.dT0y}, {P_DT0Z, &h.dT0z}, {P_PEAK, &h.str_peak}, {P_DC, &h.Dc},
        {P_C0, &h.C0}, {P_A, &h.a}, {P_B, &h.b}, {P_L, &h.L}, {P_VW, &h.Vw}, {P_STATE, &h.State},
        {P_TN, &h.Tn}, {P_TS1, &h.Ts1}, {P_TS2, &h.Ts2}, {P_T0, &h.init_t0}};
    for (auto& u : up)
      CK(cudaMemcpyAsync(ctx->pl + u.plane * nf, u.v->data(), sizeof(float) * nf, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(ctx->pl + P_CSLIP * nf, 0, sizeof(float) * 2 * nf, s));
    if (ctx->tp_T) {
      // zero columns (alloc.cu:117-118); the diffusivity from dfd_load_tp_hy, else zero
      CK(cudaMemsetAsync(ctx->tp_T, 0, sizeof(float) * p.TP_n * nf, s));
      CK(cudaMemsetAsync(ctx->tp_P, 0, sizeof(float) * p.TP_n * nf, s));
      if (ctx->tp_hy_h.size() == (size_t)p.NY * d.nk) {
        // this slab's columns of the (NZ, NY) plane
        std::vector<float> hy(nf);
        for (int k = 0; k < d.nk; k++)
          for (int j = 0; j < d.nj; j++) hy[j + (size_t)k * d.nj] = ctx->tp_hy_h[p.slab_y * d.nj + j + (size_t)k * p.NY];
        CK(cudaMemcpyAsync(ctx->tp_hy, hy.data(), sizeof(float) * nf, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
      }
      else
        CK(cudaMemsetAsync(ctx->tp_hy, 0, sizeof(float) * nf, s));
    }
    struct { int plane; std::vector<int>* v; } iup[] = {
        {I_UNITED, &h.united}, {I_FAULTGRID, &h.faultgrid}, {I_RUPY, &h.rupy}, {I_RUPZ, &h.rupz}};
    ctx->n_band_columns = 0;
    for (int v : h.united) ctx->n_band_columns += v == 0;
    ctx->united_h = h.united;
    ctx->inodes_cached = -1;
    for (auto& u : iup)
      CK(cudaMemcpyAsync(ctx->ipl + u.plane * nf, u.v->data(), sizeof(int) * nf, cudaMemcpyHostToDevice, s));
    for (int b = 0; b < 2; b++) CK(cudaMemsetAsync(ctx->FW[b], 0, sizeof(float) * 18 * d.nyz, s));
    CK(cudaMemsetAsync(ctx->Fm, 0, sizeof(float) * 18 * d.nyz, s));
    CK(cudaMemsetAsync(ctx->Ft, 0, sizeof(float) * 18 * d.nyz, s));
    CK(cudaMemsetAsync(ctx->T1, 0, sizeof(float) * 21 * d.nyz, s));
    CK(cudaMemsetAsync(ctx->mT1, 0, sizeof(float) * 3 * d.nyz, s));
    CK(cudaMemsetAsync(ctx->hT1, 0, sizeof(float) * 3 * d.nyz, s));
  }
  for (int b = 0; b < 4; b++) CK(cudaMemsetAsync(ctx->W[b], 0, sizeof(float) * 9 * d.nxyz, s));
  for (int f = 0; f < 6; f++)
    if (ctx->aux[f]) CK(cudaMemsetAsync(ctx->aux[f], 0, sizeof(float) * 27 * pml_fstride(d, f), s));
  CK(cudaMemsetAsync(ctx->newton, 0, 8 * sizeof(unsigned long long), s));
  CK(cudaStreamSynchronize(s));
  CK(cudaGetLastError());
  for (auto& gr : ctx->graph)
    if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
  ctx->ready = true;
  ctx->next_stage = 0;
  ctx->next_part = 0;
  return DFD_OK;
}

}  // extern "C"

static const int kFlags[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, -1, 1},
                                 {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};

// enqueue one stage on the context streams (no synchronisation)
// Arguments of the fault kernels for stage irk of a step with flag pattern `pattern`
// (main.cu:448-470: FD_Flags reversed at every stage).
static FaultArgs fault_args(dfd_ctx* ctx, int pattern, int irk) {
  const dfd_params& p = ctx->p;
  const Dims& d = ctx->d;
  int sg = (irk % 2) ? -1 : 1;
  int FX = kFlags[pattern][0] * sg, FY = kFlags[pattern][1] * sg, FZ = kFlags[pattern][2] * sg;
  static const int bin[4] = {0, 1, 2, 1}, bout[4] = {1, 2, 1, 0};
  float a_ = irk == 0 ? 0.5f : irk == 1 ? 0.5f : irk == 2 ? 1.0f : 1e10f;
  float b_ = (irk == 0 || irk == 3) ? (float)(1.0 / 6.0) : (float)(1.0 / 3.0);
  float DT = (float)p.DT;
  float rka = a_ * DT, rkb = b_ * DT;
  size_t nf = (size_t)d.nj * d.nk;
  FaultArgs fa;
  {
    memset(&fa, 0, sizeof fa);
    fa.d = d;
    fa.Win = ctx->W[bin[irk]]; fa.W0 = ctx->W[0]; fa.Wout = ctx->W[bout[irk]]; fa.T = ctx->W[3];
    fa.M = ctx->M; fa.mVx2Vz = ctx->mVx2Vz; fa.mVy2Vz = ctx->mVy2Vz;
    fa.dampx = ctx->damp[0]; fa.dampy = ctx->damp[1]; fa.dampz = ctx->damp[2];
    fa.FWin = ctx->FW[irk % 2]; fa.FWout = ctx->FW[(irk + 1) % 2]; fa.Fm = ctx->Fm; fa.Ft = ctx->Ft;
    fa.T1 = ctx->T1; fa.mT1 = ctx->mT1; fa.hT1 = ctx->hT1;
    fa.tab = ctx->tab; fa.tabf = ctx->tabf; fa.vecn = ctx->vecn; fa.vecs1 = ctx->vecs1; fa.vecs2 = ctx->vecs2;
    fa.rhof = ctx->rhof;
    float* P_ = ctx->pl;
    auto pl = [&](int k) { return P_ + k * nf; };
    fa.slip = pl(P_SLIP); fa.mslip = pl(P_MSLIP); fa.tslip = pl(P_TSLIP); fa.hslip = pl(P_HSLIP);
    fa.State = pl(P_STATE); fa.mState = pl(P_MSTATE); fa.tState = pl(P_TSTATE);
    fa.cslip = pl(P_CSLIP); fa.cState = pl(P_CSTATE);
    fa.tpP = ctx->tp_P ? pl(P_TPP0) : nullptr;  // null unless Friction_type 3
    fa.Vs1 = pl(P_VS1); fa.Vs2 = pl(P_VS2); fa.Tn = pl(P_TN); fa.Ts1 = pl(P_TS1); fa.Ts2 = pl(P_TS2);
    fa.tTn = pl(P_TTN); fa.tTs1 = pl(P_TTS1); fa.tTs2 = pl(P_TTS2);
    fa.sx = pl(P_SX); fa.sy = pl(P_SY); fa.sz = pl(P_SZ);
    fa.T0x = pl(P_T0X); fa.T0y = pl(P_T0Y); fa.T0z = pl(P_T0Z);
    fa.dT0x = pl(P_DT0X); fa.dT0y = pl(P_DT0Y); fa.dT0z = pl(P_DT0Z);
    fa.str_peak = pl(P_PEAK); fa.Dc = pl(P_DC); fa.C0 = pl(P_C0);
    fa.a = pl(P_A); fa.b = pl(P_B); fa.L = pl(P_L); fa.Vw = pl(P_VW);
    fa.init_t0 = pl(P_T0); fa.friction = pl(P_FRIC);
    fa.init_t0_flag = ctx->ipl + I_T0FLAG * nf; fa.flag_rup = ctx->ipl + I_FLAGRUP * nf;
    fa.united = ctx->ipl + I_UNITED * nf; fa.faultgrid = ctx->ipl + I_FAULTGRID * nf;
    fa.rupy = ctx->ipl + I_RUPY * nf; fa.rupz = ctx->ipl + I_RUPZ * nf;
    fa.newton = ctx->newton; fa.it_dev = ctx->it_dev; fa.guess_net = ctx->guess_net;
    fa.rec = ctx->rec; fa.rec_n = ctx->rec_n; fa.rec_cap = ctx->rec_cap; fa.rec_every = ctx->rec_every;
    fa.rDH = (float)(1.0 / p.DH); fa.DH = (float)p.DH; fa.DT = DT; fa.rka = rka; fa.rkb = rkb;
    fa.mu_d = (float)p.mu_d; fa.viscosity = (float)p.viscosity;
    fa.dDT = (double)DT; fa.smooth_load_T = (double)(float)p.smooth_load_T;
    fa.f0 = (double)(float)p.f0; fa.V0 = (double)(float)p.V0; fa.fw = (double)(float)p.fw;
    fa.Vini = (double)(float)p.Vini;
    fa.irk = irk; fa.FX = FX; fa.FY = FY; fa.FZ = FZ;
    fa.freenode = p.free_surface; fa.friction_type = p.Friction_type; fa.inport_stress = p.INPORT_STRESS_TYPE;
    fa.NY = p.NY; fa.NZ = p.NZ; fa.rs_guess = p.rs_guess; fa.jg0 = p.slab_y * d.nj;
    fa.prof = ctx->rs_prof; fa.judge = ctx->rs_judge; fa.guess_tol = p.rs_guess_tol;
  }
  (void)FX;
  return fa;
}

// Arguments of the volume kernels for the same stage.
static VolArgs vol_args(dfd_ctx* ctx, int pattern, int irk) {
  const dfd_params& p = ctx->p;
  const Dims& d = ctx->d;
  (void)pattern;
  static const int bin[4] = {0, 1, 2, 1}, bout[4] = {1, 2, 1, 0};
  float a_ = irk == 0 ? 0.5f : irk == 1 ? 0.5f : irk == 2 ? 1.0f : 1e10f;
  float b_ = (irk == 0 || irk == 3) ? (float)(1.0 / 6.0) : (float)(1.0 / 3.0);
  float DT = (float)p.DT;
  float rka = a_ * DT, rkb = b_ * DT;
  size_t nf = (size_t)d.nj * d.nk;
  VolArgs va;
  memset(&va, 0, sizeof va);
  va.d = d;
  va.Win = ctx->W[bin[irk]]; va.W0 = ctx->W[0]; va.Wout = ctx->W[bout[irk]]; va.T = ctx->W[3];
  va.M = ctx->M;
  va.rBx = ctx->rB[0]; va.rBy = ctx->rB[1]; va.rBz = ctx->rB[2];
  va.Bx = ctx->B[0]; va.By = ctx->B[1]; va.Bz = ctx->B[2];
  va.Dpx = ctx->Dp[0]; va.Dpy = ctx->Dp[1]; va.Dpz = ctx->Dp[2];
  va.Apx = ctx->Ap[0]; va.Apy = ctx->Ap[1]; va.Apz = ctx->Ap[2];
  for (int f = 0; f < 6; f++) va.aux[f] = ctx->aux[f];
  va.mVx2Vz = ctx->mVx2Vz; va.mVy2Vz = ctx->mVy2Vz;
  va.dampx = ctx->damp[0]; va.dampy = ctx->damp[1]; va.dampz = ctx->damp[2];
  va.united = p.rupture ? ctx->ipl + I_UNITED * nf : nullptr;
  va.rxa = ctx->rxa;
  va.nxhalf = p.NX / 2;
  va.rDH = (float)(1.0 / p.DH); va.rka = rka; va.rkb = rkb;
  va.irk = irk; va.freenode = p.free_surface;
  return va;
}

// nodes the interior kernel updates in a stage: its box less the fault-band nodes in it
static long long interior_nodes(dfd_ctx* ctx, const VolPlan& pl) {
  if (!(pl.tiled || pl.plain)) return 0;
  const int box[6] = {pl.lo.x, pl.lo.y, pl.lo.z, pl.hi.x, pl.hi.y, pl.hi.z};
  if (ctx->inodes_cached >= 0 && std::equal(box, box + 6, ctx->inodes_box)) return ctx->inodes_cached;
  long long n = pl.nodes;
  const Dims& d = ctx->d;
  if (ctx->p.rupture && !ctx->united_h.empty() && pl.lo.x + 3 <= d.i0 + 3 && pl.hi.x + 3 > d.i0 - 3) {
    long long cols = 0;
    for (int k = pl.lo.z; k < pl.hi.z; k++)
      for (int j = pl.lo.y; j < pl.hi.y; j++) cols += ctx->united_h[(size_t)k * d.nj + j] == 0;
    const int x0 = std::max(pl.lo.x + 3, d.i0 - 3), x1 = std::min(pl.hi.x + 3, d.i0 + 4);
    n -= cols * std::max(0, x1 - x0);
  }
  std::copy(box, box + 6, ctx->inodes_box);
  ctx->inodes_cached = n;
  return n;
}

static TpArgs tp_args(dfd_ctx* ctx) {
  const int nf = ctx->d.nj * ctx->d.nk;
  auto pl = [&](int k) { return ctx->pl + (size_t)k * nf; };
  TpArgs t;
  t.nf = nf; t.n = ctx->p.TP_n; t.DT = (float)ctx->p.DT;
  t.united = ctx->ipl + I_UNITED * nf;
  t.Vs1 = pl(P_VS1); t.Vs2 = pl(P_VS2); t.Tn = pl(P_TN); t.friction = pl(P_FRIC); t.hy = ctx->tp_hy;
  t.T = ctx->tp_T; t.P = ctx->tp_P; t.T0 = pl(P_TPT0); t.P0 = pl(P_TPP0);
  return t;
}

static SensorArgs sensor_args(dfd_ctx* ctx) {
  const int nf = ctx->d.nj * ctx->d.nk;
  SensorArgs a;
  a.nj = ctx->d.nj; a.nk = ctx->d.nk;
  // a slab of a decomposed domain: the fault grid in its local columns, and no sensor where
  // the second differences would reach past the slab (as the reference's per-rank sensor)
  const int j0 = ctx->p.slab_y * ctx->d.nj;
  for (int i = 0; i < 4; i++) a.fg[i] = ctx->p.Fault_grid[i] - (i < 2 ? j0 : 0);
  a.slab = ctx->p.slabs_y > 1;
  a.united = ctx->ipl + I_UNITED * nf;
  a.Ts1 = ctx->pl + (size_t)P_TS1 * nf;
  a.out = ctx->pl + (size_t)P_RUPS * nf;
  return a;
}

static int enqueue_stage(dfd_ctx* ctx, int pattern, int irk, cudaEvent_t* vb = nullptr, cudaEvent_t* ve = nullptr,
                         cudaEvent_t* kb = nullptr, cudaEvent_t* ke = nullptr, cudaEvent_t* nb = nullptr,
                         cudaEvent_t* ne = nullptr) {
  const dfd_params& p = ctx->p;
  int sg = (irk % 2) ? -1 : 1;
  int FX = kFlags[pattern][0] * sg, FY = kFlags[pattern][1] * sg, FZ = kFlags[pattern][2] * sg;
  static const int bin[4] = {0, 1, 2, 1};
  FaultArgs fa;
  // rupture sensor and thermal pressurisation once per step, before the stages
  // (main.cu:444-447)
  if (p.rupture && irk == 0) launch_rup_sensor(sensor_args(ctx), ctx->s0);
  if (p.rupture && irk == 0 && ctx->tp_T) launch_thermpress(tp_args(ctx), ctx->s0);
  if (p.rupture) {
    fa = fault_args(ctx, pattern, irk);
    if (nb) cudaEventRecord(*nb, ctx->s0);
    launch_fault_node(fa, ctx->s0);
    if (ne) cudaEventRecord(*ne, ctx->s0);
  }
  if (vb) cudaEventRecord(*vb, ctx->s0);
  if (ctx->serial) {
    // interior and PML kernels on s0; then the general kernel (free-surface rows) on s2
    // beside the fault band kernel on s0: two small latency-bound kernels that fit on the
    // SMs together
    VolArgs va = vol_args(ctx, pattern, irk);
    VolPlan pl;
    launch_volume_stage(va, FX, FY, FZ, ctx->s0, ctx->s2, ctx->use_tile ? &ctx->tile : nullptr, bin[irk], kb, ke,
                        &pl, &ctx->ev_fork);
    ctx->interior_nodes = interior_nodes(ctx, pl);
    cudaEventRecord(ctx->ev_join2, ctx->s2);
    if (p.rupture) launch_fault_band(fa, ctx->s0);
    cudaStreamWaitEvent(ctx->s0, ctx->ev_join2, 0);
    if (ve) cudaEventRecord(*ve, ctx->s0);
    return cuda_check(ctx, cudaGetLastError(), "stage launch");
  }
  // fork: fault band on s1, volume shell on s2, volume interior on s0
  cudaEventRecord(ctx->ev_fork, ctx->s0);
  if (p.rupture) {
    cudaStreamWaitEvent(ctx->s1, ctx->ev_fork, 0);
    launch_fault_band(fa, ctx->s1);
    cudaEventRecord(ctx->ev_join, ctx->s1);
  }
  cudaStreamWaitEvent(ctx->s2, ctx->ev_fork, 0);
  VolArgs va = vol_args(ctx, pattern, irk);
  VolPlan pl;
  launch_volume_stage(va, FX, FY, FZ, ctx->s0, ctx->s2, ctx->use_tile ? &ctx->tile : nullptr, bin[irk], kb, ke, &pl,
                      nullptr);
  ctx->interior_nodes = interior_nodes(ctx, pl);
  cudaEventRecord(ctx->ev_join2, ctx->s2);
  if (p.rupture) cudaStreamWaitEvent(ctx->s0, ctx->ev_join, 0);
  cudaStreamWaitEvent(ctx->s0, ctx->ev_join2, 0);
  if (ve) cudaEventRecord(*ve, ctx->s0);
  return cuda_check(ctx, cudaGetLastError(), "stage launch");
}

// One part of a stage, the kernels of enqueue_stage in three groups on the stepping
// stream: 0 = (stage 0: rupture sensor, thermal pressurisation) fault node kernel;
// 1 = the volume kernels, the free-surface rows joined back before the part ends;
// 2 = the fault band kernel.  Parts 0, 1, 2 compute what enqueue_stage computes.
static int enqueue_part(dfd_ctx* ctx, int pattern, int irk, int part) {
  const dfd_params& p = ctx->p;
  const int sg = (irk % 2) ? -1 : 1;
  const int FX = kFlags[pattern][0] * sg, FY = kFlags[pattern][1] * sg, FZ = kFlags[pattern][2] * sg;
  static const int bin[4] = {0, 1, 2, 1};
  if (part == 0 && p.rupture) {
    if (irk == 0) launch_rup_sensor(sensor_args(ctx), ctx->s0);
    if (irk == 0 && ctx->tp_T) launch_thermpress(tp_args(ctx), ctx->s0);
    launch_fault_node(fault_args(ctx, pattern, irk), ctx->s0);
  } else if (part == 1) {
    VolArgs va = vol_args(ctx, pattern, irk);
    VolPlan pl;
    launch_volume_stage(va, FX, FY, FZ, ctx->s0, ctx->s2, ctx->use_tile ? &ctx->tile : nullptr, bin[irk], nullptr,
                        nullptr, &pl, &ctx->ev_fork);
    ctx->interior_nodes = interior_nodes(ctx, pl);
    cudaEventRecord(ctx->ev_join2, ctx->s2);
    cudaStreamWaitEvent(ctx->s0, ctx->ev_join2, 0);
  } else if (part == 2 && p.rupture) {
    launch_fault_band(fault_args(ctx, pattern, irk), ctx->s0);
  }
  return cuda_check(ctx, cudaGetLastError(), "stage part launch");
}

extern "C" {

int dfd_stage(dfd_ctx* ctx, int it, int irk) {
  if (!ctx) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  if (irk != ctx->next_stage || ctx->next_part != 0)
    return fail(ctx, DFD_ERR_STATE, "stages must be issued in order 0..3");
  cudaSetDevice(ctx->device);
  if (irk == 0) dfd::set_it_kernel<<<1, 1, 0, ctx->s0>>>(ctx->it_dev, it);
  int r = enqueue_stage(ctx, ((it % 8) + 8) % 8, irk);
  if (r) return r;
  ctx->next_stage = (irk + 1) % 4;
  return DFD_OK;
}

int dfd_stage_part(dfd_ctx* ctx, int it, int irk, int part) {
  if (!ctx || irk < 0 || irk > 3 || part < 0 || part > 2) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  if (irk != ctx->next_stage || part != ctx->next_part)
    return fail(ctx, DFD_ERR_STATE, "stage parts must be issued in order 0..2 within stages 0..3");
  cudaSetDevice(ctx->device);
  if (irk == 0 && part == 0) dfd::set_it_kernel<<<1, 1, 0, ctx->s0>>>(ctx->it_dev, it);
  int r = enqueue_part(ctx, ((it % 8) + 8) % 8, irk, part);
  if (r) return r;
  ctx->next_part = (part + 1) % 3;
  if (part == 2) ctx->next_stage = (irk + 1) % 4;
  return DFD_OK;
}

// capture the four stages of one step (flag pattern) and the step-counter advance
static int build_graph(dfd_ctx* ctx, int pattern) {
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(ctx->s0, cudaStreamCaptureModeThreadLocal));
  int r = 0;
  for (int irk = 0; irk < 4 && !r; irk++) r = enqueue_stage(ctx, pattern, irk);
  dfd::inc_it_kernel<<<1, 1, 0, ctx->s0>>>(ctx->it_dev);
  cudaError_t e = cudaStreamEndCapture(ctx->s0, &g);
  if (r) return r;
  CK(e);
  CK(cudaGraphInstantiate(&ctx->graph[pattern], g, 0));
  cudaGraphDestroy(g);
  return DFD_OK;
}

int dfd_run(dfd_ctx* ctx, int it0, int nsteps) {
  if (!ctx) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  if (mid_step(ctx)) return fail(ctx, DFD_ERR_STATE, "a step is half done (dfd_stage)");
  cudaSetDevice(ctx->device);
  dfd::set_it_kernel<<<1, 1, 0, ctx->s0>>>(ctx->it_dev, it0);
  for (int s = 0; s < nsteps; s++) {
    int pat = (((it0 + s) % 8) + 8) % 8;
    if (!ctx->graph[pat]) {
      int r = build_graph(ctx, pat);
      if (r) return r;
    }
    CK(cudaGraphLaunch(ctx->graph[pat], ctx->s0));
  }
  return DFD_OK;
}

int dfd_step(dfd_ctx* ctx, int it) { return dfd_run(ctx, it, 1); }

static int tile_status(dfd_ctx* ctx);

int dfd_run_graph_timed(dfd_ctx* ctx, int it0, int nsteps, float* ms) {
  if (!ctx || !ms || nsteps < 1) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  if (mid_step(ctx)) return fail(ctx, DFD_ERR_STATE, "a step is half done (dfd_stage)");
  cudaSetDevice(ctx->device);
  for (int pat = 0; pat < 8; pat++)
    if (!ctx->graph[pat]) {
      int r = build_graph(ctx, pat);
      if (r) return r;
    }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, ctx->s0));
  int r = dfd_run(ctx, it0, nsteps);
  CK(cudaEventRecord(e1, ctx->s0));
  CK(cudaEventSynchronize(e1));
  CK(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  return tile_status(ctx);
}

// error flag of the tiled interior kernel (a TMA copy that did not complete in time)
static int tile_status(dfd_ctx* ctx) {
  if (ctx->sticky || !ctx->use_tile) return ctx->sticky;
  int e = 0;
  CK(cudaMemcpy(&e, ctx->tile_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) { ctx->sticky = DFD_ERR_CUDA; ctx->err = "tiled interior kernel: a TMA copy did not complete"; }
  return ctx->sticky;
}

int dfd_synchronize(dfd_ctx* ctx) {
  if (!ctx) return DFD_ERR_PARAM;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  CK(cudaStreamSynchronize(ctx->s1));
  CK(cudaStreamSynchronize(ctx->s2));
  if (ctx->s_fetch) CK(cudaStreamSynchronize(ctx->s_fetch));
  return tile_status(ctx);
}

// dense host fields (nf, nx, nz, ny) <-> pitched device fields (nf, nx, nz, py) at offset oy:
// all nf*nx*nz rows share one pitch, so one 2-D copy moves them
// dense reference layout <-> padded rows, on the stepping stream, complete on return
static int volume_copy(dfd_ctx* ctx, float* host, float* dev, int nf, bool to_host) {
  const Dims& d = ctx->d;
  size_t w = sizeof(float) * d.ny, hp = w, dp = sizeof(float) * d.py;
  size_t rows = (size_t)nf * d.nx * d.nz;
  if (to_host) CK(cudaMemcpy2DAsync(host, hp, dev + d.oy, dp, w, rows, cudaMemcpyDeviceToHost, ctx->s0));
  else CK(cudaMemcpy2DAsync(dev + d.oy, dp, host, hp, w, rows, cudaMemcpyHostToDevice, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return DFD_OK;
}

int dfd_get_wave(dfd_ctx* ctx, float* host) {
  if (!ctx || !host) return DFD_ERR_PARAM;
  if (mid_step(ctx)) return fail(ctx, DFD_ERR_STATE, "wavefield is mid-step");
  CK(cudaStreamSynchronize(ctx->s0));
  return volume_copy(ctx, host, ctx->W[0], 9, true);
}
int dfd_set_wave(dfd_ctx* ctx, const float* host) {
  if (!ctx || !host) return DFD_ERR_PARAM;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  CK(cudaStreamSynchronize(ctx->s0));
  return volume_copy(ctx, const_cast<float*>(host), ctx->W[0], 9, false);
}
int dfd_get_metric(dfd_ctx* ctx, float* host) {
  if (!ctx || !host) return DFD_ERR_PARAM;
  CK(cudaStreamSynchronize(ctx->s0));
  return volume_copy(ctx, host, ctx->M, 13, true);
}

int dfd_get_fault(dfd_ctx* ctx, int field, float* host) {
  if (!ctx || !host || field < 0 || field >= DFD_F_COUNT) return DFD_ERR_PARAM;
  if (!ctx->p.rupture) return fail(ctx, DFD_ERR_STATE, "rupture is off");
  CK(cudaStreamSynchronize(ctx->s0));
  size_t nf = (size_t)ctx->d.nj * ctx->d.nk;
  static const int map[] = {P_SLIP, P_HSLIP, P_VS1, P_VS2, P_TN, P_TS1, P_TS2, P_STATE,
                            P_T0, P_TTN, P_TTS1, P_TTS2, P_PEAK, P_FRIC};
  if (field <= DFD_F_FRICTION) {
    CK(cudaMemcpy(host, ctx->pl + map[field] * nf, sizeof(float) * nf, cudaMemcpyDeviceToHost));
  } else if (field == DFD_F_UNITED || field == DFD_F_FAULTGRID) {
    std::vector<int> t(nf);
    CK(cudaMemcpy(t.data(), ctx->ipl + (field == DFD_F_UNITED ? I_UNITED : I_FAULTGRID) * nf, sizeof(int) * nf,
                  cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < nf; i++) host[i] = (float)t[i];
  } else if (field == DFD_F_SPLIT) {
    CK(cudaMemcpy(host, ctx->FW[0], sizeof(float) * 18 * ctx->d.nyz, cudaMemcpyDeviceToHost));
  } else if (field == DFD_F_T1) {
    CK(cudaMemcpy(host, ctx->T1, sizeof(float) * 21 * ctx->d.nyz, cudaMemcpyDeviceToHost));
  } else if (field == DFD_F_HT1) {
    CK(cudaMemcpy(host, ctx->hT1, sizeof(float) * 3 * ctx->d.nyz, cudaMemcpyDeviceToHost));
  } else if (field == DFD_F_RUP_SENSOR) {
    CK(cudaMemcpy(host, ctx->pl + P_RUPS * nf, sizeof(float) * nf, cudaMemcpyDeviceToHost));
  } else {
    if (!ctx->tp_T) return fail(ctx, DFD_ERR_STATE, "thermal pressurisation is off (Friction_type != 3)");
    CK(cudaMemcpy(host, ctx->pl + (field == DFD_F_TP_T ? P_TPT0 : P_TPP0) * nf, sizeof(float) * nf,
                  cudaMemcpyDeviceToHost));
  }
  return DFD_OK;
}

// The device keeps each table as 9 planes of (nz, ny) (element-major, so neighbouring
// threads read neighbouring addresses); the caller gets the reference's node-major
// [node][9] layout (fault_coef.cu:26-1312).
static_assert(DFD_TAB_MATVZTOVXP + 1 == dfd::NTAB9, "public table names follow the device table order");
static_assert(DFD_TAB_MATMIN2PLUS3F - DFD_TAB_MATVX2VZ1 + 1 == dfd::NTABF, "free-surface tables");
int dfd_get_fault_table(dfd_ctx* ctx, int table, float* host) {
  if (!ctx || !host || table < 0 || table >= DFD_TAB_COUNT) return DFD_ERR_PARAM;
  if (!ctx->p.rupture || !ctx->tab) return fail(ctx, DFD_ERR_STATE, "rupture is off or setup has not run");
  CK(cudaStreamSynchronize(ctx->s0));
  const Dims& d = ctx->d;
  const float* src;
  size_t nodes;
  int ne;
  if (table <= DFD_TAB_MATVZTOVXP) {
    src = ctx->tab + (size_t)table * 9 * d.nyz; nodes = d.nyz; ne = 9;
  } else if (table <= DFD_TAB_MATMIN2PLUS3F) {
    src = ctx->tabf + (size_t)(table - DFD_TAB_MATVX2VZ1) * 9 * d.ny; nodes = d.ny; ne = 9;
  } else {
    src = table == DFD_TAB_VEC_N ? ctx->vecn : table == DFD_TAB_VEC_S1 ? ctx->vecs1 : ctx->vecs2;
    nodes = d.nyz; ne = 3;
  }
  std::vector<float> t(nodes * ne);
  CK(cudaMemcpy(t.data(), src, sizeof(float) * t.size(), cudaMemcpyDeviceToHost));
  for (size_t q = 0; q < nodes; q++)
    for (int e = 0; e < ne; e++) host[q * ne + e] = t[e * nodes + q];
  return DFD_OK;
}

int dfd_get_tp_columns(dfd_ctx* ctx, int which, float* host) {
  if (!ctx || !host || which < 0 || which > 1) return DFD_ERR_PARAM;
  if (!ctx->tp_T) return fail(ctx, DFD_ERR_STATE, "thermal pressurisation is off (Friction_type != 3)");
  CK(cudaStreamSynchronize(ctx->s0));
  const size_t n = ctx->p.TP_n, nf = (size_t)ctx->d.nj * ctx->d.nk;
  std::vector<float> col(n * nf);
  CK(cudaMemcpy(col.data(), which ? ctx->tp_P : ctx->tp_T, sizeof(float) * n * nf, cudaMemcpyDeviceToHost));
  // node-major on the device, plane-major (the reference's layout) for the caller
  for (size_t q = 0; q < nf; q++)
    for (size_t i = 0; i < n; i++) host[i * nf + q] = col[q * n + i];
  return DFD_OK;
}

int dfd_get_slice(dfd_ctx* ctx, int axis, int index, float* host) {
  if (!ctx || !host || axis < 0 || axis > 2) return DFD_ERR_PARAM;
  const Dims& d = ctx->d;
  int lim = axis == 0 ? d.ni : axis == 1 ? d.nj : d.nk;
  if (index < 0 || index >= lim) return DFD_ERR_PARAM;
  int na = axis == 0 ? d.nk : d.ni, nb = axis == 1 ? d.nk : d.nj;
  float* dv;
  CK(cudaMalloc(&dv, sizeof(float) * 3 * na * nb));
  dfd::slice_kernel<<<(na * nb + 255) / 256, 256, 0, ctx->s0>>>(d, ctx->W[0], axis, index, dv);
  cudaError_t e = cudaMemcpyAsync(host, dv, sizeof(float) * 3 * na * nb, cudaMemcpyDeviceToHost, ctx->s0);
  cudaStreamSynchronize(ctx->s0);
  cudaFree(dv);
  return cuda_check(ctx, e, "slice");
}

// ---- slice read-out that allocates nothing ----
// Callers that may not allocate device memory while they run (a host thread that polls
// slices between steps under a fixed memory budget, or code that must not call cudaMalloc
// or cudaFree because those synchronise the whole device) use this entry instead of
// dfd_get_slice.  The gather buffer is one file-scope device array per device, sized for
// DFD_SLICE_SCRATCH_FLOATS floats (3 components x the slice's nodes); larger slices are
// rejected with DFD_ERR_PARAM.  The gather kernel writes every element that is copied
// back, so nothing in the array has to start at zero.  The array is shared by every
// context on a device: two calls that overlap in time on the same device (from two host
// threads) race on it.  It occupies 16 MiB of device memory on every device where this
// library's module is loaded, whether or not the entry is ever called.  The host-side
// cache of its address is atomic, so first calls from several threads are safe.
static __device__ __align__(256) float g_slice_scratch[DFD_SLICE_SCRATCH_FLOATS];
static std::atomic<float*> g_slice_scratch_ptr[64] = {};

int dfd_get_slice_noalloc(dfd_ctx* ctx, int axis, int index, float* host) {
  if (!ctx || !host || axis < 0 || axis > 2) return DFD_ERR_PARAM;
  const Dims& d = ctx->d;
  int lim = axis == 0 ? d.ni : axis == 1 ? d.nj : d.nk;
  if (index < 0 || index >= lim) return DFD_ERR_PARAM;
  int na = axis == 0 ? d.nk : d.ni, nb = axis == 1 ? d.nk : d.nj;
  long long nfloat = 3LL * na * nb;
  if (nfloat > DFD_SLICE_SCRATCH_FLOATS)
    return fail(ctx, DFD_ERR_PARAM, "slice of " + std::to_string(nfloat) + " floats exceeds the " +
                                        std::to_string(DFD_SLICE_SCRATCH_FLOATS) + "-float static gather buffer");
  if (ctx->device < 0 || ctx->device >= 64) return fail(ctx, DFD_ERR_PARAM, "device ordinal out of range");
  CK(cudaSetDevice(ctx->device));
  // first call on this device: look up the array's device address (setup, done once)
  float* dv = g_slice_scratch_ptr[ctx->device].load(std::memory_order_acquire);
  if (!dv) {
    CK(cudaGetSymbolAddress((void**)&dv, g_slice_scratch));
    g_slice_scratch_ptr[ctx->device].store(dv, std::memory_order_release);
  }
  dfd::slice_kernel<<<(na * nb + 255) / 256, 256, 0, ctx->s0>>>(d, ctx->W[0], axis, index, dv);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, dv, sizeof(float) * nfloat, cudaMemcpyDeviceToHost, ctx->s0));
  return cuda_check(ctx, cudaStreamSynchronize(ctx->s0), "slice (static buffer)");
}

int dfd_check_finite(dfd_ctx* ctx) {
  if (!ctx) return DFD_ERR_PARAM;
  if (!ctx->p.rupture) return DFD_OK;
  size_t nf = (size_t)ctx->d.nj * ctx->d.nk;
  CK(cudaMemsetAsync(ctx->flag_dev, 0, sizeof(int), ctx->s0));
  dfd::nonfinite_kernel<<<64, 256, 0, ctx->s0>>>(ctx->pl, (long long)(P_TTS2 + 1) * nf, ctx->flag_dev);
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, ctx->flag_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  if (flag) return fail(ctx, DFD_ERR_NONFINITE, "NaN or Inf in the fault state");
  return DFD_OK;
}

int dfd_newton_stats(dfd_ctx* ctx, long long* iterations, long long* capped) {
  if (!ctx) return DFD_ERR_PARAM;
  unsigned long long v[2] = {0, 0};
  CK(cudaStreamSynchronize(ctx->s0));
  CK(cudaMemcpy(v, ctx->newton, sizeof v, cudaMemcpyDeviceToHost));
  if (iterations) *iterations = (long long)v[0];
  if (capped) *capped = (long long)v[1];
  return DFD_OK;
}

int dfd_fetch_outputs(dfd_ctx* ctx, float* host) {
  if (!ctx || !host) return DFD_ERR_PARAM;
  if (!ctx->p.rupture) return fail(ctx, DFD_ERR_STATE, "rupture is off");
  cudaSetDevice(ctx->device);
  const size_t bytes = sizeof(float) * 8 * (size_t)ctx->d.nj * ctx->d.nk;
  if (!ctx->s_fetch) {
    for (int b = 0; b < 2; b++) {
      CK(cudaMalloc(&ctx->fetch_stage[b], bytes));
      CK(cudaEventCreateWithFlags(&ctx->fetch_done[b], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&ctx->fetch_snap, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&ctx->s_fetch, cudaStreamNonBlocking));
  }
  // a device copy on the stepping stream (the next step cannot change it), then the copy
  // to the host on the side stream beside the next steps
  const int k = ctx->fetch_k;
  ctx->fetch_k ^= 1;
  if (ctx->fetch_used[k]) CK(cudaStreamWaitEvent(ctx->s0, ctx->fetch_done[k], 0));
  CK(cudaMemcpyAsync(ctx->fetch_stage[k], ctx->pl, bytes, cudaMemcpyDeviceToDevice, ctx->s0));
  CK(cudaEventRecord(ctx->fetch_snap, ctx->s0));
  CK(cudaStreamWaitEvent(ctx->s_fetch, ctx->fetch_snap, 0));
  CK(cudaMemcpyAsync(host, ctx->fetch_stage[k], bytes, cudaMemcpyDeviceToHost, ctx->s_fetch));
  CK(cudaEventRecord(ctx->fetch_done[k], ctx->s_fetch));
  ctx->fetch_used[k] = true;
  return DFD_OK;
}

int dfd_run_timed(dfd_ctx* ctx, int it0, int nsteps, float* total_ms, float* volume_ms, float* fault_ms) {
  if (!ctx || nsteps < 0) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready || mid_step(ctx)) return fail(ctx, DFD_ERR_STATE, "not ready for a step");
  cudaSetDevice(ctx->device);
  int nev = 8 * nsteps + 2;
  std::vector<cudaEvent_t> ev(nev, nullptr), kev(8 * nsteps, nullptr), fev(8 * nsteps, nullptr);
  // the events are destroyed on every return path, the early error returns included
  struct EventSet {
    std::vector<cudaEvent_t>* v[3];
    ~EventSet() {
      for (auto* l : v)
        for (auto e : *l)
          if (e) cudaEventDestroy(e);
    }
  } guard{{&ev, &kev, &fev}};
  for (auto& e : ev) CK(cudaEventCreate(&e));
  for (auto& e : kev) CK(cudaEventCreate(&e));
  for (auto& e : fev) CK(cudaEventCreate(&e));
  CK(cudaEventRecord(ev[0], ctx->s0));
  int k = 1;
  for (int s = 0; s < nsteps; s++) {
    int it = it0 + s;
    dfd::set_it_kernel<<<1, 1, 0, ctx->s0>>>(ctx->it_dev, it);
    for (int irk = 0; irk < 4; irk++) {
      int r = enqueue_stage(ctx, ((it % 8) + 8) % 8, irk, &ev[k], &ev[k + 1], &kev[k - 1], &kev[k],
                            ctx->p.rupture ? &fev[k - 1] : nullptr, ctx->p.rupture ? &fev[k] : nullptr);
      if (r) return r;
      k += 2;
    }
  }
  CK(cudaEventRecord(ev[nev - 1], ctx->s0));
  CK(cudaEventSynchronize(ev[nev - 1]));
  float tot = 0, vol = 0, inner = 0, node = 0;
  CK(cudaEventElapsedTime(&tot, ev[0], ev[nev - 1]));
  for (int i = 1; i + 1 < nev - 1; i += 2) {
    float m = 0;
    CK(cudaEventElapsedTime(&m, ev[i], ev[i + 1]));
    vol += m;
    CK(cudaEventElapsedTime(&m, kev[i - 1], kev[i]));
    inner += m;
    if (ctx->p.rupture) {
      CK(cudaEventElapsedTime(&m, fev[i - 1], fev[i]));
      node += m;
    }
  }
  ctx->interior_ms = inner;
  ctx->node_ms = node;
  if (total_ms) *total_ms = tot;
  if (volume_ms) *volume_ms = vol;
  if (fault_ms) *fault_ms = tot - vol;
  return tile_status(ctx);
}

int dfd_interior_stats(dfd_ctx* ctx, float* ms, long long* nodes) {
  if (!ctx) return DFD_ERR_PARAM;
  if (ms) *ms = ctx->interior_ms;
  if (nodes) *nodes = ctx->interior_nodes;
  return DFD_OK;
}

int dfd_fault_node_ms(dfd_ctx* ctx, float* ms) {
  if (!ctx || !ms) return DFD_ERR_PARAM;
  *ms = ctx->node_ms;
  return DFD_OK;
}

int dfd_set_guess_net(dfd_ctx* ctx, const float* w, int n) {
  if (!ctx || (w && n != DFD_MLP_PARAMS) || (!w && n != 0)) return DFD_ERR_PARAM;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  if (w) CK(h2d(ctx, ctx->guess_net, w, sizeof(float) * n));
  ctx->p.rs_guess = w ? 1 : 0;
  // the switch is baked into the step graphs: rebuild them
  for (auto& g : ctx->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return DFD_OK;
}

// ---- halo exchange of a slab of a domain decomposed along y
static long long halo_count(const dfd_ctx* ctx, int what) {
  const Dims& d = ctx->d;
  if (what == DFD_HALO_SETUP) return 13LL * 3 * d.nx * d.nz;
  return 9LL * 3 * d.nx * d.nz + (ctx->p.rupture ? 18LL * 3 * d.nz : 0);
}

int dfd_halo_floats(dfd_ctx* ctx, long long* floats) {
  if (!ctx || !floats) return DFD_ERR_PARAM;
  *floats = std::max(halo_count(ctx, DFD_HALO_SETUP), halo_count(ctx, 0));
  return DFD_OK;
}

static int halo_move(dfd_ctx* ctx, int what, int side, float* buf, int unpack) {
  if (!ctx || !buf || side < 0 || side > 1 || what < 0 || what > DFD_HALO_SETUP) return DFD_ERR_PARAM;
  if (ctx->sticky) return ctx->sticky;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  cudaSetDevice(ctx->device);
  const Dims& d = ctx->d;
  // leaving: the slab's first or last three columns; arriving: the ghost columns beside them
  const int jp = unpack ? (side ? d.nj + 3 : 0) : (side ? d.nj : 3);
  static const int bin[4] = {0, 1, 2, 1};  // stage inputs (the buffer cycle of the stages)
  float* vol = what == DFD_HALO_SETUP ? ctx->M : ctx->W[bin[what]];
  const int nvf = what == DFD_HALO_SETUP ? 13 : 9;
  float* fw = what < DFD_HALO_SETUP && ctx->p.rupture ? ctx->FW[what % 2] : nullptr;
  const int nff = fw ? 18 : 0;
  const long long n = halo_count(ctx, what);
  const int threads = 256;
  const int blocks = (int)std::min<long long>((n + threads - 1) / threads, 148LL * 8);
  dfd::halo_kernel<<<blocks, threads, 0, ctx->s0>>>(d, vol, nvf, fw, nff, jp, buf, unpack);
  return cuda_check(ctx, cudaGetLastError(), "halo");
}
int dfd_halo_pack(dfd_ctx* ctx, int what, int side, float* buf) { return halo_move(ctx, what, side, buf, 0); }
int dfd_halo_unpack(dfd_ctx* ctx, int what, int side, const float* buf) {
  return halo_move(ctx, what, side, const_cast<float*>(buf), 1);
}

int dfd_test_wait_drill(dfd_ctx* ctx, int on) {
  if (!ctx) return DFD_ERR_PARAM;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  ctx->tile.drill = on ? 1 : 0;
  // the switch is baked into the step graphs: rebuild them
  for (auto& g : ctx->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return DFD_OK;
}

int dfd_rs_profile(dfd_ctx* ctx, int timing, int judge) {
  if (!ctx) return DFD_ERR_PARAM;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  ctx->rs_prof = timing ? 1 : 0;
  ctx->rs_judge = judge ? 1 : 0;
  // the switches are baked into the step graphs: rebuild them
  for (auto& g : ctx->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return DFD_OK;
}

int dfd_rs_solve_stats(dfd_ctx* ctx, long long* accepted, long long* fallback, double* cycles_per_solve,
                       double* judge_max_rel) {
  if (!ctx) return DFD_ERR_PARAM;
  unsigned long long v[8] = {};
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  CK(cudaMemcpy(v, ctx->newton, sizeof v, cudaMemcpyDeviceToHost));
  if (accepted) *accepted = (long long)v[2];
  if (fallback) *fallback = (long long)v[3];
  if (cycles_per_solve) *cycles_per_solve = v[5] ? (double)v[4] / (double)v[5] : 0.0;
  if (judge_max_rel) {
    float f;
    unsigned u = (unsigned)v[6];
    memcpy(&f, &u, sizeof f);
    *judge_max_rel = f;
  }
  return DFD_OK;
}

int dfd_set_tile_rows(dfd_ctx* ctx, int rows) {
  if (!ctx || (rows != 8 && rows != 4)) return DFD_ERR_PARAM;
  if (mid_step(ctx)) return fail(ctx, DFD_ERR_STATE, "a step is half done (dfd_stage)");
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  ctx->tile.tr = rows;
  // the tile shape is baked into the step graphs: rebuild them
  for (auto& g : ctx->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return DFD_OK;
}

int dfd_newton_record(dfd_ctx* ctx, int capacity, int every) {
  if (!ctx || capacity < 0 || every < 1) return DFD_ERR_PARAM;
  ctx->rec_every = every;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  if (ctx->rec) {
    cudaFree(ctx->rec);
    ctx->rec = nullptr;
    ctx->rec_cap = 0;
  }
  if (capacity > 0) {
    CK(cudaMalloc(&ctx->rec, sizeof(float) * 5 * (size_t)capacity));
    ctx->rec_cap = capacity;
  }
  CK(cudaMemsetAsync(ctx->rec_n, 0, sizeof(unsigned), ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  // the recording buffer is baked into the step graphs: rebuild them
  for (auto& g : ctx->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return DFD_OK;
}

int dfd_newton_samples(dfd_ctx* ctx, float* host, int max, int* n) {
  if (!ctx || !n || max < 0 || (max > 0 && !host)) return DFD_ERR_PARAM;
  cudaSetDevice(ctx->device);
  CK(cudaStreamSynchronize(ctx->s0));
  unsigned got = 0;
  CK(cudaMemcpy(&got, ctx->rec_n, sizeof(unsigned), cudaMemcpyDeviceToHost));
  int m = (int)std::min<unsigned>(got, (unsigned)ctx->rec_cap);
  m = std::min(m, max);
  if (m > 0) CK(cudaMemcpy(host, ctx->rec, sizeof(float) * 5 * (size_t)m, cudaMemcpyDeviceToHost));
  *n = m;
  CK(cudaMemsetAsync(ctx->rec_n, 0, sizeof(unsigned), ctx->s0));
  CK(cudaStreamSynchronize(ctx->s0));
  return DFD_OK;
}

// ------------------------------------------------------------------ output --
// the writer thread: puts each finished record into the files, in order
static void out_writer(dfd_ctx* ctx) {
  OutState& o = *ctx->out;
  cudaSetDevice(ctx->device);
  const size_t nf = o.nf;
  std::vector<float> zero(ctx->p.rupture ? nf : 0, 0.0f);
  for (;;) {
    std::pair<int, int> r;
    {
      std::unique_lock<std::mutex> lk(o.mu);
      o.cv.wait(lk, [&] { return o.stop || !o.q.empty(); });
      if (o.q.empty()) break;
      r = o.q.front();
      o.q.pop_front();
    }
    const int rec = r.first, slot = r.second;
    int e = cudaEventSynchronize(o.done[slot]) == cudaSuccess ? 0 : DFD_ERR_CUDA;
    const float* h = o.host[slot];
    bool ok = true;
    if (!e && ctx->p.rupture) {
      for (int i = 0; i < 7; i++) ok = ok && ctx->ncf.put_record(ctx->vf[10 + i], rec, h + i * nf);
      ok = ok && ctx->ncf.put_fixed(ctx->vf[3], h + 7 * nf);
      ok = ok && ctx->ncf.put_record(17, rec, h + 8 * nf);
      ok = ok && ctx->ncf.put_record(18, rec, h + 9 * nf);
      ok = ok && ctx->ncf.put_record(19, rec, h + 10 * nf);  // rup_sensor
      // TP_T, TP_P at the fault (io_fault.cu:263-265), zero without thermal pressurisation
      ok = ok && ctx->ncf.put_record(20, rec, ctx->tp_T ? h + 11 * nf : zero.data());
      ok = ok && ctx->ncf.put_record(21, rec, ctx->tp_T ? h + 12 * nf : zero.data());
      ok = ok && ctx->ncf.sync();
    }
    for (int a = 0; a < 3 && !e; a++) {
      if (!o.slice_n[a]) continue;
      for (int c = 0; c < 3; c++)
        ok = ok && ctx->ncw[a].put_record(ctx->vw[a][c], rec, h + o.slice_off[a] + c * o.slice_n[a]);
      ok = ok && ctx->ncw[a].sync();
    }
    if (!e && !ok) e = DFD_ERR_IO;
    {
      std::lock_guard<std::mutex> lk(o.mu);
      o.busy[slot] = false;
      if (e && !o.err) o.err = e;
    }
    o.cv.notify_all();
  }
}

int dfd_output_open(dfd_ctx* ctx, const char* outdir) {
  if (!ctx || !outdir) return DFD_ERR_PARAM;
  if (!ctx->ready) return fail(ctx, DFD_ERR_STATE, "dfd_precompute has not run");
  const dfd_params& p = ctx->p;
  const Dims& d = ctx->d;
  std::string dir(outdir);
  // fault file (io_fault.cu:16-71)
  if (p.rupture) {
    NcWriter& w = ctx->ncf;
    char fn[64];
    snprintf(fn, sizeof fn, "/fault_mpi%06d.nc", p.slab_y);
    if (!w.open(dir + fn)) return fail(ctx, DFD_ERR_IO, "cannot create fault output");
    int nt = w.dim("nt", 0), nzd = w.dim("nz", d.nk), nyd = w.dim("ny", d.nj);
    std::vector<int> d2 = {nzd, nyd}, d3 = {nt, nzd, nyd};
    const char* fixed[] = {"x", "y", "z", "init_t0", "C0", "str_peak"};
    for (int i = 0; i < 6; i++) ctx->vf[i] = w.var(fixed[i], 5, d2);
    ctx->vf[6] = w.var("united", 4, d2);
    ctx->vf[7] = w.var("a", 5, d2);
    ctx->vf[8] = w.var("b", 5, d2);
    ctx->vf[9] = w.var("Vw", 5, d2);
    const char* rec[] = {"Vs1", "Vs2", "tn", "ts1", "ts2", "Us0", "State"};
    for (int i = 0; i < 7; i++) ctx->vf[10 + i] = w.var(rec[i], 5, d3);
    w.var("rup_index_y", 4, d3);
    w.var("rup_index_z", 4, d3);
    w.var("rup_sensor", 5, d3);
    w.var("TP_T", 5, d3);
    w.var("TP_P", 5, d3);
    w.enddef();
    size_t nf = (size_t)d.nj * d.nk;
    std::vector<float> x(nf), y(nf), z(nf), t(nf);
    for (int k = 0; k < d.nk; k++)
      for (int j = 0; j < d.nj; j++) {
        size_t q = j + (size_t)k * d.nj, f = (j + 3) + (size_t)(k + 3) * d.ny;
        x[q] = (float)(ctx->xl[d.i0] + ctx->fx[f]);
        y[q] = (float)ctx->fy[f];
        z[q] = (float)ctx->fz[f];
      }
    w.put_fixed(ctx->vf[0], x.data());
    w.put_fixed(ctx->vf[1], y.data());
    w.put_fixed(ctx->vf[2], z.data());
    CK(cudaMemcpy(t.data(), ctx->pl + P_C0 * nf, sizeof(float) * nf, cudaMemcpyDeviceToHost));
    w.put_fixed(ctx->vf[4], t.data());
    CK(cudaMemcpy(t.data(), ctx->pl + P_PEAK * nf, sizeof(float) * nf, cudaMemcpyDeviceToHost));
    w.put_fixed(ctx->vf[5], t.data());
    std::vector<int> u(nf);
    CK(cudaMemcpy(u.data(), ctx->ipl + I_UNITED * nf, sizeof(int) * nf, cudaMemcpyDeviceToHost));
    w.put_fixed(ctx->vf[6], u.data());
    int ab[3] = {P_A, P_B, P_VW};
    for (int i = 0; i < 3; i++) {
      CK(cudaMemcpy(t.data(), ctx->pl + ab[i] * nf, sizeof(float) * nf, cudaMemcpyDeviceToHost));
      w.put_fixed(ctx->vf[7 + i], t.data());
    }
    w.sync();
  }
  // wave slices (io_wave_xy.cu / io_wave_xz.cu / io_wave_yz.cu)
  const char* names[3] = {"wave_yz", "wave_xz", "wave_xy"};
  // the y slice in this slab's columns (written by the slab that holds it)
  int idx[3] = {p.EXPORT_WAVE_SLICE_X, p.EXPORT_WAVE_SLICE_Y - p.slab_y * d.nj, p.EXPORT_WAVE_SLICE_Z};
  int lim[3] = {d.ni, d.nj, d.nk};
  for (int a = 0; a < 3; a++) {
    if (idx[a] < 0 || idx[a] >= lim[a]) continue;
    NcWriter& w = ctx->ncw[a];
    char fn[64];
    snprintf(fn, sizeof fn, "/%s_mpi%06d.nc", names[a], p.slab_y);
    if (!w.open(dir + fn)) return fail(ctx, DFD_ERR_IO, "cannot create slice output");
    int nt = w.dim("nt", 0);
    int da, db;
    if (a == 0) { da = w.dim("nz", d.nk); db = w.dim("ny", d.nj); }
    else if (a == 1) { da = w.dim("nx", d.ni); db = w.dim("nz", d.nk); }
    else { da = w.dim("nx", d.ni); db = w.dim("ny", d.nj); }
    std::vector<int> d2 = {da, db}, d3 = {nt, da, db};
    int cx = w.var("x", 5, d2), cy = w.var("y", 5, d2), cz = w.var("z", 5, d2);
    ctx->vw[a][0] = w.var("Vx", 5, d3);
    ctx->vw[a][1] = w.var("Vy", 5, d3);
    ctx->vw[a][2] = w.var("Vz", 5, d3);
    w.enddef();
    int na = a == 0 ? d.nk : d.ni, nb = a == 1 ? d.nk : d.nj;
    std::vector<float> X((size_t)na * nb), Y(X.size()), Z(X.size());
    for (int ia = 0; ia < na; ia++)
      for (int ib = 0; ib < nb; ib++) {
        int i, j, k;
        if (a == 0) { i = idx[a]; k = ia; j = ib; }
        else if (a == 1) { j = idx[a]; i = ia; k = ib; }
        else { k = idx[a]; i = ia; j = ib; }
        size_t f = (j + 3) + (size_t)(k + 3) * d.ny, q = (size_t)ia * nb + ib;
        X[q] = (float)(ctx->xl[i + 3] + ctx->fx[f]);
        Y[q] = (float)ctx->fy[f];
        Z[q] = (float)ctx->fz[f];
      }
    w.put_fixed(cx, X.data());
    w.put_fixed(cy, Y.data());
    w.put_fixed(cz, Z.data());
    w.sync();
  }
  // staging sets, pinned host buffers, side stream and the writer thread
  OutState* o = new OutState();
  ctx->out = o;
  o->nf = (size_t)d.nj * d.nk;
  // record planes: the seven outputs, init_t0, rup_index_y/z, rup_sensor, then TP_T and
  // TP_P at the fault when thermal pressurisation is on
  size_t off = p.rupture ? (ctx->tp_T ? 13 : 11) * o->nf : 0;
  for (int a = 0; a < 3; a++) {
    if (idx[a] < 0 || idx[a] >= lim[a]) continue;
    const int na = a == 0 ? d.nk : d.ni, nb = a == 1 ? d.nk : d.nj;
    o->slice_off[a] = off;
    o->slice_n[a] = (size_t)na * nb;
    off += 3 * o->slice_n[a];
  }
  o->bytes = std::max<size_t>(off, 1) * sizeof(float);
  for (int b = 0; b < 2; b++) {
    CK(cudaMalloc(&o->dev[b], o->bytes));
    CK(cudaMallocHost(&o->host[b], o->bytes));
    CK(cudaEventCreateWithFlags(&o->done[b], cudaEventDisableTiming));
  }
  CK(cudaEventCreateWithFlags(&o->snap, cudaEventDisableTiming));
  CK(cudaStreamCreateWithFlags(&o->s, cudaStreamNonBlocking));
  o->writer = std::thread(out_writer, ctx);
  ctx->out_open = true;
  return DFD_OK;
}

// one output record (the reference writes it before the step, main.cu:425-437): a
// snapshot on the stepping stream, the copy to the host and the file writes behind it
static const int kOutPlanes[7] = {P_VS1, P_VS2, P_TN, P_TS1, P_TS2, P_SLIP, P_STATE};

int dfd_output_write(dfd_ctx* ctx, int it_skip) {
  if (!ctx || !ctx->out_open || !ctx->out) return DFD_ERR_STATE;
  if (ctx->sticky) return ctx->sticky;
  OutState& o = *ctx->out;
  const int slot = o.next;
  {
    // wait until the writer has put this slot's previous record into the files
    std::unique_lock<std::mutex> lk(o.mu);
    o.cv.wait(lk, [&] { return !o.busy[slot] || o.err; });
    if (o.err) return fail(ctx, o.err, "output: a record could not be written");
  }
  cudaSetDevice(ctx->device);
  const Dims& d = ctx->d;
  const size_t nf = o.nf;
  float* dst = o.dev[slot];
  if (ctx->p.rupture) {
    for (int i = 0; i < 7; i++)
      CK(cudaMemcpyAsync(dst + i * nf, ctx->pl + kOutPlanes[i] * nf, sizeof(float) * nf, cudaMemcpyDeviceToDevice,
                         ctx->s0));
    CK(cudaMemcpyAsync(dst + 7 * nf, ctx->pl + P_T0 * nf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, ctx->s0));
    CK(cudaMemcpyAsync(dst + 8 * nf, ctx->ipl + I_RUPY * nf, sizeof(int) * nf, cudaMemcpyDeviceToDevice, ctx->s0));
    CK(cudaMemcpyAsync(dst + 9 * nf, ctx->ipl + I_RUPZ * nf, sizeof(int) * nf, cudaMemcpyDeviceToDevice, ctx->s0));
    CK(cudaMemcpyAsync(dst + 10 * nf, ctx->pl + P_RUPS * nf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, ctx->s0));
    if (ctx->tp_T) {
      CK(cudaMemcpyAsync(dst + 11 * nf, ctx->pl + P_TPT0 * nf, sizeof(float) * 2 * nf, cudaMemcpyDeviceToDevice,
                         ctx->s0));
    }
  }
  const int idx[3] = {ctx->p.EXPORT_WAVE_SLICE_X, ctx->p.EXPORT_WAVE_SLICE_Y - ctx->p.slab_y * ctx->d.nj,
                      ctx->p.EXPORT_WAVE_SLICE_Z};
  for (int a = 0; a < 3; a++)
    if (o.slice_n[a])
      dfd::slice_kernel<<<(unsigned)((o.slice_n[a] + 255) / 256), 256, 0, ctx->s0>>>(d, ctx->W[0], a, idx[a],
                                                                                      dst + o.slice_off[a]);
  CK(cudaEventRecord(o.snap, ctx->s0));
  CK(cudaStreamWaitEvent(o.s, o.snap, 0));
  CK(cudaMemcpyAsync(o.host[slot], dst, o.bytes, cudaMemcpyDeviceToHost, o.s));
  CK(cudaEventRecord(o.done[slot], o.s));
  {
    std::lock_guard<std::mutex> lk(o.mu);
    o.busy[slot] = true;
    o.q.emplace_back(it_skip, slot);
  }
  o.cv.notify_all();
  o.next = slot ^ 1;
  return DFD_OK;
}

int dfd_output_close(dfd_ctx* ctx) {
  if (!ctx) return DFD_ERR_PARAM;
  int err = 0;
  if (ctx->out) {
    OutState* o = ctx->out;
    {
      std::lock_guard<std::mutex> lk(o->mu);
      o->stop = true;
    }
    o->cv.notify_all();
    if (o->writer.joinable()) o->writer.join();
    err = o->err;
    for (int b = 0; b < 2; b++) {
      if (o->dev[b]) cudaFree(o->dev[b]);
      if (o->host[b]) cudaFreeHost(o->host[b]);
      if (o->done[b]) cudaEventDestroy(o->done[b]);
    }
    if (o->snap) cudaEventDestroy(o->snap);
    if (o->s) cudaStreamDestroy(o->s);
    delete o;
    ctx->out = nullptr;
  }
  ctx->ncf.close();
  for (auto& w : ctx->ncw) w.close();
  ctx->out_open = false;
  return err ? fail(ctx, err, "output: a record could not be written") : DFD_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ ensemble --
// A batch of prepared scenarios (contexts on one device) stepped together: per RK stage
// one batched launch each of the fault node, fault band and general (shell) kernels over
// every scenario, and one persistent launch of the tiled interior kernel whose units span
// all scenarios.  The per-stage argument tables live in device memory (one set per flag
// pattern and stage); each step is replayed from a CUDA graph.  Scenario state stays in
// the scenarios' own contexts, so results are read with the usual getters.
struct EnsStage {
  FaultArgs* fault = nullptr;  // rupture scenarios
  int* fstart = nullptr;       // (nf + 1) block starts of the fault node kernel
  int fblocks = 0;
  int* bstart = nullptr;       // (nf + 1) block starts of the fault band kernel
  int bblocks = 0;
  VolArgs* vol = nullptr;      // all scenarios
  Boxes* boxes = nullptr;
  int* sstart = nullptr;       // (n + 1) block starts of the shell kernel, boxes below the top rows
  int sblocks = 0;
  int* tstart = nullptr;       // (n + 1) block starts of the shell kernel, free-surface rows
  int tblocks = 0;
  TileScen* tile = nullptr;    // all scenarios, interior kernel
  TileScen first;              // scenario 0, passed by value (stage-wide values)
  int nunits = 0;
  TileScen* ptile = nullptr;   // all scenarios, PML kernel
  TileScen pfirst;
  int punits = 0;
  int FX = 1, FY = 1, FZ = 1;
};

struct dfd_ens {
  std::vector<dfd_ctx*> sc;
  std::vector<int> rup;        // indices of rupture scenarios
  int device = 0;
  int nsm = 148;
  int chunk = 0;               // planes per unit of the tiled kernel (0: per-scenario plan)
  int tr = TILE_K;             // rows of the interior kernel's tiles (every scenario's)
  cudaStream_t s0 = nullptr, s1 = nullptr, s2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr;
  int* it_dev = nullptr;
  int* sched = nullptr;
  int* err = nullptr;
  std::vector<void*> allocs;
  EnsStage st[8][4];
  bool built = false;
  cudaGraphExec_t graph[8] = {};
  std::string msg;
  long long nodes = 0;
};

static int ens_fail(dfd_ens* e, int code, const std::string& m) {
  if (e) e->msg = m;
  return code;
}
#define ECK(call)                                                                          \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) return ens_fail(e, DFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <typename T>
static int ens_upload(dfd_ens* e, T** dst, const std::vector<T>& v) {
  void* p = nullptr;
  ECK(cudaMalloc(&p, sizeof(T) * std::max<size_t>(v.size(), 1)));
  e->allocs.push_back(p);
  if (!v.empty()) {
    // on the ensemble's stream and complete on return (see h2d)
    ECK(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, e->s0));
    ECK(cudaStreamSynchronize(e->s0));
  }
  *dst = (T*)p;
  return DFD_OK;
}

// tables of every (pattern, stage): argument structs, block starts, tile units
static int ens_build(dfd_ens* e) {
  for (auto& row : e->st)
    for (auto& t : row) t = EnsStage();
  for (void* p : e->allocs) cudaFree(p);
  e->allocs.clear();
  static const int bin[4] = {0, 1, 2, 1};
  const int n = (int)e->sc.size();
  for (int pat = 0; pat < 8; pat++)
    for (int irk = 0; irk < 4; irk++) {
      EnsStage& S = e->st[pat][irk];
      int sg = (irk % 2) ? -1 : 1;
      S.FX = kFlags[pat][0] * sg; S.FY = kFlags[pat][1] * sg; S.FZ = kFlags[pat][2] * sg;
      std::vector<FaultArgs> fa;
      std::vector<int> fs(1, 0), bs(1, 0);
      for (int r : e->rup) {
        FaultArgs a = fault_args(e->sc[r], pat, irk);
        a.it_dev = e->it_dev;  // one step counter for the whole ensemble
        fa.push_back(a);
        const int g = ((a.d.nj + 31) / 32) * ((a.d.nk + 3) / 4);
        fs.push_back(fs.back() + node_blocks(a.NY, a.NZ, a.freenode, a.jg0, a.d.nj));
        bs.push_back(bs.back() + 7 * g);  // the band kernel: seven parts per column block
      }
      S.fblocks = fs.back();
      S.bblocks = bs.back();
      std::vector<VolArgs> va;
      std::vector<Boxes> bx;
      std::vector<int> ss(1, 0), tt(1, 0);
      std::vector<TileScen> ts(n), ps(n);
      int units = 0, punits = 0;
      for (int i = 0; i < n; i++) {
        dfd_ctx* c = e->sc[i];
        VolArgs a = vol_args(c, pat, irk);
        VolPlan pl = plan_volume(a, c->use_tile ? &c->tile : nullptr);
        if (pl.plain || pl.ps.nunits < 0)
          return ens_fail(e, DFD_ERR_PARAM, "scenario " + std::to_string(i) + " cannot use the tiled kernels");
        va.push_back(a);
        bx.push_back(pl.bx);
        ss.push_back(ss.back() + pl.bx.start[pl.bx.ntop]);
        tt.push_back(tt.back() + pl.bx.start[pl.bx.n] - pl.bx.start[pl.bx.ntop]);
        TileSched sch;
        memset(&sch, 0, sizeof sch);
        if (pl.tiled) {
          int grid = 0;
          sch = tile_plan(pl.lo, pl.hi, e->nsm * tile_ctas_per_sm(e->tr), &grid, e->tr);
          if (e->chunk > 0) {
            sch.ci = std::min(e->chunk, pl.hi.x - pl.lo.x);
            sch.nunits = sch.ntj * sch.ntk * ((pl.hi.x - pl.lo.x + sch.ci - 1) / sch.ci);
          }
        }
        TileScen& t = ts[i];
        t.mp = tile_maps(c->tile, bin[irk], irk, e->tr);
        t.u.a = a;
        t.u.sc = sch;
        t.u.unit0 = units;
        units += sch.nunits;
        TileScen& tp = ps[i];
        tp.mp = t.mp;
        tp.u.a = a;
        tp.u.sc = pl.ps;
        tp.u.unit0 = punits;
        punits += pl.ps.nunits;
      }
      S.nunits = units;
      S.punits = punits;
      S.pfirst = ps[0];
      S.sblocks = ss.back();
      S.tblocks = tt.back();
      S.first = ts[0];
      int r = 0;
      if (!e->rup.empty()) {
        r = r ? r : ens_upload(e, &S.fault, fa);
        r = r ? r : ens_upload(e, &S.fstart, fs);
        r = r ? r : ens_upload(e, &S.bstart, bs);
      }
      r = r ? r : ens_upload(e, &S.vol, va);
      r = r ? r : ens_upload(e, &S.boxes, bx);
      r = r ? r : ens_upload(e, &S.sstart, ss);
      r = r ? r : ens_upload(e, &S.tstart, tt);
      r = r ? r : ens_upload(e, &S.tile, ts);
      r = r ? r : ens_upload(e, &S.ptile, ps);
      if (r) return r;
    }
  e->built = true;
  return DFD_OK;
}

static int ens_enqueue(dfd_ens* e, int pat, int irk) {
  const EnsStage& S = e->st[pat][irk];
  const int nr = (int)e->rup.size(), n = (int)e->sc.size();
  if (irk == 0)
    for (int r : e->rup) {
      launch_rup_sensor(sensor_args(e->sc[r]), e->s0);
      if (e->sc[r]->tp_T) launch_thermpress(tp_args(e->sc[r]), e->s0);
    }
  if (nr) launch_fault_node_batch(S.fault, S.fstart, nr, S.fblocks, S.FY, S.FZ, e->s0);
  if (e->sc[0]->serial) {
    launch_tile_batch(S.first, S.tile, n, S.nunits, e->nsm, e->tr, S.FX, S.FY, S.FZ, e->err, e->sched, e->s0);
    launch_pml_batch(S.pfirst, S.ptile, n, S.punits, e->nsm, S.FX, S.FY, S.FZ, e->err, e->sched, S.nunits > 0,
                     e->s0);
    // the general kernel beside the fault band kernel
    cudaEventRecord(e->ev_fork, e->s0);
    cudaStreamWaitEvent(e->s2, e->ev_fork, 0);
    launch_shell_batch(S.vol, S.boxes, S.sstart, n, S.sblocks, S.FX, S.FY, S.FZ, false, irk, e->s2);
    launch_shell_batch(S.vol, S.boxes, S.tstart, n, S.tblocks, S.FX, S.FY, S.FZ, true, irk, e->s2);
    cudaEventRecord(e->ev_join2, e->s2);
    if (nr) launch_fault_band_batch(S.fault, S.bstart, nr, S.bblocks, S.FX, S.FY, S.FZ, e->s0);
    cudaStreamWaitEvent(e->s0, e->ev_join2, 0);
    cudaError_t ce = cudaGetLastError();
    return ce == cudaSuccess ? DFD_OK : ens_fail(e, DFD_ERR_CUDA, std::string("ensemble stage: ") + cudaGetErrorString(ce));
  }
  cudaEventRecord(e->ev_fork, e->s0);
  if (nr) {
    cudaStreamWaitEvent(e->s1, e->ev_fork, 0);
    launch_fault_band_batch(S.fault, S.bstart, nr, S.bblocks, S.FX, S.FY, S.FZ, e->s1);
    cudaEventRecord(e->ev_join, e->s1);
  }
  cudaStreamWaitEvent(e->s2, e->ev_fork, 0);
  launch_shell_batch(S.vol, S.boxes, S.sstart, n, S.sblocks, S.FX, S.FY, S.FZ, false, irk, e->s2);
  launch_shell_batch(S.vol, S.boxes, S.tstart, n, S.tblocks, S.FX, S.FY, S.FZ, true, irk, e->s2);
  cudaEventRecord(e->ev_join2, e->s2);
  launch_tile_batch(S.first, S.tile, n, S.nunits, e->nsm, e->tr, S.FX, S.FY, S.FZ, e->err, e->sched, e->s0);
  launch_pml_batch(S.pfirst, S.ptile, n, S.punits, e->nsm, S.FX, S.FY, S.FZ, e->err, e->sched, S.nunits > 0,
                     e->s0);
  if (nr) cudaStreamWaitEvent(e->s0, e->ev_join, 0);
  cudaStreamWaitEvent(e->s0, e->ev_join2, 0);
  cudaError_t ce = cudaGetLastError();
  return ce == cudaSuccess ? DFD_OK : ens_fail(e, DFD_ERR_CUDA, std::string("ensemble stage: ") + cudaGetErrorString(ce));
}

static void ens_drop_graphs(dfd_ens* e) {
  for (auto& g : e->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static int ens_graph(dfd_ens* e, int pat) {
  cudaGraph_t g;
  ECK(cudaStreamBeginCapture(e->s0, cudaStreamCaptureModeThreadLocal));
  int r = 0;
  for (int irk = 0; irk < 4 && !r; irk++) r = ens_enqueue(e, pat, irk);
  dfd::inc_it_kernel<<<1, 1, 0, e->s0>>>(e->it_dev);
  cudaError_t ce = cudaStreamEndCapture(e->s0, &g);
  if (r) return r;
  ECK(ce);
  ECK(cudaGraphInstantiate(&e->graph[pat], g, 0));
  cudaGraphDestroy(g);
  return DFD_OK;
}

extern "C" {

int dfd_ens_create(dfd_ctx* const* scenarios, int n, dfd_ens** out) {
  if (!scenarios || n <= 0 || !out) return DFD_ERR_PARAM;
  *out = nullptr;
  dfd_ens* e = new dfd_ens();
  e->device = scenarios[0]->device;
  for (int i = 0; i < n; i++) {
    dfd_ctx* c = scenarios[i];
    if (!c || !c->ready || c->device != e->device || mid_step(c) || !c->use_tile) {
      delete e;
      return DFD_ERR_PARAM;
    }
    e->sc.push_back(c);
    if (c->p.rupture) e->rup.push_back(i);
    e->nodes += (long long)c->p.NX * c->p.NY * c->p.NZ;
  }
  cudaSetDevice(e->device);
  e->nsm = scenarios[0]->tile.nsm;
  e->tr = scenarios[0]->tile.tr;  // one batched launch: every scenario with the same tile rows
  for (int i = 1; i < n; i++)
    if (scenarios[i]->tile.tr != e->tr) {
      delete e;
      return DFD_ERR_PARAM;
    }
  auto done = [&](int rc) {
    if (rc) dfd_ens_destroy(e);
    return rc;
  };
  if (cudaStreamCreateWithFlags(&e->s0, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->s1, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->s2, cudaStreamNonBlocking) != cudaSuccess)
    return done(DFD_ERR_CUDA);
  cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&e->ev_join2, cudaEventDisableTiming);
  void* p = nullptr;
  if (cudaMalloc(&p, 6 * sizeof(int)) != cudaSuccess) return done(DFD_ERR_CUDA);
  // cleared on the ensemble's stream (a plain cudaMemset is not ordered with it)
  if (cudaMemsetAsync(p, 0, 6 * sizeof(int), e->s0) != cudaSuccess || cudaStreamSynchronize(e->s0) != cudaSuccess)
    return done(DFD_ERR_CUDA);
  e->it_dev = (int*)p;
  e->sched = e->it_dev + 1;  // unit and finished-CTA counters of the interior, then the PML kernel
  e->err = e->it_dev + 5;
  for (dfd_ctx* c : e->sc) cudaStreamSynchronize(c->s0);
  int r = ens_build(e);
  if (r) return done(r);
  *out = e;
  return DFD_OK;
}

int dfd_ens_destroy(dfd_ens* e) {
  if (!e) return DFD_OK;
  cudaSetDevice(e->device);
  ens_drop_graphs(e);
  if (e->s0) cudaStreamSynchronize(e->s0);
  if (e->s1) cudaStreamSynchronize(e->s1);
  if (e->s2) cudaStreamSynchronize(e->s2);
  for (void* p : e->allocs) cudaFree(p);
  if (e->it_dev) cudaFree(e->it_dev);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  if (e->ev_join2) cudaEventDestroy(e->ev_join2);
  if (e->s0) cudaStreamDestroy(e->s0);
  if (e->s1) cudaStreamDestroy(e->s1);
  if (e->s2) cudaStreamDestroy(e->s2);
  delete e;
  return DFD_OK;
}

int dfd_ens_run(dfd_ens* e, int it0, int nsteps) {
  if (!e) return DFD_ERR_PARAM;
  cudaSetDevice(e->device);
  dfd::set_it_kernel<<<1, 1, 0, e->s0>>>(e->it_dev, it0);
  for (int s = 0; s < nsteps; s++) {
    int pat = (((it0 + s) % 8) + 8) % 8;
    if (!e->graph[pat]) {
      int r = ens_graph(e, pat);
      if (r) return r;
    }
    ECK(cudaGraphLaunch(e->graph[pat], e->s0));
  }
  return DFD_OK;
}

int dfd_ens_synchronize(dfd_ens* e) {
  if (!e) return DFD_ERR_PARAM;
  cudaSetDevice(e->device);
  ECK(cudaStreamSynchronize(e->s0));
  ECK(cudaStreamSynchronize(e->s1));
  ECK(cudaStreamSynchronize(e->s2));
  int f = 0;
  ECK(cudaMemcpy(&f, e->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (f) return ens_fail(e, DFD_ERR_CUDA, "tiled interior kernel: a TMA copy did not complete");
  return DFD_OK;
}

int dfd_ens_run_timed(dfd_ens* e, int it0, int nsteps, float* ms) {
  if (!e || nsteps <= 0) return DFD_ERR_PARAM;
  cudaSetDevice(e->device);
  cudaEvent_t a, b;
  ECK(cudaEventCreate(&a));
  ECK(cudaEventCreate(&b));
  for (int s = 0; s < nsteps; s++) {  // graphs first, outside the timed region
    int pat = (((it0 + s) % 8) + 8) % 8;
    if (!e->graph[pat]) {
      int r = ens_graph(e, pat);
      if (r) return r;
    }
  }
  ECK(cudaEventRecord(a, e->s0));
  int r = dfd_ens_run(e, it0, nsteps);
  if (r) return r;
  ECK(cudaEventRecord(b, e->s0));
  ECK(cudaEventSynchronize(b));
  float t = 0;
  ECK(cudaEventElapsedTime(&t, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms) *ms = t;
  return dfd_ens_synchronize(e);
}

int dfd_ens_set_chunk(dfd_ens* e, int chunk) {
  if (!e || chunk < 0) return DFD_ERR_PARAM;
  cudaSetDevice(e->device);
  ECK(cudaStreamSynchronize(e->s0));
  ens_drop_graphs(e);
  e->chunk = chunk;
  return ens_build(e);
}

int dfd_ens_set_tile_rows(dfd_ens* e, int rows) {
  if (!e || (rows != 8 && rows != 4)) return DFD_ERR_PARAM;
  cudaSetDevice(e->device);
  ECK(cudaStreamSynchronize(e->s0));
  ens_drop_graphs(e);
  e->tr = rows;
  for (dfd_ctx* c : e->sc) c->tile.tr = rows;  // the scenarios' maps follow (tile_maps)
  return ens_build(e);
}

int dfd_ens_nodes(const dfd_ens* e, long long* nodes) {
  if (!e || !nodes) return DFD_ERR_PARAM;
  *nodes = e->nodes;
  return DFD_OK;
}

const char* dfd_ens_last_error(const dfd_ens* e) { return e ? e->msg.c_str() : ""; }

}  // extern "C"
