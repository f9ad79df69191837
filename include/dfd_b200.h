/*
 * dfd_b200.h -- C ABI of the B200-native curved-grid finite-difference
 * dynamic-rupture time step (drop-in for the single-rank path of
 * wenqiang-geophys/dynfd3dcuda).
 *
 * Every entry point returns an int status (DFD_OK == 0).  The library owns all device
 * memory of a context; host arrays cross the boundary in the reference's layouts:
 *   volume field    (nx, nz, ny) with y fastest, nx = NX+6 (3 ghost nodes per side),
 *                   field order Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz   (common.h:99-101)
 *   fault plane     (NZ, NY) with y fastest                        (alloc.cu:123-168)
 *   split nodes     (9, 2, nz, ny): field, side (-,+), z, y         (alloc.cu:96)
 * There is no global state: every parameter lives in the context, so several contexts
 * (one per thread or per scenario) can coexist on one GPU.
 */
#ifndef DFD_B200_H
#define DFD_B200_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
  DFD_OK = 0,
  DFD_ERR_PARAM = 1,      /* bad or unsupported parameter */
  DFD_ERR_CUDA = 2,       /* CUDA call failed (sticky in the context) */
  DFD_ERR_IO = 3,         /* file missing or malformed */
  DFD_ERR_STATE = 4,      /* call out of order (e.g. step before precompute) */
  DFD_ERR_CFL = 5,        /* DT above the stability limit 1.3 hmin / vpmax */
  DFD_ERR_NONFINITE = 6,  /* NaN/Inf found in the fault state */
  DFD_ERR_NEWTON = 7      /* rate-and-state Newton hit its iteration cap */
};

/* Job parameters: the reference's Params fields (common.h:49-84) plus the reference's
 * compile-time switches (Makefile:57-161) as runtime flags with the reference's
 * defaults.  Filled by dfd_params_default() and dfd_params_load_json(). */
typedef struct dfd_params {
  int NX, NY, NZ;
  int NT;
  double TMAX, DT, DH;
  int INPORT_GRID_TYPE, INPORT_STRESS_TYPE, Friction_type;
  int EXPORT_TIME_SKIP, EXPORT_WAVE_SLICE_X, EXPORT_WAVE_SLICE_Y, EXPORT_WAVE_SLICE_Z;
  int PML_N;
  double PML_velocity, PML_bmax, PML_fc;
  int DAMP_N;
  double mu_s, mu_d, mu_0, Dc, C0;
  double f0, V0, Vini, fw, L;
  double smooth_load_T, viscosity;
  int Fault_grid[4];
  int Asp_grid[4];
  double bi_vp1, bi_vs1, bi_rho1, bi_vp2, bi_vs2, bi_rho2;
  /* switches (reference macros): rupture (fault kernels on), free surface, PML, Cerjan
   * sponge, normal refinement of the x grid around the fault */
  int rupture, free_surface, use_pml, use_cerjan, normal_refine;
  /* 0 = plain Newton initial guess (reference), 1 = learned guess with Newton fallback */
  int rs_guess;
  char OUT[1024];
  char Fault_geometry[1024];
  char Fault_init_stress[1024];
  char Media1D[1024];
  /* points across the fault of each thermal-pressurisation column (Friction_type 3);
   * the reference's default is 1, which Friction_type 3 rejects (see dfd_load_tp_hy) */
  int TP_n;
  /* residual test of the learned guess (rs_guess 1): after each of at most two Newton
   * corrections from the guess, the corrected guess is accepted when the bound on its
   * remaining error (quadratic convergence) is at most rs_guess_tol |x|; default 1e-10,
   * which keeps the slip rate within FP32 rounding of the plain solve's */
  double rs_guess_tol;
  /* decomposition of the domain along y (the reference's PY ranks, mod_mpi.cu): slabs_y
   * equal slabs of NY / slabs_y columns, this context holding slab slab_y; NY, Fault_grid
   * and the input files stay global.  Set by the caller, not read from a job file (a
   * reference job's PX, PY, PZ are accepted and ignored: the whole domain runs in one
   * context unless the caller splits it).  slabs_y 1 (default): one domain. */
  int slabs_y;
  int slab_y;
} dfd_params;

typedef struct dfd_ctx dfd_ctx;

/* Named on-fault / split-node / layer arrays for dfd_get_fault. */
enum {
  DFD_F_SLIP = 0, DFD_F_HSLIP, DFD_F_VS1, DFD_F_VS2, DFD_F_TN, DFD_F_TS1, DFD_F_TS2, DFD_F_STATE,
  DFD_F_INIT_T0, DFD_F_TTN, DFD_F_TTS1, DFD_F_TTS2, DFD_F_STR_PEAK, DFD_F_FRICTION,
  DFD_F_UNITED, DFD_F_FAULTGRID,            /* int32 masks, returned as float */
  DFD_F_SPLIT,                               /* (9, 2, nz, ny) split-node state   */
  DFD_F_T1,                                  /* (3, 7, nz, ny) T11 T12 T13 layers */
  DFD_F_HT1,                                 /* (3, nz, ny) hT11 hT12 hT13        */
  DFD_F_TP_T, DFD_F_TP_P,                    /* thermal pressurisation: temperature and pore
                                                pressure at the fault (point 0 of each column,
                                                as io_fault.cu:263-265 writes them) */
  DFD_F_RUP_SENSOR,                          /* rupture sensor of the step start
                                                (rup_sensor.cu:8-95) */
  DFD_F_COUNT
};

/* ---- parameters (set_params.cu:56-297) ---- */
/* sizeof(dfd_params), for bindings that mirror the struct */
int dfd_params_size(void);
int dfd_params_default(dfd_params *p);
int dfd_params_load_json(const char *path, dfd_params *p);

/* ---- lifetime (replaces alloc_wave / alloc_fault / alloc_fault_coef / alloc_pml,
 *      alloc.cu:16-508, and set_device_params, set_params.cu:39-54) ---- */
int dfd_create(const dfd_params *p, int device, dfd_ctx **out);
int dfd_destroy(dfd_ctx *ctx);
int dfd_dims(const dfd_ctx *ctx, int *nx, int *ny, int *nz);

/* ---- inputs (replace construct_coord coord.cu:153-328, init_media1d media.cu:63-138,
 *      nc_read_init_stress init.cu:904-1022) ---- */
/* fault surface x,y,z: 3 planes of (NZ, NY) float32 (Fault_geometry file) */
int dfd_load_fault_geometry(dfd_ctx *ctx, const float *fxyz);
/* 1-D layered medium: n rows of depth, rho, vp, vs (Media1D file) */
int dfd_load_media1d(dfd_ctx *ctx, int n, const float *layers);
/* 15 planes of (NZ, NY): Tx Ty Tz dTx dTy dTz mu_s mu_d Dc C0 a b L Vw State */
int dfd_load_fault_init(dfd_ctx *ctx, const float *planes);
/* Friction_type 3 only: hydraulic diffusivity TP_hy (m^2/s), one plane of (NZ, NY), the
 * TP_hy variable of the Fault_init_stress file (init.cu:999-1003); zero if never loaded.
 * DFD_ERR_STATE for any other friction type. */
int dfd_load_tp_hy(dfd_ctx *ctx, const float *tp_hy);

/* ---- setup: grid, metric and media on the GPU in FP64 (no 3-D coordinate array), PML
 *      and Cerjan profiles on the host, fault and free-surface coefficient tables on the
 *      GPU in FP64 (replaces construct_coord coord.cu:153-328, cal_metric
 *      metric.cu:15-171, abs_init init_pml.cu:42-155, init_cerjan_host cerjan.cu:31-164,
 *      init_fault_coef fault_coef.cu:26-1312, init_wave_free :1320-1498, init_fault
 *      init.cu:160-849), then the CFL check of main.cu:323-345 ---- */
int dfd_precompute(dfd_ctx *ctx);

/* ---- time stepping ---- */
/* one RK stage irk (0..3) of step it: the fused replacement of state_rk, trial_sw /
 * trial_rs, fault2wave, wave_deriv, abs_deriv_{x,y,z}, fault_dvelo, fault_dstrs_{f,b},
 * wave_rk, fault_rk, apply_cerjan (main.cu:448-516).  Stages must be issued in order. */
int dfd_stage(dfd_ctx *ctx, int it, int irk);
/* One part of stage irk, for part-by-part parity with the reference's launchers; parts
 * 0, 1, 2 issued in order are dfd_stage(ctx, it, irk).  The product fuses the reference's
 * launchers into three kernel groups, so a part stands for several of them:
 *   DFD_PART_FAULT_TRIAL  state_rk, trial_sw / trial_rs, fault2wave (main.cu:458-467);
 *                         at stage 0 first cal_rup_sensor and thermpress (main.cu:444-446)
 *   DFD_PART_VOLUME       wave_deriv, abs_deriv_{x,y,z}, and for every node outside the
 *                         fault band wave_rk and apply_cerjan (main.cu:469-481,495,508)
 *   DFD_PART_FAULT_BAND   fault_dvelo, fault_dstrs_{f,b}, wave_rk, fault_rk and fault2wave
 *                         for the fault band and split nodes (main.cu:486-504)
 * DFD_ERR_STATE when a part comes out of order; dfd_step / dfd_run refuse a stage left
 * half done. */
enum { DFD_PART_FAULT_TRIAL = 0, DFD_PART_VOLUME = 1, DFD_PART_FAULT_BAND = 2 };
int dfd_stage_part(dfd_ctx *ctx, int it, int irk, int part);
/* one full step (four stages, replayed from a CUDA graph per flag pattern) */
int dfd_step(dfd_ctx *ctx, int it);
/* nsteps steps starting at it0, without host synchronisation in between */
int dfd_run(dfd_ctx *ctx, int it0, int nsteps);
int dfd_synchronize(dfd_ctx *ctx);

/* ---- state access ---- */
int dfd_get_wave(dfd_ctx *ctx, float *host);        /* 9*nx*ny*nz */
int dfd_set_wave(dfd_ctx *ctx, const float *host);  /* 9*nx*ny*nz */
int dfd_get_metric(dfd_ctx *ctx, float *host);      /* 13*nx*ny*nz: xix..ztz jac lam mu rho */
int dfd_get_fault(dfd_ctx *ctx, int field, float *host);
int dfd_get_slice(dfd_ctx *ctx, int axis, int index, float *host);  /* Vx,Vy,Vz on one slice */
/* Split-node coefficient tables of the FP64 precompute, rounded to FP32, in the layout
 * init_fault_coef leaves them on the device (fault_coef.cu:26-1312, alloc.cu:170-260):
 *   DFD_TAB_D21_1 .. DFD_TAB_MATVZTOVXP   (NZ+6, NY+6, 9)  per fault node, row-major 3x3
 *   DFD_TAB_MATVX2VZ1 .. DFD_TAB_MATMIN2PLUS3F  (NY+6, 9)  free-surface row
 *   DFD_TAB_VEC_N, _VEC_S1, _VEC_S2        (NZ+6, NY+6, 3)  fault normal and strike/dip vectors
 * The names and their order are the reference's. */
enum {
  DFD_TAB_D21_1 = 0, DFD_TAB_D22_1, DFD_TAB_D23_1, DFD_TAB_D31_1, DFD_TAB_D32_1, DFD_TAB_D33_1,
  DFD_TAB_D21_2, DFD_TAB_D22_2, DFD_TAB_D23_2, DFD_TAB_D31_2, DFD_TAB_D32_2, DFD_TAB_D33_2,
  DFD_TAB_MATMIN2PLUS1, DFD_TAB_MATMIN2PLUS2, DFD_TAB_MATMIN2PLUS3, DFD_TAB_MATMIN2PLUS4, DFD_TAB_MATMIN2PLUS5,
  DFD_TAB_MATPLUS2MIN1, DFD_TAB_MATPLUS2MIN2, DFD_TAB_MATPLUS2MIN3, DFD_TAB_MATPLUS2MIN4, DFD_TAB_MATPLUS2MIN5,
  DFD_TAB_MATT1TOVXM, DFD_TAB_MATVYTOVXM, DFD_TAB_MATVZTOVXM, DFD_TAB_MATT1TOVXP, DFD_TAB_MATVYTOVXP,
  DFD_TAB_MATVZTOVXP,
  DFD_TAB_MATVX2VZ1, DFD_TAB_MATVY2VZ1, DFD_TAB_MATVX2VZ2, DFD_TAB_MATVY2VZ2, DFD_TAB_MATPLUS2MIN1F,
  DFD_TAB_MATPLUS2MIN2F, DFD_TAB_MATPLUS2MIN3F, DFD_TAB_MATMIN2PLUS1F, DFD_TAB_MATMIN2PLUS2F,
  DFD_TAB_MATMIN2PLUS3F,
  DFD_TAB_VEC_N, DFD_TAB_VEC_S1, DFD_TAB_VEC_S2,
  DFD_TAB_COUNT
};
int dfd_get_fault_table(dfd_ctx *ctx, int table, float *host);
/* thermal pressurisation columns (Friction_type 3): which 0 = temperature TP_T, 1 = pore
 * pressure TP_P, (TP_n, NZ, NY) float32, point 0 on the fault (alloc.cu:111-116 layout) */
int dfd_get_tp_columns(dfd_ctx *ctx, int which, float *host);
/* enqueue (asynchronously, after the work already issued) a copy of the eight per-step
 * on-fault output planes Vs1 Vs2 Tn Ts1 Ts2 slip State init_t0, (8, NZ, NY), into host
 * memory (pinned for a true async copy); completes at the next dfd_synchronize */
int dfd_fetch_outputs(dfd_ctx *ctx, float *host);
/* nsteps steps issued stage by stage with CUDA events around every volume-kernel launch:
 * total device time, time inside the volume kernels, and the rest (milliseconds) */
int dfd_run_timed(dfd_ctx *ctx, int it0, int nsteps, float *total_ms, float *volume_ms, float *fault_ms);
/* dfd_run with its device time: the graphs of all eight flag patterns are built first,
 * then nsteps steps are replayed between two CUDA events on the context's stream; *ms is
 * their elapsed time (a measurement aid for the production path, which dfd_run_timed's
 * per-kernel events perturb) */
int dfd_run_graph_timed(dfd_ctx *ctx, int it0, int nsteps, float *ms);
/* device time spent in the interior (TMA-tiled) volume kernel during the last
 * dfd_run_timed (CUDA events on its stream, summed over all stages), and the nodes that
 * kernel updates per stage (the interior box minus the fault band); a measurement aid
 * with no counterpart in the reference */
int dfd_interior_stats(dfd_ctx *ctx, float *ms, long long *nodes);
/* device time of the fault node kernel (trial traction and friction solve) during the last
 * dfd_run_timed, summed over all stages; a measurement aid */
int dfd_fault_node_ms(dfd_ctx *ctx, float *ms);
/* The same slice as dfd_get_slice, gathered into a static device array instead of a
 * temporary allocation; this entry has no counterpart in the reference.  It is for callers
 * that must not allocate or free device memory while they run (fixed memory budget, or no
 * device-wide synchronisation from cudaMalloc/cudaFree between steps).  Limits: at most
 * DFD_SLICE_SCRATCH_FLOATS floats (3 x the slice's nodes), else DFD_ERR_PARAM; the first
 * call on a device looks up the array's address (setup), so make it before any stream
 * capture; the array is shared per device, so calls that overlap in time on one device
 * race.  Cost: the array holds 16 MiB of device memory on every device where the library's
 * module is loaded, whether or not this entry is called. */
#define DFD_SLICE_SCRATCH_FLOATS (1 << 22)
int dfd_get_slice_noalloc(dfd_ctx *ctx, int axis, int index, float *host);
/* Test hook of the bounded waits (no counterpart in the reference; off by default): with
 * on = 1 the interior (TMA-tiled) kernel's copy-issuing warp issues no copies, so the
 * computing warps' first wait on a copy runs out after a short bounded poll; they set the
 * context's error flag and return.  The next dfd_synchronize reports DFD_ERR_CUDA ("a TMA
 * copy did not complete"), which stays sticky in this context; the device and other
 * contexts are unaffected.  Exercises the timeout path without faulting the GPU. */
int dfd_test_wait_drill(dfd_ctx *ctx, int on);
/* ---- halo exchange of a domain decomposed along y (slabs_y > 1) (replaces exchange_array,
 *      exchange_wave and exchange_fault, mod_mpi.cu:104-281, mod_mpi_fault.cu:87-237) ----
 * A slab's ghost columns next to a neighbouring slab hold that neighbour's nodes.  Side 0
 * is the low-y side (columns 0..2 leave, ghost columns -3..-1 arrive), side 1 the high-y
 * side (the last three columns leave, the three ghost columns after them arrive).  A message is
 * dfd_halo_floats() floats, packed into and unpacked from DEVICE memory on the context's
 * stream, so that it can go to the neighbour by NCCL, by a peer copy or through the host.
 * what = DFD_HALO_SETUP once after dfd_precompute (the metric and media of the ghost
 * columns, which the fault band's traction stencils read), then before every stage irk
 * of every step what = irk (0..3): the stage's input wavefield (9 fields) and its
 * split-node fault state (18 fields).  dfd_halo_pack of side s pairs with
 * dfd_halo_unpack of side 1 - s on the neighbour.  Stepping then goes stage by stage
 * (dfd_stage) with the exchange in between. */
#define DFD_HALO_SETUP 4
int dfd_halo_floats(dfd_ctx *ctx, long long *floats);
int dfd_halo_pack(dfd_ctx *ctx, int what, int side, float *device_buf);
int dfd_halo_unpack(dfd_ctx *ctx, int what, int side, const float *device_buf);
/* host-side health check: 0 ok, DFD_ERR_NONFINITE if the fault state holds NaN/Inf */
int dfd_check_finite(dfd_ctx *ctx);
/* cumulative Newton iterations and non-converged solves of the rate-and-state trial */
int dfd_newton_stats(dfd_ctx *ctx, long long *iterations, long long *capped);

/* ---- NetCDF-classic output with the reference layout (io_fault.cu:16-285,
 *      io_wave_xy.cu:9-188): fault_mpi000000.nc and wave_{xy,xz,yz}_mpi000000.nc ----
 * dfd_output_write queues record it_skip of the current state (the reference writes it
 * before the step, main.cu:425-437) and returns: the state is copied on the context's
 * stream, the files are written by a writer thread while the steps go on.  It blocks
 * only while two earlier records still wait for the writer.  dfd_output_close writes
 * every queued record, then closes the files; an error of the writer is returned by the
 * next dfd_output_write or by dfd_output_close. */
int dfd_output_open(dfd_ctx *ctx, const char *outdir);
int dfd_output_write(dfd_ctx *ctx, int it_skip);
int dfd_output_close(dfd_ctx *ctx);

/* ---- learned initial guess of the rate-and-state Newton solve (replaces the guess of
 *      trial_ratestate.cu:695; the Newton iteration of :20-57 stays as the check and the
 *      fallback).  No counterpart in the reference beyond that guess. ---- */
/* MLP 4 -> 32 -> 32 -> 1 (tanh).  Inputs (psi/a, log10 Vhat, log10 coef, a) of the solve
 * f(x) = 2 V0 e^{-psi/a} sinh x + coef x - Vhat; output the residual
 * x* - asinh(Vhat e^{psi/a} / (2 V0)).  Parameter vector, DFD_MLP_PARAMS floats:
 * W1(32x4) b1(32) W2(32x32) b2(32) W3(32) b3 | input mean(4) scale(4) output mean scale;
 * the first DFD_MLP_TRAINABLE are trained. */
#define DFD_MLP_PARAMS 1259
#define DFD_MLP_TRAINABLE 1249
/* Tile shape of the TMA-staged interior kernel (no counterpart in the reference, whose
 * stencil kernels use fixed thread blocks): rows 8 (32 x 8 tiles, one CTA per SM, the
 * default) or 4 (32 x 4 tiles, two CTAs per SM).  Results are the same bits either way;
 * the speed depends on the grid.  Between steps only (DFD_ERR_STATE mid-step). */
int dfd_set_tile_rows(dfd_ctx *ctx, int rows);
/* load the weights and switch the learned guess on (weights NULL, n 0: switch it off) */
int dfd_set_guess_net(dfd_ctx *ctx, const float *weights, int n);
/* record (psi/a, log10 Vhat, log10 coef, a, x* residual) of one in `every` converged plain
 * Newton solves (chosen by node, step and stage) into a device buffer of `capacity`
 * samples (0 frees it); solves beyond the capacity are dropped */
int dfd_newton_record(dfd_ctx *ctx, int capacity, int every);
/* measurement aids of the rate-and-state solve: timing 1 accumulates the clock cycles of
 * the solve section (guess, network and Newton iterations) per node; judge 1 also runs the
 * plain solve after every learned one and keeps the largest relative difference of the
 * accepted values from it.  Both off by default. */
int dfd_rs_profile(dfd_ctx *ctx, int timing, int judge);
/* since the last dfd_precompute: learned guesses accepted by the residual test and those
 * that fell back to the plain solve, mean clock cycles of a timed solve (0 without
 * timing), and the judge's largest relative difference (0 without judge) */
int dfd_rs_solve_stats(dfd_ctx *ctx, long long *accepted, long long *fallback, double *cycles_per_solve,
                       double *judge_max_rel);
/* copy up to max recorded samples (5 floats each) to host, set *n, and empty the buffer */
int dfd_newton_samples(dfd_ctx *ctx, float *host, int max, int *n);
/* stand-alone training and inference on the current device, host arrays in and out:
 * initialise (Xavier weights from seed, standardisation constants), batch forward
 * (x: n x 4, y: n residuals), loss (mean squared standardised error) and its gradient
 * (DFD_MLP_TRAINABLE floats), and minibatch Adam training for `epochs` epochs */
int dfd_mlp_init(float *w, unsigned seed, const float *x_mean, const float *x_scale, float y_mean, float y_scale);
int dfd_mlp_forward(const float *w, const float *x, int n, float *y);
/* the fault node kernel's own inference of the residual on a batch: tensor_cores 0 the
 * per-thread network (hardware tanh), 1 the warp-wide network whose hidden layer runs on
 * the tensor cores (mma.sync, FP16 operands, FP32 accumulation) */
int dfd_mlp_forward_node(const float *w, const float *x, int n, int tensor_cores, float *y);
int dfd_mlp_loss_grad(const float *w, const float *x, const float *y, int n, double *loss, float *grad);
int dfd_mlp_train(const float *x, const float *y, int n, int epochs, int batch, float lr, unsigned seed, float *w,
                  float *loss_per_epoch);

/* ---- ensemble: prepared scenarios stepped together (no counterpart in the reference,
 *      which runs one job per process).  Every scenario is a context created, loaded and
 *      set up as usual on the same device; the ensemble advances all of them from step
 *      it0 with one batched launch per kernel and RK stage (fault node, fault band,
 *      general kernel) and one persistent launch of the tiled interior kernel whose units
 *      span every scenario, replayed from CUDA graphs.  Results stay in the scenarios'
 *      contexts.  Destroy the ensemble before its contexts. ---- */
typedef struct dfd_ens dfd_ens;
int dfd_ens_create(dfd_ctx *const *scenarios, int n, dfd_ens **out);
int dfd_ens_destroy(dfd_ens *e);
int dfd_ens_run(dfd_ens *e, int it0, int nsteps);
int dfd_ens_synchronize(dfd_ens *e);
/* nsteps steps timed with CUDA events on the ensemble's stream (graphs built beforehand) */
int dfd_ens_run_timed(dfd_ens *e, int it0, int nsteps, float *ms);
/* x planes per unit of the tiled kernel (0: each scenario's own plan); for autotuning */
int dfd_ens_set_chunk(dfd_ens *e, int chunk);
/* rows of the interior kernel's tiles for every scenario (dfd_set_tile_rows); for
 * autotuning together with the chunk */
int dfd_ens_set_tile_rows(dfd_ens *e, int rows);
int dfd_ens_nodes(const dfd_ens *e, long long *nodes);
const char *dfd_ens_last_error(const dfd_ens *e);

const char *dfd_error_string(int status);
const char *dfd_last_error(const dfd_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
