/*
 * libdiablo_gpu -- B200 (sm_100a) implementation of DIABLO 3's RK3 /
 * Crank-Nicolson channel-flow step behind the reference's plugin surface.
 *
 * The reference surface this replaces:
 *   fft_xz_to_fourier(v, vv)   for/fft.f90:247   -> diablo_fft_xz_to_fourier
 *   fft_xz_to_physical(vv, v)  for/fft.f90:319   -> diablo_fft_xz_to_physical
 *   rk_chan_1                  for/channel.f90:10 (called 3x per step from
 *                              for/diablo.f90:104-107) -> diablo_rk_substep,
 *                              diablo_step
 *   pre_first_step             for/advance.f90:17 -> diablo_pre_first_step
 *   apply_BC_vel_mpi_post,
 *   apply_BC_th_mpi_post       for/boundary.f90:824,841 -> diablo_apply_bc_post
 *   module state (flow.f90:20-51, init_flow :58-88, read_inputs/
 *   set_parameters parameters.f90:88-281, create_grid_chan domain.f90:209)
 *                              -> diablo_create, diablo_upload_state,
 *                                 diablo_download_state
 *
 * Array layouts at the boundary are the reference's own, Fortran order, one
 * y-rank and one z-rank (Nxp = Nx/2, Nzp = Nz, Nyp = Ny):
 *   physical  real    v(0:Nx+1, 0:Nz+1, 0:Ny+1)      (x fastest)
 *   Fourier   complex vv(0:Nx/2, 0:Nz+1, 0:Ny+1)     (same bytes; kx fastest)
 * Only the significant entries are read or written: physical i < Nx, k < Nz;
 * Fourier i < Nxp, k <= 2*Nkz (Nkx = Nx/3, Nkz = Nz/3, for/domain.f90:18-23).
 * Every other entry of a destination buffer is left as it was (the reference
 * leaves stale values there too, for/fft.f90:301-313).  Fourier modes
 * Nkx < i < Nxp are zero in every state the reference produces
 * (for/fft.f90:264-266): they are written as 0, and uploads that carry nonzero
 * values there are rejected with DIABLO_ERR_STATE.
 *
 * Every entry point returns an int status (0 = DIABLO_OK, negative = error);
 * nothing aborts the process.  One context per host thread; all device work
 * of a context is ordered on its CUDA stream.
 */
#ifndef DIABLO_GPU_H
#define DIABLO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define DIABLO_ABI_VERSION 1
#define DIABLO_MAX_TH 8

enum diablo_status {
  DIABLO_OK = 0,
  DIABLO_ERR_ARG = -1,          /* null pointer, bad enum or bad value */
  DIABLO_ERR_SIZE = -2,         /* grid size the kernels do not support */
  DIABLO_ERR_CUDA = -3,         /* a CUDA runtime call failed */
  DIABLO_ERR_NONFINITE = -4,    /* NaN/Inf found in the state */
  DIABLO_ERR_TIMEOUT = -5,      /* a bounded device wait gave up (diablo_set_wait_bound) */
  DIABLO_ERR_UNSUPPORTED = -6,  /* option not implemented on the device */
  DIABLO_ERR_STATE = -7,        /* uploaded state violates the layout contract */
  DIABLO_ERR_NOMEM = -8         /* device allocation failed */
};

enum diablo_precision { DIABLO_FP64 = 0, DIABLO_MIXED = 1 };

/* field ids for upload/download: u1, u2, u3, p, then scalar n at DIABLO_TH+n */
enum diablo_field { DIABLO_U1 = 0, DIABLO_U2 = 1, DIABLO_U3 = 2, DIABLO_P = 3, DIABLO_TH = 4 };

enum diablo_layout {
  DIABLO_LAYOUT_FOURIER = 0,   /* complex vv(0:Nx/2, 0:Nz+1, 0:Ny+1) */
  DIABLO_LAYOUT_PHYSICAL = 1   /* real v(0:Nx+1, 0:Nz+1, 0:Ny+1); transformed on the device */
};

/*
 * Run parameters: the fields of the reference's `parameters` module that the
 * step reads (for/parameters.f90:22-82) plus the compile-time grid
 * (grid_def: Nx, Ny, Nz, N_th).  Velocity BC names follow the reference's
 * internal variables: u_* -> u1, v_* -> u2 (wall-normal), w_* -> u3.
 * BC type 0 = Dirichlet, 1 = Neumann.  `ro` = +inf means no rotation.
 * `struct_size` must be sizeof(diablo_params) (ABI check).
 */
typedef struct diablo_params {
  int struct_size;
  int nx, ny, nz, n_th;
  double lx, ly, lz;
  double re, nu_v_scale, beta, ro, delta;
  double grav_x, grav_y, grav_z;
  double delta_t;
  int f_type;
  double ubulk0, px0, omega0, amp_omega0, force_start;
  int u_bc_ymin, v_bc_ymin, w_bc_ymin, u_bc_ymax, v_bc_ymax, w_bc_ymax;
  double u_bc_ymin_c1, v_bc_ymin_c1, w_bc_ymin_c1;
  double u_bc_ymax_c1, v_bc_ymax_c1, w_bc_ymax_c1;
  double pr[DIABLO_MAX_TH], ri[DIABLO_MAX_TH];
  int th_bc_ymin[DIABLO_MAX_TH], th_bc_ymax[DIABLO_MAX_TH];
  double th_bc_ymin_c1[DIABLO_MAX_TH], th_bc_ymax_c1[DIABLO_MAX_TH];
  double dthdx[DIABLO_MAX_TH], dthdz[DIABLO_MAX_TH];
  int use_les, les_model_type, create_new_flow;
  int variable_dt;
  double cfl;
  int update_dt;
  double max_dt;
  int precision;      /* DIABLO_FP64 or DIABLO_MIXED */
  int flavor_front;   /* 1 = flavor 'Front' (thermal-wind forcing) */
  /* filter_scalars (for/advance.f90:161-173): scalar n is filtered by
   * filter_chan after every step whose number is a multiple of filter_int[n]
   * when filter_th[n] is set (FILTER_TH / FILTER_INT of input.toml) */
  int filter_th[DIABLO_MAX_TH];
  int filter_int[DIABLO_MAX_TH];
} diablo_params;

typedef struct diablo_ctx diablo_ctx;

/* Create a context on the current CUDA device.  `gy` holds the Ny+1 wall-normal
 * base-grid points gy(1..Ny+1), i.e. grid.h5:/grids/y (for/domain.f90:383-527).
 * Replaces read_inputs + init_mpi + create_grid_chan + init_flow + init_fft. */
diablo_ctx* diablo_create(const diablo_params* p, const double* gy, int* status);
int diablo_destroy(diablo_ctx* ctx);

/* Copy one field between a buffer in the reference layout and the device
 * state.  `buf` may be host or device memory.  PHYSICAL uploads are
 * transformed with fft_xz_to_fourier semantics; PHYSICAL downloads with
 * fft_xz_to_physical semantics (the state itself stays in Fourier space). */
int diablo_upload_state(diablo_ctx* ctx, int field, const double* buf, int layout);
int diablo_download_state(diablo_ctx* ctx, int field, double* buf, int layout);
/* The eddy viscosity nu_t(0:Nx+1, 0:Nzp+1, 0:Nyp+1) of the last LES substep
 * (module array of for/flow.f90:50, set by les_chan, for/les.f90:235-241 and
 * :2241-2262) in the reference's physical layout; host or device `buf`.
 * All zero before the first LES substep, as the reference's array is. */
int diablo_download_nu_t(diablo_ctx* ctx, double* buf);

/*
 * The host-authoritative round trip, nsteps times: every step uploads the
 * state (u1, u2, u3, p, th_0..) from bufs[0..3+n_th], advances one step as
 * diablo_step does, and downloads the new state into the same arrays -- the
 * mode in which the Fortran arrays stay authoritative on the host between
 * steps.  bufs are HOST arrays in the reference Fourier layout (pinned memory
 * for the full link rate; device pointers return DIABLO_ERR_ARG).  Each
 * field's download goes out as soon as the field is packed, and the next
 * step's upload of that field follows it, so the two link directions work at
 * once on different fields.  The work is ordered after what is already queued
 * on the context's stream, and the call returns when the last download has
 * landed; DIABLO_ERR_STATE if an uploaded array broke the layout contract
 * (nonzero modes Nkx < i < Nxp).  The downloads write the rows' pad entries
 * (i = Nxp) as zero, as the reference's transform leaves its modes above Nkx.
 * No reference counterpart: the reference's state never leaves the host.
 */
int diablo_step_host(diablo_ctx* ctx, double* const* bufs, int nsteps);

/* for/fft.f90:247-315.  v: physical array, vv: Fourier array, both full
 * reference-size buffers (host or device); v == vv is allowed, as in the
 * reference, and the input is consumed.  Computes in FP64. */
int diablo_fft_xz_to_fourier(diablo_ctx* ctx, const double* v, double* vv);
/* for/fft.f90:319-382; vv == v allowed. */
int diablo_fft_xz_to_physical(diablo_ctx* ctx, double* vv, double* v);

/* One RK substep, rk_step in {1,2,3} (for/channel.f90:10-917). */
int diablo_rk_substep(diablo_ctx* ctx, int rk_step);
/* nsteps full steps: 3 substeps each, time += delta_t (for/diablo.f90:98-108).
 * Returns when the steps have finished on the device (it reads the column
 * step's wait status, see diablo_set_wait_bound). */
int diablo_step(diablo_ctx* ctx, int nsteps);
/* Wall values, projection, optional initial pressure (for/advance.f90:17-44). */
int diablo_pre_first_step(diablo_ctx* ctx, int compute_pressure);
/* Fourier-space wall/ghost values of u and theta (for/boundary.f90:824-855). */
int diablo_apply_bc_post(diablo_ctx* ctx);
/* filter_chan (for/channel.f90:1241-1329): the spectral filter
 * sigma0^4 (35 - 84 sigma0 + 70 sigma0^2 - 20 sigma0^3),
 * sigma0 = (1 + cos|(kx dx, kz dz)|)/2, on scalar n's rows jstart_th..jend_th.
 * diablo_step applies it itself as filter_scalars does; this entry point is
 * the subroutine on its own. */
int diablo_filter_chan(diablo_ctx* ctx, int n);

/* Plane statistics: save_stats_chan (for/statistics.f90:44-712) with
 * compute_averages, compute_TKE_diss, compute_MKE_diss, compute_TKE,
 * compute_TKE_Production, compute_Vorticity and compute_TKE_diss_les.
 * homogeneous_x is the reference's homogeneousX (for/parameters.f90:275-280:
 * 0 for IC types 5-8): with 0 the means are z-line averages at each x,
 * epsilon's x derivatives leave out the kz = 0 row, and compute_MKE_diss and
 * the production terms use the mean x gradients.  Applies the wall values
 * (apply_BC_vel/th_mpi_post) to the state first, as the reference does.  The
 * profiles are the values the reference writes to mean.h5 at j = 1..Ny (its
 * internal names; mean.h5 swaps the v/w labels).  Plane averages of products
 * are evaluated from the Fourier coefficients (Parseval), z-line averages and
 * the LES terms from physical fields, all in FP64 in both precisions.
 * With scalars, compute_BPE's background potential energy (scalar BPE), its
 * th_1 PDF and bin edges (th1PDF, th1bin) and Bin_Ystar_and_Write's bin means
 * of shear2, thw, chi, epsilon, TKE and KE on those th_1 bins are included
 * (the reference writes thw and chi once per scalar under one name, so the
 * last scalar's stand; empty bins are NaN, 0/0 as in the reference).  Not
 * computed: HDF5/movie output.  nu_sgs is the
 * plane mean of the nu_t of the most recent LES substep and eps_sgs2 uses that
 * nu_t, as compute_TKE_diss_les does; a scalar's kappa_sgs is the plane mean
 * of its kappa_t of that substep (les_chan_th's kappa_t_mean,
 * for/les.f90:1420-1448, which writes scalar 1's); all are 0 without LES.
 * Layout of `out` (diablo_stats_size doubles):
 *   profile q of the velocity set at out[q*Ny + j-1], q < DIABLO_STAT_NPROF;
 *   then, for scalar n, profile r at out[(NPROF + n*NTHPROF + r)*Ny + j-1];
 *   then the y-averaged kz = 0 spectrum of u1 (FTx_uu), Nx/2 values;
 *   then, when N_th > 0, th1PDF (Nx values), th1bin (Nx values) and the six
 *   y* bin means (Nx values each, in the order shear2, thw, chi, epsilon, TKE,
 *   KE);
 *   then DIABLO_STAT_NSCALAR scalars (BPE is 0 without scalars). */
enum {
  DIABLO_STAT_UME = 0, DIABLO_STAT_VME, DIABLO_STAT_WME, DIABLO_STAT_MKE,
  DIABLO_STAT_URMS, DIABLO_STAT_VRMS, DIABLO_STAT_WRMS,
  DIABLO_STAT_UV, DIABLO_STAT_UW, DIABLO_STAT_WV,
  DIABLO_STAT_UU_DUDX, DIABLO_STAT_VV_DVDY, DIABLO_STAT_WU_DWDX,
  DIABLO_STAT_VU_DVDX, DIABLO_STAT_UV_DUDY, DIABLO_STAT_WV_DWDY,
  DIABLO_STAT_DUDY, DIABLO_STAT_DWDY, DIABLO_STAT_CP, DIABLO_STAT_SHEAR,
  DIABLO_STAT_OMEGA_X, DIABLO_STAT_OMEGA_Y, DIABLO_STAT_OMEGA_Z,
  DIABLO_STAT_EPSILON, DIABLO_STAT_EPSILON_M, DIABLO_STAT_NU_SGS, DIABLO_STAT_EPS_SGS2,
  DIABLO_STAT_NPROF
};
enum {
  DIABLO_STAT_THME = 0, DIABLO_STAT_DTHDY, DIABLO_STAT_THRMS, DIABLO_STAT_THV,
  DIABLO_STAT_THV_M, DIABLO_STAT_PE_DISS, DIABLO_STAT_KAPPA_SGS, DIABLO_STAT_NTHPROF
};
enum {
  DIABLO_STAT_TIME = 0, DIABLO_STAT_DT, DIABLO_STAT_UBULK, DIABLO_STAT_URMS_B,
  DIABLO_STAT_VRMS_B, DIABLO_STAT_WRMS_B, DIABLO_STAT_U1Y_LEFT_B, DIABLO_STAT_BPE, DIABLO_STAT_NSCALAR
};
int diablo_stats_size(diablo_ctx* ctx);
int diablo_stats(diablo_ctx* ctx, int homogeneous_x, double* out, int len);

/* eps_sgs1 of les_chan (for/les.f90:924-1068), the plane mean of u_i times
 * the SGS stress force added to cf_i (interpolated onto GY points; written to
 * mean.h5 with sign opposite to the usual dissipation convention, as the
 * reference notes).  As in the reference, a diablo_stats call on an LES
 * context requests it (flag_save_LES, for/control.f90:95) and the next step's
 * first substep forms it from that substep's stresses; this call then copies
 * Ny values (j = 1..Ny; j = 1 is 0) into host `out` (len >= Ny).  All zero
 * when the LES gate was still off at that step (for/channel.f90:271-274);
 * DIABLO_ERR_STATE when no step of the context's own (diablo_step,
 * diablo_step_host, diablo_rk_substep with rk 1) has run since the request:
 * ensemble graph replays do not answer it. */
int diablo_les_eps_sgs1(diablo_ctx* ctx, double* out, int len);

int diablo_set_precision(diablo_ctx* ctx, int precision);
int diablo_get_time(diablo_ctx* ctx, double* time, int* time_step, double* delta_t);
int diablo_set_time(diablo_ctx* ctx, double time, int time_step, double delta_t);
/* Bind the context to an existing cudaStream_t (NULL = the context's own stream). */
int diablo_set_stream(diablo_ctx* ctx, void* stream);
int diablo_synchronize(diablo_ctx* ctx);
/* DIABLO_ERR_NONFINITE if any significant Fourier entry of the state is NaN
 * or Inf, 0 otherwise. */
int diablo_check_finite(diablo_ctx* ctx);
/* The column step can run as one persistent kernel (opt-in: environment
 * variable DIABLO_GENERAL_SOLVER=3 when the context is created; the default
 * two launches measured faster) in which each column group's projection
 * waits on a device counter until the group's three velocity solves are
 * done.  That wait always ends (it only waits on work already running), and
 * it is also bounded: after max_spins polls (100 ns apart; default 2^24,
 * about a second) the kernel records a timeout, leaves the group unprojected
 * and returns, and diablo_step, diablo_rk_substep and diablo_synchronize
 * return DIABLO_ERR_TIMEOUT (reading the record clears it; the state is then
 * invalid).  withheld_arrivals > 0 makes every projection wait for that many
 * more arrivals than will come: failure injection from the host, to test
 * that path.  No reference counterpart. */
int diablo_set_wait_bound(diablo_ctx* ctx, long long max_spins, int withheld_arrivals);
/* number of kernels this context has launched since creation */
long long diablo_kernel_launches(const diablo_ctx* ctx);

/* Per-kernel timing (tracing; no reference counterpart beyond the wall-clock
 * "Wall Seconds per Iteration" print, for/control.f90:104-109).  When on, every
 * step kernel is bracketed by CUDA events on the context's stream;
 * diablo_kernel_times returns the accumulated device time and launch count of
 * one kernel class since profiling was (re)enabled. */
int diablo_set_profiling(diablo_ctx* ctx, int enable);
int diablo_kernel_times(diablo_ctx* ctx, int slot, double* total_ms, long long* launches);
int diablo_kernel_slots(void);
const char* diablo_kernel_name(int slot);
const char* diablo_status_string(int status);
int diablo_abi_version(void);

/*
 * The library's forward xz transform without a context, for callers that
 * cannot allocate device memory.  This entry point has no counterpart in the
 * reference.  Its callers are drivers that own every device byte through
 * their own pool, code that cannot take the device-wide synchronisation of
 * cudaMalloc/cudaFree, and callers that never create a context.  It allocates
 * nothing: its scratch is one file-scope device array of
 * DIABLO_NOALLOC_SCRATCH_BYTES (plus a 28 KB twiddle table) that every GPU
 * loading the library holds until the process exits.
 * v and vv are DEVICE (or managed) arrays of the current device in the
 * reference layout (v == vv allowed); host pointers and other devices'
 * memory return DIABLO_ERR_ARG before anything is queued.  The work is queued
 * on `stream` (cudaStream_t, NULL = legacy default stream).  Grids whose
 * scratch needs exceed the array return DIABLO_ERR_SIZE (e.g. 128 x 129 x 128
 * fits, 256 x 257 x 256 does not).  A CUDA error already pending when the call
 * starts is left for the caller and the call returns DIABLO_ERR_CUDA without
 * queueing anything.
 * The first call on each device does a one-time set-up (the array's device
 * address by cudaGetSymbolAddress, the twiddle tables by cudaMemcpyToSymbol),
 * so make that first call before any stream capture begins.  All calls share
 * the one array and it keeps the last call's contents: calls whose work
 * overlaps on the GPU (different streams, or different host threads) race
 * and must be serialised by the caller.
 */
#define DIABLO_NOALLOC_SCRATCH_BYTES (64u << 20)
int diablo_fft_xz_to_fourier_noalloc(int nx, int ny, int nz, const double* v, double* vv,
                                     void* stream);

/*
 * Discrete adjoint of diablo_step.  No reference counterpart: the reference
 * has no adjoint.  For DNS contexts in FP64 with velocities and any number of
 * scalars (buoyancy, background gradients, scalar transport, the filter of
 * filter_scalars, whose real per-mode factor is its own transpose, and the
 * 'Front' flavor's thermal-wind advection), fixed delta_t; LES, mixed
 * precision and variable_dt get DIABLO_ERR_UNSUPPORTED.
 * diablo_adjoint_record advances nsteps steps exactly as diablo_step does and
 * keeps the state (u1, u2, u3, p, th_0..) every `every` steps on the device,
 * and the input fields of every substep of the last segment.
 * diablo_adjoint_run takes lam[0..3+n_th] = dJ/d(u1, u2, u3, p, th_0..) of the
 * recorded final state for any objective J and overwrites them with dJ/d of the state
 * the recording started from.  It recomputes each segment of `every` steps
 * from its checkpoint (not the last one after a fresh record: its substep
 * inputs are at hand) and runs the hand-written adjoint of every RK substep
 * backwards through it (transposed tridiagonal solves, adjoint transforms,
 * adjoint nonlinear products), and leaves the context at the recorded final
 * state.  lam arrays use the reference Fourier layout (host or device); each
 * complex entry holds (dJ/dRe, dJ/dIm) of the matching coefficient; only the
 * significant entries are read, and modes Nkx < i < Nxp are written as zero.
 * Stepping the context between the two calls makes the run fail with
 * DIABLO_ERR_STATE.
 */
int diablo_adjoint_record(diablo_ctx* ctx, int nsteps, int every);
int diablo_adjoint_run(diablo_ctx* ctx, double* const* lam);

/*
 * Ensembles of independent channels, stepped together.  No reference
 * counterpart: the reference runs one channel per MPI job.  Members are
 * contexts from diablo_create with any mix of grid sizes, parameters and
 * precisions; they stay owned by the caller and must outlive the ensemble.
 * diablo_ensemble_step advances every member by nsteps steps with one CUDA
 * graph launch per step.  In DIABLO_ENSEMBLE_PERSISTENT mode (the default
 * when every member qualifies: DNS without LES or the 'Front' forcing, the
 * default column path, Ny + 2 <= 288) each substep runs the members'
 * transforms and nonlinear terms on parallel branches of the graph and then
 * the column step of every member in ONE persistent launch per rows-per-lane
 * class: the launch walks a member table, and each projection task waits,
 * bounded by the member's diablo_set_wait_bound, for its own member's solves
 * (a wait that gives up makes diablo_ensemble_synchronize return
 * DIABLO_ERR_TIMEOUT).  In DIABLO_ENSEMBLE_BRANCHES mode each member's whole
 * step is one branch of the graph.  The graphs are captured on first use and again whenever a
 * member's state no longer matches them (a member stepped on its own, a
 * changed delta_t or precision, the LES gate opening).  Members whose kernel
 * arguments change every step are rejected with DIABLO_ERR_UNSUPPORTED:
 * variable_dt, the oscillating pressure gradient (f_type 2), the
 * time-dependent top-wall u3 (f_type 4 with a Neumann top) and filtered
 * scalars (filter_th).  A member's own
 * entry points (upload, download, step) stay usable and are ordered with the
 * ensemble's work through the member's stream.
 */
/*
 * Autotuner (no reference counterpart).  Times the candidate tile shapes of
 * the step's four transform kernels (sequences per block of the z transforms,
 * rows per block of the x transforms) for this context's grid and precision on
 * its own scratch, and keeps the fastest for the context's later steps.  The
 * choice is cached per (grid, number of fields, precision) for the life of the
 * process, so contexts of the same size tune once.  The state is not changed.
 * tiles (optional, 4 ints) receives the choice.  Not for an active LES
 * context (DIABLO_ERR_UNSUPPORTED); set the precision first (changing it
 * resets the tiles to their defaults).
 */
int diablo_autotune(diablo_ctx* ctx, int* tiles);
/* The context's current transform tiles (4 ints, 0 = default). */
int diablo_tiles(diablo_ctx* ctx, int* tiles);

typedef struct diablo_ensemble diablo_ensemble;
diablo_ensemble* diablo_ensemble_create(diablo_ctx* const* members, int n, int* status);
int diablo_ensemble_step(diablo_ensemble* e, int nsteps);
int diablo_ensemble_synchronize(diablo_ensemble* e);
/* The stream each ensemble step's graph is launched on (cudaStream_t); its
 * completion follows the whole step of every member, so events recorded on
 * it time the ensemble on the device. */
void* diablo_ensemble_stream(diablo_ensemble* e);
int diablo_ensemble_destroy(diablo_ensemble* e);
/* Stepping mode (see above): DIABLO_ENSEMBLE_PERSISTENT or
 * DIABLO_ENSEMBLE_BRANCHES.  Persistent mode is refused with
 * DIABLO_ERR_UNSUPPORTED when a member does not qualify.  The graphs are
 * captured again at the next step. */
enum diablo_ensemble_mode { DIABLO_ENSEMBLE_BRANCHES = 0, DIABLO_ENSEMBLE_PERSISTENT = 1 };
int diablo_ensemble_set_mode(diablo_ensemble* e, int mode);
int diablo_ensemble_mode(const diablo_ensemble* e);
/* Ensemble autotuner: coordinate descent over the transform tile shapes of
 * each group of same-size members (the candidates of diablo_autotune), scored
 * by the time of steps_per_trial steps of the ensemble's own graph.  The
 * members' states and clocks are restored afterwards; the tiles found stay.
 * Not for members with an active LES (DIABLO_ERR_UNSUPPORTED). */
int diablo_ensemble_autotune(diablo_ensemble* e, int steps_per_trial);

#ifdef __cplusplus
}
#endif
#endif /* DIABLO_GPU_H */
