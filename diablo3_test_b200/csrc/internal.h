// Internal declarations shared by the translation units of libdiablo_gpu:
// the context, its device buffers, per-kernel timing and the helpers every
// subsystem uses (step: step.cu, column_launch.cu; boundary copies and the
// C ABI core: core.cu; LES: les.cu; statistics: stats.cu; ensembles and the
// autotuner: ensemble.cu; adjoint: adjoint.cu).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <vector>

#include "../../include/diablo_gpu.h"
#include "common.cuh"
#include "fft.cuh"
#include "kernels_fft.cuh"
#include "solve_args.cuh"

struct FieldArgs;   // the field-split column step's arguments (kernels_field.cuh)

static_assert(DIABLO_MAX_TH <= SOLVE_MAXTH, "scalar capacity");
static_assert(3 + DIABLO_MAX_TH <= NF_MAX, "field capacity");

// ``pi = 4.*atan(1.0)`` in for/fft.f90:152 is evaluated in default (single)
// precision -- the reference build has no -fdefault-real-8 -- so its
// wavenumbers kx = i*2*pi/Lx use float32(pi) widened to double.
static const double PI_REF = 3.1415927410125732421875;

// RK3 coefficients (for/flow.f90:78-86)
static const double H_FRAC[3] = {8.0 / 15.0, 2.0 / 15.0, 5.0 / 15.0};
static const double BETA_BAR[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0};
static const double ZETA_BAR[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0};

#define CK(call)                                  \
  do {                                            \
    cudaError_t e__ = (call);                     \
    if (e__ != cudaSuccess) {                     \
      ctx->last_cuda = (int)e__;                  \
      return DIABLO_ERR_CUDA;                     \
    }                                             \
  } while (0)

struct diablo_ctx {
  diablo_params p;
  int nx, ny, nz, nth, nf;
  int nxp, nkx, nkz, nkx1, nk2, kp, nyp2, M;
  Geom g;
  double nu, ro_inv;
  int jstart, jend, jst[DIABLO_MAX_TH], jet[DIABLO_MAX_TH];
  double time, delta_t, h_bar[3];
  int time_step;
  double w_top_transient;
  int precision;
  int last_cuda;
  long long launches;
  cudaStream_t stream, own_stream;
  // grid metrics and wavenumbers (device)
  double *d_dy, *d_dyf, *d_gy, *d_gyf, *d_kx, *d_kz;
  std::vector<double> h_dy, h_dyf, h_gy, h_gyf, h_kx;
  // twiddles: exp(-2 pi i m/N) for N = Nz, M = Nx/2, Nx
  double2 *tz64, *tm64, *tx64;
  float2 *tz32, *tm32, *tx32;
  // Fourier state, double buffered: [u1, u2, u3, p, th0..]
  double2* st[2][4 + DIABLO_MAX_TH];
  double2* cf[2][3 + DIABLO_MAX_TH];
  int cur;      // index of the current state buffer
  int cf_cur;   // index of the buffer holding the last substep's cf
  // nonlinear terms and step scratch
  void* nl[3 + DIABLO_MAX_TH];
  void* phys[3 + DIABLO_MAX_TH];
  void* xs[2 * (3 + DIABLO_MAX_TH)];
  int scratch_prec;   // precision the scratch was sized for (-1 = none)
  // boundary-call scratch (FP64): one field in each internal layout + one reference array
  double* b_phys;
  double2* b_xs;
  double2* b_four;
  double* b_ref;
  int* d_flag;
  std::vector<void*> allocs;
  // opt-in per-kernel timing: events recorded around each step kernel
  int profiling;
  int generation;           // bumped whenever captured kernel arguments go stale (dt, precision, tiles)
  int tune[4];              // tile shapes of the step transforms (z inv S, x inv KT, x fwd KT, z fwd S; 0 = default)
  // column step (DIABLO_GENERAL_SOLVER): 0 the field-split kernels in two
  // launches, 1 the general kernel, 2 the fused tiled kernel, 3 the
  // field-split step in one launch with bounded waits
  int use_general_solver;
  // ensemble capture: when set, substep stores the arguments of its
  // field-split column step here (and sets defer_filled) instead of
  // launching it; the ensemble launches every member's column step at once
  FieldArgs* defer_col;
  int defer_filled;
  Solve2Args solve2;        // tile schedule of the current substep
  double* d_kc[3];          // implicit-row coefficients per RK substep [2+nth][3][n]
  double* d_met;            // Poisson and metric rows [MET_N][n]
  double* d_prof;           // U1(y), I(U1)(y) of the mixed-precision mean split [2][n]
  // variable dt (courant): solved velocities before the projection, their
  // physical FP64 copies and the per-plane maxima
  double2* ustar[3];
  double* cfl_phys[3];
  double* d_cfl;
  double* d_sigma;          // filter_chan transfer function [Nkx+1][2Nkz+1]
  double* d_stats;          // plane-statistics partial sums (diablo_stats)
  double* stats_phys[3];    // physical u1, u2, u3 for the z-line statistics
  double* stats_der[8];     // y* binning: d/dx, d/dz of u1..u3 and of the last scalar
  double* stats_thl;        // physical last scalar (z-line branch, N_th > 1)
  double* stats_thxy;       // its z-line mean [Ny+2][Nx]
  size_t stats_doubles;
  double* d_fac[3];         // factored field systems per RK substep (k_factor)
  // k_column_step's scheduler words (task counter, status, per-group counts),
  // the bound of its waits and the arrivals withheld by the failure hook
  int* d_sched;
  size_t sched_ints;
  long long wait_spins;
  int wait_withhold;
  // LES substep buffers (FP64), allocated on first use
  struct Les {
    int ready;
    double2* S[6];            // Fourier strain tensor
    double2* T[7];            // Fourier stresses and nu_t dU/dy, nu_t dW/dy
    double2* cr[3 + DIABLO_MAX_TH];
    double2* thg[2 * DIABLO_MAX_TH];
    double* Sp[6];            // physical strain / stresses
    double* tmp[2];
    double* thp[2 * DIABLO_MAX_TH];
    double* r[3 + DIABLO_MAX_TH];
    double *nu_t, *sf, *sg;
    double2* xs[NF_MAX];      // x-spectral scratch of the batched transforms
    double *d_cf, *d_cg, *d_d2f, *d_d2g, *d_sclf, *d_sclg;
    double *d_idy, *d_idyf;   // 1/dy, 1/dyf (physical-space CN rows)
    double* u64[3 + DIABLO_MAX_TH];   // FP64 velocities/scalars for the solve (mixed precision)
    int nu_t_fp32;                    // nu_t was last written by the FP32 model
    int amd_ready;            // AMD models: rotation, invariant strain, gradients
    double2 *Of[3], *SIf[6], *Gf[9], *Tf[3 * DIABLO_MAX_TH];
    double *Op[3], *SIp[6], *Gp[9], *Tp[3 * DIABLO_MAX_TH];
    double *fxp[DIABLO_MAX_TH], *fzp[DIABLO_MAX_TH], *kap[DIABLO_MAX_TH];
    double2 *fxf[DIABLO_MAX_TH], *fzf[DIABLO_MAX_TH];
    int dyn_ready;            // dynamic model: test-filter inputs and plane sums
    double* dp[DYN_NF];
    double2* df[DYN_NF];
    double* dsums;
    // eps_sgs1 (for/les.f90:924-1068): requested by a statistics save, formed
    // at the next step's first substep; blank when the LES gate is still off
    double* d_eps;
    int eps_req, eps_ready, eps_blank;
  } les;
  // discrete adjoint: checkpoints of the recorded steps and adjoint work arrays
  struct Tape {
    int ready, nsteps, every, nseg;
    int sub_seg;                      // segment whose substep inputs `sub` holds (-1: none)
    int step_end, gen_end;
    double time_end;
    std::vector<double2*> ckpt;       // (nseg + 1) x (4 + nth) fields (u1, u2, u3, p, th..); the last is the final state
    std::vector<int> ckpt_step;
    std::vector<double> ckpt_time;
    std::vector<double2*> sub;        // every x 3 substeps x (3 + nth) inputs (u1, u2, u3, th..)
    // lambdas of the state [u1, u2, u3, p, th..], of cf and NL [u1, u2, u3, th..],
    // the product adjoints (8 + 3 nth) and the physical fields of the substep
    double2 *lu[4 + DIABLO_MAX_TH], *ou[4 + DIABLO_MAX_TH], *lF[3 + DIABLO_MAX_TH], *oF[3 + DIABLO_MAX_TH];
    double2 *lnl[3 + DIABLO_MAX_TH], *pf[8 + 3 * DIABLO_MAX_TH];
    int work_ready;
    double *pp[8 + 3 * DIABLO_MAX_TH], *up[3 + DIABLO_MAX_TH], *lp3[3 + DIABLO_MAX_TH];
    double *d_cn, *d_rmask, *d_pa;    // [3 rk][3 + nth field][3][n], [3 + nth][n], [3][n]
  } tape;
  // diablo_step_host: copy streams (host-to-device, device-to-host), per-field
  // staging arrays in the reference layout and their events
  struct Xfer {
    cudaStream_t up, down;
    cudaEvent_t start, e_up[4 + DIABLO_MAX_TH], e_conv[4 + DIABLO_MAX_TH];
    cudaEvent_t e_down[4 + DIABLO_MAX_TH][4];   // per field and plane chunk
    double2 *up_stage[4 + DIABLO_MAX_TH], *down_stage[4 + DIABLO_MAX_TH];
    int ready;
  } xfer;
  struct Timed { int slot; cudaEvent_t a, b; };
  std::vector<Timed> timed;        // pending (recorded, not yet read)
  std::vector<cudaEvent_t> pool;   // free events
  double slot_ms[8];
  long long slot_n[8];
};

enum { K_ZINV = 0, K_XINV = 1, K_XFWD_NL = 2, K_ZFWD_NL = 3, K_SOLVE = 4, K_PROJ = 5, K_OTHER = 6,
       K_NSLOTS = 7 };
static const char* K_NAMES[K_NSLOTS] = {"z_inverse", "x_inverse_c2r", "products_x_forward_r2c",
                                        "z_forward_combine", "column_solve", "projection", "other"};

inline cudaEvent_t ev_get(diablo_ctx* ctx) {
  if (!ctx->pool.empty()) { cudaEvent_t e = ctx->pool.back(); ctx->pool.pop_back(); return e; }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
// Bracket one kernel launch with events when profiling is on.
struct Prof {
  diablo_ctx* ctx; int slot; cudaEvent_t a = nullptr;
  Prof(diablo_ctx* c, int s) : ctx(c), slot(s) {
    ctx->launches++;
    if (ctx->profiling) { a = ev_get(ctx); cudaEventRecord(a, ctx->stream); }
  }
  ~Prof() {
    if (!a) return;
    cudaEvent_t b = ev_get(ctx);
    cudaEventRecord(b, ctx->stream);
    ctx->timed.push_back({slot, a, b});
  }
};
inline void prof_collect(diablo_ctx* ctx) {
  for (auto& t : ctx->timed) {
    float ms = 0.f;
    cudaEventSynchronize(t.b);
    cudaEventElapsedTime(&ms, t.a, t.b);
    ctx->slot_ms[t.slot] += ms;
    ctx->slot_n[t.slot] += 1;
    ctx->pool.push_back(t.a);
    ctx->pool.push_back(t.b);
  }
  ctx->timed.clear();
}

#include "fft_launch.h"
#include "layout_launch.h"

// ---- shared helpers (core.cu) --------------------------------------------
int dev_alloc(diablo_ctx* ctx, void** p, size_t bytes);
int upload_tw(diablo_ctx* ctx, int n, int count, double2** d, float2** f);
inline size_t four_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nkx1 * c->kp; }
inline size_t xs_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nkx1 * c->nz; }
inline size_t phys_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nz * c->nx; }
inline size_t ref_doubles(const diablo_ctx* c) { return (size_t)c->nyp2 * (c->nz + 2) * (c->nx + 2); }
inline int grid1d(size_t n) { return (int)((n + 255) / 256); }
inline int rows_per_lane(int n) { int R = (n + 31) / 32; return R < 3 ? 3 : R; }
int ensure_scratch(diablo_ctx* ctx);
int ensure_bscratch(diablo_ctx* ctx);
int ensure_xs64(diablo_ctx* ctx);
int fwd_phys_to_four(diablo_ctx* ctx, const double* phys, double2* xs, double2* four);
int inv_four_to_phys(diablo_ctx* ctx, const double2* four, double2* xs, double* phys);
bool is_device_ptr(const void* p);
// batched transforms between FP64 Fourier arrays and physical arrays of
// element type P (double or float); instantiated for both in core.cu
template <typename P>
int ifft_batch_t(diablo_ctx* ctx, const double2* const* four, P* const* phys, int nf);
// acc_scale != 0 (FP64 output only): four[f] += w(m) acc_scale F(phys[f])
// instead of four[f] = F(phys[f]), w(0) = 1, w(m > 0) = 2
template <typename P>
int fft_batch_t(diablo_ctx* ctx, const P* const* phys, double2* const* four, int nf, double acc_scale = 0.0);
int ifft_batch(diablo_ctx* ctx, const double2* const* four, double* const* phys, int nf);
int fft_batch(diablo_ctx* ctx, const double* const* phys, double2* const* four, int nf);
int les_active(const diablo_ctx* ctx);
int four_in(diablo_ctx* ctx, const double* buf, double2* dst, bool check);
int four_out(diablo_ctx* ctx, const double2* src, double* buf);
int bc_post(diablo_ctx* ctx, int do_vel, int do_th);
int filter_scalars(diablo_ctx* ctx);
int filter_field(diablo_ctx* ctx, int n, double2* f);
bool filter_due(const diablo_ctx* ctx, int n, int time_step);

// ---- column solve launchers (column_launch.cu) ----------------------------
int launch_tiles(const Solve2Args& A, cudaStream_t s);
size_t factor_doubles(int n, int nf);
int launch_factor(const SolveArgs& a, const double* kc, double* out, int nf, cudaStream_t s);
int launch_solve(const SolveArgs& a, bool project_only, cudaStream_t s);
struct FieldArgs;
int launch_field_solve(const FieldArgs& A, cudaStream_t s);
int launch_project_cols(const FieldArgs& A, cudaStream_t s);
int launch_column_step(const FieldArgs& A, cudaStream_t s);
int column_step_resident(int n);   // blocks of k_column_step resident at once
// the ensemble column step (column_ens.cu): one launch for every member of a
// rows-per-lane class R (3..9); resident blocks of that launch
struct EnsColArgs;
int column_step_ens_resident(int R);
int launch_column_step_ens(const EnsColArgs& E, int R, int ntask, cudaStream_t s);
int sched_status(diablo_ctx* ctx);  // DIABLO_ERR_TIMEOUT if a device wait gave up (clears it)

// ---- the step (step.cu) ------------------------------------------------------
int upload_coefficients(diablo_ctx* ctx);
void fill_solve_args(diablo_ctx* ctx, SolveArgs& a, int rk);
void update_transient(diablo_ctx* ctx);
// mean_mask: fields whose (0,0) mode (the mean profile) stays out of the
// physical fields; instantiated for double and float in step.cu
template <typename T>
int spectral_inverse(diablo_ctx* ctx, unsigned mean_mask);
template <typename T>
int spectral_nl(diablo_ctx* ctx, bool mean_free_u1);
template <typename T>
int substep_spectral(diablo_ctx* ctx, unsigned mean_mask);
int substep(diablo_ctx* ctx, int rk);
int ensure_cfl(diablo_ctx* ctx);
int courant_phys(diablo_ctx* ctx, const double* const* u);
int courant_four(diablo_ctx* ctx, double2* const* cu);
bool courant_due(const diablo_ctx* ctx, int rk);
int poisson_p(diablo_ctx* ctx);

// ---- LES (les.cu) -------------------------------------------------------------
int ensure_les(diablo_ctx* ctx);
int ensure_amd(diablo_ctx* ctx);
int ensure_dyn(diablo_ctx* ctx);
int substep_les(diablo_ctx* ctx, int rk);

// ---- ensembles (ensemble.cu) -----------------------------------------------------
int one_step(diablo_ctx* ctx);
