// libdiablo_gpu: context, device memory, kernel orchestration and the C ABI
// declared in include/diablo_gpu.h.
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
#include "kernels_layout.cuh"
#include "kernels_solve.cuh"
#include "kernels_solve2.cuh"
#include "kernels_les.cuh"
#include "kernels_adjoint.cuh"
#include "kernels_init.cuh"
#include "kernels_stats.cuh"

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
  double2* st[2][3 + DIABLO_MAX_TH];
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
  int use_general_solver;   // 1: per-lane-load column kernel instead of the tiled one
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
  } les;
  // discrete adjoint: checkpoints of the recorded steps and adjoint work arrays
  struct Tape {
    int ready, nsteps, every, nseg;
    int step_end, gen_end;
    double time_end;
    std::vector<double2*> ckpt;       // (nseg + 1) x 4 fields (u1, u2, u3, p); the last is the final state
    std::vector<int> ckpt_step;
    std::vector<double> ckpt_time;
    std::vector<double2*> sub;        // every x 3 substeps x 3 velocity inputs
    double2 *lu[4], *ou[4], *lF[3], *oF[3], *lnl[3], *pf[8], *lf3[3];
    int work_ready;
    double *pp[8], *up[3], *lp3[3];
    double *d_cn, *d_rmask, *d_pa;    // [3 rk][3 field][3][n], [3][n], [3][n]
  } tape;
  struct Timed { int slot; cudaEvent_t a, b; };
  std::vector<Timed> timed;        // pending (recorded, not yet read)
  std::vector<cudaEvent_t> pool;   // free events
  double slot_ms[8];
  long long slot_n[8];
};

enum { K_ZINV = 0, K_XINV = 1, K_XFWD_NL = 2, K_ZFWD_NL = 3, K_SOLVE = 4, K_OTHER = 5, K_NSLOTS = 6 };
static const char* K_NAMES[K_NSLOTS] = {"z_inverse", "x_inverse_c2r", "products_x_forward_r2c",
                                        "z_forward_combine", "column_solve", "other"};

static cudaEvent_t ev_get(diablo_ctx* ctx) {
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
static void prof_collect(diablo_ctx* ctx) {
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

// ---- column solve ----
template <int R>
static void launch_solve_t(const SolveArgs& a, bool project_only, cudaStream_t s) {
  const int warps = 4;
  dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
  if (project_only) k_rem_div<R><<<grd, blk, 0, s>>>(a);
  else k_column_solve<R><<<grd, blk, 0, s>>>(a);
}
template <int R>
static void launch_tiles_t(const Solve2Args& A, cudaStream_t s) {
  const int smem = (T2_STAGES * A.s.n * T2_PITCH + T2_COLS * 32 * (R | 1)) * (int)sizeof(double2) +
                   (A.mean_split ? 2 * A.s.n * (int)sizeof(double) : 0);
  cudaFuncSetAttribute(k_column_tiles<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int ngroups = (A.s.nk2 + T2_COLS - 1) / T2_COLS;
  k_column_tiles<R><<<A.s.nkx1 * ngroups, 32 * T2_COLS, smem, s>>>(A);
}
static int launch_tiles(const Solve2Args& A, cudaStream_t s) {
  int R = (A.s.n + 31) / 32;
  if (R < 3) R = 3;
  switch (R) {
#define X(r) case r: launch_tiles_t<r>(A, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

template <int R>
static size_t factor_doubles_t(int nf) { return (size_t)nf * Fac<R>::N * 32; }
template <int R>
static void launch_factor_t(const SolveArgs& a, const double* kc, double* out, int nf, cudaStream_t s) {
  k_factor<R><<<nf, 32, 0, s>>>(a, kc, out);
}
static int rows_per_lane(int n) { int R = (n + 31) / 32; return R < 3 ? 3 : R; }
static size_t factor_doubles(int n, int nf) {
  switch (rows_per_lane(n)) {
#define X(r) case r: return factor_doubles_t<r>(nf);
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return 0;
  }
}
static int launch_factor(const SolveArgs& a, const double* kc, double* out, int nf, cudaStream_t s) {
  switch (rows_per_lane(a.n)) {
#define X(r) case r: launch_factor_t<r>(a, kc, out, nf, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

static int launch_solve(const SolveArgs& a, bool project_only, cudaStream_t s) {
  int R = (a.n + 31) / 32;
  if (R < 3) R = 3;
  switch (R) {
#define X(r) case r: launch_solve_t<r>(a, project_only, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

// launchers shared with other translation units (layout_launch.h)
void launch_ref_to_phys(const double* ref, double* out, int nx, int nz, int nyp2, cudaStream_t s) {
  size_t tot = (size_t)nyp2 * nz * nx;
  k_ref_to_phys<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(ref, out, nx, nz, nyp2, nz + 2);
}
void launch_four_to_ref(const double2* in, double2* ref, const Geom& g, int nxp, cudaStream_t s) {
  size_t tot = (size_t)g.nyp2 * g.nk2 * nxp;
  k_four_to_ref<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(in, ref, g, nxp, nxp + 1, g.nz + 2);
}

// --------------------------------------------------------------------------
static int dev_alloc(diablo_ctx* ctx, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    ctx->last_cuda = (int)e;
    cudaGetLastError();
    return DIABLO_ERR_NOMEM;
  }
  ctx->allocs.push_back(*p);
  e = cudaMemsetAsync(*p, 0, bytes, ctx->stream);
  if (e != cudaSuccess) { ctx->last_cuda = (int)e; return DIABLO_ERR_CUDA; }
  return 0;
}

static void twiddles(int n, int count, std::vector<double2>& d, std::vector<float2>& f) {
  const long double pi = 3.141592653589793238462643383279502884L;
  d.resize(count);
  f.resize(count);
  for (int m = 0; m < count; ++m) {
    long double ang = 2.0L * pi * (long double)m / (long double)n;
    double c = (double)cosl(ang), s = (double)-sinl(ang);
    d[m] = make_double2(c, s);
    f[m] = make_float2((float)cosl(ang), (float)-sinl(ang));
  }
}

static int upload_tw(diablo_ctx* ctx, int n, int count, double2** d, float2** f) {
  std::vector<double2> hd;
  std::vector<float2> hf;
  twiddles(n, count, hd, hf);
  int rc = dev_alloc(ctx, (void**)d, count * sizeof(double2));
  if (rc) return rc;
  rc = dev_alloc(ctx, (void**)f, count * sizeof(float2));
  if (rc) return rc;
  CK(cudaMemcpyAsync(*d, hd.data(), count * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(*f, hf.data(), count * sizeof(float2), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

static size_t four_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nkx1 * c->kp; }
static size_t xs_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nkx1 * c->nz; }
static size_t phys_elems(const diablo_ctx* c) { return (size_t)c->nyp2 * c->nz * c->nx; }
static size_t ref_doubles(const diablo_ctx* c) { return (size_t)c->nyp2 * (c->nz + 2) * (c->nx + 2); }

static int ensure_scratch(diablo_ctx* ctx) {
  if (ctx->scratch_prec == ctx->precision) return 0;
  if (ctx->scratch_prec >= 0) return DIABLO_ERR_UNSUPPORTED;  // resized below on first use only
  const size_t cs = ctx->precision == DIABLO_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t rs = cs / 2;
  for (int f = 0; f < ctx->nf; ++f) {
    // nl[0] is FP64 in both precisions (the mean-split u1 equation, mixed)
    int rc = dev_alloc(ctx, &ctx->nl[f], four_elems(ctx) * (f == 0 ? sizeof(double2) : cs));
    if (rc) return rc;
    rc = dev_alloc(ctx, &ctx->phys[f], phys_elems(ctx) * rs);
    if (rc) return rc;
  }
  for (int f = 0; f < 2 * ctx->nf; ++f) {
    int rc = dev_alloc(ctx, &ctx->xs[f], xs_elems(ctx) * cs);
    if (rc) return rc;
  }
  ctx->scratch_prec = ctx->precision;
  return 0;
}

static int ensure_bscratch(diablo_ctx* ctx) {
  if (ctx->b_phys) return 0;
  int rc;
  if ((rc = dev_alloc(ctx, (void**)&ctx->b_phys, phys_elems(ctx) * sizeof(double)))) return rc;
  if ((rc = dev_alloc(ctx, (void**)&ctx->b_xs, xs_elems(ctx) * sizeof(double2)))) return rc;
  if ((rc = dev_alloc(ctx, (void**)&ctx->b_four, four_elems(ctx) * sizeof(double2)))) return rc;
  if ((rc = dev_alloc(ctx, (void**)&ctx->b_ref, ref_doubles(ctx) * sizeof(double)))) return rc;
  return 0;
}

// --------------------------------------------------------------------------
// FP64 transforms between internal layouts (one field)
static int fwd_phys_to_four(diablo_ctx* ctx, const double* phys, double2* xs, double2* four) {
  XFwdArgs<double> xa;
  memset(&xa, 0, sizeof(xa));
  xa.in[0] = phys;
  xa.outA[0] = xs;
  xa.j0 = 0;
  xa.g = ctx->g;
  xa.twM = ctx->tm64;
  xa.twX = ctx->tx64;
  xa.kx = ctx->d_kx;
  xa.gm = GridMetrics{ctx->d_dy, ctx->d_dyf};
  xa.scale = 1.0 / ctx->nx;
  int rc = launch_xfwd<double, false>(xa, ctx->M, ctx->nyp2, 1, ctx->stream);
  if (rc) return rc;
  ctx->launches++;
  ZFwdArgs<double2, double2> za;
  memset(&za, 0, sizeof(za));
  za.srcA[0] = xs;
  za.dst[0] = four;
  za.q0 = 0;
  za.nseq = ctx->nyp2 * ctx->nkx1;
  za.g = ctx->g;
  za.tw = ctx->tz64;
  za.kz = ctx->d_kz;
  za.scale = 1.0 / ctx->nz;
  rc = launch_zfwd<double2, double2, false>(za, ctx->nz, 1, ctx->stream);
  if (rc) return rc;
  ctx->launches++;
  return 0;
}

static int inv_four_to_phys(diablo_ctx* ctx, const double2* four, double2* xs, double* phys) {
  ZInvArgs<double2> za;
  memset(&za, 0, sizeof(za));
  za.src[0] = four;
  za.dst[0] = xs;
  za.q0 = 0;
  za.nseq = ctx->nyp2 * ctx->nkx1;
  za.g = ctx->g;
  za.tw = ctx->tz64;
  int rc = launch_zinv<double2>(za, ctx->nz, 1, ctx->stream);
  if (rc) return rc;
  ctx->launches++;
  XInvArgs<double2> xa;
  memset(&xa, 0, sizeof(xa));
  xa.src[0] = xs;
  xa.dst[0] = phys;
  xa.j0 = 0;
  xa.g = ctx->g;
  xa.twM = ctx->tm64;
  xa.twX = ctx->tx64;
  rc = launch_xinv<double2>(xa, ctx->M, ctx->nyp2, 1, ctx->stream);
  if (rc) return rc;
  ctx->launches++;
  return 0;
}

static int grid1d(size_t n) { return (int)((n + 255) / 256); }

static bool is_device_ptr(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

static void fill_solve_args(diablo_ctx* ctx, SolveArgs& a, int rk);

// --------------------------------------------------------------------------
// Row coefficients of the implicit solves, evaluated with the reference's
// expressions (for/channel.f90:664-670 scalars, :726-733 u2, :782-788 and
// :838-845 u1/u3, :969-976 rem_div), for each RK substep.
static int upload_coefficients(diablo_ctx* ctx) {
  const int n = ctx->nyp2, ny = ctx->ny, nk = 2 + ctx->nth;
  const std::vector<double>& dy = ctx->h_dy;
  const std::vector<double>& dyf = ctx->h_dyf;
  const double nuv = ctx->p.nu_v_scale;
  for (int rk = 0; rk < 3; ++rk) {
    std::vector<double> kc((size_t)nk * 3 * n, 0.0);
    const double temp1 = 0.5 * ctx->nu * ctx->h_bar[rk];
    for (int kind = 0; kind < nk; ++kind) {
      double* A = &kc[(size_t)kind * 3 * n];
      double* B = A + n;
      double* C = B + n;
      for (int j = 0; j < n; ++j) B[j] = 1.0;
      if (kind == 0) {
        for (int j = 1; j <= ny; ++j) {
          A[j] = -temp1 * nuv / (dy[j] * dyf[j]);
          B[j] = 1. - temp1 * nuv * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
          C[j] = -temp1 * nuv / (dy[j + 1] * dyf[j]);
        }
      } else if (kind == 1) {
        for (int j = 2; j <= ny; ++j) {
          A[j] = -temp1 * nuv / (dyf[j - 1] * dy[j]);
          B[j] = 1. + temp1 * nuv / (dyf[j] * dy[j]) + temp1 * nuv / (dyf[j - 1] * dy[j]);
          C[j] = -temp1 * nuv / (dyf[j] * dy[j]);
        }
      } else {
        const double tm = temp1 / ctx->p.pr[kind - 2] * nuv;
        for (int j = 1; j <= ny; ++j) {
          A[j] = -tm / (dy[j] * dyf[j]);
          B[j] = 1. + tm / (dy[j + 1] * dyf[j]) + tm / (dy[j] * dyf[j]);
          C[j] = -tm / (dy[j + 1] * dyf[j]);
        }
      }
    }
    if (!ctx->d_kc[rk]) {
      int rc = dev_alloc(ctx, (void**)&ctx->d_kc[rk], kc.size() * sizeof(double));
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(ctx->d_kc[rk], kc.data(), kc.size() * sizeof(double), cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  // the met rows (below) are not used by the factorisation, the kc rows are
  for (int rk = 0; rk < 3; ++rk) {
    if (!ctx->d_fac[rk]) {
      int rc = dev_alloc(ctx, (void**)&ctx->d_fac[rk], factor_doubles(n, ctx->nf) * sizeof(double));
      if (rc) return rc;
    }
    SolveArgs a;
    fill_solve_args(ctx, a, rk + 1);
    int rc = launch_factor(a, ctx->d_kc[rk], ctx->d_fac[rk], ctx->nf, ctx->stream);
    if (rc) return rc;
    ctx->launches++;
    CK(cudaGetLastError());
  }
  std::vector<double> met((size_t)MET_N * n, 0.0);
  for (int j = 1; j <= ny; ++j) {
    met[MET_PA * n + j] = 1. / (dy[j] * dyf[j]);
    met[MET_PC * n + j] = 1. / (dy[j + 1] * dyf[j]);
    met[MET_PB0 * n + j] = -1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]);
    met[MET_IDYF * n + j] = 1.0 / dyf[j];
  }
  for (int j = 1; j <= ny + 1; ++j) met[MET_IDY * n + j] = 1.0 / dy[j];
  for (int j = 2; j <= ny; ++j) {
    met[MET_WB1 * n + j] = dyf[j - 1] / (2.0 * dy[j]);
    met[MET_WB2 * n + j] = dyf[j] / (2.0 * dy[j]);
  }
  if (!ctx->d_met) {
    int rc = dev_alloc(ctx, (void**)&ctx->d_met, met.size() * sizeof(double));
    if (rc) return rc;
  }
  if (!ctx->d_prof) {
    int rc = dev_alloc(ctx, (void**)&ctx->d_prof, 2 * (size_t)n * sizeof(double));
    if (rc) return rc;
  }
  CK(cudaMemcpyAsync(ctx->d_met, met.data(), met.size() * sizeof(double), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

static void fill_solve_args(diablo_ctx* ctx, SolveArgs& a, int rk) {
  memset(&a, 0, sizeof(a));
  const diablo_params& p = ctx->p;
  a.nyp = ctx->ny;
  a.n = ctx->nyp2;
  a.nkx1 = ctx->nkx1;
  a.nk2 = ctx->nk2;
  a.kp = ctx->kp;
  a.ncol = ctx->nkx1 * ctx->nk2;
  a.nth = ctx->nth;
  a.rk = rk;
  const double h = ctx->h_bar[rk - 1];
  a.temp1 = 0.5 * ctx->nu * h;
  a.temp2 = 0.5 * h;
  a.temp3 = ZETA_BAR[rk - 1] * h;
  a.temp4 = h;
  a.temp5 = BETA_BAR[rk - 1] * h;
  a.nu = ctx->nu;
  a.beta = p.beta;
  a.nu_v = p.nu_v_scale;
  a.roinvd = ctx->ro_inv / p.delta;
  a.grav_x = p.grav_x;
  a.grav_y = p.grav_y;
  a.grav_z = p.grav_z;
  if (p.f_type == 1) a.px = a.temp4 * p.px0;
  else if (p.f_type == 2) a.px = a.temp4 * (p.px0 + p.amp_omega0 * cos(p.omega0 * ctx->time));
  a.jstart = ctx->jstart;
  a.jend = ctx->jend;
  a.ubc[0] = p.u_bc_ymin; a.ubc[1] = p.u_bc_ymax;
  a.vbc[0] = p.v_bc_ymin; a.vbc[1] = p.v_bc_ymax;
  a.wbc[0] = p.w_bc_ymin; a.wbc[1] = p.w_bc_ymax;
  a.uc1[0] = p.u_bc_ymin_c1; a.uc1[1] = p.u_bc_ymax_c1;
  a.vc1[0] = p.v_bc_ymin_c1; a.vc1[1] = p.v_bc_ymax_c1;
  a.wc1[0] = p.w_bc_ymin_c1;
  a.wc1[1] = p.w_bc_ymax == 0 ? p.w_bc_ymax_c1 : ctx->w_top_transient;
  a.front = (p.flavor_front && ctx->ro_inv != 0.0) ? 1 : 0;
  a.ly = p.ly;
  a.front_coef = ctx->ro_inv != 0.0 ? p.delta / ctx->ro_inv : 0.0;
  for (int n = 0; n < ctx->nth; ++n) {
    a.jst[n] = ctx->jst[n];
    a.jet[n] = ctx->jet[n];
    a.thbc[n][0] = p.th_bc_ymin[n];
    a.thbc[n][1] = p.th_bc_ymax[n];
    a.thc1[n][0] = p.th_bc_ymin_c1[n];
    a.thc1[n][1] = p.th_bc_ymax_c1[n];
    a.pr[n] = p.pr[n];
    a.dthdx[n] = p.dthdx[n];
    a.dthdz[n] = p.dthdz[n];
  }
  a.dy = ctx->d_dy;
  a.dyf = ctx->d_dyf;
  a.gy = ctx->d_gy;
  a.gyf = ctx->d_gyf;
  a.kx = ctx->d_kx;
  a.kz = ctx->d_kz;
}

// Update the time-dependent top value of u3 (apply_BC_3_upper, for/channel.f90:1775)
static void update_transient(diablo_ctx* ctx) {
  const diablo_params& p = ctx->p;
  if (p.w_bc_ymax != 0 && p.f_type == 4)
    ctx->w_top_transient = p.w_bc_ymax_c1 + p.amp_omega0 *
        sin(p.omega0 * (ctx->ro_inv / p.delta * ctx->time - p.force_start));
}

// mean_mask: fields whose (0,0) mode (the mean profile) stays out of the
// physical fields; its products are added in FP64 further on.
template <typename T>
static int spectral_inverse(diablo_ctx* ctx, unsigned mean_mask = 0) {
  typedef typename CT<T>::C C;
  const int nf = ctx->nf;
  const int c = ctx->cur;
  const C* tz = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tz64 : (const void*)ctx->tz32);
  const C* tm = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tm64 : (const void*)ctx->tm32);
  const C* tx = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tx64 : (const void*)ctx->tx32);
  int rc;
  // 1. z inverse of u1, u2, u3, th_n (all planes) -> x-spectral
  {
    ZInvArgs<C> a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < nf; ++f) {
      a.src[f] = ctx->st[c][f < 3 ? f : f + 1];
      a.dst[f] = (C*)ctx->xs[f];
    }
    a.q0 = 0;
    a.nseq = ctx->nyp2 * ctx->nkx1;
    a.g = ctx->g;
    a.tw = tz;
    a.mean_mask = mean_mask;
    Prof pr(ctx, K_ZINV);
    if ((rc = launch_zinv<C>(a, ctx->nz, nf, ctx->stream, ctx->tune[0]))) return rc;
  }
  // 2. x inverse -> physical
  {
    XInvArgs<C> a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < nf; ++f) {
      a.src[f] = (const C*)ctx->xs[f];
      a.dst[f] = (T*)ctx->phys[f];
    }
    a.j0 = 0;
    a.g = ctx->g;
    a.twM = tm;
    a.twX = tx;
    Prof pr(ctx, K_XINV);
    if ((rc = launch_xinv<C>(a, ctx->M, ctx->nyp2, nf, ctx->stream, ctx->tune[1]))) return rc;
  }
  return 0;
}

template <typename T>
static int spectral_nl(diablo_ctx* ctx, bool mean_free_u1 = false) {
  typedef typename CT<T>::C C;
  const int nf = ctx->nf;
  const int c = ctx->cur;
  const C* tz = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tz64 : (const void*)ctx->tz32);
  const C* tm = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tm64 : (const void*)ctx->tm32);
  const C* tx = (const C*)(sizeof(T) == 8 ? (const void*)ctx->tx64 : (const void*)ctx->tx32);
  int rc;
  // 3. nonlinear products + x forward (planes 1..Ny)
  {
    XFwdArgs<T> a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < nf; ++f) {
      a.in[f] = (const T*)ctx->phys[f];
      a.outA[f] = (C*)ctx->xs[f];
      a.outB[f] = (C*)ctx->xs[nf + f];
    }
    a.j0 = 1;
    a.g = ctx->g;
    a.twM = tm;
    a.twX = tx;
    a.kx = ctx->d_kx;
    a.gm = GridMetrics{ctx->d_dy, ctx->d_dyf};
    a.scale = 1.0 / ctx->nx;
    Prof pr(ctx, K_XFWD_NL);
    if ((rc = launch_xfwd<T, true>(a, ctx->M, ctx->ny, nf, ctx->stream, ctx->tune[2]))) return rc;
  }
  // 4. z forward + combine -> NL (planes 1..Ny)
  {
    ZFwdArgs<C, C> a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < nf; ++f) {
      a.srcA[f] = (const C*)ctx->xs[f];
      a.srcB[f] = (const C*)ctx->xs[nf + f];
      a.dst[f] = (C*)ctx->nl[f];
    }
    a.q0 = ctx->nkx1;
    a.nseq = ctx->ny * ctx->nkx1;
    a.g = ctx->g;
    a.tw = tz;
    a.kz = ctx->d_kz;
    a.scale = 1.0 / ctx->nz;
    if (mean_free_u1) {
      // the u1 equation takes the FP64 mean epilogue into its FP64 NL array
      for (int q = 0; q < 3; ++q) a.cu[q] = ctx->st[c][q];
      a.kx = ctx->d_kx;
      a.dy = ctx->d_dy;
      a.dyf = ctx->d_dyf;
      a.prof = ctx->d_prof;
      a.fps = (size_t)ctx->nkx1 * ctx->kp;
    }
    Prof pr(ctx, K_ZFWD_NL);
    if ((rc = launch_zfwd<C, C, true>(a, ctx->nz, nf, ctx->stream, ctx->tune[3]))) return rc;
  }
  return 0;
}

template <typename T>
static int substep_spectral(diablo_ctx* ctx, unsigned mean_mask) {
  int rc = spectral_inverse<T>(ctx, mean_mask);
  return rc ? rc : spectral_nl<T>(ctx, (mean_mask & 1u) != 0);
}

// ==========================================================================
// LES substep (FP64): the reference's physical-space path, for/channel.f90
// :29-911 with les_chan/les_chan_th (for/les.f90:20-1200)

static const double LES_C_SMAG = 0.17;   // for/les.f90:38
static const double LES_BETA = 3.0;      // for/les.f90:58
static const double LES_C_AMD = 0.2887;  // for/les.f90:42

// FP64 x-spectral scratch of the batched transforms (LES and adjoint)
static int ensure_xs64(diablo_ctx* ctx) {
  diablo_ctx::Les& L = ctx->les;
  if (L.xs[0]) return 0;
  for (int i = 0; i < NF_MAX; ++i) {
    int rc = dev_alloc(ctx, (void**)&L.xs[i], xs_elems(ctx) * sizeof(double2));
    if (rc) return rc;
  }
  return 0;
}

static int ensure_les(diablo_ctx* ctx) {
  diablo_ctx::Les& L = ctx->les;
  if (L.ready) return 0;
  const size_t fe = four_elems(ctx) * sizeof(double2), pe = phys_elems(ctx) * sizeof(double);
  int rc;
#define AL(ptr, bytes) if ((rc = dev_alloc(ctx, (void**)&(ptr), (bytes)))) return rc
  for (int i = 0; i < 6; ++i) { AL(L.S[i], fe); AL(L.Sp[i], pe); }
  for (int i = 0; i < 7; ++i) AL(L.T[i], fe);
  for (int f = 0; f < ctx->nf; ++f) { AL(L.cr[f], fe); AL(L.r[f], pe); AL(L.u64[f], pe); }
  for (int i = 0; i < 2 * ctx->nth; ++i) { AL(L.thg[i], fe); AL(L.thp[i], pe); }
  AL(L.tmp[0], pe); AL(L.tmp[1], pe);
  AL(L.nu_t, pe); AL(L.sf, pe); AL(L.sg, pe);

  if ((rc = ensure_xs64(ctx))) return rc;
  const int n = ctx->nyp2;
  AL(L.d_cf, n * sizeof(double)); AL(L.d_cg, n * sizeof(double));
  AL(L.d_d2f, n * sizeof(double)); AL(L.d_d2g, n * sizeof(double));
  AL(L.d_sclf, n * sizeof(double)); AL(L.d_sclg, n * sizeof(double));
  AL(L.d_idy, n * sizeof(double)); AL(L.d_idyf, n * sizeof(double));
#undef AL
  // filter widths Delta^2 and the constant-model scalings (for/les.f90:224-245)
  std::vector<double> d2f(n, 0.0), d2g(n, 0.0), cf(n, 0.0), cg(n, 0.0), sclf(n, 1.0), sclg(n, 1.0);
  const double dx1 = ctx->p.lx / ctx->nx, dz1 = ctx->p.lz / ctx->nz;
  const double c2 = pow(LES_C_SMAG, 2.0);
  for (int j = 1; j <= ctx->ny; ++j)
    d2f[j] = pow(dx1 * LES_BETA * ctx->h_dyf[j] * 1.0 * dz1 * LES_BETA, 2.0 / 3.0);
  for (int j = 1; j <= ctx->ny + 1; ++j)
    d2g[j] = pow(dx1 * LES_BETA * ctx->h_dy[j] * 2.0 * dz1 * LES_BETA, 2.0 / 3.0);
  const int model = ctx->p.les_model_type;
  if (model == 1) {
    for (int j = 0; j < n; ++j) {
      cf[j] = c2; cg[j] = c2;
      sclf[j] = -2.0 * c2 * d2f[j];
      sclg[j] = -2.0 * c2 * d2g[j];
    }
  } else if (model == 4 || model == 5) {
    // AMD: delta_yf, delta_y of for/les.f90:500-516 (4) and :776-797 (5);
    // nu_t = -0.5 delta_y temp, carried as cg with unit Delta^2
    for (int j = 1; j <= ctx->ny + 1; ++j) {
      if (model == 4) {
        sclf[j] = -2.0 * pow(LES_C_AMD, 2.0);
        sclg[j] = -2.0 * pow(LES_C_AMD, 2.0);
      } else {
        const double ix = 1.0 / pow(dx1 * LES_BETA, 2.0), iz = 1.0 / pow(dz1 * LES_BETA, 2.0);
        sclf[j] = -2.0 * pow(LES_C_AMD, 2.0) * 3.0 / (ix + 1.0 / pow(ctx->h_dyf[j] * 2.0, 2.0) + iz);
        sclg[j] = -2.0 * pow(LES_C_AMD, 2.0) * 3.0 / (ix + 1.0 / pow(ctx->h_dy[j] * 2.0, 2.0) + iz);
      }
      cg[j] = -0.5 * sclg[j];
    }
    for (int j = 0; j < n; ++j) d2g[j] = 1.0;
  }
  CK(cudaMemcpyAsync(L.d_d2f, d2f.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_d2g, d2g.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_cf, cf.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_cg, cg.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_sclf, sclf.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_sclg, sclg.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  // 1/dy, 1/dyf for the physical-space CN rows (dy(0) is not a grid spacing)
  std::vector<double> idy(n, 0.0), idyf(n, 0.0);
  for (int j = 1; j < n; ++j) idy[j] = 1.0 / ctx->h_dy[j];
  for (int j = 0; j < n; ++j) idyf[j] = 1.0 / ctx->h_dyf[j];
  CK(cudaMemcpyAsync(L.d_idy, idy.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(L.d_idyf, idyf.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  L.ready = 1;
  return 0;
}

// batched FP64 transforms between the internal Fourier and physical layouts
// Batched transforms between FP64 Fourier arrays and physical arrays of
// element type P (double, or float for the mixed-precision LES model).
template <typename P>
static int ifft_batch_t(diablo_ctx* ctx, const double2* const* four, P* const* phys, int nf) {
  typedef typename CT<P>::C C;
  const C* tz = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tz64 : (const void*)ctx->tz32);
  const C* tm = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tm64 : (const void*)ctx->tm32);
  const C* tx = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tx64 : (const void*)ctx->tx32);
  for (int b = 0; b < nf; b += NF_MAX) {
    const int m = nf - b < NF_MAX ? nf - b : NF_MAX;
    ZInvArgs<C> za;
    memset(&za, 0, sizeof(za));
    XInvArgs<C> xa;
    memset(&xa, 0, sizeof(xa));
    for (int f = 0; f < m; ++f) {
      za.src[f] = four[b + f];
      za.dst[f] = (C*)ctx->les.xs[f];
      xa.src[f] = (const C*)ctx->les.xs[f];
      xa.dst[f] = phys[b + f];
    }
    za.nseq = ctx->nyp2 * ctx->nkx1;
    za.g = ctx->g;
    za.tw = tz;
    xa.g = ctx->g;
    xa.twM = tm;
    xa.twX = tx;
    int rc;
    { Prof pr(ctx, K_ZINV); if ((rc = launch_zinv<C>(za, ctx->nz, m, ctx->stream))) return rc; }
    { Prof pr(ctx, K_XINV); if ((rc = launch_xinv<C>(xa, ctx->M, ctx->nyp2, m, ctx->stream))) return rc; }
  }
  return 0;
}

template <typename P>
static int fft_batch_t(diablo_ctx* ctx, const P* const* phys, double2* const* four, int nf) {
  typedef typename CT<P>::C C;
  const C* tz = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tz64 : (const void*)ctx->tz32);
  const C* tm = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tm64 : (const void*)ctx->tm32);
  const C* tx = (const C*)(sizeof(P) == 8 ? (const void*)ctx->tx64 : (const void*)ctx->tx32);
  for (int b = 0; b < nf; b += NF_MAX) {
    const int m = nf - b < NF_MAX ? nf - b : NF_MAX;
    XFwdArgs<P> xa;
    memset(&xa, 0, sizeof(xa));
    ZFwdArgs<C, double2> za;
    memset(&za, 0, sizeof(za));
    for (int f = 0; f < m; ++f) {
      xa.in[f] = phys[b + f];
      xa.outA[f] = (C*)ctx->les.xs[f];
      za.srcA[f] = (const C*)ctx->les.xs[f];
      za.dst[f] = four[b + f];
    }
    xa.g = ctx->g;
    xa.twM = tm;
    xa.twX = tx;
    xa.kx = ctx->d_kx;
    xa.gm = GridMetrics{ctx->d_dy, ctx->d_dyf};
    xa.scale = 1.0 / ctx->nx;
    za.nseq = ctx->nyp2 * ctx->nkx1;
    za.g = ctx->g;
    za.tw = tz;
    za.kz = ctx->d_kz;
    za.scale = 1.0 / ctx->nz;
    int rc;
    { Prof pr(ctx, K_OTHER); if ((rc = launch_xfwd<P, false>(xa, ctx->M, ctx->nyp2, m, ctx->stream))) return rc; }
    { Prof pr(ctx, K_OTHER); if ((rc = launch_zfwd<C, double2, false>(za, ctx->nz, m, ctx->stream))) return rc; }
  }
  return 0;
}

static int ifft_batch(diablo_ctx* ctx, const double2* const* four, double* const* phys, int nf) {
  return ifft_batch_t<double>(ctx, four, phys, nf);
}
static int fft_batch(diablo_ctx* ctx, const double* const* phys, double2* const* four, int nf) {
  return fft_batch_t<double>(ctx, phys, four, nf);
}

static int les_active(const diablo_ctx* ctx) {
  // for/channel.f90:259: LES only after 100 steps of a newly created flow
  return ctx->p.use_les && (!ctx->p.create_new_flow || ctx->time_step > 100);
}

template <typename P>
static int dynamic_coefficient(diablo_ctx* ctx);
extern "C" {
static int bc_post(diablo_ctx* ctx, int do_vel, int do_th);
}

static int ensure_amd(diablo_ctx* ctx) {
  diablo_ctx::Les& L = ctx->les;
  if (L.amd_ready) return 0;
  const size_t fe = four_elems(ctx) * sizeof(double2), pe = phys_elems(ctx) * sizeof(double);
  const bool m5 = ctx->p.les_model_type == 5;
  int rc;
#define AL(ptr, bytes) if ((rc = dev_alloc(ctx, (void**)&(ptr), (bytes)))) return rc
  for (int q = 0; q < 3; ++q) { AL(L.Of[q], fe); AL(L.Op[q], pe); }
  if (m5) {
    for (int q = 0; q < 6; ++q) { AL(L.SIf[q], fe); AL(L.SIp[q], pe); }
    for (int q = 0; q < 9; ++q) { AL(L.Gf[q], fe); AL(L.Gp[q], pe); }
    for (int q = 0; q < 3 * ctx->nth; ++q) { AL(L.Tf[q], fe); AL(L.Tp[q], pe); }
    for (int n = 0; n < ctx->nth; ++n) {
      AL(L.fxp[n], pe); AL(L.fzp[n], pe); AL(L.fxf[n], fe); AL(L.fzf[n], fe); AL(L.kap[n], pe);
    }
  }
#undef AL
  L.amd_ready = 1;
  return 0;
}

static int ensure_cfl(diablo_ctx* ctx);
static int courant_phys(diablo_ctx* ctx, const double* const* u);
static bool courant_due(const diablo_ctx* ctx, int rk);

// batched transforms of LES work arrays (allocated as FP64, used as P)
template <typename P>
static int ifft_to(diablo_ctx* ctx, double2* const* four, double* const* phys, int nf) {
  P* d[64];
  for (int f = 0; f < nf; ++f) d[f] = reinterpret_cast<P*>(phys[f]);
  return ifft_batch_t<P>(ctx, four, d, nf);
}
template <typename P>
static int fft_from(diablo_ctx* ctx, double* const* phys, double2* const* four, int nf) {
  const P* sp[64];
  for (int f = 0; f < nf; ++f) sp[f] = reinterpret_cast<const P*>(phys[f]);
  return fft_batch_t<P>(ctx, sp, four, nf);
}

template <typename P>
static int substep_les_t(diablo_ctx* ctx, int rk) {
  auto PP = [](double* q) { return reinterpret_cast<P*>(q); };
  ctx->les.nu_t_fp32 = sizeof(P) == 4;
  diablo_ctx::Les& L = ctx->les;
  const int nf = ctx->nf, nth = ctx->nth;
  const int c = ctx->cur, nx_ = 1 - c;
  int rc;
  if ((rc = ensure_scratch(ctx)) || (rc = ensure_les(ctx))) return rc;
  update_transient(ctx);
  const FGeom fg{ctx->ny, ctx->nyp2, ctx->nkx1, ctx->nk2, ctx->kp, (size_t)ctx->nkx1 * ctx->kp};
  const size_t ftot = four_elems(ctx), ptot = phys_elems(ctx);
  SolveArgs a;
  fill_solve_args(ctx, a, rk);
  for (int q = 0; q < 3; ++q) { a.cu_in[q] = ctx->st[c][q]; a.cu_out[q] = ctx->st[nx_][q]; }
  a.cp_in = ctx->st[c][3];
  a.cp_out = ctx->st[nx_][3];
  for (int n = 0; n < nth; ++n) { a.cth_in[n] = ctx->st[c][4 + n]; a.cth_out[n] = ctx->st[nx_][4 + n]; }
  double2* cf_out[3 + DIABLO_MAX_TH];
  for (int f = 0; f < nf; ++f) {
    a.cf_in[f] = ctx->cf[ctx->cf_cur][f];
    a.cf_out[f] = cf_out[f] = ctx->cf[1 - ctx->cf_cur][f];
  }
  // 1. explicit RK terms from the state before the LES wall/ghost updates
  {
    ExplicitArgs2 E;
    memset(&E, 0, sizeof(E));
    E.s = a;
    for (int f = 0; f < nf; ++f) E.cr[f] = L.cr[f];
    Prof pr(ctx, K_OTHER);
    k_explicit2<<<grid1d(ftot), 256, 0, ctx->stream>>>(E);
  }
  // 2. apply_BC_vel/th_mpi_post and apply_BC_les/th_les on the state (for/les.f90:80-90)
  if ((rc = bc_post(ctx, 1, 1))) return rc;
  {
    LesBcArgs b;
    memset(&b, 0, sizeof(b));
    for (int q = 0; q < 3; ++q) b.cu[q] = ctx->st[c][q];
    for (int n = 0; n < nth; ++n) {
      b.cth[n] = ctx->st[c][4 + n];
      b.thbc[n][0] = ctx->p.th_bc_ymin[n];
      b.thbc[n][1] = ctx->p.th_bc_ymax[n];
    }
    b.nth = nth; b.nyp = ctx->ny; b.nkx1 = ctx->nkx1; b.nk2 = ctx->nk2; b.kp = ctx->kp;
    b.ubc[0] = ctx->p.u_bc_ymin; b.ubc[1] = ctx->p.u_bc_ymax;
    b.wbc[0] = ctx->p.w_bc_ymin; b.wbc[1] = ctx->p.w_bc_ymax;
    Prof pr(ctx, K_OTHER);
    k_les_bc<<<(ctx->nkx1 * ctx->nk2 + 127) / 128, 128, 0, ctx->stream>>>(b);
  }
  // 3. strain tensor, 4. strain and u, th to physical space
  {
    StrainArgs sa;
    for (int q = 0; q < 3; ++q) sa.cu[q] = ctx->st[c][q];
    for (int i = 0; i < 6; ++i) sa.S[i] = L.S[i];
    sa.kx = ctx->d_kx; sa.kz = ctx->d_kz; sa.dy = ctx->d_dy; sa.dyf = ctx->d_dyf; sa.g = fg;
    Prof pr(ctx, K_OTHER);
    k_strain<<<grid1d(ftot), 256, 0, ctx->stream>>>(sa);
  }
  if ((rc = ifft_to<P>(ctx, L.S, L.Sp, 6))) return rc;
  const int model = ctx->p.les_model_type;
  const bool amd = model == 4 || model == 5;
  const double dxb = ctx->p.lx / ctx->nx * LES_BETA, dzb = ctx->p.lz / ctx->nz * LES_BETA;
  if (amd) {
    // rotation (and for model 5 the invariant strain and all gradients), to physical
    if ((rc = ensure_amd(ctx))) return rc;
    AmdFourierArgs af;
    memset(&af, 0, sizeof(af));
    for (int q = 0; q < 3; ++q) { af.cu[q] = ctx->st[c][q]; af.O[q] = L.Of[q]; }
    for (int n = 0; n < nth; ++n) af.cth[n] = ctx->st[c][4 + n];
    if (model == 5) {
      for (int q = 0; q < 6; ++q) af.SI[q] = L.SIf[q];
      for (int q = 0; q < 9; ++q) af.G[q] = L.Gf[q];
      for (int q = 0; q < 3 * nth; ++q) af.T[q] = L.Tf[q];
    }
    af.kx = ctx->d_kx; af.kz = ctx->d_kz; af.dy = ctx->d_dy; af.dyf = ctx->d_dyf;
    af.deltax = dxb; af.deltaz = dzb;
    af.model = model; af.nth = nth; af.g = fg;
    { Prof pr(ctx, K_OTHER); k_amd_fourier<<<grid1d(ftot), 256, 0, ctx->stream>>>(af); }
    if ((rc = ifft_to<P>(ctx, L.Of, L.Op, 3))) return rc;
    if (model == 5) {
      if ((rc = ifft_to<P>(ctx, L.SIf, L.SIp, 6))) return rc;
      if ((rc = ifft_to<P>(ctx, L.Gf, L.Gp, 9))) return rc;
      if (nth > 0 && (rc = ifft_to<P>(ctx, L.Tf, L.Tp, 3 * nth))) return rc;
    }
  }
  if ((rc = spectral_inverse<P>(ctx))) return rc;            // u, th -> ctx->phys
  P* const* up = (P* const*)ctx->phys;
  // 5. |S|, the coefficient (dynamic model), eddy viscosity and stresses
  {
    LesPointArgs<P> pa;
    memset(&pa, 0, sizeof(pa));
    for (int i = 0; i < 6; ++i) pa.S[i] = PP(L.Sp[i]);
    pa.u1 = up[0]; pa.u3 = up[2];
    pa.nu_t = PP(L.nu_t);
    pa.tmp[0] = PP(L.tmp[0]); pa.tmp[1] = PP(L.tmp[1]);
    pa.dy = ctx->d_dy; pa.dyf = ctx->d_dyf;
    pa.cf = L.d_cf; pa.cg = L.d_cg; pa.d2f = L.d_d2f; pa.d2g = L.d_d2g;
    pa.nx = ctx->nx; pa.nz = ctx->nz; pa.nyp = ctx->ny;
    pa.dynamic = model == 2;
    pa.amd = amd;
    if (amd) {
      AmdCoefArgs<P> ca;
      for (int q = 0; q < 6; ++q) ca.S[q] = PP(model == 5 ? L.SIp[q] : L.Sp[q]);
      for (int q = 0; q < 3; ++q) ca.O[q] = PP(L.Op[q]);
      ca.dy = ctx->d_dy; ca.dyf = ctx->d_dyf;
      ca.sf = PP(L.sf); ca.sg = PP(L.sg);
      ca.wx = pow(dxb, 2.0); ca.wz = pow(dzb, 2.0);
      ca.model = model; ca.nyp = ctx->ny; ca.jstart = ctx->jstart; ca.jend = ctx->jend;
      ca.ps = (size_t)ctx->nz * ctx->nx;
      Prof pr(ctx, K_OTHER);
      k_amd_coef<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(ca);
    } else {
      Prof pr(ctx, K_OTHER);
      k_les_norms<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(pa, PP(L.sf), PP(L.sg));
    }
    if (model == 2 && (rc = dynamic_coefficient<P>(ctx))) return rc;
    { Prof pr(ctx, K_OTHER); k_les_point<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(pa, PP(L.sf), PP(L.sg)); }
  }
  // 6. stresses to Fourier space, divergence into cf (for/les.f90:245-274, 850-880)
  {
    const P* src[7] = {PP(L.Sp[0]), PP(L.Sp[2]), PP(L.Sp[3]), PP(L.Sp[4]), PP(L.Sp[5]), PP(L.tmp[0]), PP(L.tmp[1])};
    if ((rc = fft_batch_t<P>(ctx, src, L.T, 7))) return rc;
    LesDivArgs da;
    for (int i = 0; i < 7; ++i) da.T[i] = L.T[i];
    for (int q = 0; q < 3; ++q) da.cf[q] = cf_out[q];
    da.kx = ctx->d_kx; da.kz = ctx->d_kz; da.dyf = ctx->d_dyf;
    da.sf = L.d_sclf; da.sg = L.d_sclg; da.g = fg;
    da.j1 = ctx->jstart; da.j2 = ctx->ny - 1;
    Prof pr(ctx, K_OTHER);
    k_les_div<<<grid1d(ftot), 256, 0, ctx->stream>>>(da);
  }
  // 7. scalar SGS flux: the AMD scalar model (model 5, for/les.f90:1219-1412)
  // or kappa_t = nu_t (for/les.f90:1130-1200)
  if (nth > 0 && model == 5) {
    AmdThArgs<P> ta;
    memset(&ta, 0, sizeof(ta));
    for (int q = 0; q < 9; ++q) ta.G[q] = PP(L.Gp[q]);
    for (int q = 0; q < 3 * nth; ++q) ta.T[q] = PP(L.Tp[q]);
    for (int n = 0; n < nth; ++n) {
      ta.fx[n] = PP(L.fxp[n]); ta.fz[n] = PP(L.fzp[n]); ta.kap[n] = PP(L.kap[n]);
      ta.jst[n] = ctx->jst[n]; ta.jet[n] = ctx->jet[n];
    }
    ta.dy = ctx->d_dy; ta.dyf = ctx->d_dyf; ta.hdy = L.d_cg;
    ta.deltax = dxb; ta.deltaz = dzb;
    ta.nth = nth; ta.nyp = ctx->ny; ta.ps = (size_t)ctx->nz * ctx->nx;
    { Prof pr(ctx, K_OTHER); k_amd_th<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(ta); }
    P* srcp[2 * DIABLO_MAX_TH];
    double2* dstf[2 * DIABLO_MAX_TH];
    for (int n = 0; n < nth; ++n) {
      srcp[2 * n] = PP(L.fxp[n]); srcp[2 * n + 1] = PP(L.fzp[n]);
      dstf[2 * n] = L.fxf[n]; dstf[2 * n + 1] = L.fzf[n];
    }
    if ((rc = fft_batch_t<P>(ctx, srcp, dstf, 2 * nth))) return rc;
    AmdThDivArgs da;
    memset(&da, 0, sizeof(da));
    for (int n = 0; n < nth; ++n) {
      da.fx[n] = L.fxf[n]; da.fz[n] = L.fzf[n]; da.cfth[n] = cf_out[3 + n];
      da.jst[n] = ctx->jst[n]; da.jet[n] = ctx->jet[n];
    }
    da.kx = ctx->d_kx; da.kz = ctx->d_kz; da.dlyf = L.d_sclf; da.g = fg; da.nth = nth;
    Prof pr(ctx, K_OTHER);
    k_amd_th_div<<<grid1d(ftot), 256, 0, ctx->stream>>>(da);
  } else if (nth > 0) {
    ThGradArgs ga;
    memset(&ga, 0, sizeof(ga));
    for (int n = 0; n < nth; ++n) { ga.cth[n] = ctx->st[c][4 + n]; ga.gx[n] = L.thg[2 * n]; ga.gz[n] = L.thg[2 * n + 1]; }
    ga.kx = ctx->d_kx; ga.kz = ctx->d_kz; ga.g = fg; ga.nth = nth;
    { Prof pr(ctx, K_OTHER); k_th_grad<<<grid1d(ftot), 256, 0, ctx->stream>>>(ga); }
    if ((rc = ifft_to<P>(ctx, L.thg, L.thp, 2 * nth))) return rc;
    {
      ScaleArgs<P> sa;
      memset(&sa, 0, sizeof(sa));
      for (int q = 0; q < 2 * nth; ++q) sa.f[q] = PP(L.thp[q]);
      sa.nfield = 2 * nth;
      sa.w = PP(L.nu_t);                                   // kappa_t = nu_t (:1130-1140)
      sa.ps = (size_t)ctx->nz * ctx->nx;
      sa.nyp = ctx->ny;
      Prof pr(ctx, K_OTHER);
      k_scale_by<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(sa);
    }
    if ((rc = fft_from<P>(ctx, L.thp, L.thg, 2 * nth))) return rc;
    ThDivArgs ta;
    memset(&ta, 0, sizeof(ta));
    for (int n = 0; n < nth; ++n) {
      ta.fx[n] = L.thg[2 * n]; ta.fz[n] = L.thg[2 * n + 1]; ta.cfth[n] = cf_out[3 + n];
      ta.jst[n] = ctx->jst[n]; ta.jet[n] = ctx->jet[n];
    }
    ta.kx = ctx->d_kx; ta.kz = ctx->d_kz; ta.g = fg; ta.nth = nth;
    Prof pr(ctx, K_OTHER);
    k_th_div<<<grid1d(ftot), 256, 0, ctx->stream>>>(ta);
  }
  // 8. nonlinear terms (as the DNS step), cf -= NL, cr += beta h cf
  if ((rc = spectral_nl<P>(ctx))) return rc;
  {
    CfFinishArgs fa;
    memset(&fa, 0, sizeof(fa));
    for (int f = 0; f < nf; ++f) { fa.cf[f] = cf_out[f]; fa.cr[f] = L.cr[f]; fa.nl[f] = ctx->nl[f]; }
    fa.lo[0] = fa.lo[2] = ctx->jstart; fa.hi[0] = fa.hi[2] = ctx->jend;
    fa.lo[1] = 2; fa.hi[1] = ctx->ny;
    for (int n = 0; n < nth; ++n) { fa.lo[3 + n] = ctx->jst[n]; fa.hi[3 + n] = ctx->jet[n]; }
    fa.nf = nf; fa.temp5 = a.temp5; fa.g = fg;
    fa.nl_fp32 = sizeof(P) == 4;
    Prof pr(ctx, K_OTHER);
    k_cf_finish<<<grid1d(ftot), 256, 0, ctx->stream>>>(fa);
  }
  // 9. r = IFFT(cr); CN in y per physical column; 10. u, th back to Fourier
  if ((rc = ifft_batch(ctx, L.cr, L.r, nf))) return rc;
  // the solve runs in FP64: with the FP32 model, the post-wall-update state
  // is transformed once more in FP64 for it
  double* u64[3 + DIABLO_MAX_TH];
  if (sizeof(P) == 8) {
    for (int f = 0; f < nf; ++f) u64[f] = reinterpret_cast<double*>(up[f]);
  } else {
    const double2* src[3 + DIABLO_MAX_TH];
    for (int f = 0; f < nf; ++f) { src[f] = ctx->st[c][f < 3 ? f : f + 1]; u64[f] = L.u64[f]; }
    if ((rc = ifft_batch(ctx, src, u64, nf))) return rc;
  }
  {
    PhysSolveArgs<P> sa;
    memset(&sa, 0, sizeof(sa));
    for (int f = 0; f < nf; ++f) { sa.r[f] = L.r[f]; sa.u[f] = u64[f]; }
    sa.nu_t = PP(L.nu_t);
    for (int n = 0; n < nth; ++n) sa.kap[n] = PP(model == 5 ? L.kap[n] : L.nu_t);
    sa.dy = ctx->d_dy; sa.dyf = ctx->d_dyf; sa.idy = L.d_idy; sa.idyf = L.d_idyf;
    sa.nf = nf; sa.nth = nth; sa.n = ctx->nyp2; sa.nyp = ctx->ny; sa.cols = ctx->nz * ctx->nx;
    sa.temp1 = a.temp1; sa.temp2 = a.temp2; sa.nu_v = a.nu_v;
    sa.jstart = ctx->jstart; sa.jend = ctx->jend;
    for (int n = 0; n < nth; ++n) {
      sa.jst[n] = ctx->jst[n]; sa.jet[n] = ctx->jet[n]; sa.pr[n] = ctx->p.pr[n];
      sa.thbc[n][0] = a.thbc[n][0]; sa.thbc[n][1] = a.thbc[n][1];
      sa.thc1[n][0] = a.thc1[n][0]; sa.thc1[n][1] = a.thc1[n][1];
    }
    for (int i = 0; i < 2; ++i) {
      sa.ubc[i] = a.ubc[i]; sa.vbc[i] = a.vbc[i]; sa.wbc[i] = a.wbc[i];
      sa.uc1[i] = a.uc1[i]; sa.vc1[i] = a.vc1[i]; sa.wc1[i] = a.wc1[i];
    }
    // one warp per (field, column); PS_W adjacent columns per block through
    // shared-memory tiles when a field's columns split evenly into them
    const size_t threads = (size_t)nf * sa.cols * 32;
    const bool tiled = sa.cols % PS_W == 0;
    const int tpb = tiled ? 32 * PS_W : 128;
    const unsigned blocks = (unsigned)((threads + tpb - 1) / tpb);
    const int tsm = tiled ? 3 * sa.n * PS_W * (int)sizeof(double) : 0;
    Prof pr(ctx, K_SOLVE);
    switch (std::max(3, (sa.n + 31) / 32)) {
#define X(r)                                                                                            \
  case r:                                                                                               \
    if (tiled) {                                                                                        \
      if (tsm > 48 * 1024)                                                                              \
        CK(cudaFuncSetAttribute(k_phys_solve<P, r, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, tsm)); \
      k_phys_solve<P, r, true><<<blocks, tpb, tsm, ctx->stream>>>(sa);                                  \
    } else {                                                                                            \
      k_phys_solve<P, r, false><<<blocks, tpb, 0, ctx->stream>>>(sa);                                   \
    }                                                                                                   \
    break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: return DIABLO_ERR_SIZE;
    }
  }
  // variable dt: courant on the solved physical velocities (for/channel.f90:885-888)
  if (courant_due(ctx, rk)) {
    if ((rc = ensure_cfl(ctx)) || (rc = courant_phys(ctx, u64))) return rc;
  }
  {
    double2* dst[3 + DIABLO_MAX_TH];
    for (int f = 0; f < nf; ++f) dst[f] = ctx->st[nx_][f < 3 ? f : f + 1];
    if ((rc = fft_batch(ctx, u64, dst, nf))) return rc;
  }
  // 11. projection and pressure update on the new state (for/channel.f90:901-911)
  {
    const int R = rows_per_lane(ctx->nyp2);
    const int warps = 4;
    dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
    Prof pr(ctx, K_OTHER);
    switch (R) {
#define X(r) case r: k_project<r><<<grd, blk, 0, ctx->stream>>>(a); break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: return DIABLO_ERR_SIZE;
    }
  }
  CK(cudaGetLastError());
  ctx->cur = nx_;
  if (rk < 3) ctx->cf_cur = 1 - ctx->cf_cur;
  return 0;
}

static int ensure_dyn(diablo_ctx* ctx) {
  diablo_ctx::Les& L = ctx->les;
  if (L.dyn_ready) return 0;
  const size_t ptot = phys_elems(ctx), ftot = four_elems(ctx);
  int rc;
  for (int q = 0; q < DYN_NF; ++q) {
    if ((rc = dev_alloc(ctx, (void**)&L.dp[q], ptot * sizeof(double)))) return rc;
    if ((rc = dev_alloc(ctx, (void**)&L.df[q], ftot * sizeof(double2)))) return rc;
  }
  if ((rc = dev_alloc(ctx, (void**)&L.dsums, (size_t)ctx->nyp2 * DYN_MAX_SLICES * 12 * sizeof(double))))
    return rc;
  L.dyn_ready = 1;
  return 0;
}

// Dynamic Smagorinsky coefficient C(y) into les.d_cf (GYF) and les.d_cg (GY):
// build the 21 Germano/Lilly inputs, test-filter them in Fourier space,
// contract and average over x-z planes.  Needs les.Sp (raw strain), les.sf
// and the physical velocities in ctx->phys.
template <typename P>
static int dynamic_coefficient(diablo_ctx* ctx) {
  auto PP = [](double* q) { return reinterpret_cast<P*>(q); };
  diablo_ctx::Les& L = ctx->les;
  int rc;
  const size_t ptot = phys_elems(ctx), ftot = four_elems(ctx);
  if ((rc = ensure_dyn(ctx))) return rc;
  const size_t ps = (size_t)ctx->nz * ctx->nx;
  {
    DynPrepArgs<P> pa;
    for (int q = 0; q < 3; ++q) pa.u[q] = (const P*)ctx->phys[q];
    for (int q = 0; q < 6; ++q) pa.S[q] = PP(L.Sp[q]);
    pa.sf = PP(L.sf);
    for (int q = 0; q < DYN_NF; ++q) pa.out[q] = PP(L.dp[q]);
    pa.nyp = ctx->ny;
    pa.ps = ps;
    Prof pr(ctx, K_OTHER);
    k_dyn_prep<P><<<grid1d(ptot), 256, 0, ctx->stream>>>(pa);
  }
  if ((rc = fft_from<P>(ctx, L.dp, L.df, DYN_NF))) return rc;
  const FGeom fg{ctx->ny, ctx->nyp2, ctx->nkx1, ctx->nk2, ctx->kp, (size_t)ctx->nkx1 * ctx->kp};
  for (int b = 0; b < DYN_NF; b += NF_MAX) {
    MaskArgs ma;
    memset(&ma, 0, sizeof(ma));
    ma.nfield = DYN_NF - b < NF_MAX ? DYN_NF - b : NF_MAX;
    for (int q = 0; q < ma.nfield; ++q) ma.f[q] = L.df[b + q];
    ma.mx = ctx->nkx / 2;
    ma.mz = ctx->nkz / 2;
    ma.nkz = ctx->nkz;
    ma.g = fg;
    Prof pr(ctx, K_OTHER);
    k_test_mask<<<grid1d(ftot), 256, 0, ctx->stream>>>(ma);
  }
  if ((rc = ifft_to<P>(ctx, L.df, L.dp, DYN_NF))) return rc;
  int nslice_dyn = 1;
  {
    DynContractArgs<P> ca;
    for (int q = 0; q < DYN_NF; ++q) ca.F[q] = PP(L.dp[q]);
    for (int q = 0; q < 3; ++q) ca.u[q] = (const P*)ctx->phys[q];
    ca.d2f = L.d_d2f;
    ca.sums = L.dsums;
    ca.nyp = ctx->ny;
    // about four blocks per SM over the planes
    ca.nslice = std::max(1, std::min({DYN_MAX_SLICES, (4 * 148 + ctx->ny - 1) / ctx->ny,
                                      (int)((ps + 255) / 256)}));
    ca.ps = ps;
    ca.ratio2 = 4.0;   // (2 Delta / Delta)^2
    Prof pr(ctx, K_OTHER);
    k_dyn_contract<P><<<dim3(ca.nslice, ctx->ny), 256, 0, ctx->stream>>>(ca);
    nslice_dyn = ca.nslice;
  }
  {
    Prof pr(ctx, K_OTHER);
    k_dyn_coef<<<(ctx->nyp2 + 127) / 128, 128, 0, ctx->stream>>>(L.dsums, ctx->d_dy, ctx->d_dyf, L.d_cf, L.d_cg,
                                                                  ctx->ny, nslice_dyn, (double)ps);
  }
  CK(cudaGetLastError());
  return 0;
}

// courant (for/advance.f90:47-158) from the velocities u (physical FP64,
// planes 1..Ny): the new delta_t and RK coefficients for the steps that follow.
static int ensure_cfl(diablo_ctx* ctx) {
  if (ctx->d_cfl) return 0;
  int rc;
  for (int q = 0; q < 3; ++q) {
    if ((rc = dev_alloc(ctx, (void**)&ctx->ustar[q], four_elems(ctx) * sizeof(double2)))) return rc;
    if ((rc = dev_alloc(ctx, (void**)&ctx->cfl_phys[q], phys_elems(ctx) * sizeof(double)))) return rc;
  }
  return dev_alloc(ctx, (void**)&ctx->d_cfl, (size_t)5 * ctx->nyp2 * sizeof(double));
}

static int courant_phys(diablo_ctx* ctx, const double* const* u) {
  const diablo_params& p = ctx->p;
  const size_t ps = (size_t)ctx->nz * ctx->nx;
  {
    Prof pr(ctx, K_OTHER);
    k_plane_range<<<ctx->ny, 256, 0, ctx->stream>>>(u[0], u[1], u[2], ctx->d_cfl, ps);
  }
  std::vector<double> mx((size_t)5 * ctx->nyp2);
  CK(cudaMemcpyAsync(mx.data(), ctx->d_cfl, mx.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  double dt = p.max_dt;
  if (ctx->ro_inv != 0.0) dt = fmin(dt, 2.0 * PI_REF / fabs(ctx->ro_inv / p.delta) / 20.0);
  for (int n = 0; n < ctx->nth; ++n) {
    const double nmax = sqrt(fabs(p.th_bc_ymin_c1[n]));
    // the literal 0.1 is default (single-precision) REAL in the reference
    if (nmax > 0) dt = fmin(dt, (double)0.1f * 2.0 * PI_REF / nmax);
  }
  const double cx = p.cfl * (p.lx / ctx->nx), cz = p.cfl * (p.lz / ctx->nz);
  // max |u - a| over plane j from its range
  auto dev = [&](int j, int q, double a) {   // q = 0: u1, q = 3: u3
    return fmax(mx[(size_t)j * 5 + q + 1] - a, a - mx[(size_t)j * 5 + q]);
  };
  if (p.flavor_front) {
    // 'Front': the thermal wind added to u1 and u3, rows jstart..jend, for
    // each scalar (for/advance.f90:76-89); no velocity limit without scalars
    const double rd = ctx->ro_inv / p.delta;
    for (int n = 0; n < ctx->nth; ++n)
      for (int j = ctx->jstart; j <= ctx->jend; ++j) {
        const double m1 = dev(j, 0, p.dthdz[n] * ctx->h_gyf[j] / rd);
        const double m3 = dev(j, 3, -(1.0 / rd) * p.dthdx[n] * (ctx->h_gyf[j] - 0.5 * p.ly));
        const double m2 = mx[(size_t)j * 5 + 2];
        if (m1 > 0) dt = fmin(dt, cx / m1);
        if (m2 > 0) dt = fmin(dt, p.cfl * ctx->h_dy[j] / m2);
        if (m3 > 0) dt = fmin(dt, cz / m3);
      }
  } else {
    double m1 = 0.0, m3 = 0.0, dty = INFINITY;
    for (int j = 1; j <= ctx->ny; ++j) {
      m1 = fmax(m1, dev(j, 0, 0.0));
      m3 = fmax(m3, dev(j, 3, 0.0));
      const double m2 = mx[(size_t)j * 5 + 2];
      if (m2 > 0) dty = fmin(dty, p.cfl * ctx->h_dy[j] / m2);
    }
    const double dtx = m1 > 0 ? cx / m1 : INFINITY, dtz = m3 > 0 ? cz / m3 : INFINITY;
    dt = fmin(fmin(dt, dtx), fmin(dty, dtz));
  }
  double nd;
  if (dt <= 0) nd = 0.00001;
  else if (dt >= 1000.) nd = 1000.;
  else nd = dt;
  if (nd != ctx->delta_t) {
    ctx->delta_t = nd;
    for (int r = 0; r < 3; ++r) ctx->h_bar[r] = H_FRAC[r] * nd;
    ctx->generation++;
    int rc = upload_coefficients(ctx);
    if (rc) return rc;
  }
  return 0;
}

static int courant_four(diablo_ctx* ctx, double2* const* cu) {
  int rc;
  if ((rc = ensure_xs64(ctx)) || (rc = ensure_cfl(ctx))) return rc;
  if ((rc = ifft_batch(ctx, cu, ctx->cfl_phys, 3))) return rc;
  return courant_phys(ctx, ctx->cfl_phys);
}

static bool courant_due(const diablo_ctx* ctx, int rk) {
  return ctx->p.variable_dt && rk == 3 && ctx->p.update_dt > 0 && ctx->time_step % ctx->p.update_dt == 0;
}

// poisson_p_chan (for/channel.f90:1026-1234): cp from the current velocity
// (and scalars), FP64; its work arrays live only for the call.
static int poisson_p(diablo_ctx* ctx) {
  int rc;
  if ((rc = ensure_xs64(ctx))) return rc;
  const size_t fe = four_elems(ctx) * sizeof(double2), pe = phys_elems(ctx) * sizeof(double);
  std::vector<void*> mine;
  auto alloc = [&](void** p, size_t b) -> int {
    int r = dev_alloc(ctx, p, b);
    if (!r) mine.push_back(*p);
    return r;
  };
  auto release = [&]() {
    cudaStreamSynchronize(ctx->stream);
    for (void* p : mine) {
      for (size_t i = 0; i < ctx->allocs.size(); ++i)
        if (ctx->allocs[i] == p) { ctx->allocs.erase(ctx->allocs.begin() + i); break; }
      cudaFree(p);
    }
  };
  double2* Gf[9];
  double* Gp[9];
  double2* Qf[6];
  double* Qp[6];
  rc = 0;
  for (int q = 0; q < 9 && !rc; ++q) rc = alloc((void**)&Gf[q], fe) || alloc((void**)&Gp[q], pe);
  for (int q = 0; q < 6 && !rc; ++q) rc = alloc((void**)&Qf[q], fe) || alloc((void**)&Qp[q], pe);
  if (rc) { release(); return DIABLO_ERR_NOMEM; }
  const FGeom fg{ctx->ny, ctx->nyp2, ctx->nkx1, ctx->nk2, ctx->kp, (size_t)ctx->nkx1 * ctx->kp};
  const int c = ctx->cur;
  {
    PpGradArgs a;
    for (int q = 0; q < 3; ++q) a.cu[q] = ctx->st[c][q];
    for (int q = 0; q < 9; ++q) a.G[q] = Gf[q];
    a.kx = ctx->d_kx; a.kz = ctx->d_kz; a.dyf = ctx->d_dyf; a.g = fg;
    Prof pr(ctx, K_OTHER);
    k_pp_grad<<<grid1d(four_elems(ctx)), 256, 0, ctx->stream>>>(a);
  }
  if (!rc) rc = ifft_batch(ctx, Gf, Gp, 9);
  if (!rc) {
    PpProdArgs a;
    for (int q = 0; q < 9; ++q) a.G[q] = Gp[q];
    for (int q = 0; q < 6; ++q) a.Q[q] = Qp[q];
    a.nyp = ctx->ny;
    a.ps = (size_t)ctx->nz * ctx->nx;
    Prof pr(ctx, K_OTHER);
    k_pp_prod<<<grid1d(phys_elems(ctx)), 256, 0, ctx->stream>>>(a);
  }
  if (!rc) rc = fft_batch(ctx, Qp, Qf, 6);
  if (!rc) {
    PpSolveArgs a;
    memset(&a, 0, sizeof(a));
    for (int q = 0; q < 6; ++q) a.Q[q] = Qf[q];
    for (int n = 0; n < ctx->nth; ++n) { a.cth[n] = ctx->st[c][4 + n]; a.ri[n] = ctx->p.ri[n]; }
    a.cp = ctx->st[c][3];
    a.kx = ctx->d_kx; a.kz = ctx->d_kz; a.met = ctx->d_met; a.gyf = ctx->d_gyf;
    a.nth = ctx->nth; a.n = ctx->nyp2; a.nyp = ctx->ny; a.nkx1 = ctx->nkx1; a.nk2 = ctx->nk2; a.kp = ctx->kp;
    a.ncol = ctx->nkx1 * ctx->nk2;
    const int warps = 4;
    dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
    Prof pr(ctx, K_OTHER);
    switch (rows_per_lane(ctx->nyp2)) {
#define X(r) case r: k_pp_solve<r><<<grd, blk, 0, ctx->stream>>>(a); break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: rc = DIABLO_ERR_SIZE;
    }
  }
  if (!rc && cudaGetLastError() != cudaSuccess) rc = DIABLO_ERR_CUDA;
  release();
  return rc;
}

static int substep(diablo_ctx* ctx, int rk) {
  if (les_active(ctx)) {
    const int m = ctx->p.les_model_type;
    if (m != 1 && m != 2 && m != 4 && m != 5) return DIABLO_ERR_UNSUPPORTED;
    // mixed precision: the LES model and its transforms in FP32, the
    // Crank-Nicolson solves, projection and state in FP64
    return ctx->precision == DIABLO_FP64 ? substep_les_t<double>(ctx, rk) : substep_les_t<float>(ctx, rk);
  }
  int rc = ensure_scratch(ctx);
  if (rc) return rc;
  update_transient(ctx);
  SolveArgs a;
  fill_solve_args(ctx, a, rk);
  // Mixed precision with the tiled kernel: the physical u1 of the FP32
  // products is u1 minus its mean profile U1(y).  The products with U1 are
  // linear in the state and are added in FP64: by the z-forward epilogue for
  // the u1 equation (whose NL is then FP64), by the column kernel for the
  // others.  This keeps the large mean-flow products out of FP32.
  const bool tiled = !a.front && !ctx->use_general_solver;
  const bool mean_split = ctx->precision == DIABLO_MIXED && tiled;
  rc = ctx->precision == DIABLO_FP64 ? substep_spectral<double>(ctx, 0u)
                                     : substep_spectral<float>(ctx, mean_split ? 0x1u : 0u);
  if (rc) return rc;
  const int c = ctx->cur, nx_ = 1 - c;
  for (int q = 0; q < 3; ++q) {
    a.cu_in[q] = ctx->st[c][q];
    a.cu_out[q] = ctx->st[nx_][q];
  }
  a.cp_in = ctx->st[c][3];
  a.cp_out = ctx->st[nx_][3];
  for (int n = 0; n < ctx->nth; ++n) {
    a.cth_in[n] = ctx->st[c][4 + n];
    a.cth_out[n] = ctx->st[nx_][4 + n];
  }
  for (int f = 0; f < ctx->nf; ++f) {
    a.cf_in[f] = ctx->cf[ctx->cf_cur][f];
    a.cf_out[f] = ctx->cf[1 - ctx->cf_cur][f];
    if (ctx->precision == DIABLO_FP64) a.nl64[f] = (const double2*)ctx->nl[f];
    else a.nl32[f] = (const float2*)ctx->nl[f];
  }
  a.store_cf = rk < 3 ? 1 : 0;
  // tiled kernel: the schedule of tiles this substep needs
  Solve2Args& A = ctx->solve2;
  A.s = a;
  A.kc = ctx->d_kc[rk - 1];
  A.met = ctx->d_met;
  A.fac = ctx->d_fac[rk - 1];
  A.mean_split = mean_split ? 1 : 0;
  A.prof = ctx->d_prof;
  A.nstep = 0;
  bool fits = true;
  auto add = [&](int op, int arg, double coef, const void* src, void* dst, const void* src2) {
    if (A.nstep >= T2_MAXSTEPS) { fits = false; return; }
    A.steps[A.nstep++] = TileStep{op, arg, coef, src, dst, src2};
  };
  const diablo_params& p = ctx->p;
  const int f32 = ctx->precision == DIABLO_FP64 ? 0 : 1;
  for (int comp = 0; comp < 3; comp += 2) {
    add(OP_OWN_U13, comp, 0, a.cu_in[comp], nullptr, nullptr);
    if (a.roinvd != 0.0) add(OP_ADD_CF, 0, comp == 0 ? a.roinvd : -a.roinvd, a.cu_in[2 - comp], nullptr, nullptr);
    const double g = comp == 0 ? p.grav_x : p.grav_z;
    if (g != 0.0)
      for (int n = 0; n < ctx->nth; ++n) add(OP_ADD_CF, 0, g, a.cth_in[n], nullptr, nullptr);
    add(OP_NL, (comp == 0 && mean_split) ? 0 : f32, 0, ctx->nl[comp], a.store_cf ? a.cf_out[comp] : nullptr,
        nullptr);
    if (rk > 1) add(OP_CFOLD, 0, 0, a.cf_in[comp], nullptr, nullptr);
    add(OP_SOLVE, comp, 0, a.cp_in, a.cu_out[comp], a.cu_in[comp]);   // tile: the pressure
  }
  add(OP_OWN_U2, 1, 0, a.cu_in[1], nullptr, nullptr);
  if (p.grav_y != 0.0)
    for (int n = 0; n < ctx->nth; ++n) add(OP_BUOY, 0, p.grav_y, a.cth_in[n], nullptr, nullptr);
  add(OP_NL, f32, 0, ctx->nl[1], a.store_cf ? a.cf_out[1] : nullptr, nullptr);
  if (rk > 1) add(OP_CFOLD, 0, 0, a.cf_in[1], nullptr, nullptr);
  add(OP_SOLVE, 1, 0, a.cp_in, a.cu_out[1], a.cu_in[1]);
  for (int n = 0; n < ctx->nth; ++n) {
    add(OP_OWN_TH, n, 0, a.cth_in[n], nullptr, nullptr);
    if (p.dthdx[n] != 0.0) add(OP_ADD_CF, 0, -p.dthdx[n], a.cu_in[0], nullptr, nullptr);
    if (p.dthdz[n] != 0.0) add(OP_ADD_CF, 0, -p.dthdz[n], a.cu_in[2], nullptr, nullptr);
    add(OP_NL, f32, 0, ctx->nl[3 + n], a.store_cf ? a.cf_out[3 + n] : nullptr, nullptr);
    if (rk > 1) add(OP_CFOLD, 0, 0, a.cf_in[3 + n], nullptr, nullptr);
    add(OP_SOLVE, 3 + n, 0, nullptr, a.cth_out[n], a.cth_in[n]);
  }
  add(OP_POISSON, 0, 0, nullptr, nullptr, nullptr);
  const bool cfl = courant_due(ctx, rk);
  if (cfl && (rc = ensure_cfl(ctx))) return rc;
  add(OP_PROJ, 0, 0, a.cu_out[0], a.cu_out[0], cfl ? ctx->ustar[0] : nullptr);
  add(OP_PROJ, 2, 0, a.cu_out[2], a.cu_out[2], cfl ? ctx->ustar[2] : nullptr);
  add(OP_PROJ, 1, 0, a.cu_out[1], a.cu_out[1], cfl ? ctx->ustar[1] : nullptr);
  add(OP_CP, 0, 0, a.cp_in, a.cp_out, nullptr);
  {
    Prof pr(ctx, K_SOLVE);
    // thermal-wind forcing (flavor 'Front') keeps the general kernel
    if (fits && tiled) rc = launch_tiles(A, ctx->stream);
    else if (mean_split) rc = DIABLO_ERR_UNSUPPORTED;
    else {
      if (cfl)
        for (int q = 0; q < 3; ++q) a.keep[q] = ctx->ustar[q];
      rc = launch_solve(a, false, ctx->stream);
    }
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  ctx->cur = nx_;
  if (a.store_cf) ctx->cf_cur = 1 - ctx->cf_cur;
  // variable dt: courant on the solved velocities (for/channel.f90:885-888)
  if (cfl) return courant_four(ctx, ctx->ustar);
  return 0;
}

// ==========================================================================
// C ABI
extern "C" {

int diablo_abi_version(void) { return DIABLO_ABI_VERSION; }

const char* diablo_status_string(int s) {
  switch (s) {
    case DIABLO_OK: return "ok";
    case DIABLO_ERR_ARG: return "invalid argument";
    case DIABLO_ERR_SIZE: return "unsupported grid size";
    case DIABLO_ERR_CUDA: return "CUDA runtime error";
    case DIABLO_ERR_NONFINITE: return "non-finite value in state";
    case DIABLO_ERR_TIMEOUT: return "bounded device wait timed out";
    case DIABLO_ERR_UNSUPPORTED: return "option not supported on the device";
    case DIABLO_ERR_STATE: return "state violates the layout contract";
    case DIABLO_ERR_NOMEM: return "device allocation failed";
    default: return "unknown status";
  }
}

static int validate(const diablo_params* p) {
  if (!p || p->struct_size != (int)sizeof(diablo_params)) return DIABLO_ERR_ARG;
  if (p->nx < 8 || (p->nx % 2) || p->ny < 4 || p->nz < 8) return DIABLO_ERR_SIZE;
  if (p->n_th < 0 || p->n_th > DIABLO_MAX_TH) return DIABLO_ERR_ARG;
  int a, b;
  if (!factor(p->nz, &a, &b) || !factor(p->nx / 2, &a, &b)) return DIABLO_ERR_SIZE;
  if ((p->ny + 2 + 31) / 32 > 17) return DIABLO_ERR_SIZE;
  if (!(p->re > 0) || !(p->delta_t > 0) || !(p->lx > 0) || !(p->lz > 0)) return DIABLO_ERR_ARG;
  if (p->precision != DIABLO_FP64 && p->precision != DIABLO_MIXED) return DIABLO_ERR_ARG;
  for (int n = 0; n < p->n_th; ++n)
    if (!(p->pr[n] > 0)) return DIABLO_ERR_ARG;
  return 0;
}

diablo_ctx* diablo_create(const diablo_params* p, const double* gy, int* status) {
  int dummy;
  if (!status) status = &dummy;
  *status = validate(p);
  if (*status) return nullptr;
  if (!gy) { *status = DIABLO_ERR_ARG; return nullptr; }
  diablo_ctx* ctx = new diablo_ctx();  // value-initialised: scalars and pointers are zero
  ctx->p = *p;
  ctx->scratch_prec = -1;
  ctx->nx = p->nx; ctx->ny = p->ny; ctx->nz = p->nz; ctx->nth = p->n_th;
  ctx->nf = 3 + p->n_th;
  ctx->nxp = p->nx / 2;
  ctx->M = p->nx / 2;
  ctx->nkx = p->nx / 3;
  ctx->nkz = p->nz / 3;
  ctx->nkx1 = ctx->nkx + 1;
  ctx->nk2 = 2 * ctx->nkz + 1;
  ctx->kp = ctx->nk2;
  ctx->nyp2 = p->ny + 2;
  ctx->g = Geom{ctx->nx, ctx->nz, ctx->nyp2, ctx->nkx1, ctx->nkz, ctx->nk2, ctx->kp};
  ctx->nu = 1.0 / p->re;
  ctx->ro_inv = isinf(p->ro) ? 0.0 : 1.0 / p->ro;
  ctx->jstart = p->u_bc_ymin == 1 ? 1 : 2;
  ctx->jend = p->ny;
  for (int n = 0; n < p->n_th; ++n) {
    ctx->jst[n] = p->th_bc_ymin[n] == 1 ? 1 : 2;
    ctx->jet[n] = p->ny;
  }
  ctx->delta_t = p->delta_t;
  for (int r = 0; r < 3; ++r) ctx->h_bar[r] = H_FRAC[r] * p->delta_t;
  ctx->w_top_transient = p->w_bc_ymax_c1;
  ctx->precision = p->precision;
  {
    const char* e = getenv("DIABLO_GENERAL_SOLVER");
    ctx->use_general_solver = (e && e[0] == '1') ? 1 : 0;
  }
  int rc = 0;
#define FAIL(code) do { *status = (code); diablo_destroy(ctx); return nullptr; } while (0)
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    FAIL(DIABLO_ERR_CUDA);
  }
  ctx->stream = ctx->own_stream;
  // grid metrics exactly as ReadGridHDF5 / create_grid_chan (for/domain.f90:230-248,501-527)
  const int ny = p->ny;
  std::vector<double> hgy(ny + 2, 0.0), hgyf(ny + 2, 0.0), hdy(ny + 2, 0.0), hdyf(ny + 2, 0.0);
  for (int j = 1; j <= ny + 1; ++j) hgy[j] = gy[j - 1];
  for (int j = 1; j <= ny; ++j) hgyf[j] = 0.5 * (hgy[j] + hgy[j + 1]);
  hgyf[0] = 2.0 * hgyf[1] - hgyf[2];
  hgyf[ny + 1] = 2.0 * hgyf[ny] - hgyf[ny - 1];
  for (int j = 1; j <= ny + 1; ++j) hdy[j] = hgyf[j] - hgyf[j - 1];
  for (int j = 1; j <= ny; ++j) hdyf[j] = hgy[j + 1] - hgy[j];
  hdyf[0] = hdyf[1];
  hdyf[ny + 1] = hdyf[ny];
  for (int j = 1; j <= ny + 1; ++j)
    if (!(hdy[j] > 0) || (j <= ny && !(hdyf[j] > 0))) FAIL(DIABLO_ERR_ARG);
  ctx->h_gy = hgy; ctx->h_gyf = hgyf; ctx->h_dy = hdy; ctx->h_dyf = hdyf;
  // wavenumbers (init_fft, for/fft.f90:213-230), with the reference's float32 pi
  std::vector<double> hkx(ctx->nkx1), hkz(ctx->nk2);
  for (int i = 0; i < ctx->nkx1; ++i) hkx[i] = i * (2. * PI_REF) / p->lx;
  for (int k = 0; k <= ctx->nkz; ++k) hkz[k] = k * (2. * PI_REF) / p->lz;
  for (int k = 1; k <= ctx->nkz; ++k) hkz[2 * ctx->nkz + 1 - k] = -k * (2. * PI_REF) / p->lz;
  ctx->h_kx = hkx;
  auto up = [&](double** d, const std::vector<double>& h) -> int {
    int r = dev_alloc(ctx, (void**)d, h.size() * sizeof(double));
    if (r) return r;
    if (cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess) return DIABLO_ERR_CUDA;
    return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? 0 : DIABLO_ERR_CUDA;
  };
  if ((rc = up(&ctx->d_gy, hgy)) || (rc = up(&ctx->d_gyf, hgyf)) || (rc = up(&ctx->d_dy, hdy)) ||
      (rc = up(&ctx->d_dyf, hdyf)) || (rc = up(&ctx->d_kx, hkx)) || (rc = up(&ctx->d_kz, hkz)))
    FAIL(rc);
  if ((rc = upload_tw(ctx, ctx->nz, ctx->nz, &ctx->tz64, &ctx->tz32)) ||
      (rc = upload_tw(ctx, ctx->M, ctx->M, &ctx->tm64, &ctx->tm32)) ||
      (rc = upload_tw(ctx, ctx->nx, ctx->M + 1, &ctx->tx64, &ctx->tx32)))
    FAIL(rc);
  for (int b = 0; b < 2; ++b) {
    for (int f = 0; f < 4 + ctx->nth; ++f)
      if ((rc = dev_alloc(ctx, (void**)&ctx->st[b][f], four_elems(ctx) * sizeof(double2)))) FAIL(rc);
    for (int f = 0; f < ctx->nf; ++f)
      if ((rc = dev_alloc(ctx, (void**)&ctx->cf[b][f], four_elems(ctx) * sizeof(double2)))) FAIL(rc);
  }
  if ((rc = dev_alloc(ctx, (void**)&ctx->d_flag, sizeof(int)))) FAIL(rc);
  if ((rc = upload_coefficients(ctx))) FAIL(rc);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) FAIL(DIABLO_ERR_CUDA);
#undef FAIL
  *status = 0;
  return ctx;
}

int diablo_destroy(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (void* p : ctx->allocs) cudaFree(p);
  for (auto& t : ctx->timed) { cudaEventDestroy(t.a); cudaEventDestroy(t.b); }
  for (auto e : ctx->pool) cudaEventDestroy(e);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  cudaGetLastError();
  delete ctx;
  return 0;
}

static int field_index(const diablo_ctx* ctx, int field) {
  if (field >= DIABLO_U1 && field <= DIABLO_P) return field;
  if (field >= DIABLO_TH && field < DIABLO_TH + ctx->nth) return field;
  return -1;
}

// ---- boundary copies --------------------------------------------------------
// Host buffers move only their significant box, one copy per field: Fourier
// i < Nxp, k <= 2Nkz (uploads also carry each row's pad entry, which is not
// read); physical i < Nx, k < Nz.
static cudaMemcpy3DParms box_parms(void* dst, size_t dpitch, size_t dheight, const void* src,
                                   size_t spitch, size_t sheight, size_t wbytes, size_t rows,
                                   size_t planes, cudaMemcpyKind kind) {
  cudaMemcpy3DParms m;
  memset(&m, 0, sizeof(m));
  m.srcPtr = make_cudaPitchedPtr(const_cast<void*>(src), spitch, wbytes, sheight);
  m.dstPtr = make_cudaPitchedPtr(dst, dpitch, wbytes, dheight);
  m.extent = make_cudaExtent(wbytes, rows, planes);
  m.kind = kind;
  return m;
}

// significant Fourier box of `buf` -> internal layout `dst`
static int four_in(diablo_ctx* ctx, const double* buf, double2* dst, bool check) {
  const double2* src;
  int rp, rows;
  if (is_device_ptr(buf)) {
    src = (const double2*)buf;
    rp = ctx->nxp + 1;
    rows = ctx->nz + 2;
  } else {
    // rows k = 0..2Nkz of a plane are contiguous in the host array (with the
    // pad entry i = Nxp of each row): one 2D copy of nyp2 such blocks.  A 3D
    // copy of the Nxp-wide box instead ran at a third of the link's H2D rate.
    const size_t rowb = (size_t)(ctx->nxp + 1) * sizeof(double2);
    CK(cudaMemcpy2DAsync(ctx->b_ref, rowb * ctx->nk2, buf, rowb * (ctx->nz + 2), rowb * ctx->nk2,
                         ctx->nyp2, cudaMemcpyHostToDevice, ctx->stream));
    src = (const double2*)ctx->b_ref;
    rp = ctx->nxp + 1;
    rows = ctx->nk2;
  }
  CK(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  size_t tot = (size_t)ctx->nyp2 * ctx->nk2 * ctx->nxp;
  {
    Prof pr(ctx, K_OTHER);
    k_ref_to_four<<<grid1d(tot), 256, 0, ctx->stream>>>(src, dst, ctx->g, ctx->nxp, rp, rows,
                                                         ctx->d_flag);
  }
  if (check) {
    int bad = 0;
    CK(cudaMemcpyAsync(&bad, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (bad) return DIABLO_ERR_STATE;
  }
  return 0;
}

// internal Fourier `src` -> significant box of `buf`
static int four_out(diablo_ctx* ctx, const double2* src, double* buf) {
  const bool dev = is_device_ptr(buf);
  double2* dst = dev ? (double2*)buf : (double2*)ctx->b_ref;
  int rp = dev ? ctx->nxp + 1 : ctx->nxp, rows = dev ? ctx->nz + 2 : ctx->nk2;
  size_t tot = (size_t)ctx->nyp2 * ctx->nk2 * ctx->nxp;
  {
    Prof pr(ctx, K_OTHER);
    k_four_to_ref<<<grid1d(tot), 256, 0, ctx->stream>>>(src, dst, ctx->g, ctx->nxp, rp, rows);
  }
  if (!dev) {
    cudaMemcpy3DParms m = box_parms(buf, (ctx->nxp + 1) * sizeof(double2), ctx->nz + 2, ctx->b_ref,
                                    ctx->nxp * sizeof(double2), ctx->nk2, ctx->nxp * sizeof(double2),
                                    ctx->nk2, ctx->nyp2, cudaMemcpyDeviceToHost);
    CK(cudaMemcpy3DAsync(&m, ctx->stream));
  }
  return 0;
}

// significant physical box of `buf` -> internal physical `dst`
static int phys_in(diablo_ctx* ctx, const double* buf, double* dst) {
  const double* src = buf;
  int rows = ctx->nz + 2;
  if (!is_device_ptr(buf)) {
    // rows k < Nz of a plane are contiguous in the host array: one 2D copy of
    // those blocks (a 3D copy of the Nx-wide box is several times slower H2D)
    const size_t rowb = (size_t)(ctx->nx + 2) * sizeof(double);
    CK(cudaMemcpy2DAsync(ctx->b_ref, rowb * ctx->nz, buf, rowb * (ctx->nz + 2), rowb * ctx->nz,
                         ctx->nyp2, cudaMemcpyHostToDevice, ctx->stream));
    src = ctx->b_ref;
    rows = ctx->nz;
  }
  Prof pr(ctx, K_OTHER);
  k_ref_to_phys<<<grid1d(phys_elems(ctx)), 256, 0, ctx->stream>>>(src, dst, ctx->nx, ctx->nz, ctx->nyp2,
                                                                  rows);
  return 0;
}

// internal physical `src` -> significant box of `buf`
static int phys_out(diablo_ctx* ctx, const double* src, double* buf) {
  if (is_device_ptr(buf)) {
    Prof pr(ctx, K_OTHER);
    k_phys_to_ref<<<grid1d(phys_elems(ctx)), 256, 0, ctx->stream>>>(src, buf, ctx->nx, ctx->nz,
                                                                    ctx->nyp2);
  } else {
    cudaMemcpy3DParms m = box_parms(buf, (ctx->nx + 2) * sizeof(double), ctx->nz + 2, src,
                                    ctx->nx * sizeof(double), ctx->nz, ctx->nx * sizeof(double),
                                    ctx->nz, ctx->nyp2, cudaMemcpyDeviceToHost);
    CK(cudaMemcpy3DAsync(&m, ctx->stream));
  }
  return 0;
}

int diablo_upload_state(diablo_ctx* ctx, int field, const double* buf, int layout) {
  if (!ctx || !buf) return DIABLO_ERR_ARG;
  int fi = field_index(ctx, field);
  if (fi < 0) return DIABLO_ERR_ARG;
  int rc = ensure_bscratch(ctx);
  if (rc) return rc;
  double2* dst = ctx->st[ctx->cur][fi];
  if (layout == DIABLO_LAYOUT_FOURIER) {
    if ((rc = four_in(ctx, buf, dst, true))) return rc;
  } else if (layout == DIABLO_LAYOUT_PHYSICAL) {
    if ((rc = phys_in(ctx, buf, ctx->b_phys))) return rc;
    if ((rc = fwd_phys_to_four(ctx, ctx->b_phys, ctx->b_xs, dst))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
  } else {
    return DIABLO_ERR_ARG;
  }
  CK(cudaGetLastError());
  return 0;
}

int diablo_download_state(diablo_ctx* ctx, int field, double* buf, int layout) {
  if (!ctx || !buf) return DIABLO_ERR_ARG;
  int fi = field_index(ctx, field);
  if (fi < 0) return DIABLO_ERR_ARG;
  int rc = ensure_bscratch(ctx);
  if (rc) return rc;
  const double2* src = ctx->st[ctx->cur][fi];
  if (layout == DIABLO_LAYOUT_FOURIER) {
    if ((rc = four_out(ctx, src, buf))) return rc;
  } else if (layout == DIABLO_LAYOUT_PHYSICAL) {
    if ((rc = inv_four_to_phys(ctx, src, ctx->b_xs, ctx->b_phys))) return rc;
    if ((rc = phys_out(ctx, ctx->b_phys, buf))) return rc;
  } else {
    return DIABLO_ERR_ARG;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

int diablo_download_nu_t(diablo_ctx* ctx, double* buf) {
  if (!ctx || !buf) return DIABLO_ERR_ARG;
  int rc = ensure_bscratch(ctx);
  if (rc) return rc;
  const double* src = ctx->les.nu_t;
  if (!ctx->les.ready) {
    CK(cudaMemsetAsync(ctx->b_phys, 0, phys_elems(ctx) * sizeof(double), ctx->stream));
    src = ctx->b_phys;
  } else if (ctx->les.nu_t_fp32) {
    k_widen<<<grid1d(phys_elems(ctx)), 256, 0, ctx->stream>>>(reinterpret_cast<const float*>(ctx->les.nu_t),
                                                             ctx->b_phys, phys_elems(ctx));
    src = ctx->b_phys;
  }
  if ((rc = phys_out(ctx, src, buf))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

int diablo_fft_xz_to_fourier(diablo_ctx* ctx, const double* v, double* vv) {
  if (!ctx || !v || !vv) return DIABLO_ERR_ARG;
  int rc = ensure_bscratch(ctx);
  if (rc) return rc;
  if ((rc = phys_in(ctx, v, ctx->b_phys))) return rc;
  if ((rc = fwd_phys_to_four(ctx, ctx->b_phys, ctx->b_xs, ctx->b_four))) return rc;
  if ((rc = four_out(ctx, ctx->b_four, vv))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

int diablo_fft_xz_to_physical(diablo_ctx* ctx, double* vv, double* v) {
  if (!ctx || !v || !vv) return DIABLO_ERR_ARG;
  int rc = ensure_bscratch(ctx);
  if (rc) return rc;
  // modes above Nkx are zeroed by the reference before the x transform
  // (for/fft.f90:372-378), so they are not checked here
  if ((rc = four_in(ctx, vv, ctx->b_four, false))) return rc;
  if ((rc = inv_four_to_phys(ctx, ctx->b_four, ctx->b_xs, ctx->b_phys))) return rc;
  if ((rc = phys_out(ctx, ctx->b_phys, v))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

int diablo_rk_substep(diablo_ctx* ctx, int rk_step) {
  if (!ctx || rk_step < 1 || rk_step > 3) return DIABLO_ERR_ARG;
  return substep(ctx, rk_step);
}

static int filter_chan(diablo_ctx* ctx, int n) {
  if (!ctx->d_sigma) {
    const int nkx1 = ctx->nkx1, nk2 = ctx->nk2;
    std::vector<double> sg((size_t)nkx1 * nk2), kx(nkx1), kz(nk2);
    CK(cudaMemcpy(kx.data(), ctx->d_kx, nkx1 * sizeof(double), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(kz.data(), ctx->d_kz, nk2 * sizeof(double), cudaMemcpyDeviceToHost));
    const double fx = (double)(float)ctx->nx, fz = (double)(float)ctx->nz;
    for (int m = 0; m < nkx1; ++m)
      for (int q = 0; q < nk2; ++q) {
        const double s0 = 0.5 * (1.0 + cos(sqrt(pow(kx[m] * ctx->p.lx * 1.0 / fx, 2.0) +
                                                pow(kz[q] * ctx->p.lz * 1.0 / fz, 2.0))));
        sg[(size_t)m * nk2 + q] = pow(s0, 4.0) * (35.0 - 84.0 * s0 + 70.0 * pow(s0, 2.0) - 20.0 * pow(s0, 3.0));
      }
    int rc = dev_alloc(ctx, (void**)&ctx->d_sigma, sg.size() * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpyAsync(ctx->d_sigma, sg.data(), sg.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
  }
  const int j0 = ctx->jst[n], j1 = ctx->jet[n];
  const size_t tot = (size_t)(j1 - j0 + 1) * ctx->nkx1 * ctx->kp;
  Prof pr(ctx, K_OTHER);
  k_filter_th<<<grid1d(tot), 256, 0, ctx->stream>>>(ctx->st[ctx->cur][4 + n], ctx->d_sigma, j0, j1, ctx->nkx1,
                                                    ctx->nk2, ctx->kp);
  CK(cudaGetLastError());
  return 0;
}

// filter_scalars (for/advance.f90:161-173), after each step
static int filter_scalars(diablo_ctx* ctx) {
  for (int n = 0; n < ctx->nth; ++n)
    if (ctx->p.filter_th[n] && ctx->p.filter_int[n] > 0 && ctx->time_step % ctx->p.filter_int[n] == 0) {
      int rc = filter_chan(ctx, n);
      if (rc) return rc;
    }
  return 0;
}

int diablo_filter_chan(diablo_ctx* ctx, int n) {
  if (!ctx || n < 0 || n >= ctx->nth) return DIABLO_ERR_ARG;
  return filter_chan(ctx, n);
}

// ---------------------------------------------------------------------------
// Plane statistics (save_stats_chan, for/statistics.f90:44-712)

int diablo_stats_size(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  return ctx->ny * (DIABLO_STAT_NPROF + ctx->nth * DIABLO_STAT_NTHPROF) + ctx->nx / 2 +
         (ctx->nth > 0 ? (2 + ZS_N) * ctx->nx : 0) + DIABLO_STAT_NSCALAR;
}

int diablo_stats(diablo_ctx* ctx, int homogeneous_x, double* out, int len) {
  if (!ctx || !out) return DIABLO_ERR_ARG;
  if (len < diablo_stats_size(ctx)) return DIABLO_ERR_ARG;
  const diablo_params& p = ctx->p;
  int rc;
  // apply_BC_vel_mpi_post / apply_BC_th_mpi_post on the state (:63-64)
  if ((rc = bc_post(ctx, 1, 1))) return rc;
  const int ny = ctx->ny, nyp2 = ctx->nyp2, nth = ctx->nth, nkx1 = ctx->nkx1, nx = ctx->nx;
  const int nmodes = nkx1 * ctx->nk2;
  const size_t pn = (size_t)ctx->nz * nx;
  // x-inhomogeneous branch (IC types 5-8): z-line means when Nz > 1 (:749),
  // epsilon's x derivatives without the kz = 0 row (:862-866), compute_MKE_diss
  const bool nonhom = !homogeneous_x;
  const bool zline = nonhom && ctx->nz > 1;
  int dev = 0, nsm = 148;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  // about four blocks per SM over all planes
  int nslice = (4 * nsm + nyp2 - 1) / nyp2;
  nslice = std::max(1, std::min(nslice, (nmodes + STAT_THREADS - 1) / STAT_THREADS));
  int lslice = (4 * nsm + nyp2 - 1) / nyp2;
  lslice = std::max(1, std::min<int>(lslice, (int)((pn + STAT_THREADS - 1) / STAT_THREADS)));
  // sub-buffer sizes in doubles, each rounded up to an even count so that
  // every sub-buffer (the double2 rows among them) starts 16-byte aligned
  auto even = [](size_t v) { return (v + 1) & ~(size_t)1; };
  const size_t n_part = even((size_t)nyp2 * nslice * STAT_NQ), n_means = even((size_t)nyp2 * (4 + nth));
  const size_t n_spec = even((size_t)nyp2 * nkx1), n_les = even((size_t)nyp2 * lslice * 2);
  const size_t n_rows = (size_t)nyp2 * (3 + nth) * nkx1 * 2, n_bpe = even((size_t)nx);
  const size_t n_zs = even((size_t)(1 + ZS_N) * nx);
  const size_t n_xy = (size_t)XY_N * nyp2 * nx;
  const size_t total = n_part + n_means + n_spec + n_les + n_rows + n_bpe + n_zs + n_xy;
  if (ctx->stats_doubles < total) {
    if ((rc = dev_alloc(ctx, (void**)&ctx->d_stats, total * sizeof(double)))) return rc;
    ctx->stats_doubles = total;
  }
  double* d_part = ctx->d_stats;
  double* d_means = d_part + n_part;
  double* d_spec = d_means + n_means;
  double* d_les = d_spec + n_spec;
  double* d_rows = d_les + n_les;
  double* d_bpe = d_rows + n_rows;
  double* d_zs = d_bpe + n_bpe;
  double* d_xy = d_zs + n_zs;
  CK(cudaMemsetAsync(ctx->d_stats, 0, total * sizeof(double), ctx->stream));
  const double d0 = nth > 0 ? p.dthdx[0] : 0.0;
  // (1/(Ro_inv/delta)) dTHdX(1), the thermal-wind shear; 0 without a background gradient
  const double tws = d0 == 0.0 ? 0.0 : (1.0 / (ctx->ro_inv / p.delta)) * d0;
  {
    StatsArgs a;
    memset(&a, 0, sizeof(a));
    for (int q = 0; q < 3; ++q) a.cu[q] = ctx->st[ctx->cur][q];
    for (int n = 0; n < nth; ++n) {
      a.cth[n] = ctx->st[ctx->cur][4 + n];
      a.dthdx[n] = p.dthdx[n];
      a.dthdz[n] = p.dthdz[n];
    }
    a.cp = ctx->st[ctx->cur][3];
    a.kx = ctx->d_kx;
    a.kz = ctx->d_kz;
    a.dy = ctx->d_dy;
    a.dyf = ctx->d_dyf;
    a.gy = ctx->d_gy;
    a.gyf = ctx->d_gyf;
    a.tws = tws;
    a.nth = nth;
    a.nyp = ny;
    a.nkx1 = nkx1;
    a.nk2 = ctx->nk2;
    a.kp = ctx->kp;
    a.nslice = nslice;
    a.rowmean = zline ? 1 : 0;
    a.kstart1 = nonhom ? 1 : 0;
    a.ps = (size_t)nkx1 * ctx->kp;
    a.part = d_part;
    a.means = d_means;
    a.spec = d_spec;
    a.rows = reinterpret_cast<double2*>(d_rows);
    Prof pr(ctx, K_OTHER);
    const dim3 grid(nslice, nyp2);
    if (nth == 0) k_stats_modes<0><<<grid, STAT_THREADS, 0, ctx->stream>>>(a);
    else if (nth == 1) k_stats_modes<1><<<grid, STAT_THREADS, 0, ctx->stream>>>(a);
    else if (nth == 2) k_stats_modes<2><<<grid, STAT_THREADS, 0, ctx->stream>>>(a);
    else if (nth <= 4) k_stats_modes<4><<<grid, STAT_THREADS, 0, ctx->stream>>>(a);
    else k_stats_modes<DIABLO_MAX_TH><<<grid, STAT_THREADS, 0, ctx->stream>>>(a);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  const bool les = p.use_les && ctx->les.ready;
  double* uphys[3] = {nullptr, nullptr, nullptr};
  if (les || zline || nth > 0) {
    // physical u1, u2, u3 (all planes): LES work arrays when present, else
    // three buffers kept for the statistics
    if (les) {
      for (int q = 0; q < 3; ++q) uphys[q] = ctx->les.r[q];
      const double2* four[3] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2]};
      if ((rc = ifft_batch(ctx, four, uphys, 3))) return rc;
    } else {
      if ((rc = ensure_bscratch(ctx))) return rc;
      for (int q = 0; q < 3; ++q) {
        if (!ctx->stats_phys[q] &&
            (rc = dev_alloc(ctx, (void**)&ctx->stats_phys[q], phys_elems(ctx) * sizeof(double))))
          return rc;
        uphys[q] = ctx->stats_phys[q];
        if ((rc = inv_four_to_phys(ctx, ctx->st[ctx->cur][q], ctx->b_xs, uphys[q]))) return rc;
      }
    }
  }
  if (les) {
    diablo_ctx::Les& L = ctx->les;
    const double* nt = L.nu_t;
    if (L.nu_t_fp32) {
      if ((rc = ensure_bscratch(ctx))) return rc;
      k_widen<<<grid1d(phys_elems(ctx)), 256, 0, ctx->stream>>>(reinterpret_cast<const float*>(L.nu_t),
                                                               ctx->b_phys, phys_elems(ctx));
      ctx->launches++;
      nt = ctx->b_phys;
    }
    StatsLesArgs b;
    memset(&b, 0, sizeof(b));
    for (int q = 0; q < 3; ++q) b.u[q] = uphys[q];
    b.nu_t = nt;
    b.dy = ctx->d_dy;
    b.dyf = ctx->d_dyf;
    b.nyp = ny;
    b.nslice = lslice;
    b.pn = pn;
    b.part = d_les;
    Prof pr(ctx, K_OTHER);
    k_stats_les<<<dim3(lslice, nyp2), STAT_THREADS, 0, ctx->stream>>>(b);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  if (zline) {
    StatsXyArgs c;
    memset(&c, 0, sizeof(c));
    for (int q = 0; q < 3; ++q) c.u[q] = uphys[q];
    c.dy = ctx->d_dy;
    c.dyf = ctx->d_dyf;
    c.nx = nx;
    c.nz = ctx->nz;
    c.nyp = ny;
    c.out = d_xy;
    Prof pr(ctx, K_OTHER);
    k_stats_xy<<<dim3((nx + 127) / 128, nyp2), 128, 0, ctx->stream>>>(c);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  // compute_BPE on th_1 (:1755-1876, called for n = 1): its physical FP64 field
  // in b_phys, after every earlier reader of b_phys in stream order
  const int nbin = nx;
  double bthmin = 0.0, bthmax = 0.0, bdth = 0.0, broden = 0.0;
  if (nth > 0) {
    if ((rc = ensure_bscratch(ctx))) return rc;
    if ((rc = inv_four_to_phys(ctx, ctx->st[ctx->cur][4], ctx->b_xs, ctx->b_phys))) return rc;
    StatsBpeArgs e;
    memset(&e, 0, sizeof(e));
    e.th = ctx->b_phys;
    e.dyf = ctx->d_dyf;
    e.dthdx = p.dthdx[0];
    e.lx = p.lx;
    e.even = nonhom ? 1 : 0;
    if (nonhom) {
      // the literal 1.1 is single precision in the reference
      bthmin = -p.dthdx[0] * 0.5 * p.lx * (double)1.1f;
      bthmax = p.dthdx[0] * 0.5 * p.lx * (double)1.1f;
      bdth = (bthmax - bthmin) / nbin + 1.e-14;
    } else {
      bthmin = -ctx->ro_inv;
      bthmax = ctx->ro_inv;
      broden = ctx->ro_inv + 1.e-14;
    }
    e.thmin = bthmin;
    e.thmax = bthmax;
    e.dth = bdth;
    e.roden = broden;
    e.pi_ref = PI_REF;
    e.nx = nx;
    e.nz = ctx->nz;
    e.jlo = ctx->jst[0];
    e.jhi = ctx->jet[0];
    e.nbin = nbin;
    e.pdf = d_bpe;
    Prof pr(ctx, K_OTHER);
    k_stats_bpe<<<4 * nsm, 256, nbin * sizeof(double), ctx->stream>>>(e);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  if (nth > 0) {
    // Bin_Ystar_and_Write (:1877-1972) of six pointwise fields: their spectral
    // derivatives in physical space first, one field at a time through b_four
    const size_t pe = phys_elems(ctx) * sizeof(double), ftot = four_elems(ctx);
    for (int q = 0; q < 8; ++q)
      if (!ctx->stats_der[q] && (rc = dev_alloc(ctx, (void**)&ctx->stats_der[q], pe))) return rc;
    const int last = nth - 1;
    for (int q = 0; q < 8; ++q) {
      const double2* src = q < 6 ? ctx->st[ctx->cur][q % 3] : ctx->st[ctx->cur][4 + last];
      const int axis = q < 6 ? q / 3 : q - 6;
      // epsilon's x derivatives leave out the kz = 0 row outside the homogeneous branch
      const int drop0 = (q < 3 && nonhom) ? 1 : 0;
      k_spec_deriv<<<grid1d(ftot), 256, 0, ctx->stream>>>(src, ctx->b_four, ctx->d_kx, ctx->d_kz, axis, drop0,
                                                         nkx1, ctx->nk2, ctx->kp, ftot);
      ctx->launches++;
      if ((rc = inv_four_to_phys(ctx, ctx->b_four, ctx->b_xs, ctx->stats_der[q]))) return rc;
    }
    const double* thxy = nullptr;
    if (zline) {
      if (!ctx->stats_thxy &&
          (rc = dev_alloc(ctx, (void**)&ctx->stats_thxy, (size_t)nyp2 * nx * sizeof(double))))
        return rc;
      const double* thl = ctx->b_phys;   // th_1 when it is the last scalar
      if (nth > 1) {
        if (!ctx->stats_thl && (rc = dev_alloc(ctx, (void**)&ctx->stats_thl, pe))) return rc;
        if ((rc = inv_four_to_phys(ctx, ctx->st[ctx->cur][4 + last], ctx->b_xs, ctx->stats_thl))) return rc;
        thl = ctx->stats_thl;
      }
      k_zmean<<<dim3((nx + 127) / 128, nyp2), 128, 0, ctx->stream>>>(thl, ctx->stats_thxy, nx, ctx->nz, nyp2);
      ctx->launches++;
      thxy = ctx->stats_thxy;
    }
    StatsZstarArgs z;
    memset(&z, 0, sizeof(z));
    for (int q = 0; q < 3; ++q) z.u[q] = uphys[q];
    z.th1 = ctx->b_phys;
    for (int q = 0; q < 6; ++q) z.du[q] = ctx->stats_der[q];
    z.dthd[0] = ctx->stats_der[6];
    z.dthd[1] = ctx->stats_der[7];
    z.means = d_means;
    z.xy = zline ? d_xy : nullptr;
    z.thxy = thxy;
    z.dy = ctx->d_dy;
    z.dyf = ctx->d_dyf;
    z.gy = ctx->d_gy;
    z.gyf = ctx->d_gyf;
    z.nu = ctx->nu;
    z.dthdx0 = p.dthdx[0];
    z.dthdx_l = p.dthdx[last];
    z.dthdz_l = p.dthdz[last];
    z.lx = p.lx;
    z.thmin = bthmin;
    z.thmax = bthmax;
    z.dth = bdth;
    z.roden = broden;
    z.pi_ref = PI_REF;
    z.nx = nx;
    z.nz = ctx->nz;
    z.nyp = ny;
    z.nth = nth;
    z.jlo = ctx->jst[0];
    z.jhi = ctx->jet[0];
    z.nbin = nbin;
    z.even = nonhom ? 1 : 0;
    z.hist = d_zs;
    const int zsm = (1 + ZS_N) * nbin * (int)sizeof(double);
    if (zsm > 48 * 1024) CK(cudaFuncSetAttribute(k_stats_zstar, cudaFuncAttributeMaxDynamicSharedMemorySize, zsm));
    Prof pr(ctx, K_OTHER);
    k_stats_zstar<<<4 * nsm, 256, zsm, ctx->stream>>>(z);
    ctx->launches++;
    CK(cudaGetLastError());
  }
  // the z-line arrays come back only when they were formed
  std::vector<double> h(total);
  CK(cudaMemcpyAsync(h.data(), ctx->d_stats, (zline ? total : total - n_xy) * sizeof(double),
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());

  // host finish, O(Ny Nx) (+ O(Ny Nx Nkx) for the mean x gradients of the
  // inhomogeneous branch)
  const double* part = h.data();
  const double* means = part + n_part;
  const double* spec = means + n_means;
  const double* lpart = spec + n_spec;
  const double* rows = lpart + n_les;
  const double* hpdf = rows + n_rows;
  const double* hzs = hpdf + n_bpe;
  const double* xyd = hzs + n_zs;
  auto Q = [&](int j, int q) {
    double s = 0.0;
    for (int sl = 0; sl < nslice; ++sl) s += part[((size_t)j * nslice + sl) * STAT_NQ + q];
    return s;
  };
  auto LQ = [&](int j, int q) {
    double s = 0.0;
    for (int sl = 0; sl < lslice; ++sl) s += lpart[((size_t)j * lslice + sl) * 2 + q];
    return s;
  };
  const std::vector<double>&gy = ctx->h_gy, &gyf = ctx->h_gyf, &dy = ctx->h_dy, &dyf = ctx->h_dyf;
  auto integrate_y = [&](const std::vector<double>& v) {   // integrate_y_var (:1974-1990)
    double r = 0.0;
    for (int j = 2; j <= ny; ++j) r = r + 0.5 * (v[j] + v[j - 1]) * dy[j];
    return r / p.ly;
  };
  std::vector<double> ume(nyp2), vme(nyp2), wme(nyp2);
  for (int j = 0; j < nyp2; ++j) {
    ume[j] = means[(size_t)j * (4 + nth) + 0];
    vme[j] = means[(size_t)j * (4 + nth) + 1];
    wme[j] = means[(size_t)j * (4 + nth) + 2];
  }
  const double nn = (double)nx * ctx->nz;
  for (int i = 0, ntot = diablo_stats_size(ctx); i < ntot; ++i) out[i] = 0.0;
  auto set = [&](int q, int j, double v) { out[(size_t)q * ny + (j - 1)] = v; };
  std::vector<double> uu(nyp2, 0.0), vv(nyp2, 0.0), ww(nyp2, 0.0), uw(nyp2, 0.0), uv(nyp2, 0.0),
      wv(nyp2, 0.0);
  for (int j = 1; j <= ny; ++j) {
    uu[j] = Q(j, SQ_UU);
    vv[j] = Q(j, SQ_VV);
    ww[j] = Q(j, SQ_WW);
    uw[j] = Q(j, SQ_UW);
    if (j >= 2) { uv[j] = Q(j, SQ_UV); wv[j] = Q(j, SQ_WV); }
  }
  // z-line means and covariances at each x, [j][i] (the plane values repeated
  // along x in the homogeneous branch, :811-836)
  typedef std::vector<double> Vec;
  const size_t xyn = (size_t)nyp2 * nx;
  // (held only in the z-line branch; elsewhere XY falls back to the profile)
  Vec ume_xy, vme_xy, wme_xy, uu_xy, vv_xy, uw_xy, uv_xy, wv_xy;
  auto XY = [&](const Vec& v, const Vec& prof, int j, int i) {
    return v.empty() ? prof[j] : v[(size_t)j * nx + i];
  };
  if (zline) {
    Vec* dst[XY_N] = {&ume_xy, &vme_xy, &wme_xy, &uu_xy, &vv_xy, &uw_xy, &uv_xy, &wv_xy};
    for (int q = 0; q < XY_N; ++q) dst[q]->assign(xyd + q * xyn, xyd + (q + 1) * xyn);
  }
  const Vec zero(nyp2, 0.0);
  // x profiles of the kz = 0 rows: value or x derivative (ikx, reference
  // wavenumbers) at x_i, the C2R sum Re c_0 + 2 sum_m Re(c_m e^{2 pi i m i/Nx})
  const std::vector<double>& hkx = ctx->h_kx;
  std::vector<double> ctab(nx), stab(nx);
  for (int t = 0; t < nx; ++t) {
    ctab[t] = cos(2.0 * M_PI * t / nx);
    stab[t] = sin(2.0 * M_PI * t / nx);
  }
  auto xprof = [&](int field, bool deriv, Vec& dst) {
    for (int j = 0; j < nyp2; ++j) {
      const double* r = rows + ((size_t)j * (3 + nth) + field) * nkx1 * 2;
      for (int i = 0; i < nx; ++i) {
        double s = deriv ? 0.0 : r[0];
        for (int m = 1; m < nkx1; ++m) {
          const int t = (int)(((long long)m * i) % nx);
          double cr = r[2 * m], ci = r[2 * m + 1];
          if (deriv) { const double k = hkx[m]; const double tr = -k * ci; ci = k * cr; cr = tr; }
          s += 2.0 * (cr * ctab[t] - ci * stab[t]);
        }
        dst[(size_t)j * nx + i] = s;
      }
    }
  };
  Vec dudx_m, dvdx_m, dwdx_m;
  if (nonhom) {
    dudx_m.assign(xyn, 0.0); dvdx_m.assign(xyn, 0.0); dwdx_m.assign(xyn, 0.0);
    xprof(0, true, dudx_m);
    xprof(1, true, dvdx_m);
    xprof(2, true, dwdx_m);
  }
  for (int j = 1; j <= ny; ++j) {
    set(DIABLO_STAT_UME, j, ume[j]);
    set(DIABLO_STAT_VME, j, vme[j]);
    set(DIABLO_STAT_WME, j, wme[j]);
    set(DIABLO_STAT_URMS, j, sqrt(uu[j]));
    set(DIABLO_STAT_VRMS, j, sqrt(vv[j]));
    set(DIABLO_STAT_WRMS, j, sqrt(ww[j]));
    set(DIABLO_STAT_UW, j, uw[j]);
    set(DIABLO_STAT_DUDY, j, (ume[j] - ume[j - 1]) / (gyf[j] - gyf[j - 1]));
    set(DIABLO_STAT_DWDY, j, (wme[j] - wme[j - 1]) / (gyf[j] - gyf[j - 1]));
    set(DIABLO_STAT_CP, j, means[(size_t)j * (4 + nth) + 3]);
    set(DIABLO_STAT_SHEAR, j, Q(j, SQ_SHEAR));
    set(DIABLO_STAT_OMEGA_X, j, sqrt(Q(j, SQ_OX)));
    set(DIABLO_STAT_OMEGA_Y, j, sqrt(Q(j, SQ_OY)));
    set(DIABLO_STAT_OMEGA_Z, j, sqrt(Q(j, SQ_OZ)));
    if (les) set(DIABLO_STAT_NU_SGS, j, LQ(j, 0) / nn);
    if (ctx->nz > 1) {   // production terms on GYF (:1486-1494)
      double a = 0.0, b = 0.0;
      for (int i = 0; i < nx; ++i) {
        a += XY(uu_xy, uu, j, i) * XY(dudx_m, zero, j, i);
        b += XY(uw_xy, uw, j, i) * XY(dwdx_m, zero, j, i);
      }
      set(DIABLO_STAT_UU_DUDX, j, a / nx);
      set(DIABLO_STAT_WU_DWDX, j, b / nx);
    }
    if (nonhom) {   // compute_MKE_diss (:1150-1262), rows 1..Ny
      double e = 0.0;
      for (int i = 0; i < nx; ++i) {
        const double su = XY(dudx_m, zero, j, i), sum_ = j >= 2 ? XY(dudx_m, zero, j - 1, i) : 0.0;
        const double sw = XY(dwdx_m, zero, j, i), swm = j >= 2 ? XY(dwdx_m, zero, j - 1, i) : 0.0;
        e += (dyf[j - 1] * su * su + dyf[j] * sum_ * sum_) / (2.0 * dy[j]);
        e += XY(dvdx_m, zero, j, i) * XY(dvdx_m, zero, j, i);
        e += (dyf[j - 1] * sw * sw + dyf[j] * swm * swm) / (2.0 * dy[j]);
        if (j >= 2) {
          const double tu = (XY(ume_xy, ume, j, i) - XY(ume_xy, ume, j - 1, i)) / dy[j];
          const double tv = (XY(vme_xy, vme, j + 1, i) - XY(vme_xy, vme, j - 1, i)) / (gy[j + 1] - gy[j - 1]);
          const double tw = (XY(wme_xy, wme, j, i) - XY(wme_xy, wme, j - 1, i)) / dy[j] + tws;
          e += tu * tu + tv * tv + tw * tw;
        }
      }
      set(DIABLO_STAT_EPSILON_M, j, ctx->nu * e / nx);
    }
    if (j < 2) continue;
    // GY-grid rows (j >= 2)
    set(DIABLO_STAT_UV, j, uv[j]);
    set(DIABLO_STAT_WV, j, wv[j]);
    set(DIABLO_STAT_EPSILON, j, ctx->nu * Q(j, SQ_EPS));
    if (les) set(DIABLO_STAT_EPS_SGS2, j, LQ(j, 1) / nn);
    if (ctx->nz > 1) {   // production terms on GY (:1496-1532)
      double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
      for (int i = 0; i < nx; ++i) {
        a += XY(uv_xy, uv, j, i) * XY(dvdx_m, zero, j, i);
        b += (XY(vme_xy, vme, j + 1, i) - XY(vme_xy, vme, j - 1, i)) / (gy[j + 1] - gy[j - 1]) * XY(vv_xy, vv, j, i);
        c += (XY(ume_xy, ume, j, i) - XY(ume_xy, ume, j - 1, i)) / dy[j] * XY(uv_xy, uv, j, i);
        d += ((XY(wme_xy, wme, j, i) - XY(wme_xy, wme, j - 1, i)) / dy[j] + tws) * XY(wv_xy, wv, j, i);
      }
      set(DIABLO_STAT_VU_DVDX, j, a / nx);
      set(DIABLO_STAT_VV_DVDY, j, b / nx);
      set(DIABLO_STAT_UV_DUDY, j, c / nx);
      set(DIABLO_STAT_WV_DWDY, j, d / nx);
    }
    // MKE on GY (:133-150)
    double mk = 0.0;
    for (int i = 0; i < nx; ++i) {
      const double u0 = XY(ume_xy, ume, j, i), u1m = XY(ume_xy, ume, j - 1, i);
      const double wa = XY(wme_xy, wme, j, i) + tws * (gyf[j] - 0.5 * p.ly);
      const double wb = XY(wme_xy, wme, j - 1, i) + tws * (gyf[j - 1] - 0.5 * p.ly);
      const double v0 = XY(vme_xy, vme, j, i);
      mk += (dyf[j - 1] * u0 * u0 + dyf[j] * u1m * u1m) / (2.0 * dy[j]) +
            (dyf[j - 1] * wa * wa + dyf[j] * wb * wb) / (2.0 * dy[j]) + v0 * v0;
    }
    set(DIABLO_STAT_MKE, j, 0.5 * mk / nx);
  }
  double* sc = out + (size_t)ny * (DIABLO_STAT_NPROF + nth * DIABLO_STAT_NTHPROF) + nx / 2 +
               (nth > 0 ? (2 + ZS_N) * nx : 0);
  sc[DIABLO_STAT_TIME] = ctx->time;
  sc[DIABLO_STAT_DT] = ctx->delta_t;
  sc[DIABLO_STAT_UBULK] = integrate_y(ume);
  sc[DIABLO_STAT_URMS_B] = sqrt(integrate_y(uu));
  sc[DIABLO_STAT_VRMS_B] = sqrt(integrate_y(vv));
  sc[DIABLO_STAT_WRMS_B] = sqrt(integrate_y(ww));
  Vec thme_xy;
  for (int n = 0; n < nth; ++n) {
    double* base = out + (size_t)ny * (DIABLO_STAT_NPROF + n * DIABLO_STAT_NTHPROF);
    auto tset = [&](int r, int j, double v) { base[(size_t)r * ny + (j - 1)] = v; };
    std::vector<double> thme(nyp2);
    for (int j = 0; j < nyp2; ++j) thme[j] = means[(size_t)j * (4 + nth) + 4 + n];
    if (zline) {
      thme_xy.assign(xyn, 0.0);
      xprof(3 + n, false, thme_xy);
    }
    for (int j = 1; j <= ny; ++j) {
      const int q0 = STAT_NQV + STAT_NQT * n;
      tset(DIABLO_STAT_THME, j, thme[j]);
      tset(DIABLO_STAT_DTHDY, j, (thme[j] - thme[j - 1]) / (gyf[j] - gyf[j - 1]));
      tset(DIABLO_STAT_THRMS, j, sqrt(Q(j, q0)));
      tset(DIABLO_STAT_THV, j, Q(j, q0 + 1));
      tset(DIABLO_STAT_PE_DISS, j, Q(j, q0 + 2));
      // thv_m (:377-385), gx(i) = i Lx / Nx
      double s = 0.0;
      for (int i = 0; i < nx; ++i)
        s = s + (XY(thme_xy, thme, j, i) + p.dthdx[n] * ((i * p.lx) / nx - 0.5 * p.lx)) *
                    (0.5 * (XY(vme_xy, vme, j, i) + XY(vme_xy, vme, j + 1, i)));
      tset(DIABLO_STAT_THV_M, j, s / nx);
    }
  }
  if (nth > 0) {   // u1z_x0 (:418-430)
    std::vector<double> u1yl(nyp2, 0.0);
    for (int j = 1; j <= ny; ++j) u1yl[j] = gyf[j] * Q(j, SQ_U1YL);
    sc[DIABLO_STAT_U1Y_LEFT_B] = integrate_y(u1yl);
  }
  if (nth > 0) {   // compute_BPE's finish (:1840-1860)
    double* pdf = out + (size_t)ny * (DIABLO_STAT_NPROF + nth * DIABLO_STAT_NTHPROF) + nx / 2;
    double* bin = pdf + nx;
    std::vector<double> thb(nbin + 1), yr(nbin + 1, 0.0);
    for (int i = 0; i <= nbin; ++i)
      thb[i] = nonhom ? bthmin + i * bdth : -(ctx->ro_inv + 1.e-14) * cos(i * PI_REF / nbin);
    double tot = 0.0;
    for (int i = 0; i < nbin; ++i) tot += hpdf[i];
    for (int i = 0; i < nbin; ++i) pdf[i] = hpdf[i] / tot;
    for (int i = 1; i <= nbin; ++i) yr[i] = yr[i - 1] + pdf[i - 1];
    for (int i = 0; i <= nbin; ++i) yr[i] = yr[i] * p.ly;
    double bpe = 0.0;
    for (int i = 0; i < nbin; ++i)
      bpe = bpe - (0.5 * (thb[i + 1] + thb[i]) * 0.5 * (yr[i + 1] + yr[i])) * (yr[i + 1] - yr[i]) / p.ly;
    for (int i = 0; i < nbin; ++i) bin[i] = thb[i];
    sc[DIABLO_STAT_BPE] = bpe;
    // the y* bin means: field sums over the (unnormalised) dyf sums; an empty
    // bin is 0/0 = NaN, as the reference writes it
    double* zs = bin + nx;
    for (int q = 0; q < ZS_N; ++q)
      for (int i = 0; i < nbin; ++i) zs[(size_t)q * nx + i] = hzs[(size_t)(1 + q) * nbin + i] / hzs[i];
  }
  // FTx_uu (:650-675): kz = 0 row of u1, integrated over y
  double* sp = out + (size_t)ny * (DIABLO_STAT_NPROF + nth * DIABLO_STAT_NTHPROF);
  for (int m = 0; m < nkx1 && m < nx / 2; ++m) {
    double s = 0.0;
    for (int j = 2; j <= ny; ++j)
      s += 0.5 * (spec[(size_t)j * nkx1 + m] + spec[(size_t)(j - 1) * nkx1 + m]) * dy[j];
    sp[m] = s / p.ly;
  }
  return 0;
}

int diablo_step(diablo_ctx* ctx, int nsteps) {
  if (!ctx || nsteps < 0) return DIABLO_ERR_ARG;
  for (int s = 0; s < nsteps; ++s) {
    ctx->time_step += 1;
    for (int rk = 1; rk <= 3; ++rk) {
      int rc = substep(ctx, rk);
      if (rc) return rc;
    }
    ctx->time += ctx->delta_t;
    int rc = filter_scalars(ctx);
    if (rc) return rc;
  }
  return 0;
}

static int bc_post(diablo_ctx* ctx, int do_vel, int do_th) {
  const diablo_params& p = ctx->p;
  update_transient(ctx);
  BcPostArgs a;
  memset(&a, 0, sizeof(a));
  for (int q = 0; q < 3; ++q) a.cu[q] = ctx->st[ctx->cur][q];
  for (int n = 0; n < ctx->nth; ++n) {
    a.cth[n] = ctx->st[ctx->cur][4 + n];
    a.thbc[n][0] = p.th_bc_ymin[n];
    a.thbc[n][1] = p.th_bc_ymax[n];
    a.thc1[n][0] = p.th_bc_ymin_c1[n];
    a.thc1[n][1] = p.th_bc_ymax_c1[n];
  }
  a.nth = ctx->nth;
  a.nyp = ctx->ny;
  a.nkx1 = ctx->nkx1;
  a.nk2 = ctx->nk2;
  a.kp = ctx->kp;
  a.ubc[0] = p.u_bc_ymin; a.ubc[1] = p.u_bc_ymax;
  a.vbc[0] = p.v_bc_ymin; a.vbc[1] = p.v_bc_ymax;
  a.wbc[0] = p.w_bc_ymin; a.wbc[1] = p.w_bc_ymax;
  a.uc1[0] = p.u_bc_ymin_c1; a.uc1[1] = p.u_bc_ymax_c1;
  a.vc1[0] = p.v_bc_ymin_c1; a.vc1[1] = p.v_bc_ymax_c1;
  a.wc1[0] = p.w_bc_ymin_c1;
  a.wc1[1] = p.w_bc_ymax == 0 ? p.w_bc_ymax_c1 : ctx->w_top_transient;
  a.dy = ctx->d_dy;
  a.dyf = ctx->d_dyf;
  a.do_vel = do_vel;
  a.do_th = do_th;
  int tot = ctx->nkx1 * ctx->nk2;
  k_bc_post<<<(tot + 127) / 128, 128, 0, ctx->stream>>>(a);
  ctx->launches++;
  CK(cudaGetLastError());
  return 0;
}

int diablo_apply_bc_post(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  return bc_post(ctx, 1, 1);
}

int diablo_pre_first_step(diablo_ctx* ctx, int compute_pressure) {
  if (!ctx) return DIABLO_ERR_ARG;
  // pre_first_step applies the velocity wall values only (for/advance.f90:25)
  int rc = bc_post(ctx, 1, 0);
  if (rc) return rc;
  SolveArgs a;
  fill_solve_args(ctx, a, 1);
  for (int q = 0; q < 3; ++q) a.cu_out[q] = ctx->st[ctx->cur][q];
  if ((rc = launch_solve(a, true, ctx->stream))) return rc;
  ctx->launches++;
  CK(cudaGetLastError());
  // poisson_p_chan for the initial pressure (for/advance.f90:31-33)
  if (compute_pressure && (rc = poisson_p(ctx))) return rc;
  // courant on the projected initial field (for/advance.f90:36-41)
  if (ctx->p.variable_dt) {
    double2* cu[3] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2]};
    if ((rc = courant_four(ctx, cu))) return rc;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int diablo_set_precision(diablo_ctx* ctx, int precision) {
  if (!ctx || (precision != DIABLO_FP64 && precision != DIABLO_MIXED)) return DIABLO_ERR_ARG;
  if (ctx->scratch_prec >= 0 && ctx->scratch_prec != precision) {
    // release step scratch sized for the other precision
    CK(cudaStreamSynchronize(ctx->stream));
    for (int f = 0; f < ctx->nf; ++f) {
      for (void** pp : {&ctx->nl[f], &ctx->phys[f]}) {
        for (size_t i = 0; i < ctx->allocs.size(); ++i)
          if (ctx->allocs[i] == *pp) { ctx->allocs.erase(ctx->allocs.begin() + i); break; }
        cudaFree(*pp);
        *pp = nullptr;
      }
    }
    for (int f = 0; f < 2 * ctx->nf; ++f) {
      for (size_t i = 0; i < ctx->allocs.size(); ++i)
        if (ctx->allocs[i] == ctx->xs[f]) { ctx->allocs.erase(ctx->allocs.begin() + i); break; }
      cudaFree(ctx->xs[f]);
      ctx->xs[f] = nullptr;
    }
    ctx->scratch_prec = -1;
  }
  ctx->precision = precision;
  ctx->p.precision = precision;
  for (int q = 0; q < 4; ++q) ctx->tune[q] = 0;   // tiles are per precision
  ctx->generation++;
  return 0;
}

int diablo_get_time(diablo_ctx* ctx, double* time, int* time_step, double* delta_t) {
  if (!ctx) return DIABLO_ERR_ARG;
  if (time) *time = ctx->time;
  if (time_step) *time_step = ctx->time_step;
  if (delta_t) *delta_t = ctx->delta_t;
  return 0;
}

int diablo_set_time(diablo_ctx* ctx, double time, int time_step, double delta_t) {
  if (!ctx || !(delta_t > 0)) return DIABLO_ERR_ARG;
  ctx->time = time;
  ctx->time_step = time_step;
  const bool changed = delta_t != ctx->delta_t;
  ctx->delta_t = delta_t;
  for (int r = 0; r < 3; ++r) ctx->h_bar[r] = H_FRAC[r] * delta_t;
  if (changed) ctx->generation++;
  return changed ? upload_coefficients(ctx) : 0;
}

int diablo_set_stream(diablo_ctx* ctx, void* stream) {
  if (!ctx) return DIABLO_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return 0;
}

int diablo_synchronize(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

int diablo_check_finite(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  CK(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  for (int f = 0; f < 4 + ctx->nth; ++f) {
    k_check_finite<<<grid1d(four_elems(ctx)), 256, 0, ctx->stream>>>(ctx->st[ctx->cur][f], ctx->g,
                                                                      ctx->d_flag);
    ctx->launches++;
  }
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return bad ? DIABLO_ERR_NONFINITE : 0;
}

long long diablo_kernel_launches(const diablo_ctx* ctx) { return ctx ? ctx->launches : -1; }

int diablo_set_profiling(diablo_ctx* ctx, int enable) {
  if (!ctx) return DIABLO_ERR_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  prof_collect(ctx);
  ctx->profiling = enable ? 1 : 0;
  for (int i = 0; i < K_NSLOTS; ++i) { ctx->slot_ms[i] = 0.0; ctx->slot_n[i] = 0; }
  return 0;
}

int diablo_kernel_times(diablo_ctx* ctx, int slot, double* total_ms, long long* launches) {
  if (!ctx || slot < 0 || slot >= K_NSLOTS) return DIABLO_ERR_ARG;
  prof_collect(ctx);
  if (total_ms) *total_ms = ctx->slot_ms[slot];
  if (launches) *launches = ctx->slot_n[slot];
  return 0;
}

int diablo_kernel_slots(void) { return K_NSLOTS; }

const char* diablo_kernel_name(int slot) {
  return (slot >= 0 && slot < K_NSLOTS) ? K_NAMES[slot] : "";
}

}  // extern "C"

// ==========================================================================
// Ensembles: independent members stepped by one CUDA graph launch per step.
// Each member's kernel chain is one branch of the graph (its own stream
// during capture), so small members run concurrently.  Kernel arguments hold
// the double-buffer pointers, so two graphs are kept, one per buffer parity.

struct MemberKey {
  int cur, cf_cur, les, generation;
  bool operator==(const MemberKey& o) const {
    return cur == o.cur && cf_cur == o.cf_cur && les == o.les && generation == o.generation;
  }
};

struct diablo_ensemble {
  std::vector<diablo_ctx*> m;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  std::vector<MemberKey> key[2];
  std::vector<long long> nlaunch[2];
  int last_cuda = 0;
};

static MemberKey member_key(const diablo_ctx* c) {
  return MemberKey{c->cur, c->cf_cur, les_active(c), c->generation};
}

// Everything a step allocates on first use, so that capture allocates nothing.
static int prepare_member(diablo_ctx* ctx) {
  int rc;
  if ((rc = ensure_scratch(ctx))) return rc;
  if (les_active(ctx)) {
    if ((rc = ensure_les(ctx))) return rc;
    const int m = ctx->p.les_model_type;
    if ((m == 4 || m == 5) && (rc = ensure_amd(ctx))) return rc;
    if (m == 2 && (rc = ensure_dyn(ctx))) return rc;
  }
  return 0;
}

static int one_step(diablo_ctx* ctx) {
  ctx->time_step += 1;
  for (int rk = 1; rk <= 3; ++rk) {
    int rc = substep(ctx, rk);
    if (rc) return rc;
  }
  ctx->time += ctx->delta_t;
  return 0;
}

#define ECK(call)                                 \
  do {                                            \
    cudaError_t e__ = (call);                     \
    if (e__ != cudaSuccess) {                     \
      e->last_cuda = (int)e__;                    \
      return DIABLO_ERR_CUDA;                     \
    }                                             \
  } while (0)

// Capture one step of every member into exec[w], from the members' current
// host state; the host state is advanced as the step would advance it.
static int capture(diablo_ensemble* e, int w) {
  const int n = (int)e->m.size();
  std::vector<cudaStream_t> saved(n);
  std::vector<int> prof(n);
  e->key[w].resize(n);
  e->nlaunch[w].resize(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    saved[i] = c->stream;
    prof[i] = c->profiling;
    c->profiling = 0;
    c->stream = e->streams[i];
    e->key[w][i] = member_key(c);
  }
  cudaGraph_t graph = nullptr;
  int rc = 0;
  cudaError_t ce = cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    cudaEventRecord(e->fork, e->origin);
    for (int i = 0; i < n && !rc; ++i) {
      diablo_ctx* c = e->m[i];
      cudaStreamWaitEvent(e->streams[i], e->fork, 0);
      const long long l0 = c->launches;
      rc = one_step(c);
      e->nlaunch[w][i] = c->launches - l0;
      cudaEventRecord(e->joins[i], e->streams[i]);
      cudaStreamWaitEvent(e->origin, e->joins[i], 0);
    }
    ce = cudaStreamEndCapture(e->origin, &graph);
  }
  for (int i = 0; i < n; ++i) {
    e->m[i]->stream = saved[i];
    e->m[i]->profiling = prof[i];
  }
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return rc;
  }
  ECK(ce);
  if (e->exec[w]) { cudaGraphExecDestroy(e->exec[w]); e->exec[w] = nullptr; }
  ce = cudaGraphInstantiate(&e->exec[w], graph, 0);
  cudaGraphDestroy(graph);
  ECK(ce);
  return 0;
}

// (Re)capture both graphs from the members' current state, leaving the
// members' host state as it was.
static int capture_both(diablo_ensemble* e) {
  const int n = (int)e->m.size();
  struct Saved { double time; int time_step, cur, cf_cur; double wtt; };
  std::vector<Saved> sv(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    int rc = prepare_member(c);
    if (rc) return rc;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return DIABLO_ERR_CUDA;
    sv[i] = Saved{c->time, c->time_step, c->cur, c->cf_cur, c->w_top_transient};
  }
  int rc = capture(e, 0);
  if (!rc) rc = capture(e, 1);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    c->time = sv[i].time; c->time_step = sv[i].time_step;
    c->cur = sv[i].cur; c->cf_cur = sv[i].cf_cur; c->w_top_transient = sv[i].wtt;
  }
  return rc;
}

extern "C" {

diablo_ensemble* diablo_ensemble_create(diablo_ctx* const* members, int n, int* status) {
  int st = 0;
  diablo_ensemble* e = nullptr;
  if (!members || n <= 0) st = DIABLO_ERR_ARG;
  for (int i = 0; i < n && !st; ++i) {
    const diablo_ctx* c = members[i];
    if (!c) { st = DIABLO_ERR_ARG; break; }
    for (int k = 0; k < i; ++k)
      if (members[k] == c) st = DIABLO_ERR_ARG;
    // kernel arguments that change every step cannot be replayed from a graph
    if (c->p.variable_dt || c->p.f_type == 2 || (c->p.f_type == 4 && c->p.w_bc_ymax != 0))
      st = DIABLO_ERR_UNSUPPORTED;
    for (int q = 0; q < c->nth; ++q)
      if (c->p.filter_th[q]) st = DIABLO_ERR_UNSUPPORTED;   // filtered on some steps only
  }
  if (!st) {
    e = new diablo_ensemble();
    e->m.assign(members, members + n);
    bool ok = cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
    e->streams.assign(n, nullptr);
    e->joins.assign(n, nullptr);
    for (int i = 0; i < n && ok; ++i)
      ok = cudaStreamCreateWithFlags(&e->streams[i], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&e->joins[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) { st = DIABLO_ERR_CUDA; diablo_ensemble_destroy(e); e = nullptr; }
  }
  if (status) *status = st;
  return e;
}

int diablo_ensemble_step(diablo_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return DIABLO_ERR_ARG;
  const int n = (int)e->m.size();
  for (int s = 0; s < nsteps; ++s) {
    // the graph captured for this parity must match every member's state
    int w = -1;
    for (int k = 0; k < 2 && w < 0; ++k) {
      if (!e->exec[k] || (int)e->key[k].size() != n) continue;
      bool ok = true;
      for (int i = 0; i < n && ok; ++i) ok = member_key(e->m[i]) == e->key[k][i];
      if (ok) w = k;
    }
    if (w < 0) {
      int rc = capture_both(e);
      if (rc) return rc;
      w = 0;
    }
    // order the graph after each member's earlier work on its own stream
    for (int i = 0; i < n; ++i) {
      ECK(cudaEventRecord(e->joins[i], e->m[i]->stream));
      ECK(cudaStreamWaitEvent(e->origin, e->joins[i], 0));
    }
    ECK(cudaGraphLaunch(e->exec[w], e->origin));
    ECK(cudaEventRecord(e->fork, e->origin));
    for (int i = 0; i < n; ++i) {
      diablo_ctx* c = e->m[i];
      ECK(cudaStreamWaitEvent(c->stream, e->fork, 0));
      c->time_step += 1;
      c->time += c->delta_t;
      c->cur ^= 1;                 // three substeps flip the state buffer
      c->launches += e->nlaunch[w][i];
    }
  }
  return 0;
}

void* diablo_ensemble_stream(diablo_ensemble* e) { return e ? (void*)e->origin : nullptr; }

int diablo_ensemble_synchronize(diablo_ensemble* e) {
  if (!e) return DIABLO_ERR_ARG;
  ECK(cudaStreamSynchronize(e->origin));
  for (diablo_ctx* c : e->m) ECK(cudaStreamSynchronize(c->stream));
  ECK(cudaGetLastError());
  return 0;
}

int diablo_ensemble_destroy(diablo_ensemble* e) {
  if (!e) return DIABLO_ERR_ARG;
  if (e->origin) cudaStreamSynchronize(e->origin);
  for (int k = 0; k < 2; ++k)
    if (e->exec[k]) cudaGraphExecDestroy(e->exec[k]);
  for (cudaStream_t s : e->streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t v : e->joins)
    if (v) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->origin) cudaStreamDestroy(e->origin);
  delete e;
  return 0;
}

}  // extern "C"

// ==========================================================================
// Discrete adjoint of diablo_step (velocity-only DNS, FP64), with
// checkpoint-and-recompute: diablo_adjoint_record stores the state every
// `every` steps; diablo_adjoint_run recomputes each segment from its
// checkpoint (keeping the velocities entering every substep) and runs the
// substep adjoints backwards through it.

static int adj_free(diablo_ctx* ctx) {
  diablo_ctx::Tape& T = ctx->tape;
  auto rel = [&](void* p) {
    if (!p) return;
    for (size_t i = 0; i < ctx->allocs.size(); ++i)
      if (ctx->allocs[i] == p) { ctx->allocs.erase(ctx->allocs.begin() + i); break; }
    cudaFree(p);
  };
  for (double2* p : T.ckpt) rel(p);
  for (double2* p : T.sub) rel(p);
  T.ckpt.clear();
  T.sub.clear();
  T.ready = 0;
  return 0;
}

// host-built rows of the substep systems (the forward's expressions)
static void adj_rows(diablo_ctx* ctx, std::vector<double>& cn, std::vector<double>& rmask,
                     std::vector<double>& pa) {
  const diablo_params& p = ctx->p;
  const int n = ctx->nyp2, nyp = ctx->ny;
  const std::vector<double>& dy = ctx->h_dy;
  const std::vector<double>& dyf = ctx->h_dyf;
  cn.assign((size_t)3 * 3 * 3 * n, 0.0);
  rmask.assign((size_t)3 * n, 0.0);
  pa.assign((size_t)3 * n, 0.0);
  for (int j = 2; j <= nyp - 1; ++j) {
    pa[j] = 1. / (dy[j] * dyf[j]);
    pa[n + j] = 1. / (dy[j + 1] * dyf[j]);
    pa[2 * n + j] = -1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]);
  }
  for (int rk = 0; rk < 3; ++rk) {
    const double tc = 0.5 * ctx->nu * ctx->h_bar[rk] * p.nu_v_scale;
    for (int f = 0; f < 3; ++f) {
      double* A = &cn[((size_t)rk * 3 + f) * 3 * n];
      double* B = A + n;
      double* C = B + n;
      double* rm = &rmask[(size_t)f * n];
      for (int j = 0; j < n; ++j) { A[j] = 0.0; B[j] = 1.0; C[j] = 0.0; }
      if (f != 1) {
        for (int j = ctx->jstart; j <= ctx->jend; ++j) {
          A[j] = -tc / (dy[j] * dyf[j]);
          B[j] = 1. - tc * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
          C[j] = -tc / (dy[j + 1] * dyf[j]);
          rm[j] = 1.0;
        }
        const int bmin = f == 0 ? p.u_bc_ymin : p.w_bc_ymin, bmax = f == 0 ? p.u_bc_ymax : p.w_bc_ymax;
        A[0] = 0; B[0] = 1; C[0] = 0;
        if (bmin == 0) { A[1] = 0; B[1] = 1; C[1] = 0; } else { A[1] = 0; B[1] = -1; C[1] = 1; }
        A[nyp + 1] = 0; B[nyp + 1] = 1; C[nyp + 1] = 0;
        if (bmax == 0) { A[nyp] = 0; B[nyp] = 1; C[nyp] = 0; } else { A[nyp] = -1; B[nyp] = 1; C[nyp] = 0; }
        rm[0] = rm[1] = rm[nyp] = rm[nyp + 1] = 0.0;
      } else {
        for (int j = 2; j <= nyp; ++j) {
          A[j] = -tc / (dyf[j - 1] * dy[j]);
          B[j] = 1. + tc / (dyf[j] * dy[j]) + tc / (dyf[j - 1] * dy[j]);
          C[j] = -tc / (dyf[j] * dy[j]);
          rm[j] = 1.0;
        }
        if (p.v_bc_ymin == 0) {
          for (int r = 1; r <= 2; ++r) { A[r] = 0; B[r] = 1; C[r] = 0; rm[r] = 0; }
        } else {
          A[1] = 0; B[1] = -1; C[1] = 1; rm[1] = 0;
        }
        A[0] = 0; B[0] = 1; C[0] = 0; rm[0] = 0;
        if (p.v_bc_ymax == 0) {
          for (int r = nyp; r <= nyp + 1; ++r) { A[r] = 0; B[r] = 1; C[r] = 0; rm[r] = 0; }
        } else {
          A[nyp + 1] = -1; B[nyp + 1] = 1; C[nyp + 1] = 0; rm[nyp + 1] = 0;
        }
      }
    }
  }
}

static int adj_supported(const diablo_ctx* ctx) {
  if (ctx->nth != 0 || ctx->p.use_les || ctx->precision != DIABLO_FP64 || ctx->p.variable_dt)
    return DIABLO_ERR_UNSUPPORTED;
  return 0;
}

static int adj_alloc(diablo_ctx* ctx, int nsteps, int every) {
  diablo_ctx::Tape& T = ctx->tape;
  const size_t fe = four_elems(ctx) * sizeof(double2), pe = phys_elems(ctx) * sizeof(double);
  int rc;
  // the checkpoint and substep buffers are kept while nsteps and every stay the same
  if (T.ckpt.empty() || T.nsteps != nsteps || T.every != every) {
    adj_free(ctx);
    T.nsteps = nsteps;
    T.every = every;
    T.nseg = (nsteps + every - 1) / every;
    T.ckpt.assign((size_t)(T.nseg + 1) * 4, nullptr);
    for (auto& p : T.ckpt) if ((rc = dev_alloc(ctx, (void**)&p, fe))) return rc;
    T.sub.assign((size_t)every * 9, nullptr);
    for (auto& p : T.sub) if ((rc = dev_alloc(ctx, (void**)&p, fe))) return rc;
    T.ckpt_step.assign(T.nseg + 1, 0);
    T.ckpt_time.assign(T.nseg + 1, 0.0);
  }
  T.ready = 0;
  if (!T.work_ready) {
#define AL(ptr, bytes) if ((rc = dev_alloc(ctx, (void**)&(ptr), (bytes)))) return rc
    for (int q = 0; q < 4; ++q) { AL(T.lu[q], fe); AL(T.ou[q], fe); }
    for (int q = 0; q < 3; ++q) { AL(T.lF[q], fe); AL(T.oF[q], fe); AL(T.lnl[q], fe); AL(T.lf3[q], fe);
                                  AL(T.up[q], pe); AL(T.lp3[q], pe); }
    for (int q = 0; q < 8; ++q) { AL(T.pf[q], fe); AL(T.pp[q], pe); }
    AL(T.d_cn, (size_t)27 * ctx->nyp2 * sizeof(double));
    AL(T.d_rmask, (size_t)3 * ctx->nyp2 * sizeof(double));
    AL(T.d_pa, (size_t)3 * ctx->nyp2 * sizeof(double));
#undef AL
    T.work_ready = 1;
  }
  std::vector<double> cn, rm, pa;
  adj_rows(ctx, cn, rm, pa);
  CK(cudaMemcpyAsync(T.d_cn, cn.data(), cn.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(T.d_rmask, rm.data(), rm.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(T.d_pa, pa.data(), pa.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

static int copy_fields(diablo_ctx* ctx, double2* const* dst, double2* const* src, int nf) {
  const size_t fe = four_elems(ctx) * sizeof(double2);
  for (int q = 0; q < nf; ++q) CK(cudaMemcpyAsync(dst[q], src[q], fe, cudaMemcpyDeviceToDevice, ctx->stream));
  return 0;
}

// Adjoint of substep rk: T.lu (lambda of the substep's output state) and
// T.lF (lambda of its cf) become the lambdas of its input; u_in are the
// velocities that entered the substep.
static int adj_substep(diablo_ctx* ctx, int rk, double2* const* u_in) {
  diablo_ctx::Tape& T = ctx->tape;
  const diablo_params& p = ctx->p;
  const double h = ctx->h_bar[rk - 1];
  const FGeom fg{ctx->ny, ctx->nyp2, ctx->nkx1, ctx->nk2, ctx->kp, (size_t)ctx->nkx1 * ctx->kp};
  const size_t ftot = four_elems(ctx), ptot = phys_elems(ctx);
  int rc;
  {
    AdjColArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < 3; ++f) {
      a.lu[f] = T.lu[f];
      a.lF[f] = rk < 3 ? T.lF[f] : nullptr;
      a.ou[f] = T.ou[f];
      a.oF[f] = rk > 1 ? T.oF[f] : nullptr;
      a.onl[f] = T.lnl[f];
    }
    a.lp = T.lu[3];
    a.op = T.ou[3];
    a.cn = T.d_cn + (size_t)(rk - 1) * 9 * ctx->nyp2;
    a.rmask = T.d_rmask;
    a.pa = T.d_pa;
    a.kx = ctx->d_kx; a.kz = ctx->d_kz; a.dy = ctx->d_dy; a.dyf = ctx->d_dyf;
    a.t3 = ZETA_BAR[rk - 1] * h; a.t4 = h; a.t5 = BETA_BAR[rk - 1] * h;
    a.tc = 0.5 * ctx->nu * h * p.nu_v_scale;
    a.nu = ctx->nu; a.roinvd = ctx->ro_inv / p.delta; a.beta = p.beta;
    a.n = ctx->nyp2; a.nyp = ctx->ny; a.nkx1 = ctx->nkx1; a.nk2 = ctx->nk2; a.kp = ctx->kp;
    a.ncol = ctx->nkx1 * ctx->nk2;
    a.jstart = ctx->jstart; a.jend = ctx->jend; a.rk = rk;
    Prof pr(ctx, K_OTHER);
    const int warps = 4;
    dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
    switch (rows_per_lane(ctx->nyp2)) {
#define X(r) case r: k_adj_column<r><<<grd, blk, 0, ctx->stream>>>(a); break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: return DIABLO_ERR_SIZE;
    }
  }
  {
    AdjNlPrepArgs a;
    for (int f = 0; f < 3; ++f) a.lnl[f] = T.lnl[f];
    for (int q = 0; q < 8; ++q) a.out[q] = T.pf[q];
    a.kx = ctx->d_kx; a.kz = ctx->d_kz;
    a.inv = 1.0 / ((double)ctx->nx * ctx->nz);
    a.g = fg;
    Prof pr(ctx, K_OTHER);
    k_adj_nl_prep<<<grid1d(ftot), 256, 0, ctx->stream>>>(a);
  }
  if ((rc = ifft_batch(ctx, T.pf, T.pp, 8))) return rc;
  if ((rc = ifft_batch(ctx, u_in, T.up, 3))) return rc;
  {
    AdjNlPointArgs a;
    for (int q = 0; q < 8; ++q) a.P[q] = T.pp[q];
    a.u1 = T.up[0]; a.u2 = T.up[1]; a.u3 = T.up[2];
    a.o1 = T.lp3[0]; a.o2 = T.lp3[1]; a.o3 = T.lp3[2];
    a.dy = ctx->d_dy; a.dyf = ctx->d_dyf;
    a.nyp = ctx->ny;
    a.ps = (size_t)ctx->nz * ctx->nx;
    Prof pr(ctx, K_OTHER);
    k_adj_nl_point<<<grid1d(ptot), 256, 0, ctx->stream>>>(a);
  }
  if ((rc = fft_batch(ctx, T.lp3, T.lf3, 3))) return rc;
  {
    AdjAccArgs a;
    for (int f = 0; f < 3; ++f) { a.ou[f] = T.ou[f]; a.add[f] = T.lf3[f]; }
    a.scale = (double)ctx->nx * ctx->nz;
    a.g = fg;
    Prof pr(ctx, K_OTHER);
    k_adj_acc<<<grid1d(ftot), 256, 0, ctx->stream>>>(a);
  }
  CK(cudaGetLastError());
  for (int q = 0; q < 4; ++q) std::swap(T.lu[q], T.ou[q]);
  for (int q = 0; q < 3; ++q) std::swap(T.lF[q], T.oF[q]);
  return 0;
}

extern "C" {

int diablo_adjoint_record(diablo_ctx* ctx, int nsteps, int every) {
  if (!ctx || nsteps <= 0 || every <= 0) return DIABLO_ERR_ARG;
  int rc;
  if ((rc = adj_supported(ctx))) return rc;
  if ((rc = ensure_scratch(ctx)) || (rc = ensure_xs64(ctx))) return rc;
  if ((rc = adj_alloc(ctx, nsteps, every))) return rc;
  diablo_ctx::Tape& T = ctx->tape;
  for (int s = 0; s < nsteps; ++s) {
    if (s % every == 0) {
      const int k = s / every;
      double2* src[4] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2], ctx->st[ctx->cur][3]};
      if ((rc = copy_fields(ctx, &T.ckpt[(size_t)k * 4], src, 4))) return rc;
      T.ckpt_step[k] = ctx->time_step;
      T.ckpt_time[k] = ctx->time;
    }
    if ((rc = one_step(ctx))) return rc;
  }
  double2* src[4] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2], ctx->st[ctx->cur][3]};
  if ((rc = copy_fields(ctx, &T.ckpt[(size_t)T.nseg * 4], src, 4))) return rc;
  T.ckpt_step[T.nseg] = ctx->time_step;
  T.ckpt_time[T.nseg] = ctx->time;
  T.step_end = ctx->time_step;
  T.time_end = ctx->time;
  T.gen_end = ctx->generation;
  T.ready = 1;
  return 0;
}

int diablo_adjoint_run(diablo_ctx* ctx, double* const* lam) {
  if (!ctx || !lam) return DIABLO_ERR_ARG;
  for (int q = 0; q < 4; ++q) if (!lam[q]) return DIABLO_ERR_ARG;
  diablo_ctx::Tape& T = ctx->tape;
  if (!T.ready || ctx->time_step != T.step_end || ctx->generation != T.gen_end) return DIABLO_ERR_STATE;
  int rc;
  if ((rc = ensure_bscratch(ctx))) return rc;
  const size_t fe = four_elems(ctx) * sizeof(double2);
  for (int q = 0; q < 4; ++q)
    if ((rc = four_in(ctx, lam[q], T.lu[q], false))) return rc;
  for (int q = 0; q < 3; ++q) CK(cudaMemsetAsync(T.lF[q], 0, fe, ctx->stream));
  for (int k = T.nseg - 1; k >= 0; --k) {
    // recompute the segment from its checkpoint, keeping each substep's input velocities
    double2* dst[4] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2], ctx->st[ctx->cur][3]};
    if ((rc = copy_fields(ctx, dst, &T.ckpt[(size_t)k * 4], 4))) return rc;
    ctx->time_step = T.ckpt_step[k];
    ctx->time = T.ckpt_time[k];
    const int s0 = k * T.every, s1 = std::min(T.nsteps, s0 + T.every);
    for (int s = s0; s < s1; ++s) {
      ctx->time_step += 1;
      for (int rk = 1; rk <= 3; ++rk) {
        double2** keep = &T.sub[((size_t)(s - s0) * 3 + (rk - 1)) * 3];
        double2* cu[3] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2]};
        if ((rc = copy_fields(ctx, keep, cu, 3))) return rc;
        if ((rc = substep(ctx, rk))) return rc;
      }
      ctx->time += ctx->delta_t;
    }
    for (int s = s1 - 1; s >= s0; --s)
      for (int rk = 3; rk >= 1; --rk)
        if ((rc = adj_substep(ctx, rk, &T.sub[((size_t)(s - s0) * 3 + (rk - 1)) * 3]))) return rc;
  }
  // back to the recorded final state
  double2* dst[4] = {ctx->st[ctx->cur][0], ctx->st[ctx->cur][1], ctx->st[ctx->cur][2], ctx->st[ctx->cur][3]};
  if ((rc = copy_fields(ctx, dst, &T.ckpt[(size_t)T.nseg * 4], 4))) return rc;
  ctx->time_step = T.step_end;
  ctx->time = T.time_end;
  for (int q = 0; q < 4; ++q)
    if ((rc = four_out(ctx, T.lu[q], lam[q]))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

}  // extern "C"

// ==========================================================================
// Autotuner: the tile shapes of the four step transforms (sequences per
// block of the z kernels, rows per block of the x kernels) are timed on the
// context's own scratch for its grid and precision, and the fastest kept.
// Results are cached per (grid, fields, precision) for the process.

#include <map>
#include <mutex>
#include <tuple>

static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int, int>, std::array<int, 4>> g_tune_cache;

extern "C" {

int diablo_tiles(diablo_ctx* ctx, int* tiles) {
  if (!ctx || !tiles) return DIABLO_ERR_ARG;
  for (int q = 0; q < 4; ++q) tiles[q] = ctx->tune[q];
  return 0;
}

int diablo_autotune(diablo_ctx* ctx, int* tiles) {
  if (!ctx) return DIABLO_ERR_ARG;
  int rc;
  if (les_active(ctx)) return DIABLO_ERR_UNSUPPORTED;
  if ((rc = ensure_scratch(ctx))) return rc;
  const auto key = std::make_tuple(ctx->nx, ctx->ny, ctx->nz, ctx->nf, ctx->precision);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      for (int q = 0; q < 4; ++q) ctx->tune[q] = it->second[q];
      ctx->generation++;
      if (tiles) for (int q = 0; q < 4; ++q) tiles[q] = ctx->tune[q];
      return 0;
    }
  }
  const bool fp32 = ctx->precision != DIABLO_FP64;
  SolveArgs sa;
  fill_solve_args(ctx, sa, 1);
  const bool mean_split = fp32 && !sa.front && !ctx->use_general_solver;
  int cand[4][3], nc[4];
  for (int k = 0; k < 4; ++k) {
    nc[k] = fft_tile_candidates(k, (k == 0 || k == 3) ? ctx->nz : ctx->M, fp32, cand[k]);
    if (nc[k] <= 0) return DIABLO_ERR_SIZE;
  }
  const int slot[4] = {K_ZINV, K_XINV, K_XFWD_NL, K_ZFWD_NL};
  double best[4] = {1e300, 1e300, 1e300, 1e300};
  int pick[4] = {0, 0, 0, 0};
  const int saved_prof = ctx->profiling;
  auto run = [&]() -> int {
    return fp32 ? substep_spectral<float>(ctx, mean_split ? 0x1u : 0u) : substep_spectral<double>(ctx, 0u);
  };
  for (int i = 0; i < 3; ++i) {
    for (int k = 0; k < 4; ++k) ctx->tune[k] = cand[k][i < nc[k] ? i : nc[k] - 1];
    ctx->profiling = 0;
    if ((rc = run())) { ctx->profiling = saved_prof; return rc; }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    ctx->profiling = 1;
    for (int sl = 0; sl < K_NSLOTS; ++sl) { ctx->slot_ms[sl] = 0.0; ctx->slot_n[sl] = 0; }
    for (int r = 0; r < 3 && !rc; ++r) rc = run();
    if (rc) { ctx->profiling = saved_prof; return rc; }
    CK(cudaStreamSynchronize(ctx->stream));
    prof_collect(ctx);
    for (int k = 0; k < 4; ++k) {
      if (i >= nc[k]) continue;
      const double t = ctx->slot_ms[slot[k]];
      if (t < best[k]) { best[k] = t; pick[k] = cand[k][i]; }
    }
  }
  for (int sl = 0; sl < K_NSLOTS; ++sl) { ctx->slot_ms[sl] = 0.0; ctx->slot_n[sl] = 0; }
  ctx->profiling = saved_prof;
  for (int k = 0; k < 4; ++k) ctx->tune[k] = pick[k];
  ctx->generation++;
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune_cache[key] = {pick[0], pick[1], pick[2], pick[3]};
  }
  if (tiles) for (int q = 0; q < 4; ++q) tiles[q] = pick[q];
  return 0;
}

}  // extern "C"

// ==========================================================================
// Ensemble autotuner: coordinate descent over the transform tiles of each
// group of same-size members, scored by the time of the ensemble's own graph
// (the members' kernels run concurrently there, so isolated kernel times are
// not the objective).  Member states are restored afterwards.

extern "C" {

int diablo_ensemble_autotune(diablo_ensemble* e, int steps_per_trial) {
  if (!e || steps_per_trial <= 0) return DIABLO_ERR_ARG;
  const int n = (int)e->m.size();
  int rc;
  // snapshot every member (state fields, counters, tiles)
  struct Snap { std::vector<double2*> f; double time; int step, cur, cf_cur; int tune[4]; };
  std::vector<Snap> snap(n);
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    if ((rc = ensure_scratch(c))) return rc;
    if (les_active(c)) return DIABLO_ERR_UNSUPPORTED;
    const size_t fe = four_elems(c) * sizeof(double2);
    snap[i].f.assign(4 + c->nth, nullptr);
    for (int q = 0; q < 4 + c->nth; ++q) {
      if ((rc = dev_alloc(c, (void**)&snap[i].f[q], fe))) return rc;
      if (cudaMemcpyAsync(snap[i].f[q], c->st[c->cur][q], fe, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess)
        return DIABLO_ERR_CUDA;
    }
    snap[i].time = c->time; snap[i].step = c->time_step; snap[i].cur = c->cur; snap[i].cf_cur = c->cf_cur;
    for (int q = 0; q < 4; ++q) snap[i].tune[q] = c->tune[q];
  }
  // groups of members sharing a tile configuration
  std::vector<std::vector<int>> groups;
  std::vector<std::tuple<int, int, int, int, int>> gkey;
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    auto k = std::make_tuple(c->nx, c->ny, c->nz, c->nf, c->precision);
    size_t g = 0;
    while (g < gkey.size() && gkey[g] != k) ++g;
    if (g == gkey.size()) { gkey.push_back(k); groups.emplace_back(); }
    groups[g].push_back(i);
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto trial = [&](float* ms) -> int {
    int r = diablo_ensemble_step(e, 1);      // captures if needed, warms
    if (r) return r;
    ECK(cudaEventRecord(t0, e->origin));
    if ((r = diablo_ensemble_step(e, steps_per_trial))) return r;
    ECK(cudaEventRecord(t1, e->origin));
    ECK(cudaEventSynchronize(t1));
    ECK(cudaEventElapsedTime(ms, t0, t1));
    return 0;
  };
  float best = 0.f;
  rc = trial(&best);
  for (size_t g = 0; g < groups.size() && !rc; ++g) {
    diablo_ctx* c0 = e->m[groups[g][0]];
    const bool fp32 = c0->precision != DIABLO_FP64;
    for (int k = 0; k < 4 && !rc; ++k) {
      int cand[3];
      const int nc = fft_tile_candidates(k, (k == 0 || k == 3) ? c0->nz : c0->M, fp32, cand);
      const int keep = c0->tune[k];
      int pick = keep;
      for (int ci = 0; ci < nc && !rc; ++ci) {
        if (cand[ci] == keep || (keep == 0 && ci == 0)) continue;   // the current choice is already scored
        for (int i : groups[g]) { e->m[i]->tune[k] = cand[ci]; e->m[i]->generation++; }
        float ms = 0.f;
        if ((rc = trial(&ms))) break;
        if (ms < best) { best = ms; pick = cand[ci]; }
      }
      for (int i : groups[g]) { e->m[i]->tune[k] = pick; e->m[i]->generation++; }
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  // restore the members' states (the tiles found are kept)
  for (int i = 0; i < n; ++i) {
    diablo_ctx* c = e->m[i];
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = rc ? rc : DIABLO_ERR_CUDA;
    c->cur = snap[i].cur; c->cf_cur = snap[i].cf_cur; c->time = snap[i].time; c->time_step = snap[i].step;
    const size_t fe = four_elems(c) * sizeof(double2);
    for (int q = 0; q < 4 + c->nth; ++q) {
      cudaMemcpyAsync(c->st[c->cur][q], snap[i].f[q], fe, cudaMemcpyDeviceToDevice, c->stream);
      cudaStreamSynchronize(c->stream);
      for (size_t a = 0; a < c->allocs.size(); ++a)
        if (c->allocs[a] == snap[i].f[q]) { c->allocs.erase(c->allocs.begin() + a); break; }
      cudaFree(snap[i].f[q]);
    }
    if (rc) for (int q = 0; q < 4; ++q) c->tune[q] = snap[i].tune[q];
    c->generation++;
  }
  return rc;
}

}  // extern "C"
