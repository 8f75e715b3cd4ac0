// The RK3/Crank-Nicolson substep of DNS (rk_chan_1, for/channel.f90:10-917):
// implicit-row coefficients, transforms, nonlinear terms and the column
// kernel schedule; courant (variable dt) and poisson_p_chan.
#include "internal.h"
#include "kernels_init.cuh"
#include "kernels_field.cuh"


// --------------------------------------------------------------------------
// Row coefficients of the implicit solves, evaluated with the reference's
// expressions (for/channel.f90:664-670 scalars, :726-733 u2, :782-788 and
// :838-845 u1/u3, :969-976 rem_div), for each RK substep.
int upload_coefficients(diablo_ctx* ctx) {
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

void fill_solve_args(diablo_ctx* ctx, SolveArgs& a, int rk) {
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
void update_transient(diablo_ctx* ctx) {
  const diablo_params& p = ctx->p;
  if (p.w_bc_ymax != 0 && p.f_type == 4)
    ctx->w_top_transient = p.w_bc_ymax_c1 + p.amp_omega0 *
        sin(p.omega0 * (ctx->ro_inv / p.delta * ctx->time - p.force_start));
}

// mean_mask: fields whose (0,0) mode (the mean profile) stays out of the
// physical fields; its products are added in FP64 further on.
template <typename T>
int spectral_inverse(diablo_ctx* ctx, unsigned mean_mask) {
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
int spectral_nl(diablo_ctx* ctx, bool mean_free_u1) {
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
int substep_spectral(diablo_ctx* ctx, unsigned mean_mask) {
  int rc = spectral_inverse<T>(ctx, mean_mask);
  return rc ? rc : spectral_nl<T>(ctx, (mean_mask & 1u) != 0);
}

template int spectral_inverse<double>(diablo_ctx*, unsigned);
template int spectral_inverse<float>(diablo_ctx*, unsigned);
template int spectral_nl<double>(diablo_ctx*, bool);
template int spectral_nl<float>(diablo_ctx*, bool);
template int substep_spectral<double>(diablo_ctx*, unsigned);
template int substep_spectral<float>(diablo_ctx*, unsigned);

// courant (for/advance.f90:47-158) from the velocities u (physical FP64,
// planes 1..Ny): the new delta_t and RK coefficients for the steps that follow.
int ensure_cfl(diablo_ctx* ctx) {
  if (ctx->d_cfl) return 0;
  int rc;
  for (int q = 0; q < 3; ++q) {
    if ((rc = dev_alloc(ctx, (void**)&ctx->ustar[q], four_elems(ctx) * sizeof(double2)))) return rc;
    if ((rc = dev_alloc(ctx, (void**)&ctx->cfl_phys[q], phys_elems(ctx) * sizeof(double)))) return rc;
  }
  return dev_alloc(ctx, (void**)&ctx->d_cfl, (size_t)5 * ctx->nyp2 * sizeof(double));
}

int courant_phys(diablo_ctx* ctx, const double* const* u) {
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

int courant_four(diablo_ctx* ctx, double2* const* cu) {
  int rc;
  if ((rc = ensure_xs64(ctx)) || (rc = ensure_cfl(ctx))) return rc;
  if ((rc = ifft_batch(ctx, cu, ctx->cfl_phys, 3))) return rc;
  return courant_phys(ctx, ctx->cfl_phys);
}

bool courant_due(const diablo_ctx* ctx, int rk) {
  return ctx->p.variable_dt && rk == 3 && ctx->p.update_dt > 0 && ctx->time_step % ctx->p.update_dt == 0;
}

// poisson_p_chan (for/channel.f90:1026-1234): cp from the current velocity
// (and scalars), FP64; its work arrays live only for the call.
int poisson_p(diablo_ctx* ctx) {
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

int substep(diablo_ctx* ctx, int rk) {
  if (les_active(ctx)) {
    const int m = ctx->p.les_model_type;
    if (m != 1 && m != 2 && m != 4 && m != 5) return DIABLO_ERR_UNSUPPORTED;
    return substep_les(ctx, rk);
  }
  // LES gated off (a new flow's first 100 steps): a pending LES statistics
  // request is answered with blanks (for/channel.f90:271-274)
  if (ctx->p.use_les && rk == 1 && ctx->les.eps_req) {
    ctx->les.eps_req = 0;
    ctx->les.eps_ready = 1;
    ctx->les.eps_blank = 1;
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
  const bool tiled = !a.front && ctx->use_general_solver != 1;
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
  const bool cfl = courant_due(ctx, rk);
  if (cfl && (rc = ensure_cfl(ctx))) return rc;
  if (tiled && (ctx->use_general_solver == 0 || ctx->use_general_solver >= 3)) {
    // default: the field-split column step (kernels_field.cuh)
    FieldArgs F;
    memset(&F, 0, sizeof(F));
    F.s = a;
    if (mean_split) { F.s.nl64[0] = (const double2*)ctx->nl[0]; F.s.nl32[0] = nullptr; }
    if (cfl)
      for (int q = 0; q < 3; ++q) F.s.keep[q] = ctx->ustar[q];
    F.kc = ctx->d_kc[rk - 1];
    F.met = ctx->d_met;
    F.fac = ctx->d_fac[rk - 1];
    F.nf = ctx->nf;
    F.mean_split = mean_split ? 1 : 0;
    F.prof = ctx->d_prof;
    // Two launches (field solves, then projections) by default.  The single
    // launch (k_column_step: both, with a bounded wait per column group) is
    // opt-in: it measured slower at 256 x 257 x 256 (0.71 against 0.59 ms
    // per substep, mixed) and for the 64 x 97 x 64 adjoint case (13.9 against
    // 12.5 ms for 50 steps), and equal on the 48-member ensemble.
    if (ctx->defer_col) {
      // ensemble capture: the ensemble launches this column step with the
      // other members' (k_column_step_ens); lag is set there
      if (cfl) return DIABLO_ERR_UNSUPPORTED;
      F.sched = ctx->d_sched;
      F.need = 3 + ctx->wait_withhold;
      F.max_spins = ctx->wait_spins;
      *ctx->defer_col = F;
      ctx->defer_filled = 1;
    } else if (ctx->use_general_solver == 3) {
      const int resident = column_step_resident(ctx->nyp2);
      F.sched = ctx->d_sched;
      F.need = 3 + ctx->wait_withhold;
      F.max_spins = ctx->wait_spins;
      F.lag = std::max(1, resident / ctx->nf);
      CK(cudaMemsetAsync(ctx->d_sched + 1, 0, (ctx->sched_ints - 1) * sizeof(int), ctx->stream));
      Prof pr(ctx, K_SOLVE);
      if ((rc = launch_column_step(F, ctx->stream))) return rc;
    } else {
      {
        Prof pr(ctx, K_SOLVE);
        if ((rc = launch_field_solve(F, ctx->stream))) return rc;
      }
      {
        Prof pr(ctx, K_PROJ);
        if ((rc = launch_project_cols(F, ctx->stream))) return rc;
      }
    }
    CK(cudaGetLastError());
    ctx->cur = nx_;
    if (a.store_cf) ctx->cf_cur = 1 - ctx->cf_cur;
    if (cfl) return courant_four(ctx, ctx->ustar);
    return 0;
  }
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

