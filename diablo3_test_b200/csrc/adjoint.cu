// Discrete adjoint of diablo_step with checkpoint-and-recompute.
#include "internal.h"
#include "kernels_adjoint.cuh"

// ==========================================================================
// Discrete adjoint of diablo_step (DNS with velocities and scalars, FP64),
// with checkpoint-and-recompute: diablo_adjoint_record stores the state every
// `every` steps; diablo_adjoint_run recomputes each segment from its
// checkpoint (keeping the velocities entering every substep) and runs the
// substep adjoints backwards through it.

// Warps (columns) per block of the adjoint column kernels.  The adjoint
// workload's grids are small (946 columns at 64 x 97 x 64): fewer warps per
// block spread the columns over more SMs.
#ifndef ADJ_COLUMN_WARPS
#define ADJ_COLUMN_WARPS 2
#endif

int adj_free(diablo_ctx* ctx) {
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
  T.sub_seg = -1;
  return 0;
}

// host-built rows of the substep systems (the forward's expressions)
void adj_rows(diablo_ctx* ctx, std::vector<double>& cn, std::vector<double>& rmask,
                     std::vector<double>& pa) {
  const diablo_params& p = ctx->p;
  const int n = ctx->nyp2, nyp = ctx->ny, nfs = 3 + ctx->nth;
  const std::vector<double>& dy = ctx->h_dy;
  const std::vector<double>& dyf = ctx->h_dyf;
  cn.assign((size_t)3 * nfs * 3 * n, 0.0);
  rmask.assign((size_t)nfs * n, 0.0);
  pa.assign((size_t)3 * n, 0.0);
  for (int j = 2; j <= nyp - 1; ++j) {
    pa[j] = 1. / (dy[j] * dyf[j]);
    pa[n + j] = 1. / (dy[j + 1] * dyf[j]);
    pa[2 * n + j] = -1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]);
  }
  for (int rk = 0; rk < 3; ++rk) {
    for (int f = 0; f < nfs; ++f) {
      // scalar s = f - 3: diffusivity nu/Pr, rows jstart_th..jend_th and the
      // wall rows of apply_bc_th (for/channel.f90:657-707, 1797-1876)
      const int s = f - 3;
      const double tc = 0.5 * ctx->nu * ctx->h_bar[rk] * p.nu_v_scale / (s >= 0 ? p.pr[s] : 1.0);
      double* A = &cn[((size_t)rk * nfs + f) * 3 * n];
      double* B = A + n;
      double* C = B + n;
      double* rm = &rmask[(size_t)f * n];
      for (int j = 0; j < n; ++j) { A[j] = 0.0; B[j] = 1.0; C[j] = 0.0; }
      if (f != 1) {
        const int j0 = s >= 0 ? ctx->jst[s] : ctx->jstart, j1 = s >= 0 ? ctx->jet[s] : ctx->jend;
        for (int j = j0; j <= j1; ++j) {
          A[j] = -tc / (dy[j] * dyf[j]);
          B[j] = 1. - tc * (-1. / (dy[j + 1] * dyf[j]) - 1. / (dy[j] * dyf[j]));
          C[j] = -tc / (dy[j + 1] * dyf[j]);
          rm[j] = 1.0;
        }
        const int bmin = s >= 0 ? p.th_bc_ymin[s] : (f == 0 ? p.u_bc_ymin : p.w_bc_ymin);
        const int bmax = s >= 0 ? p.th_bc_ymax[s] : (f == 0 ? p.u_bc_ymax : p.w_bc_ymax);
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

int adj_supported(const diablo_ctx* ctx) {
  if (ctx->p.use_les || ctx->precision != DIABLO_FP64 || ctx->p.variable_dt) return DIABLO_ERR_UNSUPPORTED;
  return 0;
}

int adj_alloc(diablo_ctx* ctx, int nsteps, int every) {
  diablo_ctx::Tape& T = ctx->tape;
  const size_t fe = four_elems(ctx) * sizeof(double2), pe = phys_elems(ctx) * sizeof(double);
  int rc;
  // the checkpoint and substep buffers are kept while nsteps and every stay the same
  if (T.ckpt.empty() || T.nsteps != nsteps || T.every != every) {
    adj_free(ctx);
    T.nsteps = nsteps;
    T.every = every;
    T.nseg = (nsteps + every - 1) / every;
    T.ckpt.assign((size_t)(T.nseg + 1) * (4 + ctx->nth), nullptr);
    for (auto& p : T.ckpt) if ((rc = dev_alloc(ctx, (void**)&p, fe))) return rc;
    T.sub.assign((size_t)every * 3 * (3 + ctx->nth), nullptr);
    for (auto& p : T.sub) if ((rc = dev_alloc(ctx, (void**)&p, fe))) return rc;
    T.ckpt_step.assign(T.nseg + 1, 0);
    T.ckpt_time.assign(T.nseg + 1, 0.0);
  }
  T.ready = 0;
  T.sub_seg = -1;
  if (!T.work_ready) {
#define AL(ptr, bytes) if ((rc = dev_alloc(ctx, (void**)&(ptr), (bytes)))) return rc
    const int nfs = 3 + ctx->nth;
    for (int q = 0; q < nfs + 1; ++q) { AL(T.lu[q], fe); AL(T.ou[q], fe); }
    for (int q = 0; q < nfs; ++q) { AL(T.lF[q], fe); AL(T.oF[q], fe); AL(T.lnl[q], fe);
                                    AL(T.up[q], pe); AL(T.lp3[q], pe); }
    for (int q = 0; q < 8 + 3 * ctx->nth; ++q) { AL(T.pf[q], fe); AL(T.pp[q], pe); }
    AL(T.d_cn, (size_t)9 * nfs * ctx->nyp2 * sizeof(double));
    AL(T.d_rmask, (size_t)nfs * ctx->nyp2 * sizeof(double));
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

int copy_fields(diablo_ctx* ctx, double2* const* dst, double2* const* src, int nf) {
  const size_t fe = four_elems(ctx) * sizeof(double2);
  for (int q = 0; q < nf; ++q) CK(cudaMemcpyAsync(dst[q], src[q], fe, cudaMemcpyDeviceToDevice, ctx->stream));
  return 0;
}

// Adjoint of substep rk: T.lu (lambda of the substep's output state) and
// T.lF (lambda of its cf) become the lambdas of its input; u_in are the
// velocities and scalars that entered the substep (u1, u2, u3, th..).
int adj_substep(diablo_ctx* ctx, int rk, double2* const* u_in) {
  diablo_ctx::Tape& T = ctx->tape;
  const diablo_params& p = ctx->p;
  const double h = ctx->h_bar[rk - 1];
  const FGeom fg{ctx->ny, ctx->nyp2, ctx->nkx1, ctx->nk2, ctx->kp, (size_t)ctx->nkx1 * ctx->kp};
  const size_t ftot = four_elems(ctx), ptot = phys_elems(ctx);
  const int nth = ctx->nth, nfs = 3 + nth;
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
    a.cn = T.d_cn + (size_t)(rk - 1) * nfs * 3 * ctx->nyp2;
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
    const int warps = ADJ_COLUMN_WARPS;
    dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
    switch (rows_per_lane(ctx->nyp2)) {
#define X(r) case r: k_adj_column<r><<<grd, blk, 0, ctx->stream>>>(a); break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: return DIABLO_ERR_SIZE;
    }
  }
  for (int s = 0; s < nth; ++s) {
    // one scalar per launch: each adds its background-gradient terms to lambda u1, u3
    AdjScalarArgs a;
    memset(&a, 0, sizeof(a));
    a.lth = T.lu[4 + s];
    a.lF = rk < 3 ? T.lF[3 + s] : nullptr;
    for (int f = 0; f < 3; ++f) a.vnl[f] = T.lnl[f];
    a.oth = T.ou[4 + s];
    a.oF = rk > 1 ? T.oF[3 + s] : nullptr;
    a.onl = T.lnl[3 + s];
    a.ou1 = T.ou[0]; a.ou3 = T.ou[2];
    a.cn = T.d_cn + ((size_t)(rk - 1) * nfs + 3 + s) * 3 * ctx->nyp2;
    a.rmask = T.d_rmask + (size_t)(3 + s) * ctx->nyp2;
    a.kx = ctx->d_kx; a.kz = ctx->d_kz; a.dy = ctx->d_dy; a.dyf = ctx->d_dyf;
    a.t3 = ZETA_BAR[rk - 1] * h; a.t5 = BETA_BAR[rk - 1] * h;
    a.tc = 0.5 * ctx->nu * h * p.nu_v_scale / p.pr[s];
    a.nu_pr = ctx->nu / p.pr[s]; a.beta = p.beta;
    a.gx = p.grav_x; a.gy = p.grav_y; a.gz = p.grav_z;
    a.dthdx = p.dthdx[s]; a.dthdz = p.dthdz[s];
    a.n = ctx->nyp2; a.nyp = ctx->ny; a.nkx1 = ctx->nkx1; a.nk2 = ctx->nk2; a.kp = ctx->kp;
    a.ncol = ctx->nkx1 * ctx->nk2;
    a.jst = ctx->jst[s]; a.jet = ctx->jet[s];
    Prof pr(ctx, K_OTHER);
    const int warps = ADJ_COLUMN_WARPS;
    dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
    switch (rows_per_lane(ctx->nyp2)) {
#define X(r) case r: k_adj_scalar<r><<<grd, blk, 0, ctx->stream>>>(a); break;
      X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
      default: return DIABLO_ERR_SIZE;
    }
  }
  if (p.flavor_front && ctx->ro_inv != 0.0 && nth > 0) {
    // thermal-wind advection (for/forcing.f90:37-113), after every lambda cf
    // of this substep is known
    AdjFrontArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < 3; ++f) { a.onl[f] = T.lnl[f]; a.ou[f] = T.ou[f]; }
    for (int s = 0; s < nth; ++s) {
      a.onl[3 + s] = T.lnl[3 + s]; a.ou[3 + s] = T.ou[4 + s];
      a.dthdx[s] = p.dthdx[s]; a.dthdz[s] = p.dthdz[s];
    }
    a.kx = ctx->d_kx; a.kz = ctx->d_kz; a.gy = ctx->d_gy; a.gyf = ctx->d_gyf;
    a.ly = p.ly; a.coef = p.delta / ctx->ro_inv;
    a.nth = nth; a.n = ctx->nyp2; a.nkx1 = ctx->nkx1; a.nk2 = ctx->nk2; a.kp = ctx->kp;
    Prof pr(ctx, K_OTHER);
    k_adj_front<<<grid1d((size_t)ctx->nyp2 * ctx->nkx1 * ctx->kp), 256, 0, ctx->stream>>>(a);
  }
  const int nprod = 8 + 3 * nth;
  {
    AdjNlPrepArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < nfs; ++f) a.lnl[f] = T.lnl[f];
    for (int q = 0; q < nprod; ++q) a.out[q] = T.pf[q];
    a.kx = ctx->d_kx; a.kz = ctx->d_kz;
    a.inv = 1.0 / ((double)ctx->nx * ctx->nz);
    a.g = fg;
    a.nth = nth;
    Prof pr(ctx, K_OTHER);
    k_adj_nl_prep<<<grid1d(ftot), 256, 0, ctx->stream>>>(a);
  }
  {
    // the product adjoints and the substep's input fields in one batch
    const double2* src[8 + 3 * DIABLO_MAX_TH + 3 + DIABLO_MAX_TH];
    double* dst[8 + 3 * DIABLO_MAX_TH + 3 + DIABLO_MAX_TH];
    for (int q = 0; q < nprod; ++q) { src[q] = T.pf[q]; dst[q] = T.pp[q]; }
    for (int q = 0; q < nfs; ++q) { src[nprod + q] = u_in[q]; dst[nprod + q] = T.up[q]; }
    if ((rc = ifft_batch(ctx, src, dst, nprod + nfs))) return rc;
  }
  {
    AdjNlPointArgs a;
    memset(&a, 0, sizeof(a));
    for (int q = 0; q < nprod; ++q) a.P[q] = T.pp[q];
    a.u1 = T.up[0]; a.u2 = T.up[1]; a.u3 = T.up[2];
    a.o1 = T.lp3[0]; a.o2 = T.lp3[1]; a.o3 = T.lp3[2];
    for (int s = 0; s < nth; ++s) { a.th[s] = T.up[3 + s]; a.oth[s] = T.lp3[3 + s]; }
    a.dy = ctx->d_dy; a.dyf = ctx->d_dyf;
    a.nyp = ctx->ny;
    a.nth = nth;
    a.ps = (size_t)ctx->nz * ctx->nx;
    Prof pr(ctx, K_OTHER);
    k_adj_nl_point<<<grid1d(ptot), 256, 0, ctx->stream>>>(a);
  }
  {
    // ou += w(m) Nx Nz F(lambda physical): the inverse transform's transpose,
    // accumulated by the z forward transform itself
    double2* acc[3 + DIABLO_MAX_TH];
    for (int f = 0; f < 3; ++f) acc[f] = T.ou[f];
    for (int s = 0; s < nth; ++s) acc[3 + s] = T.ou[4 + s];
    if ((rc = fft_batch_t<double>(ctx, T.lp3, acc, nfs, (double)ctx->nx * ctx->nz))) return rc;
  }
  CK(cudaGetLastError());
  for (int q = 0; q < nfs + 1; ++q) std::swap(T.lu[q], T.ou[q]);
  for (int q = 0; q < nfs; ++q) std::swap(T.lF[q], T.oF[q]);
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
  const int ns = 4 + ctx->nth, nfs = 3 + ctx->nth;   // u1, u2, u3, p, th..
  const int slast = (T.nseg - 1) * every;             // first step of the last segment
  for (int s = 0; s < nsteps; ++s) {
    if (s % every == 0) {
      const int k = s / every;
      if ((rc = copy_fields(ctx, &T.ckpt[(size_t)k * ns], ctx->st[ctx->cur], ns))) return rc;
      T.ckpt_step[k] = ctx->time_step;
      T.ckpt_time[k] = ctx->time;
    }
    if (s < slast) {
      if ((rc = one_step(ctx)) || (rc = filter_scalars(ctx))) return rc;
      continue;
    }
    // the last segment keeps each substep's input fields as it goes, so that
    // the adjoint starts on it without recomputing it
    ctx->time_step += 1;
    for (int rk = 1; rk <= 3; ++rk) {
      double2* cu[3 + DIABLO_MAX_TH];
      for (int q = 0; q < 3; ++q) cu[q] = ctx->st[ctx->cur][q];
      for (int q = 0; q < ctx->nth; ++q) cu[3 + q] = ctx->st[ctx->cur][4 + q];
      if ((rc = copy_fields(ctx, &T.sub[((size_t)(s - slast) * 3 + (rk - 1)) * nfs], cu, nfs))) return rc;
      if ((rc = substep(ctx, rk))) return rc;
    }
    ctx->time += ctx->delta_t;
    if ((rc = filter_scalars(ctx))) return rc;
  }
  T.sub_seg = T.nseg - 1;
  if ((rc = copy_fields(ctx, &T.ckpt[(size_t)T.nseg * ns], ctx->st[ctx->cur], ns))) return rc;
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
  const int ns = 4 + ctx->nth, nfs = 3 + ctx->nth;
  for (int q = 0; q < ns; ++q) if (!lam[q]) return DIABLO_ERR_ARG;
  diablo_ctx::Tape& T = ctx->tape;
  if (!T.ready || ctx->time_step != T.step_end || ctx->generation != T.gen_end) return DIABLO_ERR_STATE;
  int rc;
  if ((rc = ensure_bscratch(ctx))) return rc;
  const size_t fe = four_elems(ctx) * sizeof(double2);
  for (int q = 0; q < ns; ++q)
    if ((rc = four_in(ctx, lam[q], T.lu[q], false))) return rc;
  for (int q = 0; q < nfs; ++q) CK(cudaMemsetAsync(T.lF[q], 0, fe, ctx->stream));
  for (int k = T.nseg - 1; k >= 0; --k) {
    // recompute the segment from its checkpoint, keeping each substep's input
    // velocities and scalars (the segment whose inputs `sub` already holds --
    // the last one, straight after the record -- is not recomputed)
    const int s0 = k * T.every, s1 = std::min(T.nsteps, s0 + T.every);
    if (T.sub_seg != k) {
      if ((rc = copy_fields(ctx, ctx->st[ctx->cur], &T.ckpt[(size_t)k * ns], ns))) return rc;
      ctx->time_step = T.ckpt_step[k];
      ctx->time = T.ckpt_time[k];
      for (int s = s0; s < s1; ++s) {
        ctx->time_step += 1;
        for (int rk = 1; rk <= 3; ++rk) {
          double2** keep = &T.sub[((size_t)(s - s0) * 3 + (rk - 1)) * nfs];
          double2* cu[3 + DIABLO_MAX_TH];
          for (int q = 0; q < 3; ++q) cu[q] = ctx->st[ctx->cur][q];
          for (int q = 0; q < ctx->nth; ++q) cu[3 + q] = ctx->st[ctx->cur][4 + q];
          if ((rc = copy_fields(ctx, keep, cu, nfs))) return rc;
          if ((rc = substep(ctx, rk))) return rc;
        }
        ctx->time += ctx->delta_t;
        if ((rc = filter_scalars(ctx))) return rc;
      }
      T.sub_seg = k;
    }
    for (int s = s1 - 1; s >= s0; --s) {
      // the scalar filter that ended step s (a real factor per mode, its own
      // transpose) acts on the scalar lambdas first
      const int ts = T.ckpt_step[k] + (s - s0) + 1;
      for (int n = 0; n < ctx->nth; ++n)
        if (filter_due(ctx, n, ts) && (rc = filter_field(ctx, n, T.lu[4 + n]))) return rc;
      for (int rk = 3; rk >= 1; --rk)
        if ((rc = adj_substep(ctx, rk, &T.sub[((size_t)(s - s0) * 3 + (rk - 1)) * nfs]))) return rc;
    }
  }
  // back to the recorded final state
  if ((rc = copy_fields(ctx, ctx->st[ctx->cur], &T.ckpt[(size_t)T.nseg * ns], ns))) return rc;
  ctx->time_step = T.step_end;
  ctx->time = T.time_end;
  for (int q = 0; q < ns; ++q)
    if ((rc = four_out(ctx, T.lu[q], lam[q]))) return rc;
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return 0;
}

}  // extern "C"

