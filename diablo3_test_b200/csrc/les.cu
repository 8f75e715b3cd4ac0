// LES substep (les_chan / les_chan_th, for/les.f90:20-1412) and the dynamic
// Smagorinsky coefficient.
#include "internal.h"
#include "kernels_les.cuh"
#include "kernels_layout.cuh"

// ==========================================================================
// LES substep (FP64): the reference's physical-space path, for/channel.f90
// :29-911 with les_chan/les_chan_th (for/les.f90:20-1200)

static const double LES_C_SMAG = 0.17;   // for/les.f90:38
static const double LES_BETA = 3.0;      // for/les.f90:58
static const double LES_C_AMD = 0.2887;  // for/les.f90:42

// FP64 x-spectral scratch of the batched transforms (LES and adjoint)
int ensure_xs64(diablo_ctx* ctx) {
  diablo_ctx::Les& L = ctx->les;
  if (L.xs[0]) return 0;
  for (int i = 0; i < NF_MAX; ++i) {
    int rc = dev_alloc(ctx, (void**)&L.xs[i], xs_elems(ctx) * sizeof(double2));
    if (rc) return rc;
  }
  return 0;
}

int ensure_les(diablo_ctx* ctx) {
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
  AL(L.d_eps, n * sizeof(double));
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


template <typename P>
int dynamic_coefficient(diablo_ctx* ctx);

int ensure_amd(diablo_ctx* ctx) {
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

int ensure_cfl(diablo_ctx* ctx);
int courant_phys(diablo_ctx* ctx, const double* const* u);
bool courant_due(const diablo_ctx* ctx, int rk);

// batched transforms of LES work arrays (allocated as FP64, used as P)
template <typename P>
int ifft_to(diablo_ctx* ctx, double2* const* four, double* const* phys, int nf) {
  P* d[64];
  for (int f = 0; f < nf; ++f) d[f] = reinterpret_cast<P*>(phys[f]);
  return ifft_batch_t<P>(ctx, four, d, nf);
}
template <typename P>
int fft_from(diablo_ctx* ctx, double* const* phys, double2* const* four, int nf) {
  const P* sp[64];
  for (int f = 0; f < nf; ++f) sp[f] = reinterpret_cast<const P*>(phys[f]);
  return fft_batch_t<P>(ctx, sp, four, nf);
}

template <typename P>
int substep_les_t(diablo_ctx* ctx, int rk) {
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
  if ((rc = spectral_inverse<P>(ctx, 0u))) return rc;            // u, th -> ctx->phys
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
  // eps_sgs1 after a statistics save, from the stresses just formed and the
  // state with the LES wall values (for/les.f90:924-1068)
  if (rk == 1 && L.eps_req) {
    EpsSgsArgs ea;
    for (int q = 0; q < 3; ++q) ea.cu[q] = ctx->st[c][q];
    for (int i = 0; i < 7; ++i) ea.T[i] = L.T[i];
    ea.kx = ctx->d_kx; ea.kz = ctx->d_kz; ea.dyf = ctx->d_dyf;
    ea.sf = L.d_sclf; ea.sg = L.d_sclg; ea.g = fg; ea.out = L.d_eps;
    {
      Prof pr(ctx, K_OTHER);
      k_eps_sgs1<<<ctx->nyp2, EPS_THREADS, 0, ctx->stream>>>(ea);
    }
    L.eps_req = 0;
    L.eps_ready = 1;
    L.eps_blank = 0;
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
  if ((rc = spectral_nl<P>(ctx, false))) return rc;
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

int ensure_dyn(diablo_ctx* ctx) {
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
int dynamic_coefficient(diablo_ctx* ctx) {
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

// mixed precision: the LES model and its transforms in FP32, the
// Crank-Nicolson solves, projection and state in FP64
int diablo_les_eps_sgs1(diablo_ctx* ctx, double* out, int len) {
  if (!ctx || !out || len < ctx->ny) return DIABLO_ERR_ARG;
  diablo_ctx::Les& L = ctx->les;
  if (!L.eps_ready) return DIABLO_ERR_STATE;
  if (L.eps_blank) {
    for (int j = 0; j < ctx->ny; ++j) out[j] = 0.0;
    return 0;
  }
  std::vector<double> h(ctx->nyp2);
  CK(cudaMemcpyAsync(h.data(), L.d_eps, ctx->nyp2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  // plane sums over the retained modes are already plane means
  for (int j = 1; j <= ctx->ny; ++j) out[j - 1] = h[j];
  return 0;
}

int substep_les(diablo_ctx* ctx, int rk) {
  return ctx->precision == DIABLO_FP64 ? substep_les_t<double>(ctx, rk) : substep_les_t<float>(ctx, rk);
}
