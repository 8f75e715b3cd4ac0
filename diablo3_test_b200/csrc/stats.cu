// Plane statistics (save_stats_chan, for/statistics.f90:44-712).
#include "internal.h"
#include "kernels_stats.cuh"
#include "kernels_layout.cuh"

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
  // flag_save_LES: eps_sgs1 is formed at the next step's first substep
  // (for/control.f90:95, for/les.f90:924)
  if (p.use_les) {
    ctx->les.eps_req = 1;
    ctx->les.eps_ready = 0;
  }
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
  const size_t n_spec = even((size_t)nyp2 * nkx1), n_les = even((size_t)nyp2 * lslice * STAT_LQ);
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
    // kappa_t: the AMD scalar model's own (model 5, in the LES precision),
    // else nu_t (for/les.f90:1130-1146)
    b.nth = nth;
    const bool amd = p.les_model_type == 5;
    b.kap32 = (amd && L.nu_t_fp32) ? 1 : 0;
    for (int n = 0; n < nth; ++n) b.kap[n] = amd ? (const void*)L.kap[n] : (const void*)nt;
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
    for (int sl = 0; sl < lslice; ++sl) s += lpart[((size_t)j * lslice + sl) * STAT_LQ + q];
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
      tset(DIABLO_STAT_KAPPA_SGS, j, les ? LQ(j, 2 + n) / nn : 0.0);
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

