// Context lifetime, device buffers, boundary copies between the reference
// layout and the internal layouts, and the core of the C ABI.
#include "internal.h"
#include "kernels_layout.cuh"
#include "kernels_init.cuh"

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
int dev_alloc(diablo_ctx* ctx, void** p, size_t bytes) {
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

void twiddles(int n, int count, std::vector<double2>& d, std::vector<float2>& f) {
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

int upload_tw(diablo_ctx* ctx, int n, int count, double2** d, float2** f) {
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


int ensure_scratch(diablo_ctx* ctx) {
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

int ensure_bscratch(diablo_ctx* ctx) {
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
int fwd_phys_to_four(diablo_ctx* ctx, const double* phys, double2* xs, double2* four) {
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

int inv_four_to_phys(diablo_ctx* ctx, const double2* four, double2* xs, double* phys) {
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


bool is_device_ptr(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

void fill_solve_args(diablo_ctx* ctx, SolveArgs& a, int rk);
// batched FP64 transforms between the internal Fourier and physical layouts
// Batched transforms between FP64 Fourier arrays and physical arrays of
// element type P (double, or float for the mixed-precision LES model).
template <typename P>
int ifft_batch_t(diablo_ctx* ctx, const double2* const* four, P* const* phys, int nf) {
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
int fft_batch_t(diablo_ctx* ctx, const P* const* phys, double2* const* four, int nf, double acc_scale) {
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
    za.acc_scale = acc_scale;
    int rc;
    { Prof pr(ctx, K_OTHER); if ((rc = launch_xfwd<P, false>(xa, ctx->M, ctx->nyp2, m, ctx->stream))) return rc; }
    { Prof pr(ctx, K_OTHER); if ((rc = launch_zfwd<C, double2, false>(za, ctx->nz, m, ctx->stream))) return rc; }
  }
  return 0;
}

template int ifft_batch_t<double>(diablo_ctx*, const double2* const*, double* const*, int);
template int ifft_batch_t<float>(diablo_ctx*, const double2* const*, float* const*, int);
template int fft_batch_t<double>(diablo_ctx*, const double* const*, double2* const*, int, double);
template int fft_batch_t<float>(diablo_ctx*, const float* const*, double2* const*, int, double);

int ifft_batch(diablo_ctx* ctx, const double2* const* four, double* const* phys, int nf) {
  return ifft_batch_t<double>(ctx, four, phys, nf);
}
int fft_batch(diablo_ctx* ctx, const double* const* phys, double2* const* four, int nf) {
  return fft_batch_t<double>(ctx, phys, four, nf);
}

int les_active(const diablo_ctx* ctx) {
  // for/channel.f90:259: LES only after 100 steps of a newly created flow
  return ctx->p.use_les && (!ctx->p.create_new_flow || ctx->time_step > 100);
}
// ==========================================================================
// C ABI
// The column step's status word: DIABLO_ERR_TIMEOUT (and the word cleared)
// if a bounded device wait gave up since the last check.  Waits for the
// context's stream.
int sched_status(diablo_ctx* ctx) {
  int v = 0;
  CK(cudaMemcpyAsync(&v, ctx->d_sched, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (!v) return 0;
  CK(cudaMemsetAsync(ctx->d_sched, 0, sizeof(int), ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return DIABLO_ERR_TIMEOUT;
}

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
    ctx->use_general_solver = (e && e[0] >= '1' && e[0] <= '3') ? e[0] - '0' : 0;
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
  // column-step scheduler: status, task counter, one count per column group
  ctx->sched_ints = 2 + (size_t)(ctx->nkx1 * ctx->nk2 + FS_COLS - 1) / FS_COLS;
  if ((rc = dev_alloc(ctx, (void**)&ctx->d_sched, ctx->sched_ints * sizeof(int)))) FAIL(rc);
  ctx->wait_spins = 1LL << 24;   // about a second of 100 ns sleeps
  ctx->wait_withhold = 0;
  if ((rc = upload_coefficients(ctx))) FAIL(rc);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) FAIL(DIABLO_ERR_CUDA);
#undef FAIL
  *status = 0;
  return ctx;
}

int diablo_destroy(diablo_ctx* ctx) {
  if (!ctx) return DIABLO_ERR_ARG;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->xfer.ready) {
    diablo_ctx::Xfer& X = ctx->xfer;
    cudaStreamSynchronize(X.up);
    cudaStreamSynchronize(X.down);
    cudaStreamDestroy(X.up);
    cudaStreamDestroy(X.down);
    cudaEventDestroy(X.start);
    for (int f = 0; f < 4 + DIABLO_MAX_TH; ++f) {
      if (X.e_up[f]) cudaEventDestroy(X.e_up[f]);
      if (X.e_conv[f]) cudaEventDestroy(X.e_conv[f]);
      for (int c = 0; c < 4; ++c)
        if (X.e_down[f][c]) cudaEventDestroy(X.e_down[f][c]);
    }
  }
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
extern "C++" int four_in(diablo_ctx* ctx, const double* buf, double2* dst, bool check) {
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
extern "C++" int four_out(diablo_ctx* ctx, const double2* src, double* buf) {
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

// Streams, events and staging arrays of diablo_step_host (once per context).
static int ensure_xfer(diablo_ctx* ctx) {
  diablo_ctx::Xfer& X = ctx->xfer;
  if (X.ready) return 0;
  const int ns = 4 + ctx->nth;
  const size_t stage = (size_t)ctx->nyp2 * ctx->nk2 * (ctx->nxp + 1) * sizeof(double2);
  int rc;
  for (int f = 0; f < ns; ++f) {
    if ((rc = dev_alloc(ctx, (void**)&X.up_stage[f], stage))) return rc;
    if ((rc = dev_alloc(ctx, (void**)&X.down_stage[f], stage))) return rc;
    // the rows' pad entries (i = Nxp) are never written by the packing
    // kernel: zero, as the reference's zeroed modes above Nkx
    CK(cudaMemsetAsync(X.down_stage[f], 0, stage, ctx->stream));
  }
  CK(cudaStreamCreateWithFlags(&X.up, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&X.down, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&X.start, cudaEventDisableTiming));
  for (int f = 0; f < ns; ++f) {
    CK(cudaEventCreateWithFlags(&X.e_up[f], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&X.e_conv[f], cudaEventDisableTiming));
    for (int c = 0; c < 4; ++c) CK(cudaEventCreateWithFlags(&X.e_down[f][c], cudaEventDisableTiming));
  }
  X.ready = 1;
  return 0;
}

int diablo_step_host(diablo_ctx* ctx, double* const* bufs, int nsteps) {
  if (!ctx || !bufs || nsteps < 0) return DIABLO_ERR_ARG;
  const int ns = 4 + ctx->nth;
  for (int f = 0; f < ns; ++f)
    if (!bufs[f] || is_device_ptr(bufs[f])) return DIABLO_ERR_ARG;
  int rc;
  if ((rc = ensure_bscratch(ctx)) || (rc = ensure_xfer(ctx))) return rc;
  diablo_ctx::Xfer& X = ctx->xfer;
  const size_t rowb = (size_t)(ctx->nxp + 1) * sizeof(double2);
  const size_t tot = (size_t)ctx->nyp2 * ctx->nk2 * ctx->nxp;
  // the copy streams start after the work already queued on the context's stream
  CK(cudaEventRecord(X.start, ctx->stream));
  CK(cudaStreamWaitEvent(X.up, X.start, 0));
  CK(cudaStreamWaitEvent(X.down, X.start, 0));
  CK(cudaMemsetAsync(ctx->d_flag, 0, sizeof(int), ctx->stream));
  // Each field moves in four chunks of planes, so that a chunk's upload can
  // follow its own download while the next chunks are still coming back: the
  // pipeline fills and drains by a quarter field, not a whole one.
  constexpr int NCH = 4;
  auto chunk = [&](int c) { return (ctx->nyp2 * c) / NCH; };   // first plane of chunk c
  const size_t hplane = (size_t)(ctx->nz + 2) * (ctx->nxp + 1);  // complex entries per host plane
  const size_t dplane = (size_t)ctx->nk2 * (ctx->nxp + 1);       // ... per staging plane
  for (int s = 0; s < nsteps; ++s) {
    // uploads: each chunk after its own download of the step before
    for (int f = 0; f < ns; ++f) {
      for (int c = 0; c < NCH; ++c) {
        const int j0 = chunk(c), nj = chunk(c + 1) - j0;
        if (nj <= 0) continue;
        if (s > 0) CK(cudaStreamWaitEvent(X.up, X.e_down[f][c], 0));
        CK(cudaMemcpy2DAsync(X.up_stage[f] + (size_t)j0 * dplane, rowb * ctx->nk2,
                             reinterpret_cast<const double2*>(bufs[f]) + (size_t)j0 * hplane,
                             rowb * (ctx->nz + 2), rowb * ctx->nk2, nj, cudaMemcpyHostToDevice, X.up));
      }
      CK(cudaEventRecord(X.e_up[f], X.up));
    }
    for (int f = 0; f < ns; ++f) {
      CK(cudaStreamWaitEvent(ctx->stream, X.e_up[f], 0));
      Prof pr(ctx, K_OTHER);
      k_ref_to_four<<<grid1d(tot), 256, 0, ctx->stream>>>(X.up_stage[f], ctx->st[ctx->cur][f], ctx->g,
                                                           ctx->nxp, ctx->nxp + 1, ctx->nk2, ctx->d_flag);
    }
    if ((rc = one_step(ctx))) return rc;
    // downloads: each field's chunks as soon as the field is packed,
    // overlapping the next step's uploads of the chunks before them
    for (int f = 0; f < ns; ++f) {
      {
        Prof pr(ctx, K_OTHER);
        k_four_to_ref<<<grid1d(tot), 256, 0, ctx->stream>>>(ctx->st[ctx->cur][f], X.down_stage[f], ctx->g,
                                                             ctx->nxp, ctx->nxp + 1, ctx->nk2);
      }
      CK(cudaEventRecord(X.e_conv[f], ctx->stream));
      CK(cudaStreamWaitEvent(X.down, X.e_conv[f], 0));
      // rows k <= 2Nkz of a plane, pad entries included, are contiguous in
      // the host array: 2D copies of such blocks (the upload's form)
      for (int c = 0; c < NCH; ++c) {
        const int j0 = chunk(c), nj = chunk(c + 1) - j0;
        if (nj <= 0) continue;
        CK(cudaMemcpy2DAsync(reinterpret_cast<double2*>(bufs[f]) + (size_t)j0 * hplane, rowb * (ctx->nz + 2),
                             X.down_stage[f] + (size_t)j0 * dplane, rowb * ctx->nk2, rowb * ctx->nk2, nj,
                             cudaMemcpyDeviceToHost, X.down));
        CK(cudaEventRecord(X.e_down[f][c], X.down));
      }
    }
  }
  // the context's stream ends after the last download
  if (nsteps > 0) {
    CK(cudaEventRecord(X.start, X.down));
    CK(cudaStreamWaitEvent(ctx->stream, X.start, 0));
  }
  int bad = 0;
  CK(cudaMemcpyAsync(&bad, ctx->d_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  return bad ? DIABLO_ERR_STATE : 0;
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
  const int rc = substep(ctx, rk_step);
  return rc ? rc : sched_status(ctx);
}

// filter_chan's transfer function applied to scalar n's planes jst..jet of
// the Fourier field f: a real factor per (kx, kz) mode, so the operation is
// its own adjoint (the discrete adjoint applies it to the scalar's lambda)
extern "C++" int filter_field(diablo_ctx* ctx, int n, double2* f) {
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
  k_filter_th<<<grid1d(tot), 256, 0, ctx->stream>>>(f, ctx->d_sigma, j0, j1, ctx->nkx1, ctx->nk2, ctx->kp);
  CK(cudaGetLastError());
  return 0;
}

static int filter_chan(diablo_ctx* ctx, int n) { return filter_field(ctx, n, ctx->st[ctx->cur][4 + n]); }

// scalars filter_scalars filters after the step that brought the counter to
// time_step (for/advance.f90:161-173)
extern "C++" bool filter_due(const diablo_ctx* ctx, int n, int time_step) {
  return ctx->p.filter_th[n] && ctx->p.filter_int[n] > 0 && time_step % ctx->p.filter_int[n] == 0;
}

// filter_scalars (for/advance.f90:161-173), after each step
extern "C++" int filter_scalars(diablo_ctx* ctx) {
  for (int n = 0; n < ctx->nth; ++n)
    if (filter_due(ctx, n, ctx->time_step)) {
      int rc = filter_chan(ctx, n);
      if (rc) return rc;
    }
  return 0;
}

int diablo_filter_chan(diablo_ctx* ctx, int n) {
  if (!ctx || n < 0 || n >= ctx->nth) return DIABLO_ERR_ARG;
  return filter_chan(ctx, n);
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
  return sched_status(ctx);
}

extern "C++" int bc_post(diablo_ctx* ctx, int do_vel, int do_th) {
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
  return sched_status(ctx);
}

int diablo_set_wait_bound(diablo_ctx* ctx, long long max_spins, int withheld_arrivals) {
  if (!ctx || max_spins < 1 || withheld_arrivals < 0) return DIABLO_ERR_ARG;
  ctx->wait_spins = max_spins;
  ctx->wait_withhold = withheld_arrivals;
  ctx->generation++;   // captured kernel arguments change
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

