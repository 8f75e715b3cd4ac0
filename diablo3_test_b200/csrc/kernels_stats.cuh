// Plane statistics of save_stats_chan (for/statistics.f90:44-712) for the
// x-homogeneous case, FP64.
//
// Every statistic the reference forms as a plane average of a product of two
// (spectrally or finite-difference derived) fields is evaluated here from the
// Fourier coefficients by Parseval's identity instead of transforming the
// fields to physical space: for fields f, g with packed coefficients F, G on
// modes kx <= Nkx, |kz| <= Nkz,
//   (1/(Nx Nz)) sum_{i,k} f g = sum_{m, kq} w(m) Re(F conj G),  w(0) = 1, w(m>0) = 2.
// The physical transform keeps only the Hermitian part of the kx = 0 column
// (the C2R x-transform ignores the anti-Hermitian part), so kx = 0
// coefficients are read as (F(kq) + conj F(-kq)) / 2.  A fluctuation about
// the plane mean is the field with its (0,0) coefficient removed.
//
// One pass reads the state once (three planes of each velocity and scalar
// per plane through L2) and writes per-block partial sums; the host adds the
// partials in a fixed order, so the result is deterministic.
#pragma once
#include "common.cuh"

constexpr int STAT_NQV = 12;   // velocity accumulators
constexpr int STAT_NQT = 3;    // accumulators per scalar
constexpr int STAT_NQ = STAT_NQV + STAT_NQT * DIABLO_MAX_TH;
constexpr int STAT_THREADS = 256;

// velocity accumulator slots
enum {
  SQ_UU = 0,   // <u1'^2>                          compute_TKE (:1296-1312)
  SQ_VV,       // <u2'^2>
  SQ_WW,       // <u3'^2>
  SQ_UW,       // <u1' u3'>                        compute_TKE_Production (:1413-1423)
  SQ_UV,       // <I(u1') u2'> on GY, j >= 2         (:1425-1447)
  SQ_WV,       // <I(u3') u2'> on GY, j >= 2
  SQ_SHEAR,    // <(du1/dy)^2 + (du3/dy)^2>, central (:159-171)
  SQ_OX,       // <(omega_x - tws)^2>              compute_Vorticity (:1557-1573)
  SQ_OY,       // <omega_y^2>                      (:1607-1620)
  SQ_OZ,       // <omega_z^2>                      (:1654-1668)
  SQ_EPS,      // sum of the nine gradient squares, j >= 2   compute_TKE_diss (:859-1062)
  SQ_U1YL      // z-mean of u1 at x = 0 (before the gyf(j) factor) (:420-426)
};

struct StatsArgs {
  const double2* cu[3];
  const double2* cth[DIABLO_MAX_TH];
  const double2* cp;
  const double* kx;
  const double* kz;
  const double* dy;
  const double* dyf;
  const double* gy;
  const double* gyf;
  double dthdx[DIABLO_MAX_TH], dthdz[DIABLO_MAX_TH];
  double tws;           // thermal-wind shear (1/(Ro_inv/delta)) dTHdX(1)
  int nth, nyp, nkx1, nk2, kp, nslice;
  // x-inhomogeneous branch (IC types 5-8): `rowmean` takes fluctuations about
  // the z-line means, i.e. drops the whole kz = 0 row instead of the (0,0)
  // mode; `kstart1` leaves the kz = 0 row out of epsilon's x derivatives
  int rowmean, kstart1;
  size_t ps;
  double* part;         // [Ny+2][nslice][STAT_NQ]
  double* means;        // [Ny+2][4 + nth]: Re of the (0,0) coefficient of u1 u2 u3 p th_n
  double* spec;         // [Ny+2][Nkx+1]: |u1(kx, kz = 0)|^2
  double2* rows;        // [Ny+2][3 + nth][Nkx+1]: the kz = 0 rows (Hermitian part at kx = 0)
};

HDI double nrm2(double2 a) { return a.x * a.x + a.y * a.y; }
HDI double re_dot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

// Sum `v[q]` (q < nq) over the block; thread 0 stores the totals to out[q].
template <int NQ>
__device__ inline void block_sum_store(double (&v)[NQ], int nq, double* out) {
  __shared__ double red[NQ][STAT_THREADS / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    if (q < nq) {
      double s = v[q];
      for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
      if (lane == 0) red[q][w] = s;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[q][k];
    out[q] = s;
  }
}

// NT: scalar capacity of the instance (nth <= NT), so the register file holds
// only the accumulators in use
template <int NT>
__global__ void __launch_bounds__(STAT_THREADS) k_stats_modes(const __grid_constant__ StatsArgs a) {
  constexpr int NQ = STAT_NQV + STAT_NQT * NT;
  const int j = blockIdx.y;
  const int nyp = a.nyp;
  const int nmodes = a.nkx1 * a.nk2;
  const size_t ps = a.ps;
  const int nq = STAT_NQV + STAT_NQT * a.nth;
  double acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
  const bool inner = j >= 1 && j <= nyp;
  const double dyj = a.dy[j], dyfj = a.dyf[j];
  const double dyfm = j >= 1 ? a.dyf[j - 1] : 0.0;
  const double dgy = inner && j >= 2 ? a.gy[j + 1] - a.gy[j - 1] : 1.0;
  const double dgyf = inner ? a.gyf[j + 1] - a.gyf[j - 1] : 1.0;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nmodes; idx += a.nslice * blockDim.x) {
    const int m = idx / a.nk2, kq = idx - m * a.nk2;
    const bool m0 = m == 0, is00 = m0 && kq == 0;
    const int kqm = kq == 0 ? 0 : a.nk2 - kq;
    const size_t col = (size_t)m * a.kp;
    // Hermitian part of the kx = 0 column
    auto ld = [&](const double2* f, int jj) -> double2 {
      const size_t o = (size_t)jj * ps + col;
      double2 v = f[o + kq];
      if (m0) {
        const double2 u = f[o + kqm];
        v = make_double2(0.5 * (v.x + u.x), 0.5 * (v.y - u.y));
      }
      return v;
    };
    const double2 c1 = ld(a.cu[0], j);
    if (kq == 0) {
      a.spec[(size_t)j * a.nkx1 + m] = nrm2(c1);
      double2* ro = a.rows + (size_t)j * (3 + a.nth) * a.nkx1 + m;
      ro[0] = c1;
      ro[a.nkx1] = ld(a.cu[1], j);
      ro[2 * a.nkx1] = ld(a.cu[2], j);
      for (int n = 0; n < a.nth; ++n) ro[(3 + n) * a.nkx1] = ld(a.cth[n], j);
    }
    if (is00) {
      double* mo = a.means + (size_t)j * (4 + a.nth);
      mo[0] = c1.x;
      mo[1] = a.cu[1][(size_t)j * ps].x;
      mo[2] = a.cu[2][(size_t)j * ps].x;
      mo[3] = a.cp[(size_t)j * ps].x;
      for (int n = 0; n < a.nth; ++n) mo[4 + n] = a.cth[n][(size_t)j * ps].x;
    }
    if (!inner) continue;
    const double w = m0 ? 1.0 : 2.0;
    const double kxm = a.kx[m], kzq = a.kz[kq];
    const double k2 = kxm * kxm + kzq * kzq;
    const double2 c1m = ld(a.cu[0], j - 1), c1p = ld(a.cu[0], j + 1);
    const double2 c2m = ld(a.cu[1], j - 1), c2 = ld(a.cu[1], j), c2p = ld(a.cu[1], j + 1);
    const double2 c3m = ld(a.cu[2], j - 1), c3 = ld(a.cu[2], j), c3p = ld(a.cu[2], j + 1);
    const double2 z = make_double2(0.0, 0.0);
    // fluctuations: the (0,0) coefficient removed, or the kz = 0 row
    const bool drop = a.rowmean ? kq == 0 : is00;
    const double2 h1 = drop ? z : c1, h2 = drop ? z : c2, h3 = drop ? z : c3;
    const double2 h1m = drop ? z : c1m, h2m = drop ? z : c2m, h3m = drop ? z : c3m;
    const double2 h2p = drop ? z : c2p;
    acc[SQ_UU] += w * nrm2(h1);
    acc[SQ_VV] += w * nrm2(h2);
    acc[SQ_WW] += w * nrm2(h3);
    acc[SQ_UW] += w * re_dot(h1, h3);
    {
      const double2 d1 = (1.0 / (2.0 * dyfj)) * (c1p - c1m), d3 = (1.0 / (2.0 * dyfj)) * (c3p - c3m);
      acc[SQ_SHEAR] += w * (nrm2(d1) + nrm2(d3));
      double2 ox = mul_ik(kzq, 0.5 * (c2p + c2)) - (1.0 / (2.0 * dyfj)) * (c3p - c3m);
      if (is00) ox.x -= a.tws;
      acc[SQ_OX] += w * nrm2(ox);
      acc[SQ_OY] += w * nrm2(mul_ik(kxm, c3) - mul_ik(kzq, c1));
      acc[SQ_OZ] += w * nrm2(d1 - mul_ik(kxm, 0.5 * (c2p + c2)));
    }
    if (j >= 2) {
      const double2 i1 = (1.0 / (2.0 * dyj)) * (dyfm * h1 + dyfj * h1m);
      const double2 i3 = (1.0 / (2.0 * dyj)) * (dyfm * h3 + dyfj * h3m);
      acc[SQ_UV] += w * re_dot(i1, h2);
      acc[SQ_WV] += w * re_dot(i3, h2);
      // du/dx, dw/dx, du/dz, dw/dz interpolated to GY; dv/dx, dv/dz at GY;
      // du/dy, dv/dy, dw/dy of the fluctuations
      // (on the kz = 0 row k2 = kx^2: the x derivatives, left out with kstart1)
      const double k2e = (a.kstart1 && kq == 0) ? 0.0 : k2;
      double e = k2e * (dyfm * (nrm2(c1) + nrm2(c3)) + dyfj * (nrm2(c1m) + nrm2(c3m))) / (2.0 * dyj);
      e += k2e * nrm2(c2);
      e += (nrm2(h1 - h1m) + nrm2(h3 - h3m)) / (dyj * dyj);
      e += nrm2(h2p - h2m) / (dgy * dgy);
      acc[SQ_EPS] += w * e;
    }
    if (kq == 0) acc[SQ_U1YL] += m0 ? c1.x : 2.0 * c1.x;
    // scalars: thrms (:275-286), thv (:331-343), pe_diss (:400-414)
    const double2 v2 = drop ? z : 0.5 * (c2 + c2p);
#pragma unroll
    for (int n = 0; n < NT; ++n) {
      if (n < a.nth) {
        const double2 ct = ld(a.cth[n], j);
        const double2 ht = drop ? z : ct;
        acc[STAT_NQV + STAT_NQT * n + 0] += w * nrm2(ht);
        acc[STAT_NQV + STAT_NQT * n + 1] += w * re_dot(ht, v2);
        // the wall-normal gradient is that of scalar 1 for every n (:316)
        const double2 r2 = (1.0 / dgyf) * (ld(a.cth[0], j + 1) - ld(a.cth[0], j - 1));
        double2 r1 = mul_ik(kxm, ct), r3 = mul_ik(kzq, ct);
        if (is00) { r1.x += a.dthdx[n]; r3.x += a.dthdz[n]; }
        acc[STAT_NQV + STAT_NQT * n + 2] += w * (nrm2(r1) + nrm2(r2) + nrm2(r3));
      }
    }
  }
  block_sum_store<NQ>(acc, nq, a.part + ((size_t)j * a.nslice + blockIdx.x) * STAT_NQ);
}

// compute_TKE_diss_les (for/statistics.f90:2054-2120), the plane mean of
// nu_t (nu_t_mean, for/les.f90:927-937) and of each scalar's kappa_t
// (kappa_t_mean, :1420-1448) from physical u1, u2, u3, nu_t and kappa_t
// ([j][k][i], Nz x Nx per plane).  Slot 0: sum of nu_t over plane j
// (1 <= j <= Ny); slot 1: sum of the GY dissipation term `temp` (2 <= j <= Ny);
// slot 2 + n: sum of scalar n's kappa_t (FP32 arrays when kap32 is set).
#define STAT_LQ (2 + DIABLO_MAX_TH)
struct StatsLesArgs {
  const double* u[3];
  const double* nu_t;
  const void* kap[DIABLO_MAX_TH];
  int nth, kap32;
  const double* dy;
  const double* dyf;
  int nyp, nslice;
  size_t pn;            // Nz * Nx
  double* part;         // [Ny+2][nslice][STAT_LQ]
};

static __global__ void __launch_bounds__(STAT_THREADS) k_stats_les(const __grid_constant__ StatsLesArgs a) {
  const int j = blockIdx.y;
  double acc[STAT_LQ];
#pragma unroll
  for (int q = 0; q < STAT_LQ; ++q) acc[q] = 0.0;
  if (j >= 1 && j <= a.nyp) {
    const size_t pn = a.pn;
    const double* u1 = a.u[0];
    const double* u2 = a.u[1];
    const double* u3 = a.u[2];
    const double* nt = a.nu_t;
    // s1 at GYF row jj (1 <= jj <= Ny) and point i
    auto s1 = [&](int jj, size_t i) -> double {
      const size_t o = (size_t)jj * pn + i, op = o + pn, om = o - pn;
      const double dyp = a.dy[jj + 1], dy0 = a.dy[jj], df = a.dyf[jj];
      return u1[o] * ((nt[op] * (u1[op] - u1[o]) / dyp - nt[o] * (u1[o] - u1[om]) / dy0) / df) +
             u3[o] * ((nt[op] * (u3[op] - u3[o]) / dyp - nt[o] * (u3[o] - u3[om]) / dy0) / df);
    };
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < pn; i += (size_t)a.nslice * blockDim.x) {
      const size_t o = (size_t)j * pn + i, op = o + pn, om = o - pn;
      acc[0] += nt[o];
#pragma unroll
      for (int n = 0; n < DIABLO_MAX_TH; ++n)
        if (n < a.nth)
          acc[2 + n] += a.kap32 ? (double)static_cast<const float*>(a.kap[n])[o]
                                : static_cast<const double*>(a.kap[n])[o];
      if (j >= 2) {
        const double t2 = u2[o] * ((0.5 * (nt[o] + nt[op]) * (u2[op] - u2[o]) / a.dyf[j] -
                                    0.5 * (nt[o] + nt[om]) * (u2[o] - u2[om]) / a.dyf[j - 1]) /
                                   a.dy[j]);
        acc[1] += 0.5 * (s1(j, i) + s1(j - 1, i)) + t2;
      }
    }
  }
  block_sum_store<STAT_LQ>(acc, 2 + a.nth, a.part + ((size_t)j * a.nslice + blockIdx.x) * STAT_LQ);
}

// Z-line statistics of the x-inhomogeneous branch from physical u1, u2, u3
// ([j][k][i]): per (j, i) the z means ume_xy, vme_xy, wme_xy
// (compute_averages, for/statistics.f90:749-786) and the z means of the
// fluctuation products the production terms weight by the mean gradients:
// uu_xy, vv_xy (compute_TKE :1296-1312), vvar_xy = <u1'u3'>, uvar_xy =
// <I(u1')u2'>, wvar_xy = <I(u3')u2'> (compute_TKE_Production :1413-1447), the
// last two on GY (j >= 2).  One thread per (j, i), two passes over k.
enum { XY_UME = 0, XY_VME, XY_WME, XY_UU, XY_VV, XY_UW, XY_UV, XY_WV, XY_N };

struct StatsXyArgs {
  const double* u[3];
  const double* dy;
  const double* dyf;
  int nx, nz, nyp;
  double* out;          // [XY_N][Ny+2][Nx]
};

static __global__ void __launch_bounds__(128) k_stats_xy(const __grid_constant__ StatsXyArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= a.nx) return;
  const size_t pn = (size_t)a.nz * a.nx;
  const size_t o = (size_t)j * pn + i;
  const bool lower = j >= 1;
  const double* u1 = a.u[0];
  const double* u2 = a.u[1];
  const double* u3 = a.u[2];
  double s1 = 0, s2 = 0, s3 = 0, s1m = 0, s3m = 0;
  for (int k = 0; k < a.nz; ++k) {
    const size_t q = o + (size_t)k * a.nx;
    s1 += u1[q];
    s2 += u2[q];
    s3 += u3[q];
    if (lower) { s1m += u1[q - pn]; s3m += u3[q - pn]; }
  }
  const double rz = 1.0 / a.nz;
  const double m1 = s1 * rz, m2 = s2 * rz, m3 = s3 * rz, m1m = s1m * rz, m3m = s3m * rz;
  const bool gy = j >= 2 && j <= a.nyp;
  const double wa = gy ? a.dyf[j - 1] / (2.0 * a.dy[j]) : 0.0, wb = gy ? a.dyf[j] / (2.0 * a.dy[j]) : 0.0;
  double uu = 0, vv = 0, uw = 0, uv = 0, wv = 0;
  for (int k = 0; k < a.nz; ++k) {
    const size_t q = o + (size_t)k * a.nx;
    const double d1 = u1[q] - m1, d2 = u2[q] - m2, d3 = u3[q] - m3;
    uu += d1 * d1;
    vv += d2 * d2;
    uw += d1 * d3;
    if (gy) {
      uv += (wa * d1 + wb * (u1[q - pn] - m1m)) * d2;
      wv += (wa * d3 + wb * (u3[q - pn] - m3m)) * d2;
    }
  }
  const size_t plane = (size_t)(a.nyp + 2) * a.nx, at = (size_t)j * a.nx + i;
  a.out[XY_UME * plane + at] = m1;
  a.out[XY_VME * plane + at] = m2;
  a.out[XY_WME * plane + at] = m3;
  a.out[XY_UU * plane + at] = uu * rz;
  a.out[XY_VV * plane + at] = vv * rz;
  a.out[XY_UW * plane + at] = uw * rz;
  a.out[XY_UV * plane + at] = uv * rz;
  a.out[XY_WV * plane + at] = wv * rz;
}

// compute_BPE (for/statistics.f90:1755-1876): the y-weighted histogram of
// s = th_1 + dTHdX(1) (gx - Lx/2) over rows jlo..jhi, into Nbin bins either
// evenly spaced from thmin (the x-inhomogeneous branch) or acos-spaced in
// [-Ro_inv, Ro_inv] with the reference's float32 pi.  Bin indices below 0 (th
// under the evenly spaced range, out of bounds in the reference) go to bin 0.
// Per-block shared-memory histograms, then one atomic add per bin.
struct StatsBpeArgs {
  const double* th;     // physical th_1, [j][k][i]
  const double* dyf;
  double dthdx, lx, thmin, thmax, dth, roden, pi_ref;
  int nx, nz, jlo, jhi, nbin, even;
  double* pdf;          // [nbin], zeroed by the caller
};

static __global__ void __launch_bounds__(256) k_stats_bpe(const __grid_constant__ StatsBpeArgs a) {
  extern __shared__ double hist[];
  for (int b = threadIdx.x; b < a.nbin; b += blockDim.x) hist[b] = 0.0;
  __syncthreads();
  const size_t pn = (size_t)a.nz * a.nx;
  const size_t tot = (size_t)(a.jhi - a.jlo + 1) * pn;
  int cur = -1;
  double accw = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    const int j = a.jlo + (int)(q / pn);
    const size_t r = q % pn;
    const int i = (int)(r % a.nx);
    const double s = a.th[(size_t)j * pn + r] + a.dthdx * ((i * a.lx) / a.nx - 0.5 * a.lx);
    double x = a.even ? (s - a.thmin) / a.dth
                      : acos(-fmin(fmax(s, a.thmin), a.thmax) / a.roden) * a.nbin / a.pi_ref;
    // truncation toward zero, then the bin range (clamping first keeps the
    // conversion in range; fmax also sends NaN to bin 0)
    x = fmin(fmax(x, 0.0), (double)(a.nbin - 1));
    const int b = (int)x;
    if (b != cur) {   // runs in one bin reach shared memory once (see k_stats_zstar)
      if (cur >= 0) atomicAdd(&hist[cur], accw);
      cur = b;
      accw = 0.0;
    }
    accw += a.dyf[j];
  }
  if (cur >= 0) atomicAdd(&hist[cur], accw);
  __syncthreads();
  for (int b = threadIdx.x; b < a.nbin; b += blockDim.x)
    if (hist[b] != 0.0) atomicAdd(&a.pdf[b], hist[b]);
}

// i k * F for the y* binning's derivative fields: axis 0 = x (kx), 1 = z (kz);
// drop0 zeroes the kz = 0 row (epsilon's x derivatives in the x-inhomogeneous
// branch, k_start = 1).  One thread per stored coefficient.
static __global__ void k_spec_deriv(const double2* __restrict__ src, double2* __restrict__ dst, const double* kx,
                             const double* kz, int axis, int drop0, int nkx1, int nk2, int kp, size_t tot) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= tot) return;
  const int kq = (int)(idx % kp);
  const int m = (int)((idx / kp) % nkx1);
  double2 v = make_double2(0.0, 0.0);
  if (kq < nk2 && !(drop0 && kq == 0)) v = mul_ik(axis == 0 ? kx[m] : kz[kq], src[idx]);
  dst[idx] = v;
}

// z mean at each (j, i) of a physical field, out[j][i]
static __global__ void k_zmean(const double* __restrict__ f, double* __restrict__ out, int nx, int nz, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= nx || j >= n) return;
  const size_t o = (size_t)j * nz * nx + i;
  double s = 0.0;
  for (int k = 0; k < nz; ++k) s += f[o + (size_t)k * nx];
  out[(size_t)j * nx + i] = s / nz;
}

// Bin_Ystar_and_Write (for/statistics.f90:1877-1972) for the six fields the
// reference bins, evaluated point by point from physical fields: shear2
// (:159-166), thw (:343-370, th_1 against the last scalar's means), chi
// (:400-423, the last scalar), epsilon (:859-1072), TKE and KE (:1296-1387).
// Bins as in k_stats_bpe.  hist[0][b] = sum of dyf, hist[1 + q][b] = sum of
// field_q dyf over the points of bin b (shared per block, then atomics).
enum { ZS_SHEAR2 = 0, ZS_THW, ZS_CHI, ZS_EPSILON, ZS_TKE, ZS_KE, ZS_N };

struct StatsZstarArgs {
  const double* u[3];
  const double* th1;
  const double* du[6];      // d/dx u1, u2, u3, then d/dz u1, u2, u3
  const double* dthd[2];    // d/dx, d/dz of the last scalar
  const double* means;      // [Ny+2][4 + nth] plane means (homogeneous means)
  const double* xy;         // [XY_N][Ny+2][Nx] z-line means (zline) or null
  const double* thxy;       // [Ny+2][Nx] z-line mean of the last scalar (zline) or null
  const double* dy;
  const double* dyf;
  const double* gy;
  const double* gyf;
  double nu, dthdx0, dthdx_l, dthdz_l, lx, thmin, thmax, dth, roden, pi_ref;
  int nx, nz, nyp, nth, jlo, jhi, nbin, even;
  double* hist;             // [1 + ZS_N][nbin], zeroed by the caller
};

static __global__ void __launch_bounds__(256) k_stats_zstar(const __grid_constant__ StatsZstarArgs a) {
  extern __shared__ double zh[];
  const int nb = a.nbin;
  for (int b = threadIdx.x; b < (1 + ZS_N) * nb; b += blockDim.x) zh[b] = 0.0;
  __syncthreads();
  const int nx = a.nx;
  const size_t pn = (size_t)a.nz * nx;
  const size_t plane = (size_t)(a.nyp + 2) * nx;
  const int stride = 4 + a.nth;
  auto UM = [&](int q, int j, int i) -> double {   // mean of u_{q+1} at (j, i)
    return a.xy ? a.xy[(size_t)q * plane + (size_t)j * nx + i] : a.means[(size_t)j * stride + q];
  };
  auto THM = [&](int j, int i) -> double {
    return a.thxy ? a.thxy[(size_t)j * nx + i] : a.means[(size_t)j * stride + 4 + a.nth - 1];
  };
  const double* u1 = a.u[0];
  const double* u2 = a.u[1];
  const double* u3 = a.u[2];
  const size_t tot = (size_t)(a.jhi - a.jlo + 1) * pn;
  int cur = -1;
  double accw = 0.0, acc[ZS_N];
#pragma unroll
  for (int k = 0; k < ZS_N; ++k) acc[k] = 0.0;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (size_t)gridDim.x * blockDim.x) {
    const int j = a.jlo + (int)(q / pn);
    const size_t r = q % pn;
    const int i = (int)(r % nx);
    const size_t o = (size_t)j * pn + r, op = o + pn, om = o - pn;
    const double s = a.th1[o] + a.dthdx0 * ((i * a.lx) / nx - 0.5 * a.lx);
    double x = a.even ? (s - a.thmin) / a.dth
                      : acos(-fmin(fmax(s, a.thmin), a.thmax) / a.roden) * nb / a.pi_ref;
    x = fmin(fmax(x, 0.0), (double)(nb - 1));
    const int b = (int)x;
    const double w = a.dyf[j];
    double f[ZS_N];
    {
      const double d1 = (u1[op] - u1[om]) / (2.0 * a.dyf[j]), d3 = (u3[op] - u3[om]) / (2.0 * a.dyf[j]);
      f[ZS_SHEAR2] = d1 * d1 + d3 * d3;
    }
    f[ZS_THW] = (a.th1[o] - THM(j, i)) * 0.5 * ((u2[o] - UM(1, j, i)) + (u2[op] - UM(1, j + 1, i)));
    {
      const double r1 = a.dthd[0][o] + a.dthdx_l, r3 = a.dthd[1][o] + a.dthdz_l;
      const double r2 = (a.th1[op] - a.th1[om]) / (a.gyf[j + 1] - a.gyf[j - 1]);
      f[ZS_CHI] = r1 * r1 + r2 * r2 + r3 * r3;
    }
    double e = 0.0;
    if (j >= 2) {
      const double wa = a.dyf[j - 1] / (2.0 * a.dy[j]), wb = a.dyf[j] / (2.0 * a.dy[j]);
      auto ip = [&](const double* sfield) { return wa * sfield[o] * sfield[o] + wb * sfield[om] * sfield[om]; };
      e += ip(a.du[0]) + a.du[1][o] * a.du[1][o] + ip(a.du[2]);
      e += ip(a.du[3]) + a.du[4][o] * a.du[4][o] + ip(a.du[5]);
      const double su = ((u1[o] - UM(0, j, i)) - (u1[om] - UM(0, j - 1, i))) / a.dy[j];
      const double sv = ((u2[op] - UM(1, j + 1, i)) - (u2[om] - UM(1, j - 1, i))) / (a.gy[j + 1] - a.gy[j - 1]);
      const double sw = ((u3[o] - UM(2, j, i)) - (u3[om] - UM(2, j - 1, i))) / a.dy[j];
      e += su * su + sv * sv + sw * sw;
    }
    f[ZS_EPSILON] = a.nu * e;
    {
      const double t1 = u1[o] - UM(0, j, i), t2 = u2[o] - UM(1, j, i), t3 = u3[o] - UM(2, j, i);
      f[ZS_TKE] = 0.5 * (t1 * t1 + t2 * t2 + t3 * t3);
      f[ZS_KE] = 0.5 * (u1[o] * u1[o] + u2[o] * u2[o] + u3[o] * u3[o]);
    }
    // runs of points in one bin accumulate in registers and reach shared
    // memory once (a flat or weakly varying th_1 puts most points in a few
    // bins, where one atomic per point would serialise)
    if (b != cur) {
      if (cur >= 0) {
        atomicAdd(&zh[cur], accw);
#pragma unroll
        for (int k = 0; k < ZS_N; ++k) atomicAdd(&zh[(1 + k) * nb + cur], acc[k]);
      }
      cur = b;
      accw = 0.0;
#pragma unroll
      for (int k = 0; k < ZS_N; ++k) acc[k] = 0.0;
    }
    accw += w;
#pragma unroll
    for (int k = 0; k < ZS_N; ++k) acc[k] += f[k] * w;
  }
  if (cur >= 0) {
    atomicAdd(&zh[cur], accw);
#pragma unroll
    for (int k = 0; k < ZS_N; ++k) atomicAdd(&zh[(1 + k) * nb + cur], acc[k]);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < (1 + ZS_N) * nb; b += blockDim.x)
    if (zh[b] != 0.0) atomicAdd(&a.hist[b], zh[b]);
}
