// Fourier-space column step split by field: the default path of the column
// solve.
//
// The implicit y operators of u1, u2, u3 and every scalar are the same in
// every (kx, kz) column (the horizontal terms are explicit, for/channel.f90
// :108-153), and a field's explicit terms read the other fields only as they
// were at the start of the substep.  So every (field, column) pair is an
// independent task until the projection, which couples the three velocities
// and the pressure through rem_div_chan (:946-1023).  The column step
// therefore runs as two kernels:
//
//   k_field_solve   one warp per (field, column): explicit RK terms
//                   (:29-249), cf for the next substep, the explicit
//                   Crank-Nicolson half (:468-514, :625-633), the pressure
//                   gradient, the wall rows and the factored implicit solve
//                   (:657-877); writes the solved velocity u* (the scalars'
//                   final value);
//   k_project_cols  one warp per column: divergence of u*, the pressure-
//                   correction Poisson solve, the projection and cp += phi/h
//                   (:901-1023).
//
// Five to seven times as many independent warps as a warp-per-column kernel
// that carries every field, and no block-wide barriers: each warp loads its
// own rows straight into registers (a lane owns R consecutive rows, its
// neighbours' edge rows come over shuffles), and the warps of a block take
// adjacent columns, so each 128-byte row segment is fetched once and served
// to its eight warps from L1/L2.
#pragma once
#include "common.cuh"
#include "kernels_solve.cuh"
#include "kernels_solve2.cuh"

#define FS_WARPS 8   // columns (warps) per block of both kernels

struct FieldArgs {
  SolveArgs s;
  const double* kc;    // implicit rows of this substep [kind][3][n] (see Solve2Args)
  const double* met;   // [MET_N][n]
  const double* fac;   // factored systems of this substep (k_factor), kinds 0..2+N_th
  int nf;              // 3 + N_th
  int mean_split;      // see Solve2Args::mean_split
  const double* prof;  // [2][n] U1(j), I(U1)(j)
};

namespace cfield {
using namespace csolve;

DI double2 ldc(const double2* p, size_t i) { return __ldg(p + i); }
DI double2 ldnl(const FieldArgs& A, int f, size_t i) {
  const SolveArgs& a = A.s;
  if (a.nl64[f]) return __ldg(a.nl64[f] + i);
  const float2 v = __ldg(a.nl32[f] + i);
  return make_double2(v.x, v.y);
}
}  // namespace cfield

// Rows per lane R = ceil((Ny+2)/32) >= 3.  Blocks per SM for the register cap:
// the explicit terms keep only a three-row window of the field, so the live
// state is the R right-hand sides.
template <int R>
constexpr int fs_min_blocks() { return R <= 5 ? 4 : 3; }

template <int R>
__global__ void __launch_bounds__(32 * FS_WARPS, fs_min_blocks<R>()) k_field_solve(const __grid_constant__ FieldArgs A) {
  using namespace cfield;
  const SolveArgs& a = A.s;
  const int nf = A.nf;
  // field fastest: the blocks of one column group run together, so the
  // pressure and coupling rows they share are read from L2
  const int f = blockIdx.x % nf;
  const int q = (blockIdx.x / nf) * FS_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= a.ncol) return;   // whole warps
  const int n = a.n, nyp = a.nyp;
  const size_t ps = (size_t)a.ncol;     // plane stride (the Fourier pitch is 2Nkz+1)
  const int m = q / a.nk2, kq = q % a.nk2;
  const bool m00 = (q == 0);
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  const double* met = A.met;

  // field kind: solve index (0 u1, 1 u2, 2 u3, 3+n scalar n), row-coefficient
  // index (0 u1/u3, 1 u2, 2+n scalar n), explicit rows [lo, hi], wall rows
  const int th = f - 3;
  const int kc_kind = f == 1 ? 1 : (f < 3 ? 0 : 2 + th);
  int lo, hi, b0, b1;
  double c0, c1;
  if (f == 0) { lo = a.jstart; hi = a.jend; b0 = a.ubc[0]; b1 = a.ubc[1]; c0 = a.uc1[0]; c1 = a.uc1[1]; }
  else if (f == 2) { lo = a.jstart; hi = a.jend; b0 = a.wbc[0]; b1 = a.wbc[1]; c0 = a.wc1[0]; c1 = a.wc1[1]; }
  else if (f == 1) { lo = 2; hi = nyp; b0 = a.vbc[0]; b1 = a.vbc[1]; c0 = a.vc1[0]; c1 = a.vc1[1]; }
  else { lo = a.jst[th]; hi = a.jet[th]; b0 = a.thbc[th][0]; b1 = a.thbc[th][1]; c0 = a.thc1[th][0]; c1 = a.thc1[th][1]; }
  const double* K = A.kc + (size_t)kc_kind * 3 * n;
  const double cfc = f >= 3 ? (a.nu / a.pr[th]) * kk : a.nu * kk;
  const double2* own = f < 3 ? a.cu_in[f] : a.cth_in[th];
  const double2* cpi = a.cp_in;
  const double v00 = m00 ? 1.0 : 0.0;
  // mean-split correction of this field: -ikx U(j) u with U = U1 (u3,
  // scalars) or its GY interpolation I(U1) (u2); none for u1
  const double* Up = (A.mean_split && f != 0) ? A.prof + (f == 1 ? n : 0) : nullptr;

  // The own field moves through a three-row window (rows j-1, j, j+1); the
  // rows next to the lane's chunk come from lanes t-1, t+1.  The pressure
  // likewise carries one row (u2 needs p(j-1)).
  auto ldo = [&](int j) -> double2 { return j < n ? ldc(own, (size_t)j * ps + q) : z2; };
  auto ldp = [&](int j) -> double2 { return j < n ? ldc(cpi, (size_t)j * ps + q) : z2; };
  const double2 u_first = ldo(j0), u_last = ldo(j0 + R - 1);
  const double2 u_lo = shfl_up2(u_last, 1);     // row j0 - 1
  const double2 u_hi = shfl_down2(u_first, 1);  // row j0 + R
  double2 p_prev = z2;
  if (f == 1) p_prev = shfl_up2(ldp(j0 + R - 1), 1);
  double2 um = u_lo, uu = u_first;

  double2 d[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    const double2 up = r == R - 1 ? u_hi : (r == R - 2 ? u_last : ldo(j + 1));
    double2 dv = z2;
    const size_t o = (size_t)j * ps + q;
    const double2 pj = (f < 3) ? ldp(j) : z2;
    if (j >= lo && j <= hi) {
      double2 cf = -cfc * uu;
      double2 cr = uu - K[2 * n + j] * (up - uu) + K[j] * (uu - um);
      if (Up) cf = cf - mul_ik(kxm * __ldg(Up + j), uu);
      // couplings through the other fields' substep-start values
      if (f == 0 || f == 2) {
        if (a.roinvd != 0.0) {
          const double2 oth = ldc(a.cu_in[2 - f], o);
          cf = cf + (f == 0 ? a.roinvd : -a.roinvd) * oth;
        }
        const double g = f == 0 ? a.grav_x : a.grav_z;
        if (g != 0.0)
          for (int t = 0; t < a.nth; ++t) cf = cf + g * ldc(a.cth_in[t], o);
      } else if (f == 1) {
        if (a.grav_y != 0.0 && !m00)
          for (int t = 0; t < a.nth; ++t)
            cf = cf + a.grav_y * (__ldg(met + MET_WB1 * n + j) * ldc(a.cth_in[t], o) +
                                  __ldg(met + MET_WB2 * n + j) * ldc(a.cth_in[t], o - ps));
      } else {
        if (a.dthdx[th] != 0.0) cf = cf + (-a.dthdx[th]) * ldc(a.cu_in[0], o);
        if (a.dthdz[th] != 0.0) cf = cf + (-a.dthdz[th]) * ldc(a.cu_in[2], o);
      }
      cf = cf - ldnl(A, f, o);
      if (a.store_cf) a.cf_out[f][o] = cf;
      cr = cr + a.temp5 * cf;
      if (a.rk > 1) cr = cr + a.temp3 * ldc(a.cf_in[f], o);
      if (f == 0) {
        cr = cr - a.temp4 * mul_ik(kxm, pj);
        if (m00) cr.x -= a.px;
      } else if (f == 2) {
        cr = cr - a.temp4 * mul_ik(kzq, pj);
      } else if (f == 1) {
        cr = cr - a.temp4 * __ldg(met + MET_IDY * n + j) * (pj - p_prev);
      }
      dv = cr;
    }
    p_prev = pj;
    um = uu;
    uu = up;
    // wall rows (for/channel.f90:1545-1876)
    if (f == 1) {
      if (b0 == 0 && (j == 1 || j == 2)) dv = make_double2(c0 * v00, 0);
      if (b0 == 1 && j == 1) dv = make_double2(a.dyf[1] * c0 * v00, 0);
      if (j == 0) dv = z2;
      if (b1 == 0 && (j == nyp || j == nyp + 1)) dv = make_double2(c1 * v00, 0);
      if (b1 == 1 && j == nyp + 1) dv = make_double2(a.dyf[nyp] * c1 * v00, 0);
    } else {
      if (j == 0 || j == nyp + 1) dv = z2;
      if (j == 1) dv = make_double2((b0 == 0 ? c0 : a.dy[2] * c0) * v00, 0);
      if (j == nyp) dv = make_double2((b1 == 0 ? c1 : a.dy[nyp] * c1) * v00, 0);
    }
    d[r] = dv;
  }
  apply_factored<R>(A.fac + (size_t)f * Fac<R>::N * 32, d, lane);
  // rows the solve writes: u2 1..Ny+1, the others lo-1..Ny+1; the rest keep
  // their input value
  const int w0 = f == 1 ? 1 : lo - 1, w1 = nyp + 1;
  double2* dst = f < 3 ? a.cu_out[f] : a.cth_out[th];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    if (j < n) dst[(size_t)j * ps + q] = (j >= w0 && j <= w1) ? d[r] : ldo(j);
  }
}

// Divergence -> pressure-correction Poisson solve -> projection -> pressure
// update of one column per warp, in place on cu (rem_div_chan,
// for/channel.f90:946-1023 with the wall rows of :1974-2015; cp += phi/h,
// :905-911).  keep[q], if set, receives the velocity before the projection
// (the field courant reads, :885-888).
template <int R>
__global__ void __launch_bounds__(32 * FS_WARPS, 2) k_project_cols(const __grid_constant__ FieldArgs A) {
  using namespace cfield;
  const SolveArgs& a = A.s;
  const int q = blockIdx.x * FS_WARPS + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= a.ncol) return;
  const int n = a.n, nyp = a.nyp;
  const size_t ps = (size_t)a.ncol;
  const int m = q / a.nk2, kq = q % a.nk2;
  const bool m00 = (q == 0);
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  const double* met = A.met;
  double2* const* cu = a.cu_out;
  // divergence ik.u1 + ik.u3 + (u2(j+1) - u2(j))/dyf(j), rows 1..Ny
  double2 d[R];
  {
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      v[r] = j < n ? ldc(cu[1], (size_t)j * ps + q) : z2;
    }
    const double2 vn = shfl_down2(v[0], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      double2 dv = z2;
      if (j >= 1 && j <= nyp) {
        const size_t o = (size_t)j * ps + q;
        const double2 vp = r == R - 1 ? vn : v[r + 1];
        dv = mul_ik(kxm, ldc(cu[0], o));
        dv = dv + mul_ik(kzq, ldc(cu[2], o));
        dv = dv + __ldg(met + MET_IDYF * n + j) * (vp - v[r]);
      }
      d[r] = dv;
    }
  }
  // Poisson rows: interior 1/(dy dyf) terms, Neumann walls, phi(1) = 0 for
  // the (0,0) mode
  double al[R], cu_[R];
  const double k2n = -kxm * kxm - kzq * kzq;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    double am = 0.0, cm = 0.0;
    if (j >= 1 && j <= nyp) { am = __ldg(met + MET_PA * n + j); cm = __ldg(met + MET_PC * n + j); }
    if (j == 1) { am = 0; cm = m00 ? 0.0 : -1.0; d[r] = z2; }
    if (j == nyp) { am = 1; cm = 0; d[r] = z2; }
    al[r] = am;
    cu_[r] = cm;
  }
  csolve2::warp_tridiag_b<R>([&](int r) -> double& { return al[r]; }, [&](int r) -> double {
    const int j = j0 + r;
    return (j == 1) ? 1.0 : (j == nyp ? -1.0 : ((j > 1 && j < nyp) ? k2n + __ldg(met + MET_PB0 * n + j) : 1.0));
  }, [&](int r) -> double& { return cu_[r]; }, d, lane);
  // d = phi from here on
  const double2 phm = shfl_up2(d[R - 1], 1);
  const double ih = 1.0 / a.temp4;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    if (j >= n) continue;
    const size_t o = (size_t)j * ps + q;
    if (j >= 1 && j <= nyp) {
      double2 u1 = ldc(cu[0], o), u2 = ldc(cu[1], o), u3 = ldc(cu[2], o);
      if (a.keep[0]) { a.keep[0][o] = u1; a.keep[1][o] = u2; a.keep[2][o] = u3; }
      cu[0][o] = u1 - mul_ik(kxm, d[r]);
      cu[2][o] = u3 - mul_ik(kzq, d[r]);
      if (j >= 2) {
        const double2 pm = r == 0 ? phm : d[r - 1];
        cu[1][o] = u2 - __ldg(met + MET_IDY * n + j) * (d[r] - pm);
      }
    }
    double2 p = ldc(a.cp_in, o);
    if (j >= a.jstart && j <= a.jend) p = p + ih * d[r];
    a.cp_out[o] = p;
  }
}
