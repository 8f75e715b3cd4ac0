// Discrete adjoint of the DNS substep with velocities and scalars (FP64).
//
// Forward substep in Fourier-column form (for/channel.f90:29-917 with
// rem_div_chan :946-1023), per (kx, kz) column, rows J = jstart..jend for
// u1/u3 and J2 = 2..Ny for u2:
//   cf  = -nu k^2b u (+/- Ro^-1/delta u3/u1) - NL(u)                  rows
//   cr  = u + zeta h cf_prev - h grad p + beta h cf (+ forcing const)   rows
//   r   = cr + t1 L u                                                  rows
//   u*  = A^-1 [r on the rows A takes it; wall-row constants]
//   u_s = u* on rows >= w0, u on rows < w0
//   phi = Lp^-1 div(u_s);  u' = u_s - grad phi;  p' = p + phi/h on J
// and per scalar th (rows Jt = jstart_th..Ny, :156-249, :553-710):
//   cf2 += grav_y I(th) (rows J2, not the (0,0) mode), cf1 += grav_x th,
//   cf3 += grav_z th (rows J)
//   cft = -nu/Pr k^2b th - dTHdX u1 - dTHdZ u3 - NL_th                 Jt
//   th' = At^-1 [th + zeta h cft_prev + beta h cft + tc/Pr L th]        Jt
// The adjoint takes lambda (the real gradient of the objective packed as a
// complex number, dJ/dRe + i dJ/dIm) of (u', p', cf) back to (u, p, cf_prev)
// and to the nonlinear terms; a complex factor a in y = a x gives
// lambda_x = conj(a) lambda_y.  The nonlinear adjoint goes through physical
// space with the transposes of the dealiased transforms:
//   (inverse)^T lambda_v = w(m) Nx Nz F(lambda_v),   w(0) = 1, w(m > 0) = 2
//   (forward)^T lambda_c = inverse(lambda_c / w(m)) / (Nx Nz)
#pragma once
#include "common.cuh"
#include "kernels_les.cuh"
#include "kernels_solve.cuh"

// Row coefficients of one substep's systems, host-built from the forward's
// expressions (wall rows included): [field 0..2][A, B, C][n] for the CN
// systems of u1, u2, u3, and rmask[field][n] = 1 on the rows whose
// right-hand side is r.  Poisson rows (mode independent part) [A, C, B0][n].
struct AdjColArgs {
  const double2* lu[3];     // in: lambda of the new u1, u2, u3
  const double2* lp;        // in: lambda of the new p
  const double2* lF[3];     // in: lambda of this substep's cf (null: none)
  double2* ou[3];           // out: linear part of lambda of the old u
  double2* op;              // out: lambda of the old p
  double2* oF[3];           // out: lambda of the previous substep's cf (null at rk 1)
  double2* onl[3];          // out: lambda of NL (rows; zero elsewhere)
  const double* cn;         // [3][3][n]
  const double* rmask;      // [3][n]
  const double* pa;         // Poisson A, C, B0 [3][n]
  const double* kx;
  const double* kz;
  const double* dy;
  const double* dyf;
  double t3, t4, t5, tc, nu, roinvd, beta;
  int n, nyp, nkx1, nk2, kp, ncol, jstart, jend;
  int rk;
};

// One warp per (kx, kz) column, rows j = lane*R + r held in registers:
// everything of the substep adjoint except the nonlinear terms.  The
// transposed systems (M^T: sub-diagonal c(j-1), diagonal b(j), super-diagonal
// a(j+1)) go through the warp partition solver of the forward column kernel.
template <int R>
__global__ void __launch_bounds__(128) k_adj_column(const __grid_constant__ AdjColArgs a) {
  using namespace csolve;
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t c0 = (size_t)m * a.kp + kq;
  const int n = a.n, nyp = a.nyp;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const bool m00 = m == 0 && kq == 0;
  const int j0 = lane * R;
  const int js = a.jstart, je = a.jend;
  const double2 z = make_double2(0.0, 0.0);
  auto ld = [&](const double2* f, int j) -> double2 { return (j >= 0 && j < n) ? f[(size_t)j * ps + c0] : z; };
  auto st = [&](double2* f, int j, double2 v) { if (j < n) f[(size_t)j * ps + c0] = v; };
  // neighbour rows across lanes
  auto up1 = [&](const double2 (&v)[R], int r) -> double2 {     // value at row j+1
    double2 nx = shfl_down2(v[0], 1);
    if (lane == 31) nx = z;
    return r + 1 < R ? v[r + 1] : nx;
  };
  auto dn1 = [&](const double2 (&v)[R], int r) -> double2 {     // value at row j-1
    double2 pv = shfl_up2(v[R - 1], 1);
    if (lane == 0) pv = z;
    return r > 0 ? v[r - 1] : pv;
  };
  auto DY = [&](int j) { return (j >= 1 && j < n) ? a.dy[j] : 1.0; };
  auto DYF = [&](int j) { return (j >= 0 && j < n) ? a.dyf[j] : 1.0; };

  double2 U1[R], U2[R], U3[R], LP[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    U1[r] = ld(a.lu[0], j); U2[r] = ld(a.lu[1], j); U3[r] = ld(a.lu[2], j); LP[r] = ld(a.lp, j);
  }
  // p' = p + phi/h on J; u' = u_s - grad phi
  double2 PH[R], OP[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    OP[r] = LP[r];
    double2 ph = z;
    if (j >= 1 && j <= nyp) {
      if (j >= js && j <= je) ph = (1.0 / a.t4) * LP[r];
      ph = ph + mul_ik(kxm, U1[r]) + mul_ik(kzq, U3[r]);
    }
    const double2 u2n = up1(U2, r);
    if (j + 1 >= 2 && j + 1 <= nyp) ph = ph + (1.0 / DY(j + 1)) * u2n;
    if (j >= 2 && j <= nyp) ph = ph - (1.0 / DY(j)) * U2[r];
    PH[r] = ph;
  }
  // lambda of the divergence: Lp^-T lambda phi, rows 1..Ny (identity elsewhere)
  {
    const double* pa = a.pa;
    auto PA = [&](int j) -> double { return (j <= 1 || j > nyp) ? 0.0 : (j == nyp ? 1.0 : pa[j]); };
    auto PC = [&](int j) -> double {
      return (j < 1 || j >= nyp) ? 0.0 : (j == 1 ? (m00 ? 0.0 : -1.0) : pa[n + j]);
    };
    auto PB = [&](int j) -> double {
      return (j < 1 || j > nyp) ? 1.0 : (j == 1 ? 1.0 : (j == nyp ? -1.0 : -kxm * kxm - kzq * kzq + pa[2 * n + j]));
    };
    double at[R], bt[R], ct[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      at[r] = PC(j - 1); bt[r] = PB(j); ct[r] = PA(j + 1);
      if (j < 1 || j > nyp) PH[r] = z;
    }
    warp_tridiag<R>(at, bt, ct, PH, lane);
  }
  // lambda u_s from the divergence rows 2..Ny-1
  double2 OU[3][R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    const bool dv = j >= 2 && j <= nyp - 1;
    const double2 lbm = dn1(PH, r);
    U1[r] = dv ? U1[r] - mul_ik(kxm, PH[r]) : U1[r];
    U3[r] = dv ? U3[r] - mul_ik(kzq, PH[r]) : U3[r];
    double2 v = U2[r];
    if (j - 1 >= 2 && j - 1 <= nyp - 1) v = v + (1.0 / DYF(j - 1)) * lbm;
    if (dv) v = v - (1.0 / DYF(j)) * PH[r];
    U2[r] = v;
    OU[0][r] = z; OU[1][r] = z; OU[2][r] = z;
  }
  double2 LC0[R];   // lambda cf of u1, for the Coriolis coupling into u3
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    double2 LS[R];
    const int w0 = f == 1 ? 1 : js - 1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      LS[r] = f == 0 ? U1[r] : (f == 1 ? U2[r] : U3[r]);
      if (j < w0) { OU[f][r] = OU[f][r] + LS[r]; LS[r] = z; }
    }
    // A^-T lambda u*
    const double* cn = a.cn + (size_t)f * 3 * n;
    const double* rm = a.rmask + (size_t)f * n;
    auto CA = [&](int j) -> double { return (j >= 0 && j < n) ? cn[j] : 0.0; };
    auto CB = [&](int j) -> double { return (j >= 0 && j < n) ? cn[n + j] : 1.0; };
    auto CC = [&](int j) -> double { return (j >= 0 && j < n) ? cn[2 * n + j] : 0.0; };
    {
      double at[R], bt[R], ct[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = j0 + r;
        at[r] = CC(j - 1); bt[r] = CB(j); ct[r] = CA(j + 1);
      }
      warp_tridiag<R>(at, bt, ct, LS, lane);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      if (!(j < n && rm[j] != 0.0)) LS[r] = z;     // LS is now lambda r (= lambda cr)
    }
    // r = cr + tc L u ; cr = u - h grad p + zeta h cf_prev + beta h cf
    const int lo = f == 1 ? 2 : js, hi = f == 1 ? nyp : je;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      const double2 lm = dn1(LS, r), lp = up1(LS, r);
      // coefficients of L at rows j-1 (for u(j) as its upper neighbour), j, j+1
      double alm, gap, al, ga;
      if (f == 1) {
        alm = 1.0 / (DYF(j - 1) * DY(j - 1)); al = 1.0 / (DYF(j) * DY(j));
        ga = 1.0 / (DYF(j - 1) * DY(j)); gap = 1.0 / (DYF(j) * DY(j + 1));
      } else {
        alm = 1.0 / (DY(j) * DYF(j - 1)); al = 1.0 / (DY(j + 1) * DYF(j));
        ga = 1.0 / (DY(j) * DYF(j)); gap = 1.0 / (DY(j + 1) * DYF(j + 1));
      }
      double2 o = OU[f][r] + LS[r] - (a.tc * (al + ga)) * LS[r];
      if (j >= 1) o = o + (a.tc * alm) * lm;
      if (j + 1 < n) o = o + (a.tc * gap) * lp;
      OU[f][r] = o;
      if (f == 0) OP[r] = OP[r] + a.t4 * mul_ik(kxm, LS[r]);
      else if (f == 2) OP[r] = OP[r] + a.t4 * mul_ik(kzq, LS[r]);
      else OP[r] = OP[r] - (a.t4 / DY(j)) * LS[r] + (a.t4 / DY(j + 1)) * lp;
      if (a.oF[f]) st(a.oF[f], j, a.t3 * LS[r]);
      double2 lcf = z;
      if (j >= lo && j <= hi) {
        lcf = a.t5 * LS[r];
        if (a.lF[f]) lcf = lcf + ld(a.lF[f], j);
      }
      st(a.onl[f], j, -1.0 * lcf);
      OU[f][r] = OU[f][r] - (a.nu * kk) * lcf;
      if (f == 0) LC0[r] = lcf;
      if (f == 2) OU[0][r] = OU[0][r] - a.roinvd * lcf;      // cf3 = ... - ro u1
    }
    if (f == 2) {
#pragma unroll
      for (int r = 0; r < R; ++r) OU[2][r] = OU[2][r] + a.roinvd * LC0[r];   // cf1 = ... + ro u3
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    st(a.ou[0], j, OU[0][r]); st(a.ou[1], j, OU[1][r]); st(a.ou[2], j, OU[2][r]);
    st(a.op, j, OP[r]);
  }
}

// Adjoint of one scalar's column work, after k_adj_column: lambda of the new
// th and of this substep's cf_th become lambda of the old th (linear part),
// of the previous cf_th and of NL_th; the buoyancy terms take lambda cf of
// the velocities (k_adj_column's -onl) into lambda th, and the background
// gradients add -dTHdX lambda cf_th to lambda u1 and -dTHdZ lambda cf_th to
// lambda u3 (read-modify-write of k_adj_column's output, so scalars run one
// launch after another).
struct AdjScalarArgs {
  const double2* lth;       // in: lambda of the new th
  const double2* lF;        // in: lambda of this substep's cf_th (null: none)
  const double2* vnl[3];    // in: lambda NL of u1, u2, u3 (= -lambda cf)
  double2* oth;             // out: linear part of lambda of the old th
  double2* oF;              // out: lambda of the previous substep's cf_th (null at rk 1)
  double2* onl;             // out: lambda of NL_th (rows Jt; zero elsewhere)
  double2* ou1;             // in/out: lambda u1 (k_adj_column's output)
  double2* ou3;             // in/out: lambda u3
  const double* cn;         // [A, B, C][n] of the scalar's CN system
  const double* rmask;      // [n]
  const double* kx;
  const double* kz;
  const double* dy;
  const double* dyf;
  double t3, t5, tc, nu_pr, beta, gx, gy, gz, dthdx, dthdz;
  int n, nyp, nkx1, nk2, kp, ncol, jst, jet;
};

template <int R>
__global__ void __launch_bounds__(128) k_adj_scalar(const __grid_constant__ AdjScalarArgs a) {
  using namespace csolve;
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t c0 = (size_t)m * a.kp + kq;
  const int n = a.n;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const bool m00 = m == 0 && kq == 0;
  const int j0 = lane * R;
  const double2 z = make_double2(0.0, 0.0);
  auto ld = [&](const double2* f, int j) -> double2 { return (j >= 0 && j < n) ? f[(size_t)j * ps + c0] : z; };
  auto st = [&](double2* f, int j, double2 v) { if (j < n) f[(size_t)j * ps + c0] = v; };
  auto up1 = [&](const double2 (&v)[R], int r) -> double2 {
    double2 nx = shfl_down2(v[0], 1);
    if (lane == 31) nx = z;
    return r + 1 < R ? v[r + 1] : nx;
  };
  auto dn1 = [&](const double2 (&v)[R], int r) -> double2 {
    double2 pv = shfl_up2(v[R - 1], 1);
    if (lane == 0) pv = z;
    return r > 0 ? v[r - 1] : pv;
  };
  auto DY = [&](int j) { return (j >= 1 && j < n) ? a.dy[j] : 1.0; };
  auto DYF = [&](int j) { return (j >= 0 && j < n) ? a.dyf[j] : 1.0; };
  double2 LS[R], OU[R];
  const int w0 = a.jst - 1;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    LS[r] = ld(a.lth, j);
    OU[r] = z;
    if (j < w0) { OU[r] = LS[r]; LS[r] = z; }
  }
  // At^-T lambda th*
  {
    const double* cn = a.cn;
    double at[R], bt[R], ct[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      at[r] = (j - 1 >= 0 && j - 1 < n) ? cn[2 * n + j - 1] : 0.0;
      bt[r] = j < n ? cn[n + j] : 1.0;
      ct[r] = j + 1 < n ? cn[j + 1] : 0.0;
    }
    warp_tridiag<R>(at, bt, ct, LS, lane);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    if (!(j < n && a.rmask[j] != 0.0)) LS[r] = z;   // now lambda r (= lambda cr)
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = j0 + r;
    const double2 lm = dn1(LS, r), lp = up1(LS, r);
    const double alm = 1.0 / (DY(j) * DYF(j - 1)), al = 1.0 / (DY(j + 1) * DYF(j));
    const double ga = 1.0 / (DY(j) * DYF(j)), gap = 1.0 / (DY(j + 1) * DYF(j + 1));
    double2 o = OU[r] + LS[r] - (a.tc * (al + ga)) * LS[r];
    if (j >= 1) o = o + (a.tc * alm) * lm;
    if (j + 1 < n) o = o + (a.tc * gap) * lp;
    if (a.oF) st(a.oF, j, a.t3 * LS[r]);
    double2 lcf = z;
    if (j >= a.jst && j <= a.jet) {
      lcf = a.t5 * LS[r];
      if (a.lF) lcf = lcf + ld(a.lF, j);
    }
    st(a.onl, j, -1.0 * lcf);
    o = o - (a.nu_pr * kk) * lcf;
    // cf_th -= dTHdX u1 + dTHdZ u3
    if (j < n && (a.dthdx != 0.0 || a.dthdz != 0.0)) {
      const size_t q = (size_t)j * ps + c0;
      if (a.dthdx != 0.0) a.ou1[q] = a.ou1[q] - a.dthdx * lcf;
      if (a.dthdz != 0.0) a.ou3[q] = a.ou3[q] - a.dthdz * lcf;
    }
    // buoyancy: lambda cf_f = -lambda NL_f, zero off each equation's rows
    o = o - a.gx * ld(a.vnl[0], j) - a.gz * ld(a.vnl[2], j);
    if (!m00 && a.gy != 0.0) {
      // cf2(i) += gy (th(i) dyf(i-1) + th(i-1) dyf(i)) / (2 dy(i)), rows 2..Ny
      const double2 b0 = ld(a.vnl[1], j), b1 = ld(a.vnl[1], j + 1);
      if (j >= 2) o = o - (a.gy * DYF(j - 1) / (2.0 * DY(j))) * b0;
      if (j + 1 >= 2 && j + 1 < n) o = o - (a.gy * DYF(j + 1) / (2.0 * DY(j + 1))) * b1;
    }
    OU[r] = o;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) st(a.oth, j0 + r, OU[r]);
}

// Adjoint of the thermal-wind advection of the 'Front' flavor
// (user_rhs_chan_fourier, for/forcing.f90:37-113), after k_adj_column and
// k_adj_scalar have written lambda cf = -onl on each field's cf rows (zero
// elsewhere).  Forward, per scalar n with c = delta / Ro_inv and
// s_n(y) = c (y - Ly/2) (dTHdX_n kz - dTHdZ_n kx):
//   cf1 -= i s_n(gyf) u1 + c (-dTHdZ_n) (u2(j) + u2(j+1)) / 2
//   cf3 -= i s_n(gyf) u3 + c dTHdX_n (u2(j) + u2(j+1)) / 2
//   cf2 -= i s_n(gy) u2,   cfth_n -= i s_n(gyf) th_n
// so lambda u += i s lambda cf (the conjugate of -i s), and lambda u2(j)
// takes -c/2 (sum -dTHdZ) (lcf1(j) + lcf1(j-1)) - c/2 (sum dTHdX) (lcf3(j) + lcf3(j-1)).
// One thread per (j, m, kq) entry; adds into the lambdas of the old state.
struct AdjFrontArgs {
  const double2* onl[3 + DIABLO_MAX_TH];   // -lambda cf of u1, u2, u3, th..
  double2* ou[3 + DIABLO_MAX_TH];          // lambda of the old u1, u2, u3, th..
  const double* kx;
  const double* kz;
  const double* gy;
  const double* gyf;
  double ly, coef;                         // Ly, delta / Ro_inv
  double dthdx[DIABLO_MAX_TH], dthdz[DIABLO_MAX_TH];
  int nth, n, nkx1, nk2, kp;
};

static __global__ void k_adj_front(const __grid_constant__ AdjFrontArgs a) {
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)a.n * ps) return;
  const int kq = idx % a.kp;
  if (kq >= a.nk2) return;
  const int m = (idx / a.kp) % a.nkx1;
  const int j = idx / ps;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double gf = a.gyf[j] - 0.5 * a.ly, gg = a.gy[j] - 0.5 * a.ly;
  double sx = 0.0, sz = 0.0;
  for (int t = 0; t < a.nth; ++t) { sx += a.dthdx[t]; sz += a.dthdz[t]; }
  // velocities: s summed over the scalars
  const double sf = a.coef * gf * (sx * kzq - sz * kxm), sg = a.coef * gg * (sx * kzq - sz * kxm);
  const double2 l1 = -1.0 * a.onl[0][idx], l2 = -1.0 * a.onl[1][idx], l3 = -1.0 * a.onl[2][idx];
  a.ou[0][idx] = a.ou[0][idx] + mul_ik(sf, l1);
  a.ou[2][idx] = a.ou[2][idx] + mul_ik(sf, l3);
  double2 o2 = a.ou[1][idx] + mul_ik(sg, l2);
  double2 s1 = l1, s3 = l3;
  if (j >= 1) {
    s1 = s1 - a.onl[0][idx - ps];
    s3 = s3 - a.onl[2][idx - ps];
  }
  o2 = o2 - (0.5 * a.coef * (-sz)) * s1 - (0.5 * a.coef * sx) * s3;
  a.ou[1][idx] = o2;
  for (int t = 0; t < a.nth; ++t) {
    const double st = a.coef * gf * (a.dthdx[t] * kzq - a.dthdz[t] * kxm);
    a.ou[3 + t][idx] = a.ou[3 + t][idx] + mul_ik(st, -1.0 * a.onl[3 + t][idx]);
  }
}

// lambda NL -> the eight physical-space product adjoints, in Fourier space,
// scaled by the forward transform's transpose (1/(NxNz), halved for kx > 0):
//   0 u1u3: -ikz l1 - ikx l3   1 u1u1: -ikx l1   2 u3u3: -ikz l3
//   3 Y(u1,u2): l1   4 Y(u3,u2): l3   5 I(u1)u2: -ikx l2   6 I(u3)u2: -ikz l2   7 V(u2): l2
// and per scalar s (NL_s = ikx F(th u1) + ikz F(th u3) + F(Y(th, u2))):
//   8+3s th u1: -ikx ls   9+3s th u3: -ikz ls   10+3s Y(th,u2): ls
struct AdjNlPrepArgs {
  const double2* lnl[3 + DIABLO_MAX_TH];
  double2* out[8 + 3 * DIABLO_MAX_TH];
  const double* kx;
  const double* kz;
  double inv;       // 1/(Nx Nz)
  FGeom g;
  int nth;
};

static __global__ void k_adj_nl_prep(const __grid_constant__ AdjNlPrepArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double w = a.inv * (m > 0 ? 0.5 : 1.0);
  const double2 l1 = a.lnl[0][idx], l2 = a.lnl[1][idx], l3 = a.lnl[2][idx];
  a.out[0][idx] = w * (mul_ik(-kzq, l1) + mul_ik(-kxm, l3));
  a.out[1][idx] = w * mul_ik(-kxm, l1);
  a.out[2][idx] = w * mul_ik(-kzq, l3);
  a.out[3][idx] = w * l1;
  a.out[4][idx] = w * l3;
  a.out[5][idx] = w * mul_ik(-kxm, l2);
  a.out[6][idx] = w * mul_ik(-kzq, l2);
  a.out[7][idx] = w * l2;
  for (int s = 0; s < a.nth; ++s) {
    const double2 ls = a.lnl[3 + s][idx];
    a.out[8 + 3 * s][idx] = w * mul_ik(-kxm, ls);
    a.out[9 + 3 * s][idx] = w * mul_ik(-kzq, ls);
    a.out[10 + 3 * s][idx] = w * ls;
  }
}

// Product rule in physical space, gathered per point (planes 0..Ny+1): the
// adjoints of u1, u2, u3 and of each scalar from the product adjoints P
// (zero off planes 1..Ny) and the forward velocities and scalars.
struct AdjNlPointArgs {
  const double* P[8 + 3 * DIABLO_MAX_TH];
  const double* u1;
  const double* u2;
  const double* u3;
  const double* th[DIABLO_MAX_TH];
  double* o1;
  double* o2;
  double* o3;
  double* oth[DIABLO_MAX_TH];
  const double* dy;
  const double* dyf;
  int nyp, nth;
  size_t ps;
};

static __global__ void k_adj_nl_point(const __grid_constant__ AdjNlPointArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  const size_t ps = a.ps;
  const int nyp = a.nyp;
  auto P = [&](int q, int jj) -> double {
    return (jj >= 1 && jj <= nyp) ? a.P[q][idx + (ptrdiff_t)(jj - j) * (ptrdiff_t)ps] : 0.0;
  };
  auto U = [&](const double* u, int jj) -> double {
    return (jj >= 0 && jj <= nyp + 1) ? u[idx + (ptrdiff_t)(jj - j) * (ptrdiff_t)ps] : 0.0;
  };
  auto D = [&](int jj) -> double { return (jj >= 1 && jj <= nyp) ? 1.0 / (2.0 * a.dyf[jj]) : 0.0; };
  const double u1 = U(a.u1, j), u3 = U(a.u3, j), v = U(a.u2, j);
  const double vp = U(a.u2, j + 1);
  double l1 = u3 * P(0, j) + 2.0 * u1 * P(1, j);
  double l3 = u1 * P(0, j) + 2.0 * u3 * P(2, j);
  double lv = 0.0;
  // Y(a, v)(j) = (a(j+1)v(j+1) + a(j)v(j+1) - a(j)v(j) - a(j-1)v(j)) / (2 dyf(j))
  l1 += v * D(j - 1) * P(3, j - 1) + (vp - v) * D(j) * P(3, j) - vp * D(j + 1) * P(3, j + 1);
  l3 += v * D(j - 1) * P(4, j - 1) + (vp - v) * D(j) * P(4, j) - vp * D(j + 1) * P(4, j + 1);
  if (j >= 1) {
    const double s1 = u1 + U(a.u1, j - 1), s3 = u3 + U(a.u3, j - 1);
    lv += s1 * (D(j - 1) * P(3, j - 1) - D(j) * P(3, j)) + s3 * (D(j - 1) * P(4, j - 1) - D(j) * P(4, j));
  }
  // I(a)(j) v(j), I(a)(j) = (dyf(j) a(j) + dyf(j-1) a(j-1)) / (2 dy(j))
  if (j >= 1 && j <= nyp) {
    const double aj = a.dyf[j] / (2.0 * a.dy[j]), bj = a.dyf[j - 1] / (2.0 * a.dy[j]);
    l1 += aj * v * P(5, j);
    l3 += aj * v * P(6, j);
    lv += (aj * u1 + bj * U(a.u1, j - 1)) * P(5, j) + (aj * u3 + bj * U(a.u3, j - 1)) * P(6, j);
  }
  if (j + 1 <= nyp) {
    const double bj1 = a.dyf[j] / (2.0 * a.dy[j + 1]);
    l1 += bj1 * vp * P(5, j + 1);
    l3 += bj1 * vp * P(6, j + 1);
  }
  // V(j) = (0.25 (v(j) + v(j+1))^2 - 0.25 (v(j) + v(j-1))^2) / dy(j)
  if (j >= 1 && j <= nyp) lv += 0.5 * (vp - U(a.u2, j - 1)) / a.dy[j] * P(7, j);
  if (j - 1 >= 1) lv += 0.5 * (U(a.u2, j - 1) + v) / a.dy[j - 1] * P(7, j - 1);
  if (j + 1 <= nyp) lv -= 0.5 * (v + vp) / a.dy[j + 1] * P(7, j + 1);
  // scalars: th u1, th u3 and Y(th, u2), the same rules as u1 u3 and Y(u1, u2)
  for (int s = 0; s < a.nth; ++s) {
    const int q = 8 + 3 * s;
    const double th = U(a.th[s], j);
    double lt = u1 * P(q, j) + u3 * P(q + 1, j);
    l1 += th * P(q, j);
    l3 += th * P(q + 1, j);
    lt += v * D(j - 1) * P(q + 2, j - 1) + (vp - v) * D(j) * P(q + 2, j) - vp * D(j + 1) * P(q + 2, j + 1);
    if (j >= 1) lv += (th + U(a.th[s], j - 1)) * (D(j - 1) * P(q + 2, j - 1) - D(j) * P(q + 2, j));
    a.oth[s][idx] = lt;
  }
  a.o1[idx] = l1;
  a.o2[idx] = lv;
  a.o3[idx] = l3;
}

