// Fourier-space column kernel of the channel step: one warp per (kx, kz)
// column does, in FP64,
//   * the explicit RK terms of every transported field
//     (for/channel.f90:29-249, the Fourier half of :468-482),
//   * the explicit half of Crank-Nicolson in y (:494-514, :625-633),
//   * the implicit y-tridiagonal solves of theta, u2, u1, u3 with their wall
//     rows (:657-877, :1545-1968),
//   * the divergence, the pressure-correction Poisson solve and the
//     projection (rem_div_chan :946-1023) and the pressure update (:905-911).
//
// Without an eddy viscosity the implicit operator is the same for every
// horizontal position, so solving it per Fourier mode is the reference's
// per-physical-column solve expressed in the other basis: the inverse FFT of
// the right-hand side and the forward FFT of the solution (:485-487,
// :891-896) cancel out.
//
// Tridiagonal solver: lane t owns rows [t*R, t*R+R).  Each lane eliminates its
// rows down to a 2-unknown interface (first and last row of its chunk, the
// "modified Thomas" sweep), the 32 lanes solve the reduced system by a one-
// step elimination plus parallel cyclic reduction over warp shuffles, and each
// lane back-substitutes its interior rows.  Rows past the system are identity.
#pragma once
#include "common.cuh"

#include "solve_args.cuh"

namespace csolve {

DI double2 shfl_up2(double2 v, int d) {
  return make_double2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
DI double2 shfl_down2(double2 v, int d) {
  return make_double2(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
}

// Solve rows [0, 32R) with lane-owned chunks; d is overwritten by x.
template <int R>
DI void warp_tridiag(double (&a)[R], double (&b)[R], double (&c)[R], double2 (&d)[R], int lane) {
  static_assert(R >= 3, "chunks need at least 3 rows");
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    double ib = 1.0 / b[r];
    a[r] *= ib; c[r] *= ib; d[r] = ib * d[r];
  }
#pragma unroll
  for (int r = 2; r < R; ++r) {
    double ib = 1.0 / (b[r] - a[r] * c[r - 1]);
    d[r] = ib * (d[r] - a[r] * d[r - 1]);
    a[r] = -ib * a[r] * a[r - 1];
    c[r] = ib * c[r];
  }
#pragma unroll
  for (int r = R - 3; r >= 1; --r) {
    d[r] = d[r] - c[r] * d[r + 1];
    a[r] = a[r] - c[r] * a[r + 1];
    c[r] = -c[r] * c[r + 1];
  }
  {
    double ib = 1.0 / (1.0 - c[0] * a[1]);
    d[0] = ib * (d[0] - c[0] * d[1]);
    a[0] = ib * a[0];
    c[0] = -ib * c[0] * c[1];
  }
  // interface system: S_t = x(first row), E_t = x(last row)
  const double as = a[0], gs = c[0];
  const double2 ds = d[0];
  const double ae = a[R - 1], ge = c[R - 1];
  const double2 de = d[R - 1];
  double ae_m = __shfl_up_sync(0xffffffffu, ae, 1);
  double ge_m = __shfl_up_sync(0xffffffffu, ge, 1);
  double2 de_m = shfl_up2(de, 1);
  if (lane == 0) { ae_m = 0.0; ge_m = 0.0; de_m = make_double2(0.0, 0.0); }
  double L = -as * ae_m;
  double D = 1.0 - as * ge_m - gs * ae;
  double U = -gs * ge;
  double2 Q = ds - as * de_m - gs * de;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    double Lm = __shfl_up_sync(0xffffffffu, L, s);
    double Dm = __shfl_up_sync(0xffffffffu, D, s);
    double Um = __shfl_up_sync(0xffffffffu, U, s);
    double2 Qm = shfl_up2(Q, s);
    double Lp = __shfl_down_sync(0xffffffffu, L, s);
    double Dp = __shfl_down_sync(0xffffffffu, D, s);
    double Up = __shfl_down_sync(0xffffffffu, U, s);
    double2 Qp = shfl_down2(Q, s);
    if (lane < s) { Lm = 0.0; Dm = 1.0; Um = 0.0; Qm = make_double2(0.0, 0.0); }
    if (lane + s >= 32) { Lp = 0.0; Dp = 1.0; Up = 0.0; Qp = make_double2(0.0, 0.0); }
    double k1 = L / Dm, k2 = U / Dp;
    L = -k1 * Lm;
    U = -k2 * Up;
    D = D - k1 * Um - k2 * Lp;
    Q = Q - k1 * Qm - k2 * Qp;
  }
  double2 S = (1.0 / D) * Q;
  double2 Sn = shfl_down2(S, 1);
  if (lane == 31) Sn = make_double2(0.0, 0.0);
  double2 E = de - ae * S - ge * Sn;
  d[0] = S;
  d[R - 1] = E;
#pragma unroll
  for (int r = 1; r < R - 1; ++r) d[r] = d[r] - a[r] * S - c[r] * E;
}

DI double2 ld(const double2* p, size_t idx) { return __ldg(p + idx); }

}  // namespace csolve

// Divergence -> pressure-correction Poisson solve -> projection of one column
// (rem_div_chan, for/channel.f90:946-1023, wall rows :1974-2015), optionally
// followed by cp += phi/h (:905-911).  Reads and writes cu in place.
template <int R>
DI void project_column(const SolveArgs& a, double2* const* cu, const double2* cp_in,
                       double2* cp_out, bool upd_cp, int lane, size_t ps, size_t cidx,
                       double kxm, double kzq, bool m00) {
  using namespace csolve;
  const int n = a.n, nyp = a.nyp;
  const int j0 = lane * R;
  const double2 z2 = make_double2(0.0, 0.0);
  double A[R], B[R], Cc[R];
  double2 Dv[R];
  {
    double2 u1v[R], u3v[R], u2v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      u1v[r] = (j < n) ? cu[0][(size_t)j * ps + cidx] : z2;
      u2v[r] = (j < n) ? cu[1][(size_t)j * ps + cidx] : z2;
      u3v[r] = (j < n) ? cu[2][(size_t)j * ps + cidx] : z2;
      // the velocity courant reads (for/channel.f90:885-888), rows 1..Ny
      if (a.keep[0] && j >= 1 && j <= nyp) {
        a.keep[0][(size_t)j * ps + cidx] = u1v[r];
        a.keep[1][(size_t)j * ps + cidx] = u2v[r];
        a.keep[2][(size_t)j * ps + cidx] = u3v[r];
      }
    }
    double2 u2n = shfl_down2(u2v[0], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      A[r] = 0.0; B[r] = 1.0; Cc[r] = 0.0; Dv[r] = z2;
      if (j >= 1 && j <= nyp) {
        const double dyj = a.dy[j], dyj1 = a.dy[j + 1], dyfj = a.dyf[j];
        double2 u2p = r == R - 1 ? u2n : u2v[r + 1];
        A[r] = 1. / (dyj * dyfj);
        B[r] = -kxm * kxm - kzq * kzq - 1. / (dyj1 * dyfj) - 1. / (dyj * dyfj);
        Cc[r] = 1. / (dyj1 * dyfj);
        Dv[r] = mul_ik(kxm, u1v[r]) + make_double2((u2p.x - u2v[r].x) / dyfj, (u2p.y - u2v[r].y) / dyfj)
                + mul_ik(kzq, u3v[r]);
      }
      if (j == 1) { A[r] = 0; B[r] = 1; Cc[r] = m00 ? 0.0 : -1.0; Dv[r] = z2; }
      if (j == nyp) { A[r] = 1; B[r] = -1; Cc[r] = 0; Dv[r] = z2; }
    }
    warp_tridiag<R>(A, B, Cc, Dv, lane);
    double2 phm = shfl_up2(Dv[R - 1], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      if (j >= n) continue;
      const double2 ph = Dv[r];
      if (j >= 1 && j <= nyp) {
        u1v[r] = u1v[r] - mul_ik(kxm, ph);
        u3v[r] = u3v[r] - mul_ik(kzq, ph);
      }
      if (j >= 2 && j <= nyp) {
        double2 pm = r == 0 ? phm : Dv[r - 1];
        u2v[r] = u2v[r] - make_double2((ph.x - pm.x) / a.dy[j], (ph.y - pm.y) / a.dy[j]);
      }
      const size_t o = (size_t)j * ps + cidx;
      cu[0][o] = u1v[r];
      cu[1][o] = u2v[r];
      cu[2][o] = u3v[r];
      if (upd_cp) {
        double2 p = ld(cp_in, o);
        if (j >= a.jstart && j <= a.jend)
          p = p + make_double2(ph.x / a.temp4, ph.y / a.temp4);
        cp_out[o] = p;
      }
    }
  }
}

template <int R>
__global__ void __launch_bounds__(128) k_column_solve(SolveArgs a) {
  using namespace csolve;
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t cidx = (size_t)m * a.kp + kq;
  const int n = a.n, nyp = a.nyp;
  const int j0 = lane * R;
  const bool m00 = (m == 0 && kq == 0);
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const double t1v = a.temp1 * a.nu_v;
  const double2 z2 = make_double2(0.0, 0.0);
  auto L = [&](const double2* p, int j) -> double2 {
    return (j >= 0 && j < n) ? ld(p, (size_t)j * ps + cidx) : z2;
  };
  auto NL = [&](int f, int j) -> double2 {
    if (a.nl64[f]) return ld(a.nl64[f], (size_t)j * ps + cidx);
    float2 v = __ldg(a.nl32[f] + (size_t)j * ps + cidx);
    return make_double2(v.x, v.y);
  };
  auto ST = [&](double2* p, int j, double2 v) {
    if (j >= 0 && j < n) p[(size_t)j * ps + cidx] = v;
  };
  double A[R], B[R], Cc[R];
  double2 Dv[R];

  // ---------------- u1 and u3 (rows jstart..jend) ----------------
#pragma unroll 1
  for (int comp = 0; comp < 3; comp += 2) {
    const double2* cu = a.cu_in[comp];
    const double2* cuo = a.cu_in[2 - comp];       // Coriolis partner
    const int f = comp;
    const int* bc = comp == 0 ? a.ubc : a.wbc;
    const double* c1 = comp == 0 ? a.uc1 : a.wc1;
    double2 uv[R];
#pragma unroll
    for (int r = 0; r < R; ++r) uv[r] = L(cu, j0 + r);
    double2 up = shfl_up2(uv[R - 1], 1), dn = shfl_down2(uv[0], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      A[r] = 0.0; B[r] = 1.0; Cc[r] = 0.0; Dv[r] = z2;
      if (j >= a.jstart && j <= a.jend) {
        const double dyj = a.dy[j], dyj1 = a.dy[j + 1], dyfj = a.dyf[j];
        double2 um = r == 0 ? up : uv[r - 1];
        double2 upp = r == R - 1 ? dn : uv[r + 1];
        double2 cp = L(a.cp_in, j);
        double2 cf = -(a.nu * kk) * uv[r];
        double2 oth = L(cuo, j);
        cf = comp == 0 ? cf + a.roinvd * oth : cf - a.roinvd * oth;
        for (int th = 0; th < a.nth; ++th)
          cf = cf + (comp == 0 ? a.grav_x : a.grav_z) * L(a.cth_in[th], j);
        if (a.front) {
          const double g = a.gyf[j] - 0.5 * a.ly;
          const double2 v2 = 0.5 * (L(a.cu_in[1], j) + L(a.cu_in[1], j + 1));
          for (int th = 0; th < a.nth; ++th) {
            const double cz = a.dthdx[th] * g * a.front_coef;
            const double cx = -1.0 * a.dthdz[th] * g * a.front_coef;
            const double cv = comp == 0 ? (-1.0 * a.dthdz[th] * a.front_coef) : (a.dthdx[th] * a.front_coef);
            cf = cf - cz * mul_ik(kzq, uv[r]) - cx * mul_ik(kxm, uv[r]) - cv * v2;
          }
        }
        cf = cf - NL(f, j);
        if (a.store_cf) ST(a.cf_out[f], j, cf);
        double2 cr = uv[r];
        if (a.rk > 1) cr = cr + a.temp3 * L(a.cf_in[f], j);
        cr = cr - a.temp4 * mul_ik(comp == 0 ? kxm : kzq, cp);
        if (comp == 0 && m00) cr.x -= a.px;
        cr = cr + a.temp5 * cf;
        double2 lap = make_double2(((upp.x - uv[r].x) / dyj1 - (uv[r].x - um.x) / dyj) / dyfj,
                                   ((upp.y - uv[r].y) / dyj1 - (uv[r].y - um.y) / dyj) / dyfj);
        cr = cr + t1v * lap;
        A[r] = -t1v / (dyj * dyfj);
        B[r] = 1. - t1v * (-1. / (dyj1 * dyfj) - 1. / (dyj * dyfj));
        Cc[r] = -t1v / (dyj1 * dyfj);
        Dv[r] = cr;
      }
      // wall rows (apply_BC_1/3_lower/upper)
      const double v00 = m00 ? 1.0 : 0.0;
      if (j == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = z2; }
      if (j == 1) {
        if (bc[0] == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(c1[0] * v00, 0); }
        else { A[r] = 0; B[r] = -1; Cc[r] = 1; Dv[r] = make_double2(a.dy[2] * c1[0] * v00, 0); }
      }
      if (j == nyp) {
        if (bc[1] == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(c1[1] * v00, 0); }
        else { A[r] = -1; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.dy[nyp] * c1[1] * v00, 0); }
      }
      if (j == nyp + 1) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = z2; }
    }
    warp_tridiag<R>(A, B, Cc, Dv, lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      ST(a.cu_out[comp], j, (j >= a.jstart - 1 && j <= a.jend + 1) ? Dv[r] : uv[r]);
    }
  }

  // ---------------- u2 (rows 2..Nyp) ----------------
  {
    const double2* cu = a.cu_in[1];
    double2 uv[R];
#pragma unroll
    for (int r = 0; r < R; ++r) uv[r] = L(cu, j0 + r);
    double2 up = shfl_up2(uv[R - 1], 1), dn = shfl_down2(uv[0], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      A[r] = 0.0; B[r] = 1.0; Cc[r] = 0.0; Dv[r] = z2;
      if (j >= 2 && j <= nyp) {
        const double dyj = a.dy[j], dyfj = a.dyf[j], dyfm = a.dyf[j - 1];
        double2 um = r == 0 ? up : uv[r - 1];
        double2 upp = r == R - 1 ? dn : uv[r + 1];
        double2 cf = -(a.nu * kk) * uv[r];
        if (!m00) {
          for (int th = 0; th < a.nth; ++th) {
            double2 tc = L(a.cth_in[th], j), tm = L(a.cth_in[th], j - 1);
            cf = cf + a.grav_y * make_double2((tc.x * dyfm + tm.x * dyfj) / (2.0 * dyj),
                                              (tc.y * dyfm + tm.y * dyfj) / (2.0 * dyj));
          }
        }
        if (a.front) {
          const double g = a.gy[j] - 0.5 * a.ly;
          for (int th = 0; th < a.nth; ++th) {
            const double cz = a.dthdx[th] * g * a.front_coef;
            const double cx = -1.0 * a.dthdz[th] * g * a.front_coef;
            cf = cf - cz * mul_ik(kzq, uv[r]) - cx * mul_ik(kxm, uv[r]);
          }
        }
        cf = cf - NL(1, j);
        if (a.store_cf) ST(a.cf_out[1], j, cf);
        double2 cr = uv[r];
        if (a.rk > 1) cr = cr + a.temp3 * L(a.cf_in[1], j);
        double2 pc = L(a.cp_in, j), pm = L(a.cp_in, j - 1);
        cr = cr - a.temp4 * make_double2((pc.x - pm.x) / dyj, (pc.y - pm.y) / dyj);
        cr = cr + a.temp5 * cf;
        double2 lap = make_double2(((upp.x - uv[r].x) / dyfj - (uv[r].x - um.x) / dyfm) / dyj,
                                   ((upp.y - uv[r].y) / dyfj - (uv[r].y - um.y) / dyfm) / dyj);
        cr = cr + t1v * lap;
        A[r] = -t1v / (dyfm * dyj);
        B[r] = 1. + t1v / (dyfj * dyj) + t1v / (dyfm * dyj);
        Cc[r] = -t1v / (dyfj * dyj);
        Dv[r] = cr;
      }
      const double v00 = m00 ? 1.0 : 0.0;
      // apply_BC_2_lower / upper (for/channel.f90:1631-1705)
      if (a.vbc[0] == 0 && (j == 1 || j == 2)) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.vc1[0] * v00, 0); }
      if (a.vbc[0] == 1 && j == 1) { A[r] = 0; B[r] = -1; Cc[r] = 1; Dv[r] = make_double2(a.dyf[1] * a.vc1[0] * v00, 0); }
      if (j == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = z2; }
      if (a.vbc[1] == 0 && (j == nyp || j == nyp + 1)) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.vc1[1] * v00, 0); }
      if (a.vbc[1] == 1 && j == nyp + 1) { A[r] = -1; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.dyf[nyp] * a.vc1[1] * v00, 0); }
    }
    warp_tridiag<R>(A, B, Cc, Dv, lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      ST(a.cu_out[1], j, (j >= 1 && j <= nyp + 1) ? Dv[r] : uv[r]);
    }
  }

  // ---------------- scalars (rows jstart_th..jend_th) ----------------
#pragma unroll 1
  for (int th = 0; th < a.nth; ++th) {
    const double2* ct = a.cth_in[th];
    const int f = 3 + th;
    const double tp = (a.temp1 / a.pr[th]) * a.nu_v;   // CN coefficient of the explicit part
    const double tm = a.temp1 / a.pr[th] * a.nu_v;     // matrix coefficient (same value)
    double2 tv[R];
#pragma unroll
    for (int r = 0; r < R; ++r) tv[r] = L(ct, j0 + r);
    double2 up = shfl_up2(tv[R - 1], 1), dn = shfl_down2(tv[0], 1);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      A[r] = 0.0; B[r] = 1.0; Cc[r] = 0.0; Dv[r] = z2;
      if (j >= a.jst[th] && j <= a.jet[th]) {
        const double dyj = a.dy[j], dyj1 = a.dy[j + 1], dyfj = a.dyf[j];
        double2 tmm = r == 0 ? up : tv[r - 1];
        double2 tpp = r == R - 1 ? dn : tv[r + 1];
        double2 cf = -((a.nu / a.pr[th]) * kk) * tv[r];
        cf = cf - a.dthdx[th] * L(a.cu_in[0], j) - a.dthdz[th] * L(a.cu_in[2], j);
        if (a.front) {
          const double g = a.gyf[j] - 0.5 * a.ly;
          cf = cf - (a.front_coef * a.dthdx[th] * g) * mul_ik(kzq, tv[r])
                  - (a.front_coef * (-1.0) * a.dthdz[th] * g) * mul_ik(kxm, tv[r]);
        }
        cf = cf - NL(f, j);
        if (a.store_cf) ST(a.cf_out[f], j, cf);
        double2 cr = tv[r];
        if (a.rk > 1) cr = cr + a.temp3 * L(a.cf_in[f], j);
        cr = cr + a.temp5 * cf;
        double2 lap = make_double2(((tpp.x - tv[r].x) / dyj1 - (tv[r].x - tmm.x) / dyj) / dyfj,
                                   ((tpp.y - tv[r].y) / dyj1 - (tv[r].y - tmm.y) / dyj) / dyfj);
        cr = cr + tp * lap;
        A[r] = -tm / (dyj * dyfj);
        B[r] = 1. + tm / (dyj1 * dyfj) + tm / (dyj * dyfj);
        Cc[r] = -tm / (dyj1 * dyfj);
        Dv[r] = cr;
      }
      const double v00 = m00 ? 1.0 : 0.0;
      if (j == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = z2; }
      if (j == 1) {
        if (a.thbc[th][0] == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.thc1[th][0] * v00, 0); }
        else { A[r] = 0; B[r] = -1; Cc[r] = 1; Dv[r] = make_double2(a.dy[2] * a.thc1[th][0] * v00, 0); }
      }
      if (j == nyp) {
        if (a.thbc[th][1] == 0) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.thc1[th][1] * v00, 0); }
        else { A[r] = -1; B[r] = 1; Cc[r] = 0; Dv[r] = make_double2(a.dy[nyp] * a.thc1[th][1] * v00, 0); }
      }
      if (j == nyp + 1) { A[r] = 0; B[r] = 1; Cc[r] = 0; Dv[r] = z2; }
    }
    warp_tridiag<R>(A, B, Cc, Dv, lane);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = j0 + r;
      ST(a.cth_out[th], j, (j >= a.jst[th] - 1 && j <= a.jet[th] + 1) ? Dv[r] : tv[r]);
    }
  }

  // ---------------- projection (rem_div_chan) ----------------
  __syncwarp();
  project_column<R>(a, a.cu_out, a.cp_in, a.cp_out, true, lane, ps, cidx, kxm, kzq, m00);
}

// Projection alone, in place on the state (pre_first_step, for/advance.f90:30).
template <int R>
__global__ void __launch_bounds__(128) k_rem_div(SolveArgs a) {
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t cidx = (size_t)m * a.kp + kq;
  project_column<R>(a, a.cu_out, nullptr, nullptr, false, lane, ps, cidx, a.kx[m], a.kz[kq],
                    m == 0 && kq == 0);
}

// Projection with the pressure update, in place on cu_out (the LES substep,
// for/channel.f90:901-911).
template <int R>
__global__ void __launch_bounds__(128) k_project(SolveArgs a) {
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t cidx = (size_t)m * a.kp + kq;
  project_column<R>(a, a.cu_out, a.cp_in, a.cp_out, true, lane, ps, cidx, a.kx[m], a.kz[kq],
                    m == 0 && kq == 0);
}
