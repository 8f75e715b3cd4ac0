// Kernels of the LES substep (eddy viscosity varies in x and z, so the
// implicit y solves run per physical column as in the reference).
//
// Substep order (for/channel.f90:29-911 with les_chan / les_chan_th,
// for/les.f90:20-1200):
//   k_explicit      Fourier explicit RK terms from the state before the LES
//                   wall/ghost updates (:29-249)
//   (BC post + apply_BC_les on the state)
//   k_strain        Fourier strain-rate tensor (compute_strain_chan)
//   inverse FFTs    S1..S6 and u, th to physical space
//   k_les_point     |S|, eddy viscosity nu_t, SGS stress components and
//                   nu_t dU/dy, nu_t dW/dy
//   forward FFTs    stresses
//   k_les_div       cf -= div(tau) (:850-880)
//   k_les_th_*      scalar SGS flux with kappa_t = nu_t (:1130-1200)
//   (nonlinear terms as in the DNS step)
//   k_cf_finish     cf -= NL, cr += beta h cf
//   inverse FFT     cr -> r
//   k_phys_solve    CN explicit half + implicit solve per physical column
//                   with the eddy-viscosity rows (:494-877)
//   forward FFT     u, th -> state; projection + pressure (:901-911)
#pragma once
#include "common.cuh"
#include "kernels_fft.cuh"
#include "kernels_solve.cuh"

#define LES_MAXF 11

// Fourier index helpers: F[j][m][kp], pitch kp
struct FGeom {
  int nyp, n;          // Nyp, Ny+2
  int nkx1, nk2, kp;
  size_t ps;           // plane stride (elements)
};

// ---------------------------------------------------------------------------
// explicit RK terms in Fourier space; one thread per (j, m, kq)
struct ExplicitArgs2 {
  SolveArgs s;
  double2* cr[SOLVE_NF];
};

static __global__ void k_explicit2(const __grid_constant__ ExplicitArgs2 E) {
  const SolveArgs& a = E.s;
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t tot = (size_t)a.n * ps;
  if (idx >= tot) return;
  const int kq = idx % a.kp;
  if (kq >= a.nk2) return;
  const int m = (idx / a.kp) % a.nkx1;
  const int j = idx / ps;
  const size_t o = idx;
  const bool m00 = (m == 0 && kq == 0);
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const int nyp = a.nyp;
  // u1 / u3 rows jstart..jend (:40-92, :128-153, :184-198)
  for (int comp = 0; comp < 3; comp += 2) {
    if (j < a.jstart || j > a.jend) continue;
    const double2 u = a.cu_in[comp][o];
    double2 cr = u;
    if (a.rk > 1) cr = cr + a.temp3 * a.cf_in[comp][o];
    cr = cr - a.temp4 * mul_ik(comp == 0 ? kxm : kzq, a.cp_in[o]);
    if (comp == 0 && m00) cr.x -= a.px;
    double2 cf = -(a.nu * kk) * u;
    const double2 oth = a.cu_in[2 - comp][o];
    cf = comp == 0 ? cf + a.roinvd * oth : cf - a.roinvd * oth;
    for (int th = 0; th < a.nth; ++th) cf = cf + (comp == 0 ? a.grav_x : a.grav_z) * a.cth_in[th][o];
    E.cr[comp][o] = cr;
    a.cf_out[comp][o] = cf;
  }
  // u2 rows 2..Nyp (:48-100, :136-182)
  if (j >= 2 && j <= nyp) {
    const double2 u = a.cu_in[1][o];
    double2 cr = u;
    if (a.rk > 1) cr = cr + a.temp3 * a.cf_in[1][o];
    const double2 pc = a.cp_in[o], pm = a.cp_in[o - ps];
    cr = cr - a.temp4 * make_double2((pc.x - pm.x) / a.dy[j], (pc.y - pm.y) / a.dy[j]);
    double2 cf = -(a.nu * kk) * u;
    if (!m00) {
      for (int th = 0; th < a.nth; ++th) {
        const double2 tc = a.cth_in[th][o], tm = a.cth_in[th][o - ps];
        cf = cf + a.grav_y * make_double2((tc.x * a.dyf[j - 1] + tm.x * a.dyf[j]) / (2.0 * a.dy[j]),
                                          (tc.y * a.dyf[j - 1] + tm.y * a.dyf[j]) / (2.0 * a.dy[j]));
      }
    }
    E.cr[1][o] = cr;
    a.cf_out[1][o] = cf;
  }
  // scalars rows jstart_th..jend_th (:209-246)
  for (int th = 0; th < a.nth; ++th) {
    if (j < a.jst[th] || j > a.jet[th]) continue;
    const double2 t = a.cth_in[th][o];
    double2 cr = t;
    if (a.rk > 1) cr = cr + a.temp3 * a.cf_in[3 + th][o];
    double2 cf = -((a.nu / a.pr[th]) * kk) * t;
    cf = cf - a.dthdx[th] * a.cu_in[0][o] - a.dthdz[th] * a.cu_in[2][o];
    E.cr[3 + th][o] = cr;
    a.cf_out[3 + th][o] = cf;
  }
}

// ---------------------------------------------------------------------------
// Neumann ghost planes for the LES gradients (apply_BC_les / apply_BC_th_les,
// for/les.f90:2001-2105), one thread per stored mode
struct LesBcArgs {
  double2* cu[3];
  double2* cth[8];
  int nth, nyp, nkx1, nk2, kp;
  int ubc[2], wbc[2];
  int thbc[8][2];
};

static __global__ void k_les_bc(LesBcArgs a) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.nkx1 * a.nk2) return;
  const int m = idx / a.nk2, kq = idx % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp, c = (size_t)m * a.kp + kq;
  const int nyp = a.nyp;
  auto P = [&](double2* f, int j) -> double2& { return f[(size_t)j * ps + c]; };
  for (int q = 0; q < 2; ++q) {
    double2* cu = a.cu[q == 0 ? 0 : 2];
    const int* b = q == 0 ? a.ubc : a.wbc;
    if (b[1] == 1) { P(cu, nyp) = P(cu, nyp - 1); P(cu, nyp + 1) = P(cu, nyp); }
    if (b[0] == 1) { P(cu, 1) = P(cu, 2); P(cu, 0) = P(cu, 1); }
  }
  for (int n = 0; n < a.nth; ++n) {
    double2* ct = a.cth[n];
    if (a.thbc[n][1] == 1) { P(ct, nyp) = P(ct, nyp - 1); P(ct, nyp + 1) = P(ct, nyp); }
    if (a.thbc[n][0] == 1) { P(ct, 1) = P(ct, 2); P(ct, 0) = P(ct, 1); }
  }
}

// ---------------------------------------------------------------------------
// strain-rate tensor in Fourier space (compute_strain_chan, :1463-1510 and the
// ghost_CS2_mpi sentinel of :2521-2527); one thread per (j, m, kq)
struct StrainArgs {
  const double2* cu[3];
  double2* S[6];
  const double* kx;
  const double* kz;
  const double* dy;
  const double* dyf;
  FGeom g;
};

static __global__ void k_strain(StrainArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double2 u1 = a.cu[0][idx], u2 = a.cu[1][idx], u3 = a.cu[2][idx];
  a.S[0][idx] = mul_ik(kxm, u1);
  a.S[2][idx] = mul_ik(kzq, u3);
  a.S[4][idx] = 0.5 * (mul_ik(kzq, u1) + mul_ik(kxm, u3));
  if (j <= a.g.nyp) {
    const double2 u2p = a.cu[1][idx + a.g.ps];
    a.S[1][idx] = make_double2((u2p.x - u2.x) / a.dyf[j], (u2p.y - u2.y) / a.dyf[j]);
  } else {
    a.S[1][idx] = make_double2(-10000.0, 0.0);
  }
  if (j >= 1) {
    const double2 u1m = a.cu[0][idx - a.g.ps], u3m = a.cu[2][idx - a.g.ps];
    a.S[3][idx] = 0.5 * (make_double2((u1.x - u1m.x) / a.dy[j], (u1.y - u1m.y) / a.dy[j]) + mul_ik(kxm, u2));
    a.S[5][idx] = 0.5 * (mul_ik(kzq, u2) + make_double2((u3.x - u3m.x) / a.dy[j], (u3.y - u3m.y) / a.dy[j]));
  } else {
    a.S[3][idx] = make_double2(0.0, 0.0);
    a.S[5][idx] = make_double2(0.0, 0.0);
  }
}

// ---------------------------------------------------------------------------
// pointwise eddy viscosity and stresses in physical space (:123-241, Smagorinsky)
// S[0..5] in: strain components (S2 is zeroed on output, as the reference
// does); out: |S| S_ij at GYF (S1, S3, S5), |S|_GY (S_ij - implicit part) at GY
// (S4, S6); tmp[0] = nu_t dU1/dy, tmp[1] = nu_t dU3/dy at GY; nu_t at GY.
template <typename P>
struct LesPointArgs {
  P* S[6];
  const P* u1;
  const P* u3;
  P* nu_t;
  P* nu_f;               // dynamic model only: clipped nu_t at GYF (may be null)
  P* tmp[2];
  const double* dy;
  const double* dyf;
  const double* cf;      // C(y) at GYF (constant model: c_s^2 for all j)
  const double* cg;      // C(y) at GY
  const double* d2f;     // Delta^2 at GYF
  const double* d2g;     // Delta^2 at GY
  int nx, nz, nyp;
  int dynamic;
  int amd;               // AMD models: the GY stresses start at j = 2 (row 1 keeps the strain)
};

// |S| at GYF point j (needs S4, S6 at j and j+1)
template <typename P>
DI double snorm_f(const LesPointArgs<P>& a, size_t o, size_t ps) {
  const double s4 = 0.5 * (a.S[3][o + ps] + a.S[3][o]);
  const double s6 = 0.5 * (a.S[5][o + ps] + a.S[5][o]);
  const double s1 = a.S[0][o], s2 = a.S[1][o], s3 = a.S[2][o], s5 = a.S[4][o];
  return sqrt(2.0 * (s1 * s1) + 4.0 * (s4 * s4) + 4.0 * (s5 * s5) + 2.0 * (s2 * s2) + 4.0 * (s6 * s6) +
              2.0 * (s3 * s3));
}
// |S| at GY point j (GYF components interpolated)
template <typename P>
DI double snorm_g(const LesPointArgs<P>& a, size_t o, size_t ps, int j) {
  const double w1 = a.dyf[j - 1], w0 = a.dyf[j], den = 2.0 * a.dy[j];
  auto I = [&](const P* f) { return (f[o] * w1 + f[o - ps] * w0) / den; };
  const double s1 = I(a.S[0]), s2 = I(a.S[1]), s3 = I(a.S[2]), s5 = I(a.S[4]);
  const double s4 = a.S[3][o], s6 = a.S[5][o];
  return sqrt(2.0 * (s1 * s1) + 4.0 * (s4 * s4) + 4.0 * (s5 * s5) + 2.0 * (s2 * s2) + 4.0 * (s6 * s6) +
              2.0 * (s3 * s3));
}

// pass 1: |S| at GYF and GY into scratch (two planes are read per point)
template <typename P>
__global__ void k_les_norms(LesPointArgs<P> a, P* sf, P* sg) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t ps = (size_t)a.nz * a.nx;
  const size_t tot = (size_t)(a.nyp + 2) * ps;
  if (idx >= tot) return;
  const int j = idx / ps;
  sf[idx] = (j >= 1 && j <= a.nyp) ? snorm_f(a, idx, ps) : 0.0;
  sg[idx] = (j >= 1 && j <= a.nyp + 1) ? snorm_g(a, idx, ps, j) : 0.0;
}

// pass 2: stresses, nu_t and the implicit-part fluxes
template <typename P>
__global__ void k_les_point(LesPointArgs<P> a, const P* sf, const P* sg) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t ps = (size_t)a.nz * a.nx;
  const size_t tot = (size_t)(a.nyp + 2) * ps;
  if (idx >= tot) return;
  const int j = idx / ps;
  const int nyp = a.nyp;
  // eddy viscosity at GY: nu_t = -0.5 delta_y |S| = C Delta^2 |S| (:235-241)
  double nt = 0.0;
  if (j >= 2 && j <= nyp) {
    nt = a.cg[j] * a.d2g[j] * sg[idx];
    if (a.dynamic) nt = fmax(nt, 0.0);
  }
  if (j >= 1 && j <= nyp) {
    const double s = sf[idx];
    if (a.dynamic) {
      const double nf = fmax(a.cf[j] * a.d2f[j] * s, 0.0);
      a.S[0][idx] = -2.0 * nf * a.S[0][idx];
      a.S[2][idx] = -2.0 * nf * a.S[2][idx];
      a.S[4][idx] = -2.0 * nf * a.S[4][idx];
    } else {
      a.S[0][idx] = s * a.S[0][idx];
      a.S[2][idx] = s * a.S[2][idx];
      a.S[4][idx] = s * a.S[4][idx];
    }
    a.S[1][idx] = 0.0;
  }
  if (j >= (a.amd ? 2 : 1) && j <= nyp + 1) {
    const double g = sg[idx];
    const double d1 = 0.5 * (a.u1[idx] - a.u1[idx - ps]) / a.dy[j];
    const double d3 = 0.5 * (a.u3[idx] - a.u3[idx - ps]) / a.dy[j];
    if (a.dynamic) {
      a.S[3][idx] = -2.0 * nt * (a.S[3][idx] - d1);
      a.S[5][idx] = -2.0 * nt * (a.S[5][idx] - d3);
    } else {
      a.S[3][idx] = g * (a.S[3][idx] - d1);
      a.S[5][idx] = g * (a.S[5][idx] - d3);
    }
  }
  // ghost_les_mpi at one rank: nu_t = 0 on planes 1, 2, Nyp, Nyp+1 (:2241-2262)
  if (j <= 2 || j >= nyp) nt = 0.0;
  a.nu_t[idx] = nt;
  if (j >= 2 && j <= nyp) {
    a.tmp[0][idx] = nt * (a.u1[idx] - a.u1[idx - ps]) / a.dy[j];
    a.tmp[1][idx] = nt * (a.u3[idx] - a.u3[idx - ps]) / a.dy[j];
  } else {
    a.tmp[0][idx] = 0.0;
    a.tmp[1][idx] = 0.0;
  }
}

// ---------------------------------------------------------------------------
// cf -= div(tau) in Fourier space (:253-274 scaling, :850-880 divergence);
// T[0..4] = tau11, tau33, tau12, tau13, tau23 (Fourier), T[5..6] = the
// transformed nu_t dU/dy, nu_t dW/dy; scale arrays are delta_yf (GYF) and
// delta_y (GY) (all ones for the dynamic model, whose stresses carry -2 nu_t)
struct LesDivArgs {
  const double2* T[7];
  double2* cf[3];
  const double* kx;
  const double* kz;
  const double* dyf;
  const double* sf;   // delta_yf
  const double* sg;   // delta_y
  FGeom g;
  int j1, j2;
};

static __global__ void k_les_div(LesDivArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  const size_t ps = a.g.ps;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  if (j >= a.j1 && j <= a.j2) {
    const double2 c1 = a.sf[j] * a.T[0][idx], c3 = a.sf[j] * a.T[1][idx], c5 = a.sf[j] * a.T[3][idx];
    const double2 c4 = a.sg[j] * a.T[2][idx], c4p = a.sg[j + 1] * a.T[2][idx + ps];
    const double2 c6 = a.sg[j] * a.T[4][idx], c6p = a.sg[j + 1] * a.T[4][idx + ps];
    const double idf = a.dyf[j];
    a.cf[0][idx] = a.cf[0][idx] - mul_ik(kxm, c1) - make_double2((c4p.x - c4.x) / idf, (c4p.y - c4.y) / idf) -
                   mul_ik(kzq, c5);
    a.cf[2][idx] = a.cf[2][idx] - mul_ik(kxm, c5) - make_double2((c6p.x - c6.x) / idf, (c6p.y - c6.y) / idf) -
                   mul_ik(kzq, c3);
  }
  if (j >= 2 && j <= a.g.nyp) {
    const double2 c4 = a.sg[j] * a.T[2][idx], c6 = a.sg[j] * a.T[4][idx];
    a.cf[1][idx] = a.cf[1][idx] - mul_ik(kxm, c4) - mul_ik(kzq, c6) + mul_ik(kxm, a.T[5][idx]) +
                   mul_ik(kzq, a.T[6][idx]);
  }
}

// ---------------------------------------------------------------------------
// eps_sgs1 (for/les.f90:924-1068): the plane mean of u_i times the SGS force
// F_i that k_les_div adds to cf_i, formed at the first substep of a step that
// follows a statistics save.  The reference transforms each F_i to physical
// space and sums u_i F_i over the plane; both factors are band-limited, so the
// plane mean is the Parseval sum over the retained modes (weight 2 for kx > 0,
// the kx = 0 column through the Hermitian part of u).  F1 and F3 live on GYF
// planes and are averaged onto GY plane j from planes j and j - 1; F2 (with
// the explicit cross terms ikx T5 + ikz T6) is on GY.  One block per plane,
// out[j] for j = 2..Nyp and 0 elsewhere.
struct EpsSgsArgs {
  const double2* cu[3];
  const double2* T[7];
  const double* kx;
  const double* kz;
  const double* dyf;
  const double* sf;   // delta_yf
  const double* sg;   // delta_y
  FGeom g;
  double* out;
};

static constexpr int EPS_THREADS = 256;

static __global__ void __launch_bounds__(EPS_THREADS) k_eps_sgs1(EpsSgsArgs a) {
  const int j = blockIdx.x;
  const int nyp = a.g.nyp;
  const size_t ps = a.g.ps;
  double acc = 0.0;
  if (j >= 2 && j <= nyp) {
    const int nmodes = a.g.nkx1 * a.g.nk2;
    for (int idx = threadIdx.x; idx < nmodes; idx += EPS_THREADS) {
      const int m = idx / a.g.nk2, kq = idx - m * a.g.nk2;
      const bool m0 = m == 0;
      const int kqm = kq == 0 ? 0 : a.g.nk2 - kq;
      const size_t col = (size_t)m * a.g.kp;
      const double kxm = a.kx[m], kzq = a.kz[kq];
      auto ld = [&](const double2* f, int jj) -> double2 {
        const size_t o = (size_t)jj * ps + col;
        double2 v = f[o + kq];
        if (m0) {
          const double2 u = f[o + kqm];
          v = make_double2(0.5 * (v.x + u.x), 0.5 * (v.y - u.y));
        }
        return v;
      };
      auto dot = [](double2 p, double2 q) { return p.x * q.x + p.y * q.y; };
      // F1, F3 on GYF plane jj (the cf1, cf3 terms of k_les_div)
      auto f13 = [&](int jj, double2& F1, double2& F3) {
        const size_t o = (size_t)jj * ps + col + kq;
        const double s = a.sf[jj], g0 = a.sg[jj], g1 = a.sg[jj + 1], idf = a.dyf[jj];
        const double2 c1 = s * a.T[0][o], c3 = s * a.T[1][o], c5 = s * a.T[3][o];
        const double2 c4 = g0 * a.T[2][o], c4p = g1 * a.T[2][o + ps];
        const double2 c6 = g0 * a.T[4][o], c6p = g1 * a.T[4][o + ps];
        F1 = make_double2(0.0, 0.0) - mul_ik(kxm, c1) - make_double2((c4p.x - c4.x) / idf, (c4p.y - c4.y) / idf) -
             mul_ik(kzq, c5);
        F3 = make_double2(0.0, 0.0) - mul_ik(kxm, c5) - make_double2((c6p.x - c6.x) / idf, (c6p.y - c6.y) / idf) -
             mul_ik(kzq, c3);
      };
      double2 F1, F3, F1m, F3m;
      f13(j, F1, F3);
      f13(j - 1, F1m, F3m);
      const size_t o = (size_t)j * ps + col + kq;
      const double2 c4 = a.sg[j] * a.T[2][o], c6 = a.sg[j] * a.T[4][o];
      const double2 F2 = make_double2(0.0, 0.0) - mul_ik(kxm, c4) - mul_ik(kzq, c6) + mul_ik(kxm, a.T[5][o]) +
                         mul_ik(kzq, a.T[6][o]);
      const double w = m0 ? 1.0 : 2.0;
      acc += w * (0.5 * (dot(ld(a.cu[0], j), F1) + dot(ld(a.cu[0], j - 1), F1m)) +
                  0.5 * (dot(ld(a.cu[2], j), F3) + dot(ld(a.cu[2], j - 1), F3m)) + dot(ld(a.cu[1], j), F2));
    }
  }
  // fixed-order block reduction: the result does not depend on scheduling
  __shared__ double red[EPS_THREADS / 32];
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < EPS_THREADS / 32; ++w) s += red[w];
    a.out[j] = s;
  }
}

// ---------------------------------------------------------------------------
// scalar SGS flux (:1144-1200): out_x = ikx cth, out_z = ikz cth on planes 1..Nyp+1
struct ThGradArgs {
  const double2* cth[8];
  double2* gx[8];
  double2* gz[8];
  const double* kx;
  const double* kz;
  FGeom g;
  int nth;
};

static __global__ void k_th_grad(ThGradArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  for (int n = 0; n < a.nth; ++n) {
    double2 t = j >= 1 ? a.cth[n][idx] : make_double2(0.0, 0.0);
    a.gx[n][idx] = mul_ik(a.kx[m], t);
    a.gz[n][idx] = mul_ik(a.kz[kq], t);
  }
}

// physical: f *= nu_t on planes 1..Nyp+1
template <typename P>
struct ScaleArgs {
  P* f[2 * 8];
  int nfield;
  const P* w;
  size_t ps;
  int nyp;
};

template <typename P>
__global__ void k_scale_by(ScaleArgs<P> a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  const double w = (j >= 1) ? a.w[idx] : 0.0;
  for (int q = 0; q < a.nfield; ++q) a.f[q][idx] = w * a.f[q][idx];
}

struct ThDivArgs {
  const double2* fx[8];
  const double2* fz[8];
  double2* cfth[8];
  const double* kx;
  const double* kz;
  FGeom g;
  int nth;
  int jst[8], jet[8];
};

static __global__ void k_th_div(ThDivArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  for (int n = 0; n < a.nth; ++n) {
    if (j < a.jst[n] || j > a.jet[n]) continue;
    a.cfth[n][idx] = a.cfth[n][idx] + mul_ik(a.kx[m], a.fx[n][idx]) + mul_ik(a.kz[kq], a.fz[n][idx]);
  }
}

// ---------------------------------------------------------------------------
// cf -= NL ; cr += temp5*cf on each field's rows (:299-459 accumulation, :468-482, :610-617)
struct CfFinishArgs {
  double2* cf[SOLVE_NF];
  double2* cr[SOLVE_NF];
  const void* nl[SOLVE_NF];
  int nl_fp32;
  int lo[SOLVE_NF], hi[SOLVE_NF];
  int nf;
  double temp5;
  FGeom g;
};

static __global__ void k_cf_finish(CfFinishArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int j = idx / a.g.ps;
  for (int f = 0; f < a.nf; ++f) {
    if (j < a.lo[f] || j > a.hi[f]) continue;
    double2 nl;
    if (a.nl_fp32) { float2 v = ((const float2*)a.nl[f])[idx]; nl = make_double2(v.x, v.y); }
    else nl = ((const double2*)a.nl[f])[idx];
    const double2 cf = a.cf[f][idx] - nl;
    a.cf[f][idx] = cf;
    a.cr[f][idx] = a.cr[f][idx] + a.temp5 * cf;
  }
}

// ---------------------------------------------------------------------------
// Crank-Nicolson in y per physical column with the eddy viscosity
// (:494-547 explicit half, :625-646 scalars, :657-877 implicit rows, Thomas
// :1335-1496).
template <typename P>
struct PhysSolveArgs {
  const double* r[SOLVE_NF];    // inverse-transformed cr
  double* u[SOLVE_NF];          // in: physical field at the start; out: solution on the write rows
  const P* nu_t;                // eddy viscosity / diffusivities (the LES model's precision)
  const P* kap[8];
  const double* dy;
  const double* dyf;
  const double* idy;            // 1/dy, 1/dyf
  const double* idyf;
  int nf, nth, n, nyp, cols;
  double temp1, temp2, nu_v;
  int jstart, jend;
  int jst[8], jet[8];
  double pr[8];
  int ubc[2], vbc[2], wbc[2];
  double uc1[2], vc1[2], wc1[2];
  int thbc[8][2];
  double thc1[8][2];
};

// One warp per (field, physical column): each lane builds R consecutive rows
// of the column's system and csolve::warp_tridiag solves it (the partition
// method of the Fourier-space solves).  Rows past Ny+1 are identity rows; the
// last real row has no upper coefficient, so they do not couple.
// TILED (when the columns of a field are a multiple of PS_W): a block of PS_W
// warps takes PS_W adjacent columns of one field and first copies their u, r
// and nu_t rows into shared memory with coalesced PS_W-wide row loads (a lane
// otherwise reads 8 scattered bytes per row); the solution goes back the same
// way.  Untiled: each warp reads its column from global memory.
constexpr int PS_W = 8;
template <typename P, int R, bool TILED>
__global__ void __launch_bounds__(TILED ? 32 * PS_W : 128) k_phys_solve(PhysSolveArgs<P> a) {
  using namespace csolve;
  extern __shared__ double ps_tile[];
  const int lane = threadIdx.x & 31;
  const size_t gid = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gid >= (size_t)a.nf * a.cols) return;   // the whole warp (TILED: block) leaves together
  const int f = gid / a.cols;
  const size_t col = gid % a.cols;
  const size_t ps = a.cols;
  const int n = a.n, nyp = a.nyp;
  const double* r = a.r[f];
  double* u = a.u[f];
  const P* nt = f < 3 ? a.nu_t : a.kap[f - 3];
  // tiles [n][PS_W] of u, r, nu_t; c = this warp's column in them
  double* tu = ps_tile;
  double* tr = tu + (size_t)n * PS_W;
  double* tn = tr + (size_t)n * PS_W;
  const int c = threadIdx.x >> 5;
  const size_t col0 = col - c;
  if (TILED) {
    for (int idx = threadIdx.x; idx < n * PS_W; idx += blockDim.x) {
      const size_t o = (size_t)(idx / PS_W) * ps + col0 + idx % PS_W;
      tu[idx] = u[o];
      tr[idx] = r[o];
      tn[idx] = (double)nt[o];
    }
    __syncthreads();
  }
  // row j (and its neighbours) of u, r, nu_t in this column
  auto U = [&](int j) -> double { return TILED ? tu[j * PS_W + c] : u[(size_t)j * ps + col]; };
  auto RR = [&](int j) -> double { return TILED ? tr[j * PS_W + c] : r[(size_t)j * ps + col]; };
  auto NT = [&](int j) -> double { return TILED ? tn[j * PS_W + c] : (double)nt[(size_t)j * ps + col]; };
  int lo, hi, w0, b0, b1;
  double c0v, c1v, tc;
  if (f == 1) { lo = 2; hi = nyp; w0 = 1; b0 = a.vbc[0]; b1 = a.vbc[1]; c0v = a.vc1[0]; c1v = a.vc1[1]; tc = a.temp1 * a.nu_v; }
  else if (f == 0 || f == 2) {
    lo = a.jstart; hi = a.jend; w0 = lo - 1;
    b0 = f == 0 ? a.ubc[0] : a.wbc[0]; b1 = f == 0 ? a.ubc[1] : a.wbc[1];
    c0v = f == 0 ? a.uc1[0] : a.wc1[0]; c1v = f == 0 ? a.uc1[1] : a.wc1[1];
    tc = a.temp1 * a.nu_v;
  } else {
    const int t = f - 3;
    lo = a.jst[t]; hi = a.jet[t]; w0 = lo - 1;
    b0 = a.thbc[t][0]; b1 = a.thbc[t][1]; c0v = a.thc1[t][0]; c1v = a.thc1[t][1];
    tc = a.temp1 / a.pr[t] * a.nu_v;
  }
  // row j of the system
  auto row = [&](int j, double& A, double& B, double& C, double& D) {
    A = 0.0; B = 1.0; C = 0.0; D = 0.0;
    if (j >= lo && j <= hi) {
      const double uc = U(j), um = U(j - 1), up = U(j + 1);
      double rhs = RR(j);
      // the reference's quotients by dy and dyf, as products with the
      // precomputed reciprocals (FP64 division is a long instruction sequence)
      if (f == 1) {
        const double idyj = a.idy[j], idyfj = a.idyf[j], idyfm = a.idyf[j - 1];
        const double ntp = 0.5 * (NT(j) + NT(j + 1)), ntm = 0.5 * (NT(j) + NT(j - 1));
        const double gp = (up - uc) * idyfj, gm = (uc - um) * idyfm;
        rhs += tc * ((gp - gm) * idyj);
        rhs += a.temp2 * ((ntp * gp - ntm * gm) * idyj);
        const double wp = idyfj * idyj, wm = idyfm * idyj;
        A = -(tc + a.temp2 * ntm) * wm;
        B = 1. + (tc + a.temp2 * ntp) * wp + (tc + a.temp2 * ntm) * wm;
        C = -(tc + a.temp2 * ntp) * wp;
      } else {
        const double idyj = a.idy[j], idyj1 = a.idy[j + 1], idyfj = a.idyf[j];
        const double ntp = NT(j + 1), ntc = NT(j);
        const double gp = (up - uc) * idyj1, gm = (uc - um) * idyj;
        rhs += tc * ((gp - gm) * idyfj);
        rhs += a.temp2 * ((ntp * gp - ntc * gm) * idyfj);
        const double wp = idyj1 * idyfj, wm = idyj * idyfj;
        A = -(tc + a.temp2 * ntc) * wm;
        B = 1. + (tc + a.temp2 * ntp) * wp + (tc + a.temp2 * ntc) * wm;
        C = -(tc + a.temp2 * ntp) * wp;
      }
      D = rhs;
    }
    if (f == 1) {
      if (b0 == 0 && (j == 1 || j == 2)) { A = 0; B = 1; C = 0; D = c0v; }
      if (b0 == 1 && j == 1) { A = 0; B = -1; C = 1; D = a.dyf[1] * c0v; }
      if (j == 0) { A = 0; B = 1; C = 0; D = 0; }
      if (b1 == 0 && (j == nyp || j == nyp + 1)) { A = 0; B = 1; C = 0; D = c1v; }
      if (b1 == 1 && j == nyp + 1) { A = -1; B = 1; C = 0; D = a.dyf[nyp] * c1v; }
    } else {
      if (j == 0 || j == nyp + 1) { A = 0; B = 1; C = 0; D = 0; }
      if (j == 1) {
        if (b0 == 0) { A = 0; B = 1; C = 0; D = c0v; }
        else { A = 0; B = -1; C = 1; D = a.dy[2] * c0v; }
      }
      if (j == nyp) {
        if (b1 == 0) { A = 0; B = 1; C = 0; D = c1v; }
        else { A = -1; B = 1; C = 0; D = a.dy[nyp] * c1v; }
      }
    }
  };
  double Am[R], Bm[R], Cm[R];
  double2 Dm[R];
#pragma unroll
  for (int rr = 0; rr < R; ++rr) {
    const int j = lane * R + rr;
    double A = 0.0, B = 1.0, C = 0.0, D = 0.0;
    if (j < n) row(j, A, B, C, D);
    Am[rr] = A; Bm[rr] = B; Cm[rr] = C; Dm[rr] = make_double2(D, 0.0);
  }
  warp_tridiag<R>(Am, Bm, Cm, Dm, lane);
  // every lane's reads of u (its rows and their neighbours) are done: write
  // the solution on the rows the reference writes
  const int w1 = nyp + 1;
  if (TILED) {
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int j = lane * R + rr;
      if (j < n && j >= w0 && j <= w1) tu[j * PS_W + c] = Dm[rr].x;
    }
    __syncthreads();
    // rows outside the write range hold the values just read: rewriting them
    // leaves them unchanged
    for (int idx = threadIdx.x; idx < n * PS_W; idx += blockDim.x)
      u[(size_t)(idx / PS_W) * ps + col0 + idx % PS_W] = tu[idx];
  } else {
    __syncwarp();
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int j = lane * R + rr;
      if (j < n && j >= w0 && j <= w1) u[(size_t)j * ps + col] = Dm[rr].x;
    }
  }
}

// ---------------------------------------------------------------------------
// Dynamic Smagorinsky coefficient (Germano identity with Lilly's least-squares
// contraction, sharp spectral test filter of width 2 Delta in x and z).  The
// reference stops on this model (for/les.f90:272-277); its commented-out test
// filters are at :1773-1990.
//
// Field order of the 21 test-filtered inputs, all at GYF points j = 1..Nyp:
//   0..2   U_a      (u1, (u2(j) + u2(j+1)) / 2, u3)
//   3..8   S_ab     (11, 22, 33, 12, 13, 23; S12, S23 averaged from GY)
//   9..14  U_a U_b  (same pair order)
//   15..20 |S| S_ab
template <typename P>
struct DynPrepArgs {
  const P* u[3];
  const P* S[6];          // raw strain components S1..S6 (physical)
  const P* sf;            // |S| at GYF
  P* out[DYN_NF];
  int nyp;
  size_t ps;              // Nx * Nz
};

__device__ __constant__ int c_pair_a[6] = {0, 1, 2, 0, 0, 1};
__device__ __constant__ int c_pair_b[6] = {0, 1, 2, 1, 2, 2};

template <typename P>
__global__ void k_dyn_prep(DynPrepArgs<P> a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  if (j < 1 || j > a.nyp) {
    for (int q = 0; q < DYN_NF; ++q) a.out[q][idx] = 0.0;
    return;
  }
  double U[3], S[6];
  U[0] = a.u[0][idx];
  U[1] = 0.5 * (a.u[1][idx] + a.u[1][idx + a.ps]);
  U[2] = a.u[2][idx];
  S[0] = a.S[0][idx];
  S[1] = a.S[1][idx];
  S[2] = a.S[2][idx];
  S[3] = 0.5 * (a.S[3][idx] + a.S[3][idx + a.ps]);
  S[4] = a.S[4][idx];
  S[5] = 0.5 * (a.S[5][idx] + a.S[5][idx + a.ps]);
  const double s = a.sf[idx];
#pragma unroll
  for (int q = 0; q < 3; ++q) a.out[q][idx] = U[q];
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    a.out[3 + q][idx] = S[q];
    a.out[9 + q][idx] = U[c_pair_a[q]] * U[c_pair_b[q]];
    a.out[15 + q][idx] = s * S[q];
  }
}

// Sharp spectral test filter: zero the stored modes with kx index > mx or
// |kz index| > mz (packed z index kq: kz = kq for kq <= Nkz, else kq - nk2).
struct MaskArgs {
  double2* f[NF_MAX];
  int nfield, mx, mz, nkz;
  FGeom g;
};

static __global__ void k_test_mask(MaskArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int kz = kq <= a.nkz ? kq : a.g.nk2 - kq;
  if (m > a.mx || kz > a.mz) {
    for (int q = 0; q < a.nfield; ++q) a.f[q][idx] = make_double2(0.0, 0.0);
  }
}

// Per-plane Germano/Lilly sums: `nslice` blocks per GYF plane j
// (blockIdx.y + 1), each summing a strided share of the plane's points, so a
// 129-plane grid still fills every SM.  sums[j][slice][0..5] = sum of
// L_ab M_ab per pair, [6..11] of M_ab^2; k_dyn_coef adds the slices in order.
constexpr int DYN_MAX_SLICES = 16;
template <typename P>
struct DynContractArgs {
  const P* F[DYN_NF];         // test-filtered fields (physical)
  const P* u[3];              // unfiltered u1, u2 (GY), u3
  const double* d2f;          // Delta^2 at GYF
  double* sums;               // [(Ny+2)][nslice][12]
  int nyp, nslice;
  size_t ps;
  double ratio2;              // (test / grid width)^2
};

template <typename P>
__global__ void __launch_bounds__(256) k_dyn_contract(DynContractArgs<P> a) {
  const int j = blockIdx.y + 1;
  const size_t base = (size_t)j * a.ps;
  double acc[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) acc[q] = 0.0;
  const double w2[6] = {1.0, 1.0, 1.0, 2.0, 2.0, 2.0};
  const double d2 = a.d2f[j];
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.ps;
       p += (size_t)a.nslice * blockDim.x) {
    const size_t o = base + p;
    double Uh[3], Sh[6];
#pragma unroll
    for (int q = 0; q < 3; ++q) Uh[q] = a.F[q][o];
#pragma unroll
    for (int q = 0; q < 6; ++q) Sh[q] = a.F[3 + q][o];
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) sum = sum + w2[q] * 2.0 * (Sh[q] * Sh[q]);
    const double sh = sqrt(sum);
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      const double L = a.F[9 + q][o] - Uh[c_pair_a[q]] * Uh[c_pair_b[q]];
      const double M = 2.0 * d2 * (a.F[15 + q][o] - a.ratio2 * sh * Sh[q]);
      acc[q] += L * M;
      acc[6 + q] += M * M;
    }
  }
  __shared__ double red[8][12];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    double v = acc[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    a.sums[((size_t)j * a.nslice + blockIdx.x) * 12 + threadIdx.x] = v;
  }
}

// C(y) at GYF from the plane sums, and interpolated to GY (for/les.f90's
// GYF-to-GY weights); one thread per plane, planes 0..Ny+1.
static __global__ void k_dyn_coef(const double* sums, const double* dy, const double* dyf, double* cf, double* cg,
                           int nyp, int nslice, double nps) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > nyp + 1) return;
  const double w2[6] = {1.0, 1.0, 1.0, 2.0, 2.0, 2.0};
  auto C = [&](int jj) -> double {
    if (jj < 1 || jj > nyp) return 0.0;
    double num = 0.0, den = 0.0;
    for (int q = 0; q < 6; ++q) {
      double sn = 0.0, sd = 0.0;
      for (int sl = 0; sl < nslice; ++sl) {
        sn += sums[((size_t)jj * nslice + sl) * 12 + q];
        sd += sums[((size_t)jj * nslice + sl) * 12 + 6 + q];
      }
      num += w2[q] * (sn / nps);
      den += w2[q] * (sd / nps);
    }
    return den > 0.0 ? num / den : 0.0;
  };
  const double cj = C(j);
  cf[j] = cj;
  cg[j] = (j >= 2 && j <= nyp) ? (cj * dyf[j - 1] + C(j - 1) * dyf[j]) / (2.0 * dy[j]) : 0.0;
}

// ---------------------------------------------------------------------------
// Anisotropic minimum dissipation models (for/les.f90:279-850): Rozema (4)
// with the plain rotation tensor, Verstappen (5) with the scaled-invariant
// strain and rotation tensors and, for the scalar, all velocity and scalar
// gradients.  Fourier inputs, one thread per (j, m, kq).
struct AmdFourierArgs {
  const double2* cu[3];
  const double2* cth[8];
  double2* O[3];          // O4, O5, O6
  double2* SI[6];         // model 5: SI1..SI6
  double2* G[9];          // model 5: du1dx du2dy du3dz du2dx du3dx du1dz du2dz du1dy du3dy
  double2* T[3 * 8];      // model 5: dth/dx, dth/dy, dth/dz per scalar
  const double* kx;
  const double* kz;
  const double* dy;
  const double* dyf;
  double deltax, deltaz;  // dx(1) beta, dz(1) beta
  int model, nth;
  FGeom g;
};

DI double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
DI double2 cdiff_over(double2 a, double2 b, double d) { return make_double2((a.x - b.x) / d, (a.y - b.y) / d); }

static __global__ void k_amd_fourier(const __grid_constant__ AmdFourierArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  const size_t ps = a.g.ps;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double2 u1 = a.cu[0][idx], u2 = a.cu[1][idx], u3 = a.cu[2][idx];
  const double2 z = make_double2(0.0, 0.0);
  const bool inv = a.model == 5;
  const double rzx = a.deltaz / a.deltax, rxz = a.deltax / a.deltaz;
  // omega_13 (:1595, :1641): all planes
  a.O[1][idx] = inv ? 0.5 * (cscale(mul_ik(kzq, u1), rzx) - cscale(mul_ik(kxm, u3), rxz))
                    : 0.5 * (mul_ik(kzq, u1) - mul_ik(kxm, u3));
  if (j >= 1) {
    const double2 d1 = cdiff_over(u1, a.cu[0][idx - ps], a.dy[j]);
    const double2 d3 = cdiff_over(u3, a.cu[2][idx - ps], a.dy[j]);
    if (inv) {
      const double dly = a.dy[j] * 2.0;
      const double ryx = dly / a.deltax, rxy = a.deltax / dly, rzy = a.deltaz / dly, ryz = dly / a.deltaz;
      a.O[0][idx] = 0.5 * (cscale(d1, ryx) - cscale(mul_ik(kxm, u2), rxy));
      a.O[2][idx] = 0.5 * (cscale(mul_ik(kzq, u2), rzy) - cscale(d3, ryz));
      a.SI[3][idx] = 0.5 * (cscale(d1, ryx) + cscale(mul_ik(kxm, u2), rxy));
      a.SI[5][idx] = 0.5 * (cscale(mul_ik(kzq, u2), rzy) + cscale(d3, ryz));
    } else {
      a.O[0][idx] = 0.5 * (d1 - mul_ik(kxm, u2));
      a.O[2][idx] = 0.5 * (mul_ik(kzq, u2) - d3);
    }
  } else {
    a.O[0][idx] = z;
    a.O[2][idx] = z;
    if (inv) { a.SI[3][idx] = z; a.SI[5][idx] = z; }
  }
  if (!inv) return;
  // scaled-invariant strain (:1514-1577)
  a.SI[0][idx] = mul_ik(kxm, u1);
  a.SI[2][idx] = mul_ik(kzq, u3);
  a.SI[4][idx] = 0.5 * (cscale(mul_ik(kzq, u1), rzx) + cscale(mul_ik(kxm, u3), rxz));
  a.SI[1][idx] = j <= a.g.nyp ? cdiff_over(a.cu[1][idx + ps], u2, a.dyf[j]) : make_double2(-10000.0, 0.0);
  // all gradients (:1681-1767)
  a.G[0][idx] = mul_ik(kxm, u1);
  a.G[2][idx] = mul_ik(kzq, u3);
  a.G[3][idx] = mul_ik(kxm, u2);
  a.G[4][idx] = mul_ik(kxm, u3);
  a.G[5][idx] = mul_ik(kzq, u1);
  a.G[6][idx] = mul_ik(kzq, u2);
  if (j >= 1) {
    a.G[7][idx] = cdiff_over(u1, a.cu[0][idx - ps], a.dy[j]);
    a.G[1][idx] = cdiff_over(u2, a.cu[1][idx - ps], a.dyf[j - 1]);   // dyf(j-1), as the reference
    a.G[8][idx] = cdiff_over(u3, a.cu[2][idx - ps], a.dy[j]);
  } else {
    a.G[7][idx] = z;
    a.G[1][idx] = z;
    a.G[8][idx] = z;
  }
  for (int n = 0; n < a.nth; ++n) {
    if (j >= 1) {
      const double2 t = a.cth[n][idx];
      a.T[3 * n][idx] = mul_ik(kxm, t);
      a.T[3 * n + 1][idx] = cdiff_over(t, a.cth[n][idx - ps], a.dy[j]);
      a.T[3 * n + 2][idx] = mul_ik(kzq, t);
    } else {
      a.T[3 * n][idx] = z;
      a.T[3 * n + 1][idx] = z;
      a.T[3 * n + 2][idx] = z;
    }
  }
}

// max(0, -(I3 - I4)) / (I1 - I2) from the six strain and three rotation
// components at one point, with direction weights (wx, wy, wz)
// (for/les.f90:300-350 form; unit weights give the :591-650 form)
DI double amd_ratio(double a1, double a2, double a3, double a4, double a5, double a6, double o4, double o5,
                    double o6, double dx, double dy, double dz) {
  const double i3 = dx * (a1 * a1 * a1) + dy * (a2 * a2 * a2) + dz * (a3 * a3 * a3) +
                    (2.0 * dx + dy) * a1 * (a4 * a4) + (2.0 * dx + dz) * a1 * (a5 * a5) +
                    (2.0 * dy + dx) * a2 * (a4 * a4) + (2.0 * dy + dz) * a2 * (a6 * a6) +
                    (2.0 * dz + dx) * a3 * (a5 * a5) + (2.0 * dz + dy) * a3 * (a6 * a6) +
                    2.0 * (dx + dy + dz) * a4 * a5 * a6;
  const double num = -i3 - dy * a1 * (o4 * o4) - dz * a1 * (o5 * o5) - dx * a2 * (o4 * o4) -
                     dz * a2 * (o6 * o6) - dx * a3 * (o5 * o5) - dy * a3 * (o6 * o6) -
                     2.0 * dz * a4 * o5 * o6 + 2.0 * dy * a5 * o4 * o6 - 2.0 * dx * a6 * o4 * o5;
  if (num <= 0.0) return 0.0;
  const double den = a1 * a1 + a2 * a2 + a3 * a3 + 2.0 * (a4 * a4) + 2.0 * (o4 * o4) + 2.0 * (a5 * a5) +
                     2.0 * (o5 * o5) + 2.0 * (a6 * a6) + 2.0 * (o6 * o6);
  return num / den;
}

// AMD coefficient at GYF (sf) and GY (sg) points, physical, one thread per point.
// Model 4: strain S, weights delta_i^2 with (2 dy(j))^2 in y, GYF rows 1..Nyp,
// GY rows 2..Nyp+1.  Model 5: invariant strain, unit weights, GYF rows
// jstart..jend, GY rows 2..Nyp.
template <typename P>
struct AmdCoefArgs {
  const P* S[6];
  const P* O[3];
  const double* dy;
  const double* dyf;
  P* sf;
  P* sg;
  double wx, wz;          // (dx beta)^2, (dz beta)^2 (model 4)
  int model, nyp, jstart, jend;
  size_t ps;
};

template <typename P>
__global__ void k_amd_coef(const __grid_constant__ AmdCoefArgs<P> a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  const size_t ps = a.ps;
  const bool m4 = a.model == 4;
  const int f0 = m4 ? 1 : a.jstart, f1 = m4 ? a.nyp : a.jend;
  const int g1 = m4 ? a.nyp + 1 : a.nyp;
  double sfv = 0.0, sgv = 0.0;
  if (j >= f0 && j <= f1) {
    const double wy = m4 ? (a.dy[j] * 2.0) * (a.dy[j] * 2.0) : 1.0;
    const double wx = m4 ? a.wx : 1.0, wz = m4 ? a.wz : 1.0;
    auto av = [&](const P* f) { return 0.5 * ((double)f[idx + ps] + (double)f[idx]); };
    sfv = amd_ratio(a.S[0][idx], a.S[1][idx], a.S[2][idx], av(a.S[3]), a.S[4][idx], av(a.S[5]), av(a.O[0]),
                    a.O[1][idx], av(a.O[2]), wx, wy, wz);
  }
  if (j >= 2 && j <= g1) {
    const double wy = m4 ? (a.dy[j] * 2.0) * (a.dy[j] * 2.0) : 1.0;
    const double wx = m4 ? a.wx : 1.0, wz = m4 ? a.wz : 1.0;
    const double w1 = a.dyf[j - 1], w0 = a.dyf[j], den = 2.0 * a.dy[j];
    auto ip = [&](const P* f) { return ((double)f[idx] * w1 + (double)f[idx - ps] * w0) / den; };
    sgv = amd_ratio(ip(a.S[0]), ip(a.S[1]), ip(a.S[2]), a.S[3][idx], ip(a.S[4]), a.S[5][idx], a.O[0][idx],
                    ip(a.O[1]), a.O[2][idx], wx, wy, wz);
  }
  a.sf[idx] = sfv;
  a.sg[idx] = sgv;
}

// Type-5 scalar model (for/les.f90:1239-1380) for every scalar: the horizontal
// fluxes s1_th dth/dx, s1_th dth/dz at GYF rows jstart_th..jend_th into fx, fz
// (zero elsewhere) and kappa_t = -0.5 delta_y temp_th at GY rows 2..Nyp, zero
// on planes 0, 1, 2, Nyp, Nyp+1 (ghost_les_th_mpi at one rank).
template <typename P>
struct AmdThArgs {
  const P* G[9];
  const P* T[3 * 8];
  P* fx[8];
  P* fz[8];
  P* kap[8];
  const double* dy;
  const double* dyf;
  const double* hdy;      // -0.5 delta_y(j)
  double deltax, deltaz;
  int nth, nyp;
  int jst[8], jet[8];
  size_t ps;
};

template <typename P>
__global__ void k_amd_th(const __grid_constant__ AmdThArgs<P> a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  const size_t ps = a.ps;
  const double dx2 = a.deltax * a.deltax, dz2 = a.deltaz * a.deltaz;
  for (int n = 0; n < a.nth; ++n) {
    const P* tx = a.T[3 * n];
    const P* ty = a.T[3 * n + 1];
    const P* tz = a.T[3 * n + 2];
    double s1 = 0.0;
    if (j >= a.jst[n] && j <= a.jet[n]) {
      const double dly = a.dyf[j] * 2.0, dy2 = dly * dly;
      const double tyf = 0.5 * (ty[idx + ps] + ty[idx]);
      const double txj = tx[idx], tzj = tz[idx];
      auto av = [&](const P* f) { return 0.5 * ((double)f[idx + ps] + (double)f[idx]); };
      const double num = -(dx2 * a.G[0][idx] * (txj * txj) + dy2 * a.G[1][idx] * (tyf * tyf) +
                           dz2 * a.G[2][idx] * (tzj * tzj) +
                           (dy2 * av(a.G[7]) + dx2 * av(a.G[3])) * txj * tyf +
                           (dz2 * a.G[5][idx] + dx2 * a.G[4][idx]) * txj * tzj +
                           (dz2 * av(a.G[6]) + dy2 * av(a.G[8])) * tyf * tzj);
      if (num > 0.0) {
        const double ex = a.deltax * txj, ey = dly * tyf, ez = a.deltaz * tzj;
        s1 = num / (ex * ex + ey * ey + ez * ez);
      }
      a.fx[n][idx] = s1 * txj;
      a.fz[n][idx] = s1 * tzj;
    } else {
      a.fx[n][idx] = 0.0;
      a.fz[n][idx] = 0.0;
    }
    double kt = 0.0;
    if (j >= 3 && j <= a.nyp - 1) {
      const double dly = a.dy[j] * 2.0, dy2 = dly * dly;
      const double w1 = a.dyf[j - 1], w0 = a.dyf[j], den = 2.0 * a.dy[j];
      auto ip = [&](const P* f) { return ((double)f[idx] * w1 + (double)f[idx - ps] * w0) / den; };
      const double txg = ip(tx), tzg = ip(tz), tyg = ty[idx];
      const double num = -(dx2 * ip(a.G[0]) * (txg * txg) + dy2 * ip(a.G[1]) * (tyg * tyg) +
                           dz2 * ip(a.G[2]) * (tzg * tzg) +
                           (dy2 * a.G[7][idx] + dx2 * a.G[3][idx]) * txg * tyg +
                           (dz2 * ip(a.G[5]) + dx2 * ip(a.G[4])) * txg * tzg +
                           (dz2 * a.G[6][idx] + dy2 * a.G[8][idx]) * tyg * tzg);
      if (num > 0.0) {
        const double ex = a.deltax * txg, ey = dly * tyg, ez = a.deltaz * tzg;
        kt = a.hdy[j] * (num / (ex * ex + ey * ey + ez * ez));
      }
    }
    a.kap[n][idx] = kt;
  }
}

// cfth -= ikx (delta_yf/2) F(fx) + ikz (delta_yf/2) F(fz) on rows jstart_th..jend_th (:1391-1412)
struct AmdThDivArgs {
  const double2* fx[8];
  const double2* fz[8];
  double2* cfth[8];
  const double* kx;
  const double* kz;
  const double* dlyf;     // delta_yf(j)
  FGeom g;
  int nth;
  int jst[8], jet[8];
};

static __global__ void k_amd_th_div(const __grid_constant__ AmdThDivArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  const double h = 0.5 * a.dlyf[j];
  for (int n = 0; n < a.nth; ++n) {
    if (j < a.jst[n] || j > a.jet[n]) continue;
    a.cfth[n][idx] = a.cfth[n][idx] - mul_ik(a.kx[m], h * a.fx[n][idx]) - mul_ik(a.kz[kq], h * a.fz[n][idx]);
  }
}

// FP32 -> FP64 copy (the mixed-precision eddy viscosity for the boundary)
