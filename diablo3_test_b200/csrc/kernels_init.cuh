// Initial pressure (poisson_p_chan, for/channel.f90:1026-1234) and the CFL
// reductions of courant (for/advance.f90:47-158), FP64.
#pragma once
#include "common.cuh"
#include "kernels_les.cuh"
#include "kernels_solve.cuh"
#include "kernels_solve2.cuh"

// Gradients whose products form the pressure source, in Fourier space on
// planes 2..Ny (zero elsewhere), in the order the reference squares and
// multiplies them (:1041-1135):
//   0 ikx u1   1 (u2(j+1) - u2(j))/dyf   2 ikz u3
//   3 (u1(j+1) - u1(j-1))/(2 dyf)   4 ikx (u2(j) + u2(j+1))/2
//   5 (u3(j+1) - u3(j-1))/(2 dyf)   6 ikz (u2(j) + u2(j+1))/2
//   7 ikz u1   8 ikx u3
struct PpGradArgs {
  const double2* cu[3];
  double2* G[9];
  const double* kx;
  const double* kz;
  const double* dyf;
  FGeom g;
};

static __global__ void k_pp_grad(const __grid_constant__ PpGradArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)a.g.n * a.g.ps;
  if (idx >= tot) return;
  const int kq = idx % a.g.kp;
  if (kq >= a.g.nk2) return;
  const int m = (idx / a.g.kp) % a.g.nkx1;
  const int j = idx / a.g.ps;
  const double2 z = make_double2(0.0, 0.0);
  if (j < 2 || j > a.g.nyp) {
    for (int q = 0; q < 9; ++q) a.G[q][idx] = z;
    return;
  }
  const size_t ps = a.g.ps;
  const double kxm = a.kx[m], kzq = a.kz[kq], d = a.dyf[j];
  const double2 u1 = a.cu[0][idx], u2 = a.cu[1][idx], u3 = a.cu[2][idx];
  const double2 u2p = a.cu[1][idx + ps];
  const double2 u1p = a.cu[0][idx + ps], u1m = a.cu[0][idx - ps];
  const double2 u3p = a.cu[2][idx + ps], u3m = a.cu[2][idx - ps];
  a.G[0][idx] = mul_ik(kxm, u1);
  a.G[1][idx] = make_double2((u2p.x - u2.x) / d, (u2p.y - u2.y) / d);
  a.G[2][idx] = mul_ik(kzq, u3);
  a.G[3][idx] = make_double2((u1p.x - u1m.x) / (2.0 * d), (u1p.y - u1m.y) / (2.0 * d));
  a.G[4][idx] = mul_ik(kxm, 0.5 * (u2 + u2p));
  a.G[5][idx] = make_double2((u3p.x - u3m.x) / (2.0 * d), (u3p.y - u3m.y) / (2.0 * d));
  a.G[6][idx] = mul_ik(kzq, 0.5 * (u2 + u2p));
  a.G[7][idx] = mul_ik(kzq, u1);
  a.G[8][idx] = mul_ik(kxm, u3);
}

// Physical products on planes 2..Ny: G0^2, G1^2, G2^2, 2 G3 G4, 2 G5 G6, 2 G7 G8
struct PpProdArgs {
  const double* G[9];
  double* Q[6];
  int nyp;
  size_t ps;
};

static __global__ void k_pp_prod(const __grid_constant__ PpProdArgs a) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t tot = (size_t)(a.nyp + 2) * a.ps;
  if (idx >= tot) return;
  const int j = idx / a.ps;
  if (j < 2 || j > a.nyp) {
    for (int q = 0; q < 6; ++q) a.Q[q][idx] = 0.0;
    return;
  }
  const double g0 = a.G[0][idx], g1 = a.G[1][idx], g2 = a.G[2][idx];
  a.Q[0][idx] = g0 * g0;
  a.Q[1][idx] = g1 * g1;
  a.Q[2][idx] = g2 * g2;
  a.Q[3][idx] = 2.0 * a.G[3][idx] * a.G[4][idx];
  a.Q[4][idx] = 2.0 * a.G[5][idx] * a.G[6][idx];
  a.Q[5][idx] = 2.0 * a.G[7][idx] * a.G[8][idx];
}

// Source and solve per (kx, kz) column, one warp per column: rows 2..Ny-1
// -(sum of the transformed products + Ri dth/dy off the mean mode), wall rows
// 1 and Ny (apply_BC_poisson, :2019-2055), complex Thomas over rows 1..Ny
// (:1408-1457); cp rows 1..Ny receive the solution.
struct PpSolveArgs {
  const double2* Q[6];
  const double2* cth[8];
  double2* cp;
  const double* kx;
  const double* kz;
  const double* met;      // MET_PA, MET_PC, MET_PB0 rows
  const double* gyf;
  double ri[8];
  int nth, n, nyp, nkx1, nk2, kp, ncol;
};

template <int R>
__global__ void __launch_bounds__(128) k_pp_solve(const __grid_constant__ PpSolveArgs a) {
  using namespace csolve;
  const int lane = threadIdx.x & 31;
  const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= a.ncol) return;
  const int m = col / a.nk2, kq = col % a.nk2;
  const size_t ps = (size_t)a.nkx1 * a.kp, c0 = (size_t)m * a.kp + kq;
  const int n = a.n, nyp = a.nyp;
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const bool m00 = m == 0 && kq == 0;
  double A[R], B[R], C[R];
  double2 D[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = lane * R + r;
    A[r] = 0.0; B[r] = 1.0; C[r] = 0.0; D[r] = make_double2(0.0, 0.0);
    if (j >= 2 && j <= nyp - 1) {
      const size_t o = (size_t)j * ps + c0;
      double2 s = a.Q[0][o] + a.Q[1][o] + a.Q[2][o];
      s = s + a.Q[3][o];
      s = s + a.Q[4][o];
      s = s + a.Q[5][o];
      if (!m00) {
        for (int q = 0; q < a.nth; ++q) {
          const double2 tp = a.cth[q][o + ps], tm = a.cth[q][o - ps];
          const double den = a.gyf[j + 1] - a.gyf[j - 1];
          s = s + a.ri[q] * make_double2((tp.x - tm.x) / den, (tp.y - tm.y) / den);
        }
      }
      A[r] = a.met[MET_PA * n + j];
      C[r] = a.met[MET_PC * n + j];
      B[r] = -kxm * kxm - kzq * kzq + a.met[MET_PB0 * n + j];
      D[r] = -1.0 * s;
    } else if (j == 1) {
      B[r] = 1.0; C[r] = m00 ? 0.0 : -1.0;
    } else if (j == nyp) {
      A[r] = 1.0; B[r] = -1.0;
    }
  }
  warp_tridiag<R>(A, B, C, D, lane);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = lane * R + r;
    if (j >= 1 && j <= nyp) a.cp[(size_t)j * ps + c0] = D[r];
  }
}

// Per plane j = 1..Ny (one block per plane): min and max of u1 and u3 and the
// largest |u2|, out[j][0..4] = (min u1, max u1, max |u2|, min u3, max u3).
// courant turns them into the CFL time step: max|u - a| over the plane is
// max(max u - a, a - min u) for any shift a, which covers both the plain
// branch (a = 0) and the 'Front' branch's thermal-wind shifts.
static __global__ void __launch_bounds__(256) k_plane_range(const double* u1, const double* u2, const double* u3,
                                                     double* out, size_t ps) {
  const int j = blockIdx.x + 1;
  const size_t base = (size_t)j * ps;
  double v[5] = {INFINITY, -INFINITY, 0.0, INFINITY, -INFINITY};
  for (size_t i = threadIdx.x; i < ps; i += blockDim.x) {
    const double a = u1[base + i], c = u3[base + i];
    v[0] = fmin(v[0], a); v[1] = fmax(v[1], a);
    v[2] = fmax(v[2], fabs(u2[base + i]));
    v[3] = fmin(v[3], c); v[4] = fmax(v[4], c);
  }
  __shared__ double red[5][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v[q], off);
      v[q] = (q == 0 || q == 3) ? fmin(v[q], o) : fmax(v[q], o);
    }
    if (lane == 0) red[q][w] = v[q];
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    const int q = threadIdx.x;
    double r = red[q][0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = (q == 0 || q == 3) ? fmin(r, red[q][k]) : fmax(r, red[q][k]);
    out[(size_t)j * 5 + q] = r;
  }
}

// filter_chan (for/channel.f90:1241-1329): cth *= sigma(m, kq) on rows j0..j1
static __global__ void k_filter_th(double2* cth, const double* sigma, int j0, int j1, int nkx1, int nk2, int kp) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t ps = (size_t)nkx1 * kp;
  const size_t tot = (size_t)(j1 - j0 + 1) * ps;
  if (idx >= tot) return;
  const int kq = idx % kp;
  if (kq >= nk2) return;
  const int m = (idx / kp) % nkx1;
  const size_t o = (size_t)j0 * ps + idx;
  cth[o] = sigma[m * nk2 + kq] * cth[o];
}
