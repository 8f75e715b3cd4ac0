// Layout conversions between the reference's aliased arrays and the internal
// layouts, plus the small Fourier-space boundary kernels.
#pragma once
#include "common.cuh"
#include "kernels_fft.cuh"

// reference physical v(0:Nx+1, 0:Nz+1, 0:Ny+1) -> internal P[j][k][i]
// (`rows` rows of Nx+2 per plane in `ref`: Nz+2 for a whole reference array,
// Nz for its significant rows staged contiguously)
static __global__ void k_ref_to_phys(const double* __restrict__ ref, double* __restrict__ out,
                              int nx, int nz, int nyp2, int rows) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)nyp2 * nz * nx;
  if (idx >= tot) return;
  int i = idx % nx;
  size_t r = idx / nx;
  int k = r % nz;
  int j = r / nz;
  out[idx] = ref[((size_t)j * rows + k) * (nx + 2) + i];
}

// internal P -> the significant box (i < Nx, k < Nz) of a reference physical array
static __global__ void k_phys_to_ref(const double* __restrict__ in, double* __restrict__ ref,
                              int nx, int nz, int nyp2) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)nyp2 * nz * nx;
  if (idx >= tot) return;
  int i = idx % nx;
  size_t r = idx / nx;
  int k = r % nz;
  int j = r / nz;
  ref[((size_t)j * (nz + 2) + k) * (nx + 2) + i] = in[idx];
}

// reference Fourier vv(0:Nxp, 0:Nz+1, 0:Ny+1) -> internal F[j][m][kp]; sets
// *bad if a significant mode above Nkx is nonzero.  The source has row pitch
// `rp` complex elements and `rows` rows per plane (Nxp+1 and Nz+2 for a full
// reference array, Nxp and 2Nkz+1 for a packed copy of its significant box).
static __global__ void k_ref_to_four(const double2* __restrict__ ref, double2* __restrict__ out,
                              Geom g, int nxp, int rp, int rows, int* bad) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)g.nyp2 * g.nk2 * nxp;
  if (idx >= tot) return;
  int i = idx % nxp;
  size_t r = idx / nxp;
  int kp = r % g.nk2;
  int j = r / g.nk2;
  double2 v = ref[((size_t)j * rows + kp) * rp + i];
  if (i < g.nkx1) {
    out[((size_t)j * g.nkx1 + i) * g.kp + kp] = v;
  } else if (v.x != 0.0 || v.y != 0.0) {
    atomicOr(bad, 1);
  }
}

// internal F -> the significant box (i < Nxp, k <= 2Nkz) of a Fourier array
// with row pitch `rp` and `rows` rows per plane; modes above Nkx written as 0
static __global__ void k_four_to_ref(const double2* __restrict__ in, double2* __restrict__ ref,
                              Geom g, int nxp, int rp, int rows) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)g.nyp2 * g.nk2 * nxp;
  if (idx >= tot) return;
  int i = idx % nxp;
  size_t r = idx / nxp;
  int k = r % g.nk2;
  int j = r / g.nk2;
  double2 v = make_double2(0.0, 0.0);
  if (i < g.nkx1) v = in[((size_t)j * g.nkx1 + i) * g.kp + k];
  ref[((size_t)j * rows + k) * rp + i] = v;
}

// any non-finite significant entry -> *bad
static __global__ void k_check_finite(const double2* __restrict__ f, Geom g, int* bad) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t tot = (size_t)g.nyp2 * g.nkx1 * g.kp;
  if (idx >= tot) return;
  if ((int)(idx % g.kp) >= g.nk2) return;
  double2 v = f[idx];
  if (!isfinite(v.x) || !isfinite(v.y)) atomicOr(bad, 1);
}

// Fourier-space wall and ghost values (for/boundary.f90:299-498, 728-821);
// one thread per stored (m, kp) mode.
struct BcPostArgs {
  double2* cu[3];
  double2* cth[8];
  int nth, nyp, nkx1, nk2, kp;
  int ubc[2], vbc[2], wbc[2];
  double uc1[2], vc1[2], wc1[2];   // wc1[1] already the transient top value when Neumann
  int thbc[8][2];
  double thc1[8][2];
  const double* dy;
  const double* dyf;
  int do_vel, do_th;   // apply_BC_vel_mpi_post / apply_BC_th_mpi_post
};

static __global__ void k_bc_post(BcPostArgs a) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= a.nkx1 * a.nk2) return;
  const int m = idx / a.nk2, kq = idx % a.nk2;
  const bool m00 = (m == 0 && kq == 0);
  const size_t ps = (size_t)a.nkx1 * a.kp, c = (size_t)m * a.kp + kq;
  const int nyp = a.nyp;
  auto P = [&](double2* f, int j) -> double2& { return f[(size_t)j * ps + c]; };
  const double2 z = make_double2(0.0, 0.0);
  const double* dy = a.dy;
  const double* dyf = a.dyf;
  if (a.do_vel) {
  // lower wall, u1 and u3
  for (int q = 0; q < 2; ++q) {
    double2* cu = a.cu[q == 0 ? 0 : 2];
    int b = q == 0 ? a.ubc[0] : a.wbc[0];
    double c1 = q == 0 ? a.uc1[0] : a.wc1[0];
    if (b == 0) {
      P(cu, 0) = z; P(cu, 1) = z;
      if (m00) { P(cu, 1) = make_double2(c1, 0); P(cu, 0) = make_double2(c1, 0); }
    } else {
      P(cu, 1) = P(cu, 2); P(cu, 0) = P(cu, 1);
      if (m00) {
        P(cu, 1) = make_double2(P(cu, 2).x - dy[2] * c1, P(cu, 2).y);
        P(cu, 0) = make_double2(P(cu, 1).x - dy[1] * c1, P(cu, 1).y);
      }
    }
  }
  {
    double2* cu = a.cu[1];
    if (a.vbc[0] == 0) {
      // every mode gets the real constant 2*c1 (for/boundary.f90:373-378)
      double2 v2 = P(cu, 2);
      P(cu, 1) = make_double2(2.0 * a.vc1[0] - v2.x, -v2.y);
      P(cu, 0) = P(cu, 1);
    } else {
      P(cu, 1) = P(cu, 2); P(cu, 0) = P(cu, 1);
      if (m00) {
        P(cu, 1) = make_double2(P(cu, 2).x - dyf[1] * a.vc1[0], P(cu, 2).y);
        P(cu, 0) = make_double2(P(cu, 1).x - dyf[1] * a.vc1[0], P(cu, 1).y);
      }
    }
  }
  // upper wall
  {
    double2* cu = a.cu[0];
    if (a.ubc[1] == 0) {
      P(cu, nyp) = z; P(cu, nyp + 1) = z;
      if (m00) { P(cu, nyp) = make_double2(a.uc1[1], 0); P(cu, nyp + 1) = make_double2(a.uc1[1], 0); }
    } else {
      P(cu, nyp) = P(cu, nyp - 1); P(cu, nyp + 1) = P(cu, nyp);
      if (m00) {
        P(cu, nyp) = make_double2(P(cu, nyp - 1).x + dy[nyp] * a.uc1[1], P(cu, nyp - 1).y);
        P(cu, nyp + 1) = make_double2(P(cu, nyp).x + dy[nyp] * a.uc1[1], P(cu, nyp).y);
      }
    }
  }
  {
    double2* cu = a.cu[2];
    if (a.wbc[1] == 0) {
      P(cu, nyp) = z; P(cu, nyp + 1) = z;
      if (m00) { P(cu, nyp) = make_double2(a.wc1[1], 0); P(cu, nyp + 1) = z; }
    } else {
      P(cu, nyp) = P(cu, nyp - 1); P(cu, nyp + 1) = P(cu, nyp);
      if (m00) {
        P(cu, nyp) = make_double2(P(cu, nyp - 1).x + dy[nyp] * a.wc1[1], P(cu, nyp - 1).y);
        P(cu, nyp + 1) = make_double2(P(cu, nyp).x + dy[nyp] * a.wc1[1], P(cu, nyp).y);
      }
    }
  }
  {
    double2* cu = a.cu[1];
    if (a.vbc[1] == 0) {
      // the reference loop body only touches the (0,0) mode (for/boundary.f90:476-480)
      if (m00) P(cu, nyp + 1) = make_double2(2.0 * a.vc1[1] - P(cu, nyp).x, -P(cu, nyp).y);
    } else {
      P(cu, nyp) = P(cu, nyp - 1); P(cu, nyp + 1) = P(cu, nyp);
      if (m00) P(cu, nyp + 1) = make_double2(P(cu, nyp).x + dy[nyp] * a.vc1[1], P(cu, nyp).y);
    }
  }
  }
  // scalars
  for (int n = 0; a.do_th && n < a.nth; ++n) {
    double2* ct = a.cth[n];
    if (a.thbc[n][0] == 0) {
      P(ct, 0) = z; P(ct, 1) = z;
      if (m00) { P(ct, 1) = make_double2(a.thc1[n][0], 0); P(ct, 0) = make_double2(a.thc1[n][0], 0); }
    } else {
      P(ct, 1) = P(ct, 2); P(ct, 0) = P(ct, 1);
      if (m00) {
        P(ct, 1) = make_double2(P(ct, 2).x - dy[2] * a.thc1[n][0], P(ct, 2).y);
        P(ct, 0) = make_double2(P(ct, 1).x - dy[1] * a.thc1[n][0], P(ct, 1).y);
      }
    }
    if (a.thbc[n][1] == 0) {
      P(ct, nyp) = z; P(ct, nyp + 1) = z;
      if (m00) { P(ct, nyp) = make_double2(a.thc1[n][1], 0); P(ct, nyp + 1) = make_double2(a.thc1[n][1], 0); }
    } else {
      P(ct, nyp) = P(ct, nyp - 1); P(ct, nyp + 1) = P(ct, nyp);
      if (m00) {
        P(ct, nyp) = make_double2(P(ct, nyp - 1).x + dy[nyp] * a.thc1[n][1], P(ct, nyp - 1).y);
        P(ct, nyp + 1) = make_double2(P(ct, nyp).x + dy[nyp] * a.thc1[n][1], P(ct, nyp).y);
      }
    }
  }
}

// FP32 -> FP64 copy of n values
static __global__ void k_widen(const float* in, double* out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)in[i];
}
