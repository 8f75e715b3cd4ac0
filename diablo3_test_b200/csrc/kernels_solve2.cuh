// Tiled Fourier-space column kernel (the default path of the column solve).
//
// Same mathematics as k_column_solve (kernels_solve.cuh): explicit RK terms,
// explicit Crank-Nicolson half, implicit y solves with wall rows, projection
// and pressure update (for/channel.f90:29-249, :468-514, :553-877, :901-911,
// rem_div_chan :946-1023), one warp per (kx, kz) column.  The difference is
// the data path: a block owns 4 adjacent kz columns of one kx, and every
// field it needs moves through shared memory as an (Ny+2) x 4 tile copied with
// cp.async (16-byte pieces, 64-byte rows) through a ring of T2_STAGES tiles,
// so the next tile is in flight while one is consumed.  Lanes then read their own rows
// (and y-neighbours) from shared memory.  The host builds the list of tiles
// (`steps`) once per substep; terms whose coefficient is zero are not loaded
// at all.  The pressure arrives as the tile of each velocity solve and of the
// pressure update rather than staying resident, which keeps a 257-row block at
// 56 KB of shared memory.
#pragma once
#include "common.cuh"
#include "kernels_solve.cuh"

namespace csolve2 {

// Shared-memory slot of tile element (row j, column c).  Lanes of a warp own
// rows R apart; a 16-byte slot index 4j + c would put them in only two of the
// eight 16-byte bank groups of a 128-byte wavefront.  XOR-ing the column with
// bits 1-2 of the row spreads any 8 consecutive rows over all eight.
DI int tix(int j, int c) { return j * T2_PITCH + (c ^ ((j >> 1) & 3)); }

DI void cp_async16(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
DI void cp_async8(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
DI void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> DI void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// issue the copies of one (n x 4) tile; element bytes 16 (double2) or 8 (float2)
DI void load_tile(void* tile, const void* g, bool fp32, size_t ps, size_t cbase, int nvalid,
                  int n, int tid, int nthr) {
  if (g) {
    for (int idx = tid; idx < n * T2_COLS; idx += nthr) {
      const int j = idx >> 2, c = idx & 3;
      if (c < nvalid) {
        if (fp32)
          cp_async8((float2*)tile + tix(j, c), (const float2*)g + j * ps + cbase + c);
        else
          cp_async16((double2*)tile + tix(j, c), (const double2*)g + j * ps + cbase + c);
      } else {
        if (fp32) ((float2*)tile)[tix(j, c)] = make_float2(0.f, 0.f);
        else ((double2*)tile)[tix(j, c)] = make_double2(0.0, 0.0);
      }
    }
  }
  cp_commit();
}

}  // namespace csolve2

namespace csolve2 {
// warp_tridiag with b supplied row by row (it is only read by the forward
// sweep) and a, c reached through accessors returning double&, so that the
// caller can keep them in registers it has no other use for at that point
template <int R, typename AF, typename BF, typename CF>
DI void warp_tridiag_b(AF a, BF bf, CF c, double2 (&d)[R], int lane) {
  using namespace csolve;
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    double ib = 1.0 / bf(r);
    a(r) *= ib; c(r) *= ib; d[r] = ib * d[r];
  }
#pragma unroll
  for (int r = 2; r < R; ++r) {
    double ib = 1.0 / (bf(r) - a(r) * c(r - 1));
    d[r] = ib * (d[r] - a(r) * d[r - 1]);
    a(r) = -ib * a(r) * a(r - 1);
    c(r) = ib * c(r);
  }
#pragma unroll
  for (int r = R - 3; r >= 1; --r) {
    d[r] = d[r] - c(r) * d[r + 1];
    a(r) = a(r) - c(r) * a(r + 1);
    c(r) = -c(r) * c(r + 1);
  }
  {
    double ib = 1.0 / (1.0 - c(0) * a(1));
    d[0] = ib * (d[0] - c(0) * d[1]);
    a(0) = ib * a(0);
    c(0) = -ib * c(0) * c(1);
  }
  const double as = a(0), gs = c(0);
  const double2 ds = d[0];
  const double ae = a(R - 1), ge = c(R - 1);
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
  for (int r = 1; r < R - 1; ++r) d[r] = d[r] - a(r) * S - c(r) * E;
}
}  // namespace csolve2


// ---- factored solves ----------------------------------------------------------
// The u1, u2, u3 and scalar systems have the same matrix in every (kx, kz)
// column (their rows depend on y only; the wall rows on the BC type only), so
// warp_tridiag's elimination multipliers are computed once per substep by
// k_factor and each column only replays them on its right-hand side.  The
// replay performs the same operations on d as warp_tridiag_b.
// Per-lane item layout (stored [item][lane]):
template <int R> struct Fac {
  static constexpr int IB = 0;            // r = 0..R-1
  static constexpr int ARAW = R;          // r = 2..R-1 (input a of the row)
  static constexpr int CF = 2 * R;        // r = 1..R-3 (c after the forward sweep)
  static constexpr int AFIN = 3 * R;      // r = 1..R-2
  static constexpr int CFIN = 4 * R;      // r = 1..R-2
  static constexpr int IB0B = 5 * R, C0F = 5 * R + 1, AS = 5 * R + 2, GS = 5 * R + 3;
  static constexpr int AE = 5 * R + 4, GE = 5 * R + 5, INVD = 5 * R + 6;
  static constexpr int K1 = 5 * R + 7, K2 = 5 * R + 12;
  static constexpr int N = 5 * R + 17;
};

// rows of field kind (0 = u1, 1 = u2, 2 = u3, 3+n = scalar n): interior rows
// from kc, wall rows of for/channel.f90:1545-1876, identity elsewhere
template <int R>
DI void system_rows(const SolveArgs& a, const double* kc, int kind, int lane, double (&Am)[R],
                    double (&Bm)[R], double (&Cm)[R]) {
  const int n = a.n, nyp = a.nyp;
  int lo, hi, b0, b1;
  const double* K;
  if (kind == 1) { lo = 2; hi = nyp; K = kc + (size_t)1 * 3 * n; b0 = a.vbc[0]; b1 = a.vbc[1]; }
  else if (kind == 0 || kind == 2) {
    lo = a.jstart; hi = a.jend; K = kc;
    b0 = kind == 0 ? a.ubc[0] : a.wbc[0];
    b1 = kind == 0 ? a.ubc[1] : a.wbc[1];
  } else {
    lo = a.jst[kind - 3]; hi = a.jet[kind - 3]; K = kc + (size_t)(kind - 1) * 3 * n;
    b0 = a.thbc[kind - 3][0]; b1 = a.thbc[kind - 3][1];
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = lane * R + r;
    Am[r] = 0.0; Bm[r] = 1.0; Cm[r] = 0.0;
    if (j >= lo && j <= hi) { Am[r] = K[j]; Bm[r] = K[n + j]; Cm[r] = K[2 * n + j]; }
    if (kind == 1) {
      if (b0 == 0 && (j == 1 || j == 2)) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
      if (b0 == 1 && j == 1) { Am[r] = 0; Bm[r] = -1; Cm[r] = 1; }
      if (j == 0) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
      if (b1 == 0 && (j == nyp || j == nyp + 1)) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
      if (b1 == 1 && j == nyp + 1) { Am[r] = -1; Bm[r] = 1; Cm[r] = 0; }
    } else {
      if (j == 0 || j == nyp + 1) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
      if (j == 1) {
        if (b0 == 0) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
        else { Am[r] = 0; Bm[r] = -1; Cm[r] = 1; }
      }
      if (j == nyp) {
        if (b1 == 0) { Am[r] = 0; Bm[r] = 1; Cm[r] = 0; }
        else { Am[r] = -1; Bm[r] = 1; Cm[r] = 0; }
      }
    }
  }
}

// warp_tridiag_b's elimination on the matrix alone, recording its multipliers
template <int R>
DI void factor_rows(double (&a)[R], double (&b)[R], double (&c)[R], int lane, double* out) {
  using F = Fac<R>;
  auto W = [&](int item, double v) { out[item * 32 + lane] = v; };
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    double ib = 1.0 / b[r];
    W(F::IB + r, ib);
    a[r] *= ib; c[r] *= ib;
  }
#pragma unroll
  for (int r = 2; r < R; ++r) {
    double ib = 1.0 / (b[r] - a[r] * c[r - 1]);
    W(F::IB + r, ib);
    W(F::ARAW + r, a[r]);
    a[r] = -ib * a[r] * a[r - 1];
    c[r] = ib * c[r];
  }
#pragma unroll
  for (int r = R - 3; r >= 1; --r) {
    W(F::CF + r, c[r]);
    a[r] = a[r] - c[r] * a[r + 1];
    c[r] = -c[r] * c[r + 1];
  }
  {
    double ib = 1.0 / (1.0 - c[0] * a[1]);
    W(F::IB0B, ib);
    W(F::C0F, c[0]);
    a[0] = ib * a[0];
    c[0] = -ib * c[0] * c[1];
  }
#pragma unroll
  for (int r = 1; r < R - 1; ++r) { W(F::AFIN + r, a[r]); W(F::CFIN + r, c[r]); }
  const double as = a[0], gs = c[0], ae = a[R - 1], ge = c[R - 1];
  W(F::AS, as); W(F::GS, gs); W(F::AE, ae); W(F::GE, ge);
  double ae_m = __shfl_up_sync(0xffffffffu, ae, 1);
  double ge_m = __shfl_up_sync(0xffffffffu, ge, 1);
  if (lane == 0) { ae_m = 0.0; ge_m = 0.0; }
  double L = -as * ae_m;
  double D = 1.0 - as * ge_m - gs * ae;
  double U = -gs * ge;
  int lev = 0;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1, ++lev) {
    double Lm = __shfl_up_sync(0xffffffffu, L, s);
    double Dm = __shfl_up_sync(0xffffffffu, D, s);
    double Um = __shfl_up_sync(0xffffffffu, U, s);
    double Lp = __shfl_down_sync(0xffffffffu, L, s);
    double Dp = __shfl_down_sync(0xffffffffu, D, s);
    double Up = __shfl_down_sync(0xffffffffu, U, s);
    if (lane < s) { Lm = 0.0; Dm = 1.0; Um = 0.0; }
    if (lane + s >= 32) { Lp = 0.0; Dp = 1.0; Up = 0.0; }
    double k1 = L / Dm, k2 = U / Dp;
    W(F::K1 + lev, k1);
    W(F::K2 + lev, k2);
    L = -k1 * Lm;
    U = -k2 * Up;
    D = D - k1 * Um - k2 * Lp;
  }
  W(F::INVD, 1.0 / D);
}

// replay of the recorded elimination on one right-hand side (d <- x)
template <int R>
DI void apply_factored(const double* __restrict__ fac, double2 (&d)[R], int lane) {
  using namespace csolve;
  using F = Fac<R>;
  auto G = [&](int item) -> double { return __ldg(fac + item * 32 + lane); };
#pragma unroll
  for (int r = 0; r < 2; ++r) d[r] = G(F::IB + r) * d[r];
#pragma unroll
  for (int r = 2; r < R; ++r) d[r] = G(F::IB + r) * (d[r] - G(F::ARAW + r) * d[r - 1]);
#pragma unroll
  for (int r = R - 3; r >= 1; --r) d[r] = d[r] - G(F::CF + r) * d[r + 1];
  d[0] = G(F::IB0B) * (d[0] - G(F::C0F) * d[1]);
  const double2 ds = d[0], de = d[R - 1];
  double2 de_m = shfl_up2(de, 1);
  if (lane == 0) de_m = make_double2(0.0, 0.0);
  double2 Q = ds - G(F::AS) * de_m - G(F::GS) * de;
  int lev = 0;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1, ++lev) {
    double2 Qm = shfl_up2(Q, s);
    double2 Qp = shfl_down2(Q, s);
    if (lane < s) Qm = make_double2(0.0, 0.0);
    if (lane + s >= 32) Qp = make_double2(0.0, 0.0);
    Q = Q - G(F::K1 + lev) * Qm - G(F::K2 + lev) * Qp;
  }
  const double2 S = G(F::INVD) * Q;
  double2 Sn = shfl_down2(S, 1);
  if (lane == 31) Sn = make_double2(0.0, 0.0);
  const double2 E = de - G(F::AE) * S - G(F::GE) * Sn;
  d[0] = S;
  d[R - 1] = E;
#pragma unroll
  for (int r = 1; r < R - 1; ++r) d[r] = d[r] - G(F::AFIN + r) * S - G(F::CFIN + r) * E;
}

// one warp per field kind: factor its system for the substep coefficients kc
template <int R>
__global__ void __launch_bounds__(32) k_factor(const __grid_constant__ SolveArgs a, const double* kc,
                                               double* out) {
  const int kind = blockIdx.x, lane = threadIdx.x;
  double Am[R], Bm[R], Cm[R];
  system_rows<R>(a, kc, kind, lane, Am, Bm, Cm);
  factor_rows<R>(Am, Bm, Cm, lane, out + (size_t)kind * Fac<R>::N * 32);
}

// Ring depth and blocks per SM.  Occupancy, not prefetch depth, decides this
// kernel's speed: at Ny = 257 (R = 9) a two-stage ring keeps a block at 56 KB
// and a 128-register cap fits four blocks (16 warps) per SM, measured 0.84 ms
// per launch against 0.90 (two stages, three blocks), 0.92 (three stages,
// three blocks) and 1.08 (four stages, two blocks).  Larger R need more
// shared memory, so fewer blocks fit and the cap is relaxed.
#ifndef T2_STAGES
#define T2_STAGES 2
#endif
template <int R>
constexpr int t2_min_blocks() { return R <= 9 ? 4 : (R <= 13 ? 3 : 2); }

template <int R>
__global__ void __launch_bounds__(128, t2_min_blocks<R>()) k_column_tiles(const __grid_constant__ Solve2Args A) {
  using namespace csolve;
  using namespace csolve2;
  const SolveArgs& a = A.s;
  extern __shared__ __align__(16) unsigned char t2_smem[];
  const int n = a.n, nyp = a.nyp;
  const int tsz = n * T2_PITCH;
  double2* Tbase = reinterpret_cast<double2*>(t2_smem);   // T2_STAGES streamed tiles
  double2* dvs = Tbase + T2_STAGES * tsz;             // lane-private divergence rows
  // a lane's rows sit (R | 1) slots apart: an odd 16-byte stride keeps the 32
  // lanes on distinct bank groups for any R
  constexpr int RP = R | 1;
  double* Um = reinterpret_cast<double*>(dvs + T2_COLS * 32 * RP);   // U1, I(U1) (mean_split)
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int lane = tid & 31, c = tid >> 5;
  const int ngroups = (a.nk2 + T2_COLS - 1) / T2_COLS;
  const int m = blockIdx.x / ngroups;
  const int kq0 = (blockIdx.x % ngroups) * T2_COLS;
  const int nvalid = min(T2_COLS, a.nk2 - kq0);
  const bool valid = c < nvalid;
  const int kq = min(kq0 + c, a.nk2 - 1);
  const size_t ps = (size_t)a.nkx1 * a.kp;
  const size_t cbase = (size_t)m * a.kp + kq0;
  const bool m00 = (m == 0 && kq == 0 && valid);
  const double kxm = a.kx[m], kzq = a.kz[kq];
  const double k2s = kxm * kxm + kzq * kzq;
  const double kk = a.beta == 1.0 ? k2s : pow(k2s, a.beta);
  const double2 z2 = make_double2(0.0, 0.0);
  const int j0 = lane * R;
  const double v00 = m00 ? 1.0 : 0.0;
  const double* met = A.met;
  double2* dv = dvs + c * (32 * RP) + lane * RP;      // this lane's R rows

  double2 cr[R], cf[R];
#pragma unroll
  for (int r = 0; r < R; ++r) { cr[r] = z2; cf[r] = z2; dv[r] = z2; }
  int lo = 0, hi = -1;           // explicit row range of the current field
  const double* K = A.kc;        // implicit rows of the current field

  if (A.mean_split)
    for (int j = tid; j < 2 * n; j += nthr) Um[j] = A.prof[j];
  for (int q = 0; q < T2_STAGES - 1; ++q) {
    const TileStep* st = q < A.nstep ? &A.steps[q] : nullptr;
    load_tile(Tbase + q * tsz, st ? st->src : nullptr, st && st->op == OP_NL && st->arg, ps, cbase,
              nvalid, n, tid, nthr);
  }
  for (int k = 0; k < A.nstep; ++k) {
    const TileStep st = A.steps[k];
    {
      const int kn = k + T2_STAGES - 1;
      const TileStep* nx = kn < A.nstep ? &A.steps[kn] : nullptr;
      load_tile(Tbase + (kn % T2_STAGES) * tsz, nx ? nx->src : nullptr,
                nx && nx->op == OP_NL && nx->arg, ps, cbase, nvalid, n, tid, nthr);
      cp_wait<T2_STAGES - 1>();
    }
    __syncthreads();
    double2* T = Tbase + (k % T2_STAGES) * tsz;
    const float2* T32 = reinterpret_cast<const float2*>(T);
    auto TV = [&](int j) -> double2 { return T[tix(j, c)]; };

    switch (st.op) {
      case OP_OWN_U13:
      case OP_OWN_U2:
      case OP_OWN_TH: {
        int kind;
        if (st.op == OP_OWN_U13) { lo = a.jstart; hi = a.jend; kind = 0; }
        else if (st.op == OP_OWN_U2) { lo = 2; hi = nyp; kind = 1; }
        else { lo = a.jst[st.arg]; hi = a.jet[st.arg]; kind = 2 + st.arg; }
        K = A.kc + (size_t)kind * 3 * n;
        const double cfc = st.op == OP_OWN_TH ? (a.nu / a.pr[st.arg]) * kk : a.nu * kk;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          cr[r] = z2; cf[r] = z2;
          if (j >= lo && j <= hi) {
            const double2 u = TV(j), um = TV(j - 1), up = TV(j + 1);
            cf[r] = -cfc * u;
            cr[r] = u - K[2 * n + j] * (up - u) + K[j] * (u - um);
            if (A.mean_split && !(kind == 0 && st.arg == 0))
              cf[r] = cf[r] - mul_ik(kxm * Um[kind == 1 ? n + j : j], u);
          }
        }
        break;
      }
      case OP_ADD_CF: {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= lo && j <= hi) cf[r] = cf[r] + st.coef * TV(j);
        }
        break;
      }
      case OP_BUOY: {
        if (!m00) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= lo && j <= hi)
              cf[r] = cf[r] + st.coef * (met[MET_WB1 * n + j] * TV(j) + met[MET_WB2 * n + j] * TV(j - 1));
          }
        }
        break;
      }
      case OP_NL: {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= lo && j <= hi) {
            double2 nl;
            if (st.arg) { float2 v = T32[tix(j, c)]; nl = make_double2(v.x, v.y); }
            else nl = TV(j);
            cf[r] = cf[r] - nl;
            cr[r] = cr[r] + a.temp5 * cf[r];
          }
        }
        if (st.dst) {  // cf for the next substep, stored through the tile
          __syncthreads();
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j < n) T[tix(j, c)] = cf[r];
          }
          __syncthreads();
          for (int idx = tid; idx < n * T2_COLS; idx += nthr) {
            const int j = idx >> 2, cc = idx & 3;
            if (cc < nvalid && j >= lo && j <= hi)
              ((double2*)st.dst)[j * ps + cbase + cc] = T[tix(j, cc)];
          }
        }
        break;
      }
      case OP_CFOLD: {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= lo && j <= hi) cr[r] = cr[r] + a.temp3 * TV(j);
        }
        break;
      }
      case OP_SOLVE: {
        // st.arg: 0 = u1, 1 = u2, 2 = u3, 3+n = scalar n
        const int kind = st.arg;
        int b0, b1;
        double c0, c1;
        if (kind == 0) { b0 = a.ubc[0]; b1 = a.ubc[1]; c0 = a.uc1[0]; c1 = a.uc1[1]; }
        else if (kind == 2) { b0 = a.wbc[0]; b1 = a.wbc[1]; c0 = a.wc1[0]; c1 = a.wc1[1]; }
        else if (kind == 1) { b0 = a.vbc[0]; b1 = a.vbc[1]; c0 = a.vc1[0]; c1 = a.vc1[1]; }
        else { b0 = a.thbc[kind - 3][0]; b1 = a.thbc[kind - 3][1]; c0 = a.thc1[kind - 3][0]; c1 = a.thc1[kind - 3][1]; }
        // right-hand side: explicit terms on the interior rows, wall values
        // on the wall rows (the matrix itself is in the factor table)
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          double2 d = z2;
          if (j >= lo && j <= hi) {
            d = cr[r];
            if (kind == 1) {
              d = d - a.temp4 * met[MET_IDY * n + j] * (TV(j) - TV(j - 1));
            } else if (kind == 0 || kind == 2) {
              d = d - a.temp4 * mul_ik(kind == 0 ? kxm : kzq, TV(j));
              if (kind == 0 && m00) d.x -= a.px;
            }
          }
          if (kind == 1) {
            if (b0 == 0 && (j == 1 || j == 2)) d = make_double2(c0 * v00, 0);
            if (b0 == 1 && j == 1) d = make_double2(a.dyf[1] * c0 * v00, 0);
            if (j == 0) d = z2;
            if (b1 == 0 && (j == nyp || j == nyp + 1)) d = make_double2(c1 * v00, 0);
            if (b1 == 1 && j == nyp + 1) d = make_double2(a.dyf[nyp] * c1 * v00, 0);
          } else {
            if (j == 0 || j == nyp + 1) d = z2;
            if (j == 1) d = make_double2((b0 == 0 ? c0 : a.dy[2] * c0) * v00, 0);
            if (j == nyp) d = make_double2((b1 == 0 ? c1 : a.dy[nyp] * c1) * v00, 0);
          }
          cr[r] = d;
        }
        apply_factored<R>(A.fac + (size_t)kind * Fac<R>::N * 32, cr, lane);
        // divergence of the new velocity (rem_div_chan RHS, for/channel.f90:980-986)
        if (kind == 0 || kind == 2) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            if (j >= 1 && j <= nyp) dv[r] = dv[r] + mul_ik(kind == 0 ? kxm : kzq, cr[r]);
          }
        } else if (kind == 1) {
          const double2 xn = shfl_down2(cr[0], 1);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int j = j0 + r;
            const double2 xp = r == R - 1 ? xn : cr[r + 1];
            if (j >= 1 && j <= nyp) dv[r] = dv[r] + met[MET_IDYF * n + j] * (xp - cr[r]);
          }
        }
        const int w0 = (kind == 1) ? 1 : lo - 1;
        const int w1 = nyp + 1;
        // the tile held the pressure (rows j and j-1 were read above, the
        // latter possibly another lane's); it now stages the solution
        __syncwarp();
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j < n) T[tix(j, c)] = cr[r];
        }
        __syncthreads();
        for (int idx = tid; idx < n * T2_COLS; idx += nthr) {
          const int j = idx >> 2, cc = idx & 3;
          if (cc >= nvalid) continue;
          const size_t o = j * ps + cbase + cc;
          ((double2*)st.dst)[o] = (j >= w0 && j <= w1) ? T[tix(j, cc)] : ((const double2*)st.src2)[o];
        }
        break;
      }
      case OP_POISSON: {
        // cf is dead here (every field's NL step has stored it and the next
        // field's own step resets it): its .x and .y hold the sub- and
        // super-diagonal, which keeps the solve within the register cap
        const double k2n = -kxm * kxm - kzq * kzq;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          double am = 0.0, cm = 0.0;
          double2 d = z2;
          if (j >= 1 && j <= nyp) {
            am = met[MET_PA * n + j];
            cm = met[MET_PC * n + j];
            d = dv[r];
          }
          if (j == 1) { am = 0; cm = m00 ? 0.0 : -1.0; d = z2; }
          if (j == nyp) { am = 1; cm = 0; d = z2; }
          cf[r] = make_double2(am, cm);
          cr[r] = d;
        }
        warp_tridiag_b<R>([&](int r) -> double& { return cf[r].x; }, [&](int r) -> double {
          const int j = j0 + r;
          return (j == 1) ? 1.0 : (j == nyp ? -1.0 : ((j > 1 && j < nyp) ? k2n + met[MET_PB0 * n + j] : 1.0));
        }, [&](int r) -> double& { return cf[r].y; }, cr, lane);  // cr = phi from here on
        break;
      }
      case OP_PROJ: {
        const int comp = st.arg;
        const double2 phm = shfl_up2(cr[R - 1], 1);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= n) continue;
          double2 u = TV(j);
          // src2: keep the solved velocity before the projection (the field
          // courant reads, for/channel.f90:885-888)
          if (st.src2 && valid && j >= 1 && j <= nyp) ((double2*)st.src2)[j * ps + cbase + c] = u;
          if (comp != 1 && j >= 1 && j <= nyp) u = u - mul_ik(comp == 0 ? kxm : kzq, cr[r]);
          if (comp == 1 && j >= 2 && j <= nyp) {
            const double2 pm = r == 0 ? phm : cr[r - 1];
            u = u - met[MET_IDY * n + j] * (cr[r] - pm);
          }
          T[tix(j, c)] = u;
        }
        __syncthreads();
        const int w0 = comp == 1 ? 2 : 1;
        for (int idx = tid; idx < n * T2_COLS; idx += nthr) {
          const int j = idx >> 2, cc = idx & 3;
          if (cc < nvalid && j >= w0 && j <= nyp) ((double2*)st.dst)[j * ps + cbase + cc] = T[tix(j, cc)];
        }
        break;
      }
      case OP_CP: {
        const double ih = 1.0 / a.temp4;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int j = j0 + r;
          if (j >= n) continue;
          double2 p = TV(j);
          if (j >= a.jstart && j <= a.jend) p = p + ih * cr[r];
          T[tix(j, c)] = p;
        }
        __syncthreads();
        for (int idx = tid; idx < n * T2_COLS; idx += nthr) {
          const int j = idx >> 2, cc = idx & 3;
          if (cc < nvalid) ((double2*)st.dst)[j * ps + cbase + cc] = T[tix(j, cc)];
        }
        break;
      }
      default:
        break;
    }
    __syncthreads();
  }
}
