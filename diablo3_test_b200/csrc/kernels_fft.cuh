// xz-FFT kernels of the channel step.
//
// Internal layouts (all contiguous, x or k fastest):
//   physical  P[j][k][i]          (Ny+2) x Nz x Nx reals
//   x-spectral X[j][m][k]          m in [0, Nkx], k in [0, Nz)      complex
//   Fourier    F[j][m][kp]         m in [0, Nkx], kp in [0, 2Nkz]   complex, pitch KP
// The x-spectral layout keeps z contiguous so the z transforms read and write
// whole columns; the x transforms move tiles of KT z-rows through shared memory
// so both sides stay coalesced.  Together the two kernels of a direction are
// the reference's x-FFT + dealias + MPI_Alltoall repack + z-FFT + pack
// (for/fft.f90:247-382): modes Nkx < m <= Nx/2 are never stored (they are the
// zeroed ones, :264-266 and :372-378) and the dealiased z band is never stored
// (the pack/unpack of :307-312 and :329-340 is the kp <-> k index map).
#pragma once
#include "common.cuh"
#include "fft.cuh"

#define NF_MAX 12  // 3 velocities + up to DIABLO_MAX_TH scalars + spare

struct Geom {
  int nx, nz, nyp2;   // Nx, Nz, Ny+2
  int nkx1;           // Nkx+1 stored x modes
  int nkz, nk2, kp;   // Nkz, 2Nkz+1, Fourier pitch (>= nk2)
};

// packed Fourier index kp of the z-mode k in [0, Nz), or -1 in the dealiased band
HDI int z_pack(int k, int nz, int nkz) {
  return k <= nkz ? k : (k >= nz - nkz ? k - nz + 2 * nkz + 1 : -1);
}

// --------------------------------------------------------------------------
// z inverse: Fourier (packed, double2) -> x-spectral (C), one column per N2 threads
template <typename C> struct ZInvArgs {
  const double2* src[NF_MAX];
  C* dst[NF_MAX];
  int q0, nseq;      // first (j, m) column and number of columns
  Geom g;
  const C* tw;       // exp(-2 pi i m / Nz)
  unsigned mean_mask;  // fields transformed without their (kx, kz) = (0, 0) mode
};

template <typename C, int N1, int N2, int S>
__global__ void __launch_bounds__(N2* S) k_zinv(ZInvArgs<C> a) {
  __shared__ C sm[S][dfft::SmemSize<N1, N2>::v];
  const int t = threadIdx.x, s = threadIdx.y;
  const int q = blockIdx.x * S + s;
  const int f = blockIdx.y;
  const bool ok = q < a.nseq;
  const double2* src = a.src[f] + (size_t)(a.q0 + q) * a.g.kp;
  // the mean-free transform leaves out kp = 0 of the m = 0 sequences
  const int kmin = (((a.mean_mask >> f) & 1u) && (a.q0 + q) % a.g.nkx1 == 0) ? 1 : 0;
  C v[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    int kp = z_pack(n1 * N2 + t, a.g.nz, a.g.nkz);
    v[n1] = (ok && kp >= kmin) ? cvt<C>(src[kp]) : czero<C>();
  }
  dfft::step1<N1, N2, +1>(v, t, a.tw, sm[s]);
  __syncthreads();
  if (!ok) return;
  C* dst = a.dst[f] + (size_t)(a.q0 + q) * a.g.nz;
  for (int k1 = t; k1 < N1; k1 += N2) {
    C u[N2];
    dfft::step2<N1, N2, +1>(u, k1, sm[s]);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) dst[k1 + N1 * k2] = u[k2];
  }
}

// --------------------------------------------------------------------------
// z forward: x-spectral -> Fourier (packed).
//   plain:   out[kp] = X^[k] / Nz                        (for/fft.f90:298-313)
//   combine: out[kp] = (i kz(kp) A^[k] + B^[k]) / Nz     (the sum of one
//            momentum/scalar equation's nonlinear terms, for/channel.f90:299-459)
template <typename C, typename CO> struct ZFwdArgs {
  const C* srcA[NF_MAX];
  const C* srcB[NF_MAX];   // null for the plain transform
  CO* dst[NF_MAX];
  int q0, nseq;
  Geom g;
  const C* tw;
  const double* kz;        // wavenumbers kz(kp), length nk2
  double scale;            // 1/Nz
  // Mean epilogue of field 0 (the u1 equation, COMBINE, when cu[0] is set):
  // its products were taken with u1 minus its mean profile U1(y), and the
  // products with U1, linear in the state, are added here in FP64
  //   ikz U1 u3 + 2 ikx U1 u1 + (U1(j+1)u2(j+1) + U1(j)u2(j+1) - U1(j)u2(j) - U1(j-1)u2(j)) / (2 dyf(j))
  // (for/channel.f90:299-335, :398-417); dst[0] is then a double2 array.
  // cu = state u1, u2, u3, fps = its plane stride.  prof[j] = U1(j) and
  // prof[Ny+2+j] = (dyf(j) U1(j) + dyf(j-1) U1(j-1)) / (2 dy(j)) are written
  // for the column kernel's own corrections.
  const double2* cu[3];
  const double* kx;
  const double* dy;
  const double* dyf;
  double* prof;
  size_t fps;
  // plain form, FP64 output: nonzero makes the kernel accumulate,
  // dst[kp] += w(m) acc_scale X^[k] / Nz with w(0) = 1, w(m > 0) = 2 (the
  // transpose of the dealiased inverse transform, which the discrete adjoint
  // adds into its lambdas)
  double acc_scale;
};

// Blocks per SM the FP32 z-forward and x-inverse kernels' register caps are
// set for, and whether k_zfwd's combine form loads B together with A, before
// A's transform.  Measured at 256 x 257 x 256 with B loaded after A's
// transform: 6 blocks (80 registers) took the combine kernel from 0.234 to
// 0.216 ms per launch; 7 (72 registers) spills and measured 0.220.  Loading B
// with A: 0.2135 ms at 5 blocks (96 registers), 0.2173 at 6 (spills) and
// 0.2215 at 4, against 0.2150 without; the FP64 combine kernel went from
// 0.327 to 0.320 ms.  The x inverse holds 64 registers and, with its single
// row buffer, fits eight blocks per SM.
#ifndef ZFWD32_MIN_BLOCKS
#define ZFWD32_MIN_BLOCKS 5
#endif
#ifndef ZFWD_PREFETCH
#define ZFWD_PREFETCH 1
#endif
// The FP64 x inverse keeps separate spectrum and tile buffers: sharing them
// measured 0.693 against 0.677 ms per launch at 256 x 257 x 256.
#ifndef XC2R_ALIAS_FP64
#define XC2R_ALIAS_FP64 0
#endif
#ifndef XC2R32_MIN_BLOCKS
#define XC2R32_MIN_BLOCKS 8
#endif

template <typename C, typename CO, int N1, int N2, int S, bool COMBINE>
__global__ void __launch_bounds__(N2* S, sizeof(C) == 8 ? ZFWD32_MIN_BLOCKS : 1) k_zfwd(ZFwdArgs<C, CO> a) {
  typedef typename CReal<C>::R T;
  __shared__ C sm[S][dfft::SmemSize<N1, N2>::v];
  const int t = threadIdx.x, s = threadIdx.y;
  const int q = blockIdx.x * S + s;
  const int f = blockIdx.y;
  const bool ok = q < a.nseq;
  constexpr int NR = (N1 + N2 - 1) / N2;  // step-2 rows per thread
  C ra[NR][N2];
  const T sc = (T)a.scale;
  // B's loads are issued with A's when ZFWD_PREFETCH is set
  constexpr bool PF = COMBINE && ZFWD_PREFETCH;
  C vb[PF ? N1 : 1];
  // transform A
  {
    const C* src = a.srcA[f] + (size_t)(a.q0 + (ok ? q : 0)) * a.g.nz;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = ok ? src[n1 * N2 + t] : czero<C>();
    if (PF) {
      const C* srcb = a.srcB[f] + (size_t)(a.q0 + (ok ? q : 0)) * a.g.nz;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) vb[PF ? n1 : 0] = ok ? srcb[n1 * N2 + t] : czero<C>();
    }
    dfft::step1<N1, N2, -1>(v, t, a.tw, sm[s]);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      int k1 = t + r * N2;
      if (k1 < N1) dfft::step2<N1, N2, -1>(ra[r], k1, sm[s]);
    }
  }
  if (COMBINE) {
    __syncthreads();
    C v[N1];
    if (PF) {
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[n1] = vb[PF ? n1 : 0];
    } else {
      const C* src = a.srcB[f] + (size_t)(a.q0 + (ok ? q : 0)) * a.g.nz;
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) v[n1] = ok ? src[n1 * N2 + t] : czero<C>();
    }
    dfft::step1<N1, N2, -1>(v, t, a.tw, sm[s]);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      int k1 = t + r * N2;
      if (k1 < N1) {
        C u[N2];
        dfft::step2<N1, N2, -1>(u, k1, sm[s]);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          int kp = z_pack(k1 + N1 * k2, a.g.nz, a.g.nkz);
          T kzv = kp >= 0 ? (T)a.kz[kp] : (T)0;
          ra[r][k2] = mul_ik(kzv, ra[r][k2]) + u[k2];
        }
      }
    }
  }
  if (!ok) return;
  CO* dst = a.dst[f] + (size_t)(a.q0 + q) * a.g.kp;
  if (COMBINE && f == 0 && a.cu[0]) {
    double2* dst64 = reinterpret_cast<double2*>(a.dst[0]) + (size_t)(a.q0 + q) * a.g.kp;
    const int j = (a.q0 + q) / a.g.nkx1, m = (a.q0 + q) % a.g.nkx1;
    const size_t ps = a.fps, o = (size_t)(a.q0 + q) * a.g.kp;
    const double U0 = a.cu[0][(size_t)j * ps].x, Um = a.cu[0][(size_t)(j - 1) * ps].x,
                 Up = a.cu[0][(size_t)(j + 1) * ps].x;
    const double kxm = a.kx[m], id = 1.0 / (2.0 * a.dyf[j]);
    if (m == 0 && t == 0) {
      a.prof[j] = U0;
      a.prof[a.g.nyp2 + j] = (a.dyf[j] * U0 + a.dyf[j - 1] * Um) / (2.0 * a.dy[j]);
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      int k1 = t + r * N2;
      if (k1 < N1) {
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          int kp = z_pack(k1 + N1 * k2, a.g.nz, a.g.nkz);
          if (kp >= 0) {
            const double2 u1 = a.cu[0][o + kp], u3 = a.cu[2][o + kp];
            const double2 vc = a.cu[1][o + kp], vp = a.cu[1][o + ps + kp];
            double2 v = cvt<double2>(sc * ra[r][k2]);
            v = v + mul_ik(a.kz[kp] * U0, u3) + mul_ik(2.0 * kxm * U0, u1);
            v.x += ((Up + U0) * vp.x - (U0 + Um) * vc.x) * id;
            v.y += ((Up + U0) * vp.y - (U0 + Um) * vc.y) * id;
            dst64[kp] = v;
          }
        }
      }
    }
    return;
  }
  if (!COMBINE && a.acc_scale != 0.0) {
    const int m = (a.q0 + q) % a.g.nkx1;
    const double w = a.acc_scale * (m > 0 ? 2.0 : 1.0);
    double2* dacc = reinterpret_cast<double2*>(dst);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      int k1 = t + r * N2;
      if (k1 < N1) {
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          int kp = z_pack(k1 + N1 * k2, a.g.nz, a.g.nkz);
          if (kp >= 0) dacc[kp] = dacc[kp] + w * cvt<double2>(sc * ra[r][k2]);
        }
      }
    }
    return;
  }
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    int k1 = t + r * N2;
    if (k1 < N1) {
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        int kp = z_pack(k1 + N1 * k2, a.g.nz, a.g.nkz);
        if (kp >= 0) dst[kp] = cvt<CO>(sc * ra[r][k2]);
      }
    }
  }
}

// --------------------------------------------------------------------------
// x inverse (c2r): x-spectral -> physical rows, KT z-rows per block.
// Length-Nx real transform as a length-M=Nx/2 complex transform with the
// standard even/odd split; only Re X[0] enters (FFTW c2r ignores Im of the
// DC and Nyquist bins), and X[m] = 0 for Nkx < m <= M (for/fft.f90:372-378).
template <typename C> struct XInvArgs {
  const C* src[NF_MAX];
  typename CReal<C>::R* dst[NF_MAX];
  int j0;            // first plane
  Geom g;
  const C* twM;      // exp(-2 pi i m / M), m < M
  const C* twX;      // exp(-2 pi i m / Nx), m <= M
};

// Spectrum loads a thread keeps in flight in k_xc2r before storing them.  At
// 256 x 257 x 256 (FP32, 16x8 tile, 16 rows) issuing them one load per
// shared store took 0.2095 ms per launch; batches of 4, 9 and all 17 took
// 0.163, 0.162 and 0.163 ms.
#ifndef XC2R_LOAD_BATCH
#define XC2R_LOAD_BATCH 32
#endif

template <typename C, int N1, int N2, int KT>
__global__ void __launch_bounds__(N2* KT, sizeof(C) == 8 ? XC2R32_MIN_BLOCKS : 1) k_xc2r(XInvArgs<C> a) {
  typedef typename CReal<C>::R T;
  constexpr int M = N1 * N2;
  constexpr int SM = dfft::SmemSize<N1, N2>::v;
  // When the N2 threads of a row share a warp (32 % N2 == 0), one row buffer
  // holds the spectrum (M + 1 entries) and then the four-step tile: a row is
  // read and rewritten only by its own threads, so a warp barrier separates
  // the two uses and the block needs half the shared memory (more blocks per
  // SM).  Otherwise the two live side by side.
  constexpr bool ALIAS = 32 % N2 == 0 && (sizeof(C) == 8 || XC2R_ALIAS_FP64);
  constexpr int ROW = ALIAS ? (SM > M + 1 ? SM : M + 1) : M + 1 + SM;
  constexpr int SMOFF = ALIAS ? 0 : M + 1;
  __shared__ C rowbuf[KT][ROW];
  auto xs = [&](int rr) -> C* { return rowbuf[rr]; };
  auto sm = [&](int rr) -> C* { return rowbuf[rr] + SMOFF; };
  const int t = threadIdx.x, r = threadIdx.y;
  const int tid = r * N2 + t;
  const int k0 = blockIdx.x * KT;
  const int j = a.j0 + blockIdx.y;
  const int f = blockIdx.z;
  const int nkx1 = a.g.nkx1, nz = a.g.nz;
  const C* src = a.src[f] + (size_t)j * nkx1 * nz;
  // a thread's spectrum loads are issued in batches of LB before their shared
  // stores, so LB loads are in flight at once
  constexpr int NT = N2 * KT, TOT = KT * (M + 1), IT = (TOT + NT - 1) / NT;
  constexpr int LB = IT < XC2R_LOAD_BATCH ? IT : XC2R_LOAD_BATCH;
#pragma unroll
  for (int i0 = 0; i0 < IT; i0 += LB) {
    C ld[LB];
#pragma unroll
    for (int i = 0; i < LB; ++i) {
      const int idx = tid + (i0 + i) * NT, rr = idx % KT, m = idx / KT;
      ld[i] = czero<C>();
      if (i0 + i < IT && idx < TOT && m < nkx1 && k0 + rr < nz) ld[i] = src[(size_t)m * nz + k0 + rr];
    }
#pragma unroll
    for (int i = 0; i < LB; ++i) {
      const int idx = tid + (i0 + i) * NT;
      if (i0 + i < IT && idx < TOT) xs(idx % KT)[idx / KT] = ld[i];
    }
  }
  __syncthreads();
  C v[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    int m = n1 * N2 + t;
    C xm = xs(r)[m];
    C xc = conj(xs(r)[M - m]);  // m == 0 reads X[M] = 0
    if (m == 0) xm.y = 0;
    C e = xm + xc;
    C o = xm - xc;
    C w = conj(a.twX[m]);           // exp(+2 pi i m / Nx)
    v[n1] = e + mul_i(cmul(w, o));
  }
  if (ALIAS) __syncwarp();
  dfft::step1<N1, N2, +1>(v, t, a.twM, sm(r));
  __syncthreads();
  if (k0 + r >= nz) return;
  T* dst = a.dst[f] + ((size_t)j * nz + k0 + r) * a.g.nx;
  C* dstc = reinterpret_cast<C*>(dst);
  for (int k1 = t; k1 < N1; k1 += N2) {
    C u[N2];
    dfft::step2<N1, N2, +1>(u, k1, sm(r));
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) dstc[k1 + N1 * k2] = u[k2];
  }
}

// --------------------------------------------------------------------------
// x forward (r2c) of physical rows, KT z-rows per block, optionally of the
// nonlinear products of the channel step.
//   plain: out0 = X / Nx for m <= Nkx (for/fft.f90:258-266)
//   NL:    for output equation f the products (A: needs d/dz, Bx: needs d/dx,
//          B0: already a y-difference) give outA = Fx(A)/Nx and
//          outB = (i kx Fx(Bx) + Fx(B0))/Nx.
struct GridMetrics {
  const double* dy;
  const double* dyf;
};

template <typename T> struct XFwdArgs {
  const T* in[NF_MAX];           // plain: field to transform; NL: u1,u2,u3,th_n
  typename CT<T>::C* outA[NF_MAX];
  typename CT<T>::C* outB[NF_MAX];
  int j0;
  Geom g;
  const typename CT<T>::C* twM;
  const typename CT<T>::C* twX;
  const double* kx;              // kx(m)
  GridMetrics gm;
  double scale;                  // 1/Nx
};

// The four kinds of nonlinear product of for/channel.f90:299-459,553-608 at
// the x pair (2n, 2n+1) of one row.  Each `fill_*` evaluates all N1 pairs of a
// thread with straight-line code, so every load of the term is in flight
// before the first product is formed.
template <typename T> struct Pair { T a, b; };

template <typename T>
DI Pair<T> ld2(const T* p) {
  typedef typename CT<T>::C C;
  C v = *reinterpret_cast<const C*>(p);
  return Pair<T>{v.x, v.y};
}

// Division of a row's products by one per-row denominator.  The FP32 build
// multiplies by the reciprocal (one rounding more, inside the mixed path's
// tolerance, and no IEEE divide sequence per element); FP64 divides, so the
// FP64 path rounds as the reference does.
template <typename T>
struct DivBy {
  T d, inv;
  DI explicit DivBy(T den) : d(den), inv((T)1 / den) {}
  DI T operator()(T x) const {
    if constexpr (sizeof(T) == 4) return x * inv;
    else return x / d;
  }
};

// x(j) * y(j)
template <typename T, int N1, int N2>
DI void fill_prod(typename CT<T>::C (&v)[N1], const T* x, const T* y, size_t off, int t) {
  Pair<T> px[N1], py[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    const size_t o = off + 2 * (n1 * N2 + t);
    px[n1] = ld2(x + o); py[n1] = ld2(y + o);
  }
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) v[n1] = CT<T>::mk(px[n1].a * py[n1].a, px[n1].b * py[n1].b);
}

// x(j)^2 (u1 u1 and u3 u3): one load per element
template <typename T, int N1, int N2>
DI void fill_sq(typename CT<T>::C (&v)[N1], const T* x, size_t off, int t) {
  Pair<T> px[N1];
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) px[n1] = ld2(x + off + 2 * (n1 * N2 + t));
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) v[n1] = CT<T>::mk(px[n1].a * px[n1].a, px[n1].b * px[n1].b);
}

// (uf(j+1)u2(j+1) + uf(j)u2(j+1) - uf(j)u2(j) - uf(j-1)u2(j)) / (2 dyf(j))
template <typename T, int N1, int N2>
DI void fill_flux(typename CT<T>::C (&v)[N1], const T* uf, const T* u2, size_t off, size_t ps,
                  T den, int t) {
  const DivBy<T> dv(den);
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    const size_t o = off + 2 * (n1 * N2 + t);
    Pair<T> p = ld2(uf + o + ps), c = ld2(uf + o), m = ld2(uf + o - ps);
    Pair<T> vp = ld2(u2 + o + ps), vc = ld2(u2 + o);
    v[n1] = CT<T>::mk(dv(p.a * vp.a + c.a * vp.a - c.a * vc.a - m.a * vc.a),
                      dv(p.b * vp.b + c.b * vp.b - c.b * vc.b - m.b * vc.b));
  }
}

// ((dyf(j) uf(j) + dyf(j-1) uf(j-1)) / (2 dy(j))) * u2(j)
template <typename T, int N1, int N2>
DI void fill_interp(typename CT<T>::C (&v)[N1], const T* uf, const T* u2, size_t off, size_t ps,
                    T dyfj, T dyfm, T den, int t) {
  const DivBy<T> dv(den);
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    const size_t o = off + 2 * (n1 * N2 + t);
    Pair<T> c = ld2(uf + o), m = ld2(uf + o - ps), w = ld2(u2 + o);
    v[n1] = CT<T>::mk(dv(dyfj * c.a + dyfm * m.a) * w.a, dv(dyfj * c.b + dyfm * m.b) * w.b);
  }
}

// (0.25 (u2(j) + u2(j+1))^2 - 0.25 (u2(j) + u2(j-1))^2) / dy(j)
template <typename T, int N1, int N2>
DI void fill_v2(typename CT<T>::C (&v)[N1], const T* u2, size_t off, size_t ps, T dyj, int t) {
  const DivBy<T> dv(dyj);
#pragma unroll
  for (int n1 = 0; n1 < N1; ++n1) {
    const size_t o = off + 2 * (n1 * N2 + t);
    Pair<T> p = ld2(u2 + o + ps), c = ld2(u2 + o), m = ld2(u2 + o - ps);
    T sa = c.a + p.a, sb = c.b + p.b, da = c.a + m.a, db = c.b + m.b;
    v[n1] = CT<T>::mk(dv((T)0.25 * (sa * sa) - (T)0.25 * (da * da)),
                      dv((T)0.25 * (sb * sb) - (T)0.25 * (db * db)));
  }
}

// term q (0: needs d/dz, 1: needs d/dx, 2: y-flux) of output equation f
// (0 = u1, 1 = u2, 2 = u3, 3+n = scalar n)
template <typename T, int N1, int N2>
DI void nl_fill(typename CT<T>::C (&v)[N1], const XFwdArgs<T>& a, int f, int q, int j, size_t off,
                size_t ps, int t) {
  const T* u1 = a.in[0];
  const T* u2 = a.in[1];
  const T* u3 = a.in[2];
  if (f == 1) {
    if (q == 2) {
      fill_v2<T, N1, N2>(v, u2, off, ps, (T)a.gm.dy[j], t);
    } else {
      fill_interp<T, N1, N2>(v, q == 0 ? u3 : u1, u2, off, ps, (T)a.gm.dyf[j], (T)a.gm.dyf[j - 1],
                             (T)(2.0 * a.gm.dy[j]), t);
    }
    return;
  }
  const T* own = f == 0 ? u1 : (f == 2 ? u3 : a.in[f]);
  if (q == 2) {
    fill_flux<T, N1, N2>(v, own, u2, off, ps, (T)(2.0 * a.gm.dyf[j]), t);
  } else if (q == 0) {
    // f=0: u3*u1; f=2: u3*u3; scalar: th*u3
    if (f == 2) fill_sq<T, N1, N2>(v, u3, off, t);
    else fill_prod<T, N1, N2>(v, f == 0 ? u3 : own, f == 0 ? u1 : u3, off, t);
  } else {
    // f=0: u1*u1; f=2: u3*u1; scalar: th*u1
    if (f == 0) fill_sq<T, N1, N2>(v, u1, off, t);
    else fill_prod<T, N1, N2>(v, own, u1, off, t);
  }
}

// 16-byte row loads for the FP32 transforms with N1 = 2 N2 (XR2C_VEC4).
// Thread t of a row loads float4 number N2 i + t (i < N1/2): the N2 threads
// of the row read 16 N2 contiguous bytes per instruction (128 bytes at
// N2 = 8, against 64 with the 8-byte pair loads), so a warp's load covers
// whole 128-byte lines.  Element e = 2i + b of the thread is then the complex
// point z[2 N2 i + 2t + b].
DI float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
template <int N1, int N2>
DI size_t v4off(int i, int t) { return (size_t)4 * (N2 * i + t); }

template <int N1, int N2>
DI void fill4_prod(float2 (&v)[N1], const float* x, const float* y, size_t off, int t) {
  float4 px[N1 / 2], py[N1 / 2];
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) { px[i] = ld4(x + off + v4off<N1, N2>(i, t)); py[i] = ld4(y + off + v4off<N1, N2>(i, t)); }
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) {
    v[2 * i] = make_float2(px[i].x * py[i].x, px[i].y * py[i].y);
    v[2 * i + 1] = make_float2(px[i].z * py[i].z, px[i].w * py[i].w);
  }
}
template <int N1, int N2>
DI void fill4_sq(float2 (&v)[N1], const float* x, size_t off, int t) {
  float4 px[N1 / 2];
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) px[i] = ld4(x + off + v4off<N1, N2>(i, t));
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) {
    v[2 * i] = make_float2(px[i].x * px[i].x, px[i].y * px[i].y);
    v[2 * i + 1] = make_float2(px[i].z * px[i].z, px[i].w * px[i].w);
  }
}
template <int N1, int N2>
DI void fill4_flux(float2 (&v)[N1], const float* uf, const float* u2, size_t off, size_t ps, float den, int t) {
  const DivBy<float> dv(den);
  auto f = [&](float p, float c, float m, float vp, float vc) { return dv(p * vp + c * vp - c * vc - m * vc); };
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) {
    const size_t o = off + v4off<N1, N2>(i, t);
    const float4 p = ld4(uf + o + ps), c = ld4(uf + o), m = ld4(uf + o - ps);
    const float4 vp = ld4(u2 + o + ps), vc = ld4(u2 + o);
    v[2 * i] = make_float2(f(p.x, c.x, m.x, vp.x, vc.x), f(p.y, c.y, m.y, vp.y, vc.y));
    v[2 * i + 1] = make_float2(f(p.z, c.z, m.z, vp.z, vc.z), f(p.w, c.w, m.w, vp.w, vc.w));
  }
}
template <int N1, int N2>
DI void fill4_interp(float2 (&v)[N1], const float* uf, const float* u2, size_t off, size_t ps, float dyfj,
                     float dyfm, float den, int t) {
  const DivBy<float> dv(den);
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) {
    const size_t o = off + v4off<N1, N2>(i, t);
    const float4 c = ld4(uf + o), m = ld4(uf + o - ps), w = ld4(u2 + o);
    v[2 * i] = make_float2(dv(dyfj * c.x + dyfm * m.x) * w.x, dv(dyfj * c.y + dyfm * m.y) * w.y);
    v[2 * i + 1] = make_float2(dv(dyfj * c.z + dyfm * m.z) * w.z, dv(dyfj * c.w + dyfm * m.w) * w.w);
  }
}
template <int N1, int N2>
DI void fill4_v2(float2 (&v)[N1], const float* u2, size_t off, size_t ps, float dyj, int t) {
  const DivBy<float> dv(dyj);
  auto f = [&](float p, float c, float m) {
    const float sa = c + p, da = c + m;
    return dv(0.25f * (sa * sa) - 0.25f * (da * da));
  };
#pragma unroll
  for (int i = 0; i < N1 / 2; ++i) {
    const size_t o = off + v4off<N1, N2>(i, t);
    const float4 p = ld4(u2 + o + ps), c = ld4(u2 + o), m = ld4(u2 + o - ps);
    v[2 * i] = make_float2(f(p.x, c.x, m.x), f(p.y, c.y, m.y));
    v[2 * i + 1] = make_float2(f(p.z, c.z, m.z), f(p.w, c.w, m.w));
  }
}
// nl_fill with the 16-byte loads (same products, same operation order)
template <int N1, int N2>
DI void nl_fill4(float2 (&v)[N1], const XFwdArgs<float>& a, int f, int q, int j, size_t off, size_t ps, int t) {
  const float* u1 = a.in[0];
  const float* u2 = a.in[1];
  const float* u3 = a.in[2];
  if (f == 1) {
    if (q == 2) {
      fill4_v2<N1, N2>(v, u2, off, ps, (float)a.gm.dy[j], t);
    } else {
      fill4_interp<N1, N2>(v, q == 0 ? u3 : u1, u2, off, ps, (float)a.gm.dyf[j], (float)a.gm.dyf[j - 1],
                           (float)(2.0 * a.gm.dy[j]), t);
    }
    return;
  }
  const float* own = f == 0 ? u1 : (f == 2 ? u3 : a.in[f]);
  if (q == 2) {
    fill4_flux<N1, N2>(v, own, u2, off, ps, (float)(2.0 * a.gm.dyf[j]), t);
  } else if (q == 0) {
    if (f == 2) fill4_sq<N1, N2>(v, u3, off, t);
    else fill4_prod<N1, N2>(v, f == 0 ? u3 : own, f == 0 ? u1 : u3, off, t);
  } else {
    if (f == 0) fill4_sq<N1, N2>(v, u1, off, t);
    else fill4_prod<N1, N2>(v, own, u1, off, t);
  }
}

// Whether k_xr2c finishes the real-to-complex split in registers.  The split
// needs Z[m] and Z[M - m] together.  With N1 = 2 N2 a thread can own step-2
// rows k1 and N1 - k1 (thread 0: rows 0 and N1/2), and row k1 holds
// Z[k1 + N1 k2] while row N1 - k1 holds Z[M - k1 - N1 k2] at k2' = N2-1-k2:
// every pair (m, M - m) then lies in one thread, and the spectrum needs no
// natural-order copy in shared memory.  At 256 x 257 x 256 (FP32 products,
// 16 rows per block) this and the accumulator pitch below took the launch
// from 0.615 to 0.494 ms; with a separate code path for thread 0 (run
// serially beside the other threads' in every warp) it had measured 0.689.
#ifndef XR2C_PAIRED
#define XR2C_PAIRED 1
#endif
#ifndef XR2C_PAD_OP
#define XR2C_PAD_OP 1
#endif
// Whether the FP32 paired transforms use the 16-byte row loads.  The loads
// give each thread the columns n2 = c0, c0 + 1 (c0 = 2t mod N2) of the
// four-step split n = n2 + N2 n1, the even n1 (t < N2/2) or the odd n1
// (t >= N2/2).  Step 1 is then a radix-2 split of the length-N1 DFT: the
// thread transforms its two half sequences (length N1/2 = N2), E_c or O_c,
// and stores E'[c][k] = E_c[k] w_M^(c k) or O'[c][k] = O_c[k] w_M^((N2+c) k);
// the step-2 thread of row k1 forms E' + O' (k1 < N1/2, k = k1) or
// (E' - O') w_M^(N2 c) (k1 >= N1/2, k = k1 - N1/2) and transforms along c.
// Tile entry (h, c, k) sits at h HP + c CP + k with CP = N2 + 1 and
// HP = N2 CP + 1: at N2 = 8 both the stores (fixed c, k per instruction)
// and the step-2 reads (fixed c, consecutive k) of the warp's four rows fill
// two 128-byte wavefronts each.
#ifndef XR2C_VEC4
#define XR2C_VEC4 1
#endif

// Shared-memory layout of k_xr2c for a given configuration.
template <typename T, int N1, int N2, int KT, bool NL = true>
struct XFwdSmem {
  typedef typename CT<T>::C C;
  static constexpr int M = N1 * N2;
  static constexpr int NKX1 = (2 * M) / 3 + 1;   // upper bound of Nkx+1
  static constexpr bool PAIRED = XR2C_PAIRED && N1 == 2 * N2;
  static constexpr bool VEC = XR2C_VEC4 && PAIRED && sizeof(T) == 4;
  static constexpr int VCP = N2 + 1, VHP = N2 * VCP + 1;
  static constexpr int VRAW = 2 * VHP;
  // the E'/O' tile padded like dfft::SmemSize: rows start 64 bytes apart modulo 128
  static constexpr int VROW = VRAW + ((((VRAW * 8) % 128) == 64) ? 0 : ((128 + 64 - (VRAW * 8) % 128) % 128) / 8);
  // per row one four-step tile (without the register split also the
  // natural-order spectrum, which needs M+1 entries)
  static constexpr int ROWC = VEC ? VROW
                            : ((PAIRED || dfft::SmemSize<N1, N2>::v > M + 1) ? dfft::SmemSize<N1, N2>::v : M + 1);
  // Pitch of the accumulated B output [m][row] of the NL form (the A output
  // goes straight to global memory).  Shared memory serves 128 bytes per
  // wavefront: W = 128 / sizeof(C) threads, that is G = W / N2 rows of N2
  // threads with consecutive modes m.  Entry (m, row) sits at m OP + row, so
  // the W threads hit distinct banks when OP / G is odd; OP is the smallest
  // such pitch >= KT (18 against KT + 1 = 17 for the FP32 products: 0.494
  // against 0.501 ms per launch).
  static constexpr int W = 128 / (int)sizeof(C);
  static constexpr int G = W / N2 > 1 ? W / N2 : 1;
  static constexpr int OPG = (KT + G - 1) / G;
  static constexpr int OP = !XR2C_PAD_OP ? KT + 1 : G * (OPG % 2 ? OPG : OPG + 1);
  static constexpr int bytes = (KT * ROWC + (NL ? NKX1 * OP : 0)) * (int)sizeof(C);
};

// Blocks per SM the FP32 products kernel's register cap is set for.  With the
// A output stored straight to global memory a block holds 30 KB of shared
// memory, so six fit; at 80 registers (40 bytes spilled) the launch measured
// 0.660 ms against 0.671 at 96 registers and five blocks (0.726 ms with both
// outputs staged in shared memory) and 0.701 at seven blocks (72 registers,
// 80 bytes spilled).
#ifndef XR2C32_MIN_BLOCKS
#define XR2C32_MIN_BLOCKS 6
#endif
// Whether k_xr2c separates the phases of one row's transform with a warp
// barrier instead of a block barrier.  The N2 threads of a row share a warp
// when 32 % N2 == 0, and every shared-memory entry a phase reads was written
// by the same row's threads; only the B output's final store reads other
// rows' entries.  At 256 x 257 x 256 (FP32, before the register split) the
// warp barrier measured 5.057 against 5.101 ms per step.
#ifndef XR2C_WARP_SYNC
#define XR2C_WARP_SYNC 1
#endif

// The FP64 products kernel (8 z-rows of 64 threads a block) holds 252
// registers unbounded, four blocks per SM.  A cap for six blocks (168
// registers, no spills) took it from 1.546 to 1.200 ms per launch at
// 256 x 257 x 256 with bit-identical output, and eight blocks (128 registers,
// 176 bytes spilled) measured 1.239 ms.  The same caps on the FP64 z forward
// combine and x inverse (168/128 registers) moved them by +-2% and are not set.
// The cap applies to that measured shape (Nx = 256, 8 rows a block) only: on
// other lengths and row counts it makes the compiler spill.
#ifndef XR2C64_MIN_BLOCKS
#define XR2C64_MIN_BLOCKS 6
#endif

template <typename T, int N1, int N2, int KT, bool NL>
__global__ void __launch_bounds__(N2* KT, NL ? (sizeof(T) == 4 ? XR2C32_MIN_BLOCKS
                                                   : (N1 == 16 && N2 == 8 && KT == 8 ? XR2C64_MIN_BLOCKS : 1))
                                             : 1)
    k_xr2c(XFwdArgs<T> a) {
  typedef typename CT<T>::C C;
  typedef XFwdSmem<T, N1, N2, KT, NL> L;
  constexpr int M = N1 * N2;
  constexpr int ROWC = L::ROWC;
  constexpr int NKX1 = L::NKX1;
  constexpr int NS = (NKX1 + N2 - 1) / N2;  // output slots per thread
  constexpr int NR = (N1 + N2 - 1) / N2;    // step-2 rows per thread
  constexpr int OP = L::OP;
  constexpr bool PAIRED = L::PAIRED;
  constexpr bool VEC = L::VEC;
  extern __shared__ __align__(16) unsigned char xr2c_smem[];
  C* smb = reinterpret_cast<C*>(xr2c_smem);          // [KT][ROWC] four-step tile / spectrum
  C* acc = smb + KT * ROWC;                            // [NKX1][OP] output B (NL)
  const int t = threadIdx.x, r = threadIdx.y;
  // field fastest: the blocks that read the same input rows run together
  const int f = blockIdx.x;
  const int k0 = blockIdx.y * KT;
  const int j = a.j0 + blockIdx.z;
  const int nz = a.g.nz, nx = a.g.nx, nkx1 = a.g.nkx1;
  const int row = min(k0 + r, nz - 1);
  const size_t ps = (size_t)nz * nx;
  const size_t rowoff = (size_t)j * ps + (size_t)row * nx;
  C* dstA = a.outA[f] + (size_t)j * nkx1 * nz;
  const T sc = (T)a.scale;
  C* sm = smb + r * ROWC;
  C* zs = sm;  // the natural-order spectrum replaces the tile after step 2
  constexpr int NQ = NL ? 3 : 1;
  constexpr bool WROW = XR2C_WARP_SYNC && 32 % N2 == 0;
  auto rowsync = [] { if constexpr (WROW) __syncwarp(); else __syncthreads(); };
  // output X[m] of transform q: A straight to global (a warp writes 32-byte
  // runs along k of 32 / N2 rows for each of its N2 modes); Bx and B0 into the
  // accumulator, each (m, row) entry always by the same thread
  auto put = [&](int q, int m, C x) {
    if (!NL || q == 0) { if (k0 + r < nz) dstA[(size_t)m * nz + k0 + r] = x; }
    else if (q == 1) acc[m * OP + r] = mul_ik((T)a.kx[m], x);
    else acc[m * OP + r] = acc[m * OP + r] + x;
  };
  // the pair (m, M - m) from zm = Z[m], zp = Z[M - m]:
  //   X[m] = sc (e - i w o),  X[M - m] = sc conj(e + i w o)
  // with e = (zm + conj zp)/2, o = (zm - conj zp)/2, w = exp(-2 pi i m / Nx)
  // (w(M - m) = -conj w(m) gives the second form)
  auto put_pair = [&](int q, int m, C zm, C zp) {
    const C zc = conj(zp);
    const C e = (T)0.5 * (zm + zc);
    const C o = (T)0.5 * (zm - zc);
    const C wo = cmul(a.twX[m], o);
    if (m < nkx1) put(q, m, sc * (e - mul_i(wo)));
    if (2 * m != M && M - m < nkx1) put(q, M - m, sc * conj(e + mul_i(wo)));
  };
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    C v[N1];
    if constexpr (VEC) {
      if (NL) {
        nl_fill4<N1, N2>(v, a, f, q, j, rowoff, ps, t);
      } else {
#pragma unroll
        for (int i = 0; i < N1 / 2; ++i) {
          const float4 x = ld4(a.in[f] + rowoff + v4off<N1, N2>(i, t));
          v[2 * i] = CT<T>::mk(x.x, x.y);
          v[2 * i + 1] = CT<T>::mk(x.z, x.w);
        }
      }
      // step 1: the half sequences of columns c0 and c0 + 1
      constexpr int H = N1 / 2, CP = L::VCP, HP = L::VHP;
      const int h = t >= N2 / 2 ? 1 : 0;
      const int c0 = 2 * (t - h * (N2 / 2));
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        C sq[H];
#pragma unroll
        for (int i = 0; i < H; ++i) sq[i] = v[2 * i + b];
        dfft::RegDFT<H, -1, C>::run(sq);
        const int c = c0 + b;
        C* dst = sm + h * HP + c * CP;
        dst[0] = sq[0];
        const int tws = h * N2 + c;
#pragma unroll
        for (int k = 1; k < H; ++k) dst[k] = cmul(sq[k], a.twM[tws * k]);
      }
    } else {
      if (NL) {
        nl_fill<T, N1, N2>(v, a, f, q, j, rowoff, ps, t);
      } else {
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1)
          v[n1] = *reinterpret_cast<const C*>(a.in[f] + rowoff + 2 * (n1 * N2 + t));
      }
      dfft::step1<N1, N2, -1>(v, t, a.twM, sm);
    }
    rowsync();
    if constexpr (PAIRED) {
      // thread t owns rows t and N1 - t; thread 0 rows 0 and N1/2
      C ua[N2], ub[N2];
      if constexpr (VEC) {
        constexpr int H = N1 / 2, CP = L::VCP, HP = L::VHP;
        const int ka = t, kb = (H - t) % H;   // rows t (< H) and N1 - t or H (>= H)
#pragma unroll
        for (int c = 0; c < N2; ++c) {
          const C ea = sm[c * CP + ka], oa = sm[HP + c * CP + ka];
          const C eb = sm[c * CP + kb], ob = sm[HP + c * CP + kb];
          ua[c] = ea + oa;
          ub[c] = c == 0 ? eb - ob : cmul(eb - ob, a.twM[N2 * c]);
        }
        dfft::RegDFT<N2, -1, C>::run(ua);
        dfft::RegDFT<N2, -1, C>::run(ub);
      } else {
        dfft::step2<N1, N2, -1>(ua, t, sm);
        dfft::step2<N1, N2, -1>(ub, t == 0 ? N1 / 2 : N1 - t, sm);
      }
      rowsync();  // the tile is free for the next transform
      // N2 pair slots per thread, the same code path in every thread (a
      // separate path for thread 0 would run serially beside the others'):
      //   t != 0:  Z[t + N1 k2] with Z[(N1 - t) + N1 (N2-1-k2)]
      //   t == 0:  slots k2 < N2/2: row N1/2, Z[N1/2 + N1 k2] with
      //            Z[N1/2 + N1 (N2-1-k2)]; slots k2 >= N2/2: row 0,
      //            Z[N1 i] with Z[N1 (N2 - i)], i = k2 - N2/2 + 1 (i = N2/2
      //            pairs Z[M/2] with itself)
      // and X[0] = sc (Re Z[0] + Im Z[0]) from thread 0 besides.
      const bool t0 = t == 0;
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) {
        constexpr int H = N2 / 2;
        const int i = k2 - H + 1;  // row-0 index of thread 0's upper slots
        C zm, zp;
        int m;
        if (k2 < H) {
          zm = t0 ? ub[k2] : ua[k2];
          zp = ub[N2 - 1 - k2];
          m = t0 ? N1 / 2 + N1 * k2 : t + N1 * k2;
        } else {
          zm = t0 ? ua[i < 0 ? 0 : i] : ua[k2];
          zp = t0 ? ua[(N2 - i) % N2] : ub[N2 - 1 - k2];
          m = t0 ? N1 * i : t + N1 * k2;
        }
        put_pair(q, m, zm, zp);
      }
      if (t0) put(q, 0, CT<T>::mk(sc * (ua[0].x + ua[0].y), (T)0));
    } else {
      C u[NR][N2];
#pragma unroll
      for (int rr = 0; rr < NR; ++rr)
        if (t + rr * N2 < N1) dfft::step2<N1, N2, -1>(u[rr], t + rr * N2, sm);
      rowsync();
#pragma unroll
      for (int rr = 0; rr < NR; ++rr) {
        const int k1 = t + rr * N2;
        if (k1 < N1) {
#pragma unroll
          for (int k2 = 0; k2 < N2; ++k2) zs[k1 + N1 * k2] = u[rr][k2];
        }
      }
      if (t == 0) zs[M] = u[0][0];
      rowsync();
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        int m = t + s * N2;
        if (m < nkx1) {
          C zm = zs[m], zc = conj(zs[M - m]);
          C e = (T)0.5 * (zm + zc);
          C o = (T)0.5 * (zm - zc);
          put(q, m, sc * (e - mul_i(cmul(a.twX[m], o))));
        }
      }
      rowsync();
    }
  }
  // B stores run along k (KT consecutive rows per mode)
  if (NL) {
    if constexpr (WROW) __syncthreads();
    C* dst = a.outB[f] + (size_t)j * nkx1 * nz;
    for (int idx = r * N2 + t; idx < nkx1 * KT; idx += N2 * KT) {
      int rr = idx % KT, m = idx / KT;
      if (k0 + rr < nz) dst[(size_t)m * nz + k0 + rr] = acc[m * OP + rr];
    }
  }
}
