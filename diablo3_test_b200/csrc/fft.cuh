// Register / shared-memory building blocks of the xz FFTs.
//
// A length-N transform (N = N1*N2, N1, N2 in {1,2,3,4,6,8,12,16}) is done as a
// four-step FFT by N2 cooperating threads:
//   step 1: thread n2 holds x[n1*N2 + n2] (n1 = 0..N1-1), does a register
//           DFT of length N1, multiplies element k1 by w_N^(n2*k1) and writes
//           it to shared memory at [k1][n2];
//   step 2: the thread owning k1 reads [k1][0..N2-1], does a register DFT of
//           length N2 and holds X[k1 + N1*k2] for k2 = 0..N2-1.
// One shared-memory exchange per transform; all other data movement is
// register renaming inside fully unrolled code.
//
// DIR = -1 is FFTW_FORWARD (exp(-2 pi i jk/N)), DIR = +1 FFTW_BACKWARD; neither
// is normalised, as in FFTW (the reference normalises by hand, for/fft.f90:262,304).
#pragma once
#include "common.cuh"

namespace dfft {

// cos(2*pi*q/48) for the angles the register DFTs of length 6, 8, 12, 16 use
// (multiples of 2*pi/16 and 2*pi/12).  Literal values are the exact
// mathematical constants rounded to double.
HDI constexpr double base_cos48(int r) {
  return r == 0 ? 1.0
       : r == 3 ? 0.92387953251128675612818318939679   // cos(pi/8)
       : r == 4 ? 0.86602540378443864676372317075294   // sqrt(3)/2
       : r == 6 ? 0.70710678118654752440084436210485   // sqrt(2)/2
       : r == 8 ? 0.5
       : r == 9 ? 0.38268343236508977172845998403040   // sin(pi/8)
       : 0.0;                                            // r == 12
}
HDI constexpr double cos48(int q) {
  return (q % 48) / 12 == 0 ? base_cos48((q % 48) % 12)
       : (q % 48) / 12 == 1 ? -base_cos48(12 - (q % 48) % 12)
       : (q % 48) / 12 == 2 ? -base_cos48((q % 48) % 12)
       : base_cos48(12 - (q % 48) % 12);
}
HDI constexpr double sin48(int q) { return cos48(q + 36); }

// exp(DIR * 2 pi i * m / R) for R in {6, 8, 12, 16}
template <int R, int DIR, int M, typename C> DI C wconst() {
  constexpr int q = (M % R) * (48 / R);
  typedef typename CReal<C>::R T;
  C w;
  w.x = (T)cos48(q);
  w.y = (T)(DIR * sin48(q));
  return w;
}

// multiply by DIR*i  (forward: -i, backward: +i)
template <int DIR, typename C> DI C mul_dir_i(C a) {
  C r;
  if (DIR < 0) { r.x = a.y; r.y = -a.x; } else { r.x = -a.y; r.y = a.x; }
  return r;
}

template <int R, int DIR, typename C> struct RegDFT;

template <int DIR, typename C> struct RegDFT<1, DIR, C> {
  DI static void run(C*) {}
};
template <int DIR, typename C> struct RegDFT<2, DIR, C> {
  DI static void run(C* x) { C t = x[0]; x[0] = t + x[1]; x[1] = t - x[1]; }
};
template <int DIR, typename C> struct RegDFT<3, DIR, C> {
  DI static void run(C* x) {
    typedef typename CReal<C>::R T;
    const T s = (T)0.86602540378443864676372317075294;  // sin(2 pi/3)
    C t1 = x[1] + x[2];
    C t2 = x[1] - x[2];
    C m1 = x[0] - (T)0.5 * t1;
    C m2 = mul_dir_i<DIR>(s * t2);
    x[0] = x[0] + t1;
    x[1] = m1 + m2;
    x[2] = m1 - m2;
  }
};
template <int DIR, typename C> struct RegDFT<4, DIR, C> {
  DI static void run(C* x) {
    C a0 = x[0] + x[2], a1 = x[0] - x[2];
    C b0 = x[1] + x[3], b1 = mul_dir_i<DIR>(x[1] - x[3]);
    x[0] = a0 + b0;
    x[2] = a0 - b0;
    x[1] = a1 + b1;
    x[3] = a1 - b1;
  }
};

// composite length R = R1*R2 (Cooley-Tukey in registers)
template <int R1, int R2, int DIR, typename C> DI void regdft_ct(C* x) {
  constexpr int R = R1 * R2;
  C t[R];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    C col[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) col[n1] = x[n1 * R2 + n2];
    RegDFT<R1, DIR, C>::run(col);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) t[k1 * R2 + n2] = col[k1];
  }
  // twiddles w_R^(n2*k1); unrolled so every index is a compile-time constant
#define DFFT_TW(N2, K1)                                                          \
  if constexpr ((N2) < R2 && (K1) < R1 && ((N2) * (K1)) % R != 0)                \
    t[(K1) * R2 + (N2)] = cmul(t[(K1) * R2 + (N2)], wconst<R, DIR, ((N2) * (K1)) % R, C>());
#define DFFT_TW_ROW(N2)                                                            \
  DFFT_TW(N2, 1) DFFT_TW(N2, 2) DFFT_TW(N2, 3) DFFT_TW(N2, 4) DFFT_TW(N2, 5)      \
  DFFT_TW(N2, 6) DFFT_TW(N2, 7) DFFT_TW(N2, 8) DFFT_TW(N2, 9) DFFT_TW(N2, 10)     \
  DFFT_TW(N2, 11) DFFT_TW(N2, 12) DFFT_TW(N2, 13) DFFT_TW(N2, 14) DFFT_TW(N2, 15)
  DFFT_TW_ROW(1) DFFT_TW_ROW(2) DFFT_TW_ROW(3) DFFT_TW_ROW(4) DFFT_TW_ROW(5)
  DFFT_TW_ROW(6) DFFT_TW_ROW(7) DFFT_TW_ROW(8) DFFT_TW_ROW(9) DFFT_TW_ROW(10)
  DFFT_TW_ROW(11) DFFT_TW_ROW(12) DFFT_TW_ROW(13) DFFT_TW_ROW(14) DFFT_TW_ROW(15)
#undef DFFT_TW_ROW
#undef DFFT_TW
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    C row[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) row[n2] = t[k1 * R2 + n2];
    RegDFT<R2, DIR, C>::run(row);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) x[k1 + R1 * k2] = row[k2];
  }
}

template <int DIR, typename C> struct RegDFT<6, DIR, C> {
  DI static void run(C* x) { regdft_ct<3, 2, DIR>(x); }
};
template <int DIR, typename C> struct RegDFT<8, DIR, C> {
  DI static void run(C* x) { regdft_ct<4, 2, DIR>(x); }
};
template <int DIR, typename C> struct RegDFT<12, DIR, C> {
  DI static void run(C* x) { regdft_ct<4, 3, DIR>(x); }
};
template <int DIR, typename C> struct RegDFT<16, DIR, C> {
  DI static void run(C* x) { regdft_ct<4, 4, DIR>(x); }
};

// ---- four-step across threads --------------------------------------------
// Shared-memory pitch of one [k1][n2] tile row (one pad element breaks the
// 16-byte bank stride of step-2 reads).
template <int N2> struct Pitch { static constexpr int v = N2 + 1; };

// Step 1 for the thread owning column n2: DFT_N1 in registers, twiddle by
// w_N^(n2*k1) (table `tw` holds exp(-2 pi i m/N), m < N), store to smem.
template <int N1, int N2, int DIR, typename C>
DI void step1(C (&v)[N1], int n2, const C* __restrict__ tw, C* sm) {
  RegDFT<N1, DIR, C>::run(v);
  constexpr int SP = Pitch<N2>::v;
  sm[n2] = v[0];
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) {
    C w = tw[n2 * k1];
    if (DIR > 0) w.y = -w.y;
    sm[k1 * SP + n2] = (N2 == 1) ? v[k1] : cmul(v[k1], w);
  }
}

// Step 2 for row k1: load [k1][0..N2-1], DFT_N2; u[k2] = X[k1 + N1*k2].
template <int N1, int N2, int DIR, typename C>
DI void step2(C (&u)[N2], int k1, const C* sm) {
  constexpr int SP = Pitch<N2>::v;
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) u[n2] = sm[k1 * SP + n2];
  RegDFT<N2, DIR, C>::run(u);
}

// Complex elements of one sequence's tile, padded so that consecutive tiles
// start 64 bytes apart modulo 128: two sequences in one warp then use
// disjoint shared-memory banks.
template <int N1, int N2> struct SmemSize {
  static constexpr int raw = N1 * Pitch<N2>::v;
  static constexpr int v = raw + ((((raw * 8) % 128) == 64) ? 0 : ((128 + 64 - (raw * 8) % 128) % 128) / 8);
};

}  // namespace dfft
