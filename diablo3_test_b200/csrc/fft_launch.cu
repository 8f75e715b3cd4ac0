// Host launchers of the xz-FFT kernels, one explicit instantiation per
// supported transform length (kept in their own translation unit).
#include "../../include/diablo_gpu.h"
#include "fft_launch.h"
#include "kernels_fft.cuh"

// --------------------------------------------------------------------------
// supported transform lengths: N = N1*N2
bool factor(int n, int* n1, int* n2) {
  switch (n) {
    case 8: *n1 = 4; *n2 = 2; return true;
    case 12: *n1 = 4; *n2 = 3; return true;
    case 16: *n1 = 4; *n2 = 4; return true;
    case 24: *n1 = 8; *n2 = 3; return true;
    case 32: *n1 = 8; *n2 = 4; return true;
    case 48: *n1 = 12; *n2 = 4; return true;
    case 64: *n1 = 8; *n2 = 8; return true;
    case 96: *n1 = 12; *n2 = 8; return true;
    case 128: *n1 = 16; *n2 = 8; return true;
    case 192: *n1 = 16; *n2 = 12; return true;
    case 256: *n1 = 16; *n2 = 16; return true;
    default: return false;
  }
}

#define FFT_SIZE_CASES(X) X(4, 2) X(4, 3) X(4, 4) X(8, 3) X(8, 4) X(12, 4) X(8, 8) X(12, 8) X(16, 8) X(16, 12) X(16, 16)

// Tile shapes.  z kernels: S sequences per block, candidates S0/2, S0, 2 S0
// with S0 = 128/N2 (64 to 512 threads).  x kernels: KT rows per block,
// candidates KT0, KT0/2, KT0/4 with KT0 the largest that fits the kernel's
// shared-memory budget.  `tile` = 0 picks S0 / KT0; any other value must be
// one of the candidates (DIABLO_ERR_ARG otherwise).

// ---- z inverse ----
template <typename C, int N1, int N2, int S>
static void launch_zinv_s(const ZInvArgs<C>& a, int nfield, cudaStream_t s) {
  dim3 blk(N2, S), grd((a.nseq + S - 1) / S, nfield);
  k_zinv<C, N1, N2, S><<<grd, blk, 0, s>>>(a);
}
template <typename C, int N1, int N2>
static int launch_zinv_t(const ZInvArgs<C>& a, int nfield, cudaStream_t s, int tile) {
  constexpr int S0 = 128 / N2 > 0 ? 128 / N2 : 1;
  constexpr int SH = S0 / 2 > 0 ? S0 / 2 : 1;
  if (tile == 0 || tile == S0) { launch_zinv_s<C, N1, N2, S0>(a, nfield, s); return 0; }
  if (tile == SH) { launch_zinv_s<C, N1, N2, SH>(a, nfield, s); return 0; }
  if constexpr (2 * S0 * dfft::SmemSize<N1, N2>::v * (int)sizeof(C) <= 49152)
    if (tile == 2 * S0) { launch_zinv_s<C, N1, N2, 2 * S0>(a, nfield, s); return 0; }
  return DIABLO_ERR_ARG;
}
template <typename C>
int launch_zinv(const ZInvArgs<C>& a, int nz, int nfield, cudaStream_t s, int tile) {
  int n1, n2;
  if (!factor(nz, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) return launch_zinv_t<C, A, B>(a, nfield, s, tile);
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- z forward ----
template <typename C, typename CO, int N1, int N2, bool COMB, int S>
static void launch_zfwd_s(const ZFwdArgs<C, CO>& a, int nfield, cudaStream_t s) {
  dim3 blk(N2, S), grd((a.nseq + S - 1) / S, nfield);
  k_zfwd<C, CO, N1, N2, S, COMB><<<grd, blk, 0, s>>>(a);
}
template <typename C, typename CO, int N1, int N2, bool COMB>
static int launch_zfwd_t(const ZFwdArgs<C, CO>& a, int nfield, cudaStream_t s, int tile) {
  constexpr int S0 = 128 / N2 > 0 ? 128 / N2 : 1;
  constexpr int SH = S0 / 2 > 0 ? S0 / 2 : 1;
  if (tile == 0 || tile == S0) { launch_zfwd_s<C, CO, N1, N2, COMB, S0>(a, nfield, s); return 0; }
  if (tile == SH) { launch_zfwd_s<C, CO, N1, N2, COMB, SH>(a, nfield, s); return 0; }
  if constexpr (2 * S0 * dfft::SmemSize<N1, N2>::v * (int)sizeof(C) <= 49152)
    if (tile == 2 * S0) { launch_zfwd_s<C, CO, N1, N2, COMB, 2 * S0>(a, nfield, s); return 0; }
  return DIABLO_ERR_ARG;
}
template <typename C, typename CO, bool COMB>
int launch_zfwd(const ZFwdArgs<C, CO>& a, int nz, int nfield, cudaStream_t s, int tile) {
  int n1, n2;
  if (!factor(nz, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) return launch_zfwd_t<C, CO, A, B, COMB>(a, nfield, s, tile);
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- x inverse ----
template <typename C, int N1, int N2, int KT>
static void launch_xinv_k(const XInvArgs<C>& a, int nplanes, int nfield, cudaStream_t s) {
  dim3 blk(N2, KT), grd((a.g.nz + KT - 1) / KT, nplanes, nfield);
  k_xc2r<C, N1, N2, KT><<<grd, blk, 0, s>>>(a);
}
template <typename C, int N1, int N2>
static int launch_xinv_t(const XInvArgs<C>& a, int nplanes, int nfield, cudaStream_t s, int tile) {
  constexpr int M = N1 * N2;
  constexpr int ROW = (M + 1 + dfft::SmemSize<N1, N2>::v) * (int)sizeof(C);
  constexpr int KT0 = (40 * 1024) / ROW;
  constexpr int KT = KT0 >= 16 ? 16 : (KT0 >= 8 ? 8 : (KT0 >= 4 ? 4 : 2));
  constexpr int K2 = KT / 2 > 0 ? KT / 2 : 1, K4 = KT / 4 > 0 ? KT / 4 : 1;
  if (tile == 0 || tile == KT) { launch_xinv_k<C, N1, N2, KT>(a, nplanes, nfield, s); return 0; }
  if (tile == K2) { launch_xinv_k<C, N1, N2, K2>(a, nplanes, nfield, s); return 0; }
  if (tile == K4) { launch_xinv_k<C, N1, N2, K4>(a, nplanes, nfield, s); return 0; }
  return DIABLO_ERR_ARG;
}
template <typename C>
int launch_xinv(const XInvArgs<C>& a, int m, int nplanes, int nfield, cudaStream_t s, int tile) {
  int n1, n2;
  if (!factor(m, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) return launch_xinv_t<C, A, B>(a, nplanes, nfield, s, tile);
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- x forward ----
template <typename T, int N1, int N2, bool NL, int KT>
static void launch_xfwd_k(const XFwdArgs<T>& a, int nplanes, int nfield, cudaStream_t s) {
  constexpr int SMB = XFwdSmem<T, N1, N2, KT, NL>::bytes;
  cudaFuncSetAttribute(k_xr2c<T, N1, N2, KT, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMB);
  dim3 blk(N2, KT), grd(nfield, (a.g.nz + KT - 1) / KT, nplanes);
  k_xr2c<T, N1, N2, KT, NL><<<grd, blk, SMB, s>>>(a);
}
template <typename T, int N1, int N2, bool NL>
static int launch_xfwd_t(const XFwdArgs<T>& a, int nplanes, int nfield, cudaStream_t s, int tile) {
  // rows per block: as many as fit ~56 KB of shared memory, at most 16
  constexpr int KT = XFwdSmem<T, N1, N2, 16>::bytes <= 57344 ? 16
                   : (XFwdSmem<T, N1, N2, 8>::bytes <= 57344 ? 8 : 4);
  constexpr int K2 = KT / 2, K4 = KT / 4 > 0 ? KT / 4 : 1;
  if (tile == 0 || tile == KT) { launch_xfwd_k<T, N1, N2, NL, KT>(a, nplanes, nfield, s); return 0; }
  if (tile == K2) { launch_xfwd_k<T, N1, N2, NL, K2>(a, nplanes, nfield, s); return 0; }
  if (tile == K4) { launch_xfwd_k<T, N1, N2, NL, K4>(a, nplanes, nfield, s); return 0; }
  return DIABLO_ERR_ARG;
}
template <typename T, bool NL>
int launch_xfwd(const XFwdArgs<T>& a, int m, int nplanes, int nfield, cudaStream_t s, int tile) {
  int n1, n2;
  if (!factor(m, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) return launch_xfwd_t<T, A, B, NL>(a, nplanes, nfield, s, tile);
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// candidate tiles of each launcher for a transform length (for the autotuner),
// from the same constants the launchers use
static int uniq(int* out, int k, int v) {
  for (int i = 0; i < k; ++i) if (out[i] == v) return k;
  out[k] = v;
  return k + 1;
}
template <typename C, int N1, int N2>
static int z_cand(int* out) {
  constexpr int S0 = 128 / N2 > 0 ? 128 / N2 : 1;
  constexpr int SH = S0 / 2 > 0 ? S0 / 2 : 1;
  int k = uniq(out, 0, S0);
  k = uniq(out, k, SH);
  if (2 * S0 * dfft::SmemSize<N1, N2>::v * (int)sizeof(C) <= 49152) k = uniq(out, k, 2 * S0);
  return k;
}
template <typename C, int N1, int N2>
static int xi_cand(int* out) {
  constexpr int M = N1 * N2;
  constexpr int ROW = (M + 1 + dfft::SmemSize<N1, N2>::v) * (int)sizeof(C);
  constexpr int KT0 = (40 * 1024) / ROW;
  constexpr int KT = KT0 >= 16 ? 16 : (KT0 >= 8 ? 8 : (KT0 >= 4 ? 4 : 2));
  int k = uniq(out, 0, KT);
  k = uniq(out, k, KT / 2 > 0 ? KT / 2 : 1);
  return uniq(out, k, KT / 4 > 0 ? KT / 4 : 1);
}
template <typename T, int N1, int N2>
static int xf_cand(int* out) {
  constexpr int KT = XFwdSmem<T, N1, N2, 16>::bytes <= 57344 ? 16
                   : (XFwdSmem<T, N1, N2, 8>::bytes <= 57344 ? 8 : 4);
  int k = uniq(out, 0, KT);
  k = uniq(out, k, KT / 2);
  return uniq(out, k, KT / 4 > 0 ? KT / 4 : 1);
}
int fft_tile_candidates(int kind, int n, bool fp32, int* out) {
  int n1, n2;
  if (!factor(n, &n1, &n2)) return 0;
#define X(A, B)                                                                  \
  if (n1 == A && n2 == B) {                                                      \
    if (kind == 0 || kind == 3) return fp32 ? z_cand<float2, A, B>(out) : z_cand<double2, A, B>(out); \
    if (kind == 1) return fp32 ? xi_cand<float2, A, B>(out) : xi_cand<double2, A, B>(out); \
    return fp32 ? xf_cand<float, A, B>(out) : xf_cand<double, A, B>(out);        \
  }
  FFT_SIZE_CASES(X)
#undef X
  return 0;
}

// explicit instantiations used by the host code
template int launch_zinv<double2>(const ZInvArgs<double2>&, int, int, cudaStream_t, int);
template int launch_zinv<float2>(const ZInvArgs<float2>&, int, int, cudaStream_t, int);
template int launch_zfwd<double2, double2, false>(const ZFwdArgs<double2, double2>&, int, int, cudaStream_t, int);
template int launch_zfwd<double2, double2, true>(const ZFwdArgs<double2, double2>&, int, int, cudaStream_t, int);
template int launch_zfwd<float2, float2, true>(const ZFwdArgs<float2, float2>&, int, int, cudaStream_t, int);
template int launch_xinv<double2>(const XInvArgs<double2>&, int, int, int, cudaStream_t, int);
template int launch_xinv<float2>(const XInvArgs<float2>&, int, int, int, cudaStream_t, int);
template int launch_xfwd<double, false>(const XFwdArgs<double>&, int, int, int, cudaStream_t, int);
template int launch_xfwd<double, true>(const XFwdArgs<double>&, int, int, int, cudaStream_t, int);
template int launch_xfwd<float, true>(const XFwdArgs<float>&, int, int, int, cudaStream_t, int);
template int launch_xfwd<float, false>(const XFwdArgs<float>&, int, int, int, cudaStream_t, int);
template int launch_zfwd<float2, double2, false>(const ZFwdArgs<float2, double2>&, int, int, cudaStream_t, int);
