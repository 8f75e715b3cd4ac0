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

// ---- z inverse ----
template <typename C, int N1, int N2>
static void launch_zinv_t(const ZInvArgs<C>& a, int nfield, cudaStream_t s) {
  constexpr int S = 128 / N2 > 0 ? 128 / N2 : 1;
  dim3 blk(N2, S), grd((a.nseq + S - 1) / S, nfield);
  k_zinv<C, N1, N2, S><<<grd, blk, 0, s>>>(a);
}
template <typename C>
int launch_zinv(const ZInvArgs<C>& a, int nz, int nfield, cudaStream_t s) {
  int n1, n2;
  if (!factor(nz, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) { launch_zinv_t<C, A, B>(a, nfield, s); return 0; }
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- z forward ----
template <typename C, typename CO, int N1, int N2, bool COMB>
static void launch_zfwd_t(const ZFwdArgs<C, CO>& a, int nfield, cudaStream_t s) {
  constexpr int S = 128 / N2 > 0 ? 128 / N2 : 1;
  dim3 blk(N2, S), grd((a.nseq + S - 1) / S, nfield);
  k_zfwd<C, CO, N1, N2, S, COMB><<<grd, blk, 0, s>>>(a);
}
template <typename C, typename CO, bool COMB>
int launch_zfwd(const ZFwdArgs<C, CO>& a, int nz, int nfield, cudaStream_t s) {
  int n1, n2;
  if (!factor(nz, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) { launch_zfwd_t<C, CO, A, B, COMB>(a, nfield, s); return 0; }
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- x inverse ----
template <typename C, int N1, int N2>
static void launch_xinv_t(const XInvArgs<C>& a, int nplanes, int nfield, cudaStream_t s) {
  constexpr int M = N1 * N2;
  constexpr int ROW = (M + 1 + dfft::SmemSize<N1, N2>::v) * (int)sizeof(C);
  constexpr int KT0 = (40 * 1024) / ROW;
  constexpr int KT = KT0 >= 16 ? 16 : (KT0 >= 8 ? 8 : (KT0 >= 4 ? 4 : 2));
  dim3 blk(N2, KT), grd((a.g.nz + KT - 1) / KT, nplanes, nfield);
  k_xc2r<C, N1, N2, KT><<<grd, blk, 0, s>>>(a);
}
template <typename C>
int launch_xinv(const XInvArgs<C>& a, int m, int nplanes, int nfield, cudaStream_t s) {
  int n1, n2;
  if (!factor(m, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) { launch_xinv_t<C, A, B>(a, nplanes, nfield, s); return 0; }
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}

// ---- x forward ----
template <typename T, int N1, int N2, bool NL>
static void launch_xfwd_t(const XFwdArgs<T>& a, int nplanes, int nfield, cudaStream_t s) {
  // rows per block: as many as fit ~56 KB of shared memory, at most 16
  constexpr int KT = XFwdSmem<T, N1, N2, 16>::bytes <= 57344 ? 16
                   : (XFwdSmem<T, N1, N2, 8>::bytes <= 57344 ? 8 : 4);
  constexpr int SMB = XFwdSmem<T, N1, N2, KT>::bytes;
  cudaFuncSetAttribute(k_xr2c<T, N1, N2, KT, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMB);
  dim3 blk(N2, KT), grd(nfield, (a.g.nz + KT - 1) / KT, nplanes);
  k_xr2c<T, N1, N2, KT, NL><<<grd, blk, SMB, s>>>(a);
}
template <typename T, bool NL>
int launch_xfwd(const XFwdArgs<T>& a, int m, int nplanes, int nfield, cudaStream_t s) {
  int n1, n2;
  if (!factor(m, &n1, &n2)) return DIABLO_ERR_SIZE;
#define X(A, B) if (n1 == A && n2 == B) { launch_xfwd_t<T, A, B, NL>(a, nplanes, nfield, s); return 0; }
  FFT_SIZE_CASES(X)
#undef X
  return DIABLO_ERR_SIZE;
}


// explicit instantiations used by the host code
template int launch_zinv<double2>(const ZInvArgs<double2>&, int, int, cudaStream_t);
template int launch_zinv<float2>(const ZInvArgs<float2>&, int, int, cudaStream_t);
template int launch_zfwd<double2, double2, false>(const ZFwdArgs<double2, double2>&, int, int, cudaStream_t);
template int launch_zfwd<double2, double2, true>(const ZFwdArgs<double2, double2>&, int, int, cudaStream_t);
template int launch_zfwd<float2, float2, true>(const ZFwdArgs<float2, float2>&, int, int, cudaStream_t);
template int launch_xinv<double2>(const XInvArgs<double2>&, int, int, int, cudaStream_t);
template int launch_xinv<float2>(const XInvArgs<float2>&, int, int, int, cudaStream_t);
template int launch_xfwd<double, false>(const XFwdArgs<double>&, int, int, int, cudaStream_t);
template int launch_xfwd<double, true>(const XFwdArgs<double>&, int, int, int, cudaStream_t);
template int launch_xfwd<float, true>(const XFwdArgs<float>&, int, int, int, cudaStream_t);
