// Declarations of the xz-FFT launchers (defined in fft_launch.cu).
#pragma once
#include <cuda_runtime.h>
#include "kernels_fft.cuh"

// supported transform lengths N = N1*N2 (N1, N2 register-DFT sizes)
bool factor(int n, int* n1, int* n2);

// `tile`: 0 = the default tile shape, else one of fft_tile_candidates()
template <typename C>
int launch_zinv(const ZInvArgs<C>& a, int nz, int nfield, cudaStream_t s, int tile = 0);
template <typename C, typename CO, bool COMB>
int launch_zfwd(const ZFwdArgs<C, CO>& a, int nz, int nfield, cudaStream_t s, int tile = 0);
template <typename C>
int launch_xinv(const XInvArgs<C>& a, int m, int nplanes, int nfield, cudaStream_t s, int tile = 0);
template <typename T, bool NL>
int launch_xfwd(const XFwdArgs<T>& a, int m, int nplanes, int nfield, cudaStream_t s, int tile = 0);
// candidate tiles of launcher `kind` (0 z inverse, 1 x inverse, 2 x forward,
// 3 z forward: the step's order) for transform length n; returns their count (at most 3)
int fft_tile_candidates(int kind, int n, bool fp32, int* out);
