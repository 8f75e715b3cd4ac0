// Host launchers of the reference-layout gather/scatter kernels (defined in
// diablo_gpu.cu next to the kernels) for use from other translation units.
#pragma once
#include <cuda_runtime.h>
#include "kernels_fft.cuh"

// reference physical array (pitch Nx+2, Nz+2 rows) -> internal P[j][k][i]
void launch_ref_to_phys(const double* ref, double* out, int nx, int nz, int nyp2, cudaStream_t s);
// internal Fourier F[j][m][kp] -> significant box of a reference Fourier array
void launch_four_to_ref(const double2* in, double2* ref, const Geom& g, int nxp, cudaStream_t s);
