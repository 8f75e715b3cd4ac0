// diablo_fft_xz_to_fourier_noalloc: the FP64 forward xz transform for callers
// that must not allocate device memory.
//
// Who cannot allocate: a Fortran or C driver that hands the library a
// preallocated device buffer pool (its own allocator owns every byte, and a
// hidden cudaMalloc would break its accounting or exceed its budget); code
// that runs between other work on a stream and cannot accept the device-wide
// synchronisation a cudaMalloc/cudaFree can cause; and callers that have not
// created (and will not create) a diablo_ctx, whose creation allocates the
// whole step state.  This entry point uses no context: its scratch lives in
// one file-scope device array that the library image carries, so it exists on
// every GPU that loads libdiablo_gpu.so until the process exits.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>

#include "../../include/diablo_gpu.h"
#include "fft_launch.h"
#include "kernels_fft.cuh"
#include "layout_launch.h"

namespace {

constexpr size_t kScratchBytes = DIABLO_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The shared scratch.  Host code may not use this name as a device address
// (on the host it is only a stand-in symbol); the address of each device's
// copy comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {nullptr};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Twiddle table exp(-2 pi i m / n), m < count, into `out` (host stack memory).
void twiddles(int n, int count, double2* out) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < count; ++m) {
    long double ang = 2.0L * pi * (long double)m / (long double)n;
    out[m] = make_double2((double)cosl(ang), (double)-sinl(ang));
  }
}

}  // namespace

extern "C" int diablo_fft_xz_to_fourier_noalloc(int nx, int ny, int nz, const double* v, double* vv,
                                                void* stream) {
  if (!v || !vv || nx < 8 || (nx % 2) || ny < 4 || nz < 8) return DIABLO_ERR_ARG;
  int a1, a2;
  if (!factor(nz, &a1, &a2) || !factor(nx / 2, &a1, &a2)) return DIABLO_ERR_SIZE;
  if (nz > 256 || nx / 2 > 256) return DIABLO_ERR_SIZE;
  cudaStream_t s = (cudaStream_t)stream;
  // set-up, once per device, with that device current
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DIABLO_ERR_CUDA;
  }
  unsigned char* base;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return DIABLO_ERR_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    base = (unsigned char*)g_scratch_addr[dev];
  }
  // carve the scratch: twiddles, internal physical, x-spectral, Fourier
  const int nyp2 = ny + 2, M = nx / 2, nkx1 = nx / 3 + 1, nkz = nz / 3, nk2 = 2 * nkz + 1;
  const Geom g{nx, nz, nyp2, nkx1, nkz, nk2, nk2};
  const size_t b_tz = align256(sizeof(double2) * nz);
  const size_t b_tm = align256(sizeof(double2) * M);
  const size_t b_tx = align256(sizeof(double2) * (M + 1));
  const size_t b_ph = align256(sizeof(double) * (size_t)nyp2 * nz * nx);
  const size_t b_xs = align256(sizeof(double2) * (size_t)nyp2 * nkx1 * nz);
  const size_t b_fo = align256(sizeof(double2) * (size_t)nyp2 * nkx1 * nk2);
  if (b_tz + b_tm + b_tx + b_ph + b_xs + b_fo > kScratchBytes) return DIABLO_ERR_SIZE;
  double2* tz = (double2*)base;
  double2* tm = (double2*)(base + b_tz);
  double2* tx = (double2*)(base + b_tz + b_tm);
  double* phys = (double*)(base + b_tz + b_tm + b_tx);
  double2* xs = (double2*)(base + b_tz + b_tm + b_tx + b_ph);
  double2* four = (double2*)(base + b_tz + b_tm + b_tx + b_ph + b_xs);
  // every scratch region is written in full below before it is read, so
  // nothing left by an earlier call leaks into this one
  double2 htw[256 + 256 + 257];
  twiddles(nz, nz, htw);
  twiddles(M, M, htw + nz);
  twiddles(nx, M + 1, htw + nz + M);
  if (cudaMemcpyAsync(tz, htw, sizeof(double2) * nz, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(tm, htw + nz, sizeof(double2) * M, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(tx, htw + nz + M, sizeof(double2) * (M + 1), cudaMemcpyHostToDevice, s) != cudaSuccess) {
    cudaGetLastError();
    return DIABLO_ERR_CUDA;
  }
  launch_ref_to_phys(v, phys, nx, nz, nyp2, s);
  XFwdArgs<double> xa = {};
  xa.in[0] = phys;
  xa.outA[0] = xs;
  xa.j0 = 0;
  xa.g = g;
  xa.twM = tm;
  xa.twX = tx;
  xa.scale = 1.0 / nx;
  int rc = launch_xfwd<double, false>(xa, M, nyp2, 1, s);
  if (rc) return rc;
  ZFwdArgs<double2, double2> za = {};
  za.srcA[0] = xs;
  za.dst[0] = four;
  za.q0 = 0;
  za.nseq = nyp2 * nkx1;
  za.g = g;
  za.tw = tz;
  za.scale = 1.0 / nz;
  rc = launch_zfwd<double2, double2, false>(za, nz, 1, s);
  if (rc) return rc;
  launch_four_to_ref(four, (double2*)vv, g, nx / 2, s);
  if (cudaGetLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
  return 0;
}
