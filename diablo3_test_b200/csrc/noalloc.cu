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
// file-scope device arrays that the library image carries, so they exist on
// every GPU that loads libdiablo_gpu.so until the process exits.
//
// Set-up, once per device with that device current (the first call on the
// device): the scratch array's device address is looked up with
// cudaGetSymbolAddress, and the twiddle tables of every supported transform
// length are written into their own device array with cudaMemcpyToSymbol.
// After that a call only queues kernels on the caller's stream.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include <vector>

#include "../../include/diablo_gpu.h"
#include "fft_launch.h"
#include "kernels_fft.cuh"
#include "layout_launch.h"

namespace {

constexpr size_t kScratchBytes = DIABLO_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// Transform lengths the register FFTs support (factor() in fft_launch.cu).
constexpr int kLengths[] = {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256};
constexpr int kNumLengths = sizeof(kLengths) / sizeof(kLengths[0]);
constexpr int sum_lengths() {
  int s = 0;
  for (int i = 0; i < kNumLengths; ++i) s += kLengths[i];
  return s;
}
// Table layout: for each supported L, exp(-2 pi i m / L) for m < L (the z
// and half-length x transforms); then for each L, exp(-2 pi i m / (2L)) for
// m <= L (the r2c split of an x transform of length 2L).
constexpr int kTwiddleEntries = 2 * sum_lengths() + kNumLengths;

// The shared scratch and the twiddle tables.  Host code may not use these
// names as device addresses (on the host they are only stand-in symbols); the
// address of each device's copy comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ __align__(256) double2 g_noalloc_twiddles[kTwiddleEntries];

struct DeviceTables {
  unsigned char* scratch = nullptr;
  double2* twiddles = nullptr;
};
std::mutex g_setup_mutex;
DeviceTables g_tables[kMaxDevices];

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int length_index(int n) {
  for (int i = 0; i < kNumLengths; ++i)
    if (kLengths[i] == n) return i;
  return -1;
}
// offset of the table exp(-2 pi i m / L) (half = false) or of
// exp(-2 pi i m / (2L)) (half = true) for the supported length L = kLengths[i]
int table_offset(int i, bool half) {
  int o = half ? sum_lengths() : 0;
  for (int q = 0; q < i; ++q) o += kLengths[q] + (half ? 1 : 0);
  return o;
}

void fill_twiddles(std::vector<double2>& h) {
  const long double pi = 3.141592653589793238462643383279502884L;
  h.assign(kTwiddleEntries, make_double2(0.0, 0.0));
  for (int i = 0; i < kNumLengths; ++i) {
    const int L = kLengths[i];
    for (int half = 0; half < 2; ++half) {
      const int n = half ? 2 * L : L, count = half ? L + 1 : L;
      double2* out = h.data() + table_offset(i, half != 0);
      for (int m = 0; m < count; ++m) {
        long double ang = 2.0L * pi * (long double)m / (long double)n;
        out[m] = make_double2((double)cosl(ang), (double)-sinl(ang));
      }
    }
  }
}

// Once per device, with that device current: the device addresses of the
// scratch and twiddle arrays, and the twiddle tables themselves.
int setup_device(int dev, DeviceTables* out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  DeviceTables& t = g_tables[dev];
  if (!t.scratch) {
    void* s = nullptr;
    void* w = nullptr;
    if (cudaGetSymbolAddress(&s, g_noalloc_scratch) != cudaSuccess || !s ||
        cudaGetSymbolAddress(&w, g_noalloc_twiddles) != cudaSuccess || !w) {
      cudaGetLastError();
      return DIABLO_ERR_CUDA;
    }
    std::vector<double2> h;
    fill_twiddles(h);
    if (cudaMemcpyToSymbol(g_noalloc_twiddles, h.data(), h.size() * sizeof(double2)) != cudaSuccess) {
      cudaGetLastError();
      return DIABLO_ERR_CUDA;
    }
    t.twiddles = (double2*)w;
    t.scratch = (unsigned char*)s;
  }
  *out = t;
  return 0;
}

// v and vv must be device (or managed) memory of the current device
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (at.type == cudaMemoryTypeDevice && at.device == dev) || at.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int diablo_fft_xz_to_fourier_noalloc(int nx, int ny, int nz, const double* v, double* vv,
                                                void* stream) {
  if (!v || !vv || nx < 8 || (nx % 2) || ny < 4 || nz < 8) return DIABLO_ERR_ARG;
  const int M = nx / 2;
  const int iz = length_index(nz), im = length_index(M);
  if (iz < 0 || im < 0) return DIABLO_ERR_SIZE;
  // scratch need: internal physical, x-spectral and Fourier arrays
  const int nyp2 = ny + 2, nkx1 = nx / 3 + 1, nkz = nz / 3, nk2 = 2 * nkz + 1;
  const size_t b_ph = align256(sizeof(double) * (size_t)nyp2 * nz * nx);
  const size_t b_xs = align256(sizeof(double2) * (size_t)nyp2 * nkx1 * nz);
  const size_t b_fo = align256(sizeof(double2) * (size_t)nyp2 * nkx1 * nk2);
  if (b_ph + b_xs + b_fo > kScratchBytes) return DIABLO_ERR_SIZE;
  // an error left pending by earlier work stays the caller's: nothing is queued
  if (cudaPeekAtLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DIABLO_ERR_CUDA;
  }
  if (!on_device(v, dev) || !on_device(vv, dev)) return DIABLO_ERR_ARG;
  DeviceTables t;
  int rc = setup_device(dev, &t);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const Geom g{nx, nz, nyp2, nkx1, nkz, nk2, nk2};
  const double2* tz = t.twiddles + table_offset(iz, false);
  const double2* tm = t.twiddles + table_offset(im, false);
  const double2* tx = t.twiddles + table_offset(im, true);
  double* phys = (double*)t.scratch;
  double2* xs = (double2*)(t.scratch + b_ph);
  double2* four = (double2*)(t.scratch + b_ph + b_xs);
  // every scratch region is written in full below before it is read, so
  // nothing left by an earlier call leaks into this one
  launch_ref_to_phys(v, phys, nx, nz, nyp2, s);
  if (cudaGetLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
  XFwdArgs<double> xa = {};
  xa.in[0] = phys;
  xa.outA[0] = xs;
  xa.j0 = 0;
  xa.g = g;
  xa.twM = tm;
  xa.twX = tx;
  xa.scale = 1.0 / nx;
  rc = launch_xfwd<double, false>(xa, M, nyp2, 1, s);
  if (rc) return rc;
  if (cudaGetLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
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
  if (cudaGetLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
  launch_four_to_ref(four, (double2*)vv, g, M, s);
  if (cudaGetLastError() != cudaSuccess) return DIABLO_ERR_CUDA;
  return 0;
}
