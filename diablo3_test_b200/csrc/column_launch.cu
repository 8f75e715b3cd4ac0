// Launchers of the Fourier-space column kernels (k_column_tiles, k_column_solve,
// k_rem_div, k_factor), instantiated per rows-per-lane R.
#include "internal.h"
#include "kernels_solve.cuh"
#include "kernels_solve2.cuh"
#include "kernels_field.cuh"


// ---- column solve ----
template <int R>
static void launch_solve_t(const SolveArgs& a, bool project_only, cudaStream_t s) {
  const int warps = 4;
  dim3 blk(32 * warps), grd((a.ncol + warps - 1) / warps);
  if (project_only) k_rem_div<R><<<grd, blk, 0, s>>>(a);
  else k_column_solve<R><<<grd, blk, 0, s>>>(a);
}
template <int R>
static void launch_tiles_t(const Solve2Args& A, cudaStream_t s) {
  const int smem = (T2_STAGES * A.s.n * T2_PITCH + T2_COLS * 32 * (R | 1)) * (int)sizeof(double2) +
                   (A.mean_split ? 2 * A.s.n * (int)sizeof(double) : 0);
  cudaFuncSetAttribute(k_column_tiles<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  const int ngroups = (A.s.nk2 + T2_COLS - 1) / T2_COLS;
  k_column_tiles<R><<<A.s.nkx1 * ngroups, 32 * T2_COLS, smem, s>>>(A);
}
int launch_tiles(const Solve2Args& A, cudaStream_t s) {
  int R = (A.s.n + 31) / 32;
  if (R < 3) R = 3;
  switch (R) {
#define X(r) case r: launch_tiles_t<r>(A, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

template <int R>
static size_t factor_doubles_t(int nf) { return (size_t)nf * Fac<R>::N * 32; }
template <int R>
static void launch_factor_t(const SolveArgs& a, const double* kc, double* out, int nf, cudaStream_t s) {
  k_factor<R><<<nf, 32, 0, s>>>(a, kc, out);
}
size_t factor_doubles(int n, int nf) {
  switch (rows_per_lane(n)) {
#define X(r) case r: return factor_doubles_t<r>(nf);
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return 0;
  }
}
int launch_factor(const SolveArgs& a, const double* kc, double* out, int nf, cudaStream_t s) {
  switch (rows_per_lane(a.n)) {
#define X(r) case r: launch_factor_t<r>(a, kc, out, nf, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

int launch_solve(const SolveArgs& a, bool project_only, cudaStream_t s) {
  int R = (a.n + 31) / 32;
  if (R < 3) R = 3;
  switch (R) {
#define X(r) case r: launch_solve_t<r>(a, project_only, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}

// ---- field-split column step (kernels_field.cuh) ----
// Both kernels are persistent: as many blocks as fit on the device at once
// (two per SM at Ny = 257), each walking its share of the tasks.  The shared-
// memory attribute and the resident block count are set up once per device
// and instantiation, for the largest system of its R (32 R rows), so a launch
// makes no extra runtime calls beyond cudaGetDevice.
template <typename K>
static int resident_blocks(K kernel, int smem, int* cache) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  int v = __atomic_load_n(&cache[dev], __ATOMIC_ACQUIRE);
  if (v > 0) return v;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int sms = 0, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, FS_THREADS, smem);
  v = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);
  __atomic_store_n(&cache[dev], v, __ATOMIC_RELEASE);
  return v;
}
template <int R>
static void launch_column_step_t(const FieldArgs& A, cudaStream_t s) {
  static int cache[64];
  const int resident = resident_blocks(k_column_step<R>, (int)field_smem_bytes(32 * R), cache);
  const int groups = (A.s.ncol + FS_COLS - 1) / FS_COLS;
  k_column_step<R><<<std::min(groups * (A.nf + 1), resident), FS_THREADS, field_smem_bytes(A.s.n), s>>>(A);
}
template <int R>
static void launch_field_t(const FieldArgs& A, cudaStream_t s) {
  static int cache[64];
  const int resident = resident_blocks(k_field_solve<R>, (int)field_smem_bytes(32 * R), cache);
  const int tasks = ((A.s.ncol + FS_COLS - 1) / FS_COLS) * A.nf;
  k_field_solve<R><<<std::min(tasks, resident), FS_THREADS, field_smem_bytes(A.s.n), s>>>(A);
}
template <int R>
static void launch_project_t(const FieldArgs& A, cudaStream_t s) {
  static int cache[64];
  const int resident = resident_blocks(k_project_cols<R>, (int)field_smem_bytes(32 * R), cache);
  const int groups = (A.s.ncol + FS_COLS - 1) / FS_COLS;
  k_project_cols<R><<<std::min(groups, resident), FS_THREADS, field_smem_bytes(A.s.n), s>>>(A);
}
int launch_field_solve(const FieldArgs& A, cudaStream_t s) {
  switch (rows_per_lane(A.s.n)) {
#define X(r) case r: launch_field_t<r>(A, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}
int launch_project_cols(const FieldArgs& A, cudaStream_t s) {
  switch (rows_per_lane(A.s.n)) {
#define X(r) case r: launch_project_t<r>(A, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}
int column_step_resident(int n) {
  switch (rows_per_lane(n)) {
#define X(r) case r: { static int cache[64]; return resident_blocks(k_column_step<r>, (int)field_smem_bytes(32 * r), cache); }
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return 0;
  }
}
int launch_column_step(const FieldArgs& A, cudaStream_t s) {
  switch (rows_per_lane(A.s.n)) {
#define X(r) case r: launch_column_step_t<r>(A, s); return 0;
    X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}
