// Launchers of the ensemble column step (k_column_step_ens): the column
// step of many members in one persistent launch per rows-per-lane class.
#include "internal.h"
#include "kernels_field.cuh"

// Zero every member's per-group counts (and the unused per-member counter)
// and the launch's task counter: one block per member.
static __global__ void k_ens_zero_sched(const __grid_constant__ EnsColArgs E) {
  const FieldArgs& A = E.mem[blockIdx.x];
  const int ngroup = (A.s.ncol + FS_COLS - 1) / FS_COLS;
  for (int k = threadIdx.x; k < 1 + ngroup; k += blockDim.x) A.sched[SCHED_COUNTER + k] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *E.counter = 0;
}

template <int R>
static int ens_resident() {
  static int cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  int v = __atomic_load_n(&cache[dev], __ATOMIC_ACQUIRE);
  if (v > 0) return v;
  const int smem = (int)field_smem_bytes(32 * R);
  cudaFuncSetAttribute(k_column_step_ens<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  int sms = 0, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_column_step_ens<R>, FS_THREADS, smem);
  v = (per > 0 ? per : 1) * (sms > 0 ? sms : 1);
  __atomic_store_n(&cache[dev], v, __ATOMIC_RELEASE);
  return v;
}

// The systems the ensemble kernel is built for: R = 3 .. 9 rows per lane
// (Ny + 2 <= 288); other members keep the per-member graph branches.
#define ENS_R_CASES(X) X(3) X(4) X(5) X(6) X(7) X(8) X(9)

int column_step_ens_resident(int R) {
  switch (R) {
#define X(r) case r: return ens_resident<r>();
    ENS_R_CASES(X)
#undef X
    default: return 0;
  }
}

int launch_column_step_ens(const EnsColArgs& E, int R, int ntask, cudaStream_t s) {
  if (E.nmem <= 0 || ntask <= 0) return 0;
  k_ens_zero_sched<<<E.nmem, 128, 0, s>>>(E);
  switch (R) {
#define X(r)                                                                                 \
    case r: {                                                                                \
      const int res = ens_resident<r>();                                                     \
      k_column_step_ens<r><<<std::min(ntask, res), FS_THREADS, field_smem_bytes(32 * r), s>>>(E); \
      return 0;                                                                              \
    }
    ENS_R_CASES(X)
#undef X
    default: return DIABLO_ERR_SIZE;
  }
}
