// Launcher of the precision-form kernel (compiled with fused multiply-adds).
#include <cuda_runtime.h>

#include "launch.hpp"
#include "perturb_f32.cuh"

namespace fdk {

static int per_sm(int occupancy, int cap) { return cap > 0 && cap < occupancy ? cap : occupancy; }

template <bool D, bool L>
static cudaError_t launch_t(const Params &p, const Entry32 *orbit, int sm_count, int cap, cudaStream_t st,
                            int *cache) {
  if (*cache == 0) {
    int b = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, perturb_f32_kernel<D, L>, 128, 0);
    if (e != cudaSuccess) return e;
    *cache = b > 0 ? b : 1;
  }
  perturb_f32_kernel<D, L><<<sm_count * per_sm(*cache, cap), 128, 0, st>>>(p, orbit);
  return cudaGetLastError();
}

cudaError_t launch_f32(const Params &p, const void *orbit32, bool deriv, bool bla, int sm_count, int cap,
                       cudaStream_t st, int *blocks_per_sm) {
  const Entry32 *o = (const Entry32 *)orbit32;
  int v = (deriv ? 2 : 0) | (bla ? 1 : 0);
  switch (v) {
    case 0: return launch_t<false, false>(p, o, sm_count, cap, st, blocks_per_sm + 0);
    case 1: return launch_t<false, true>(p, o, sm_count, cap, st, blocks_per_sm + 1);
    case 2: return launch_t<true, false>(p, o, sm_count, cap, st, blocks_per_sm + 2);
    default: return launch_t<true, true>(p, o, sm_count, cap, st, blocks_per_sm + 3);
  }
}

template <bool D, bool L>
static cudaError_t batch_t(const Params *jobs, const unsigned long long *starts, uint32_t njobs,
                           unsigned long long total, unsigned long long *queue, Counters *per_job, int sm_count,
                           int cap, uint32_t defer, cudaStream_t st, int *cache) {
  if (*cache == 0) {
    int b = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, perturb_f32_batch_kernel<D, L>, 128, 0);
    if (e != cudaSuccess) return e;
    *cache = b > 0 ? b : 1;
  }
  perturb_f32_batch_kernel<D, L>
      <<<sm_count * per_sm(*cache, cap), 128, 0, st>>>(jobs, starts, njobs, total, queue, per_job, defer);
  return cudaGetLastError();
}

cudaError_t launch_f32_batch(const Params *jobs, const unsigned long long *starts, uint32_t njobs,
                             unsigned long long total, unsigned long long *queue, Counters *per_job, bool deriv,
                             bool bla, int sm_count, int cap, uint32_t defer, cudaStream_t st, int *blocks_per_sm) {
  int v = (deriv ? 2 : 0) | (bla ? 1 : 0);
  switch (v) {
    case 0: return batch_t<false, false>(jobs, starts, njobs, total, queue, per_job, sm_count, cap, defer, st, blocks_per_sm + 0);
    case 1: return batch_t<false, true>(jobs, starts, njobs, total, queue, per_job, sm_count, cap, defer, st, blocks_per_sm + 1);
    case 2: return batch_t<true, false>(jobs, starts, njobs, total, queue, per_job, sm_count, cap, defer, st, blocks_per_sm + 2);
    default: return batch_t<true, true>(jobs, starts, njobs, total, queue, per_job, sm_count, cap, defer, st, blocks_per_sm + 3);
  }
}

}  // namespace fdk
