// Kernel launchers shared between the route's translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace fdk {
struct Params;
struct Counters;
// Precision-form kernel (perturb_f32.cu): orbit32 holds the 32-byte entries
// (zr, zi in f64; zr, zi in f32, NaN where |Z| < 2^-60; r^2 of the 2-step block at m).
// cap: at most this many blocks per SM (0: the occupancy limit, cached in blocks_per_sm).
cudaError_t launch_f32(const Params &p, const void *orbit32, bool deriv, bool bla, int sm_count, int cap,
                       cudaStream_t st, int *blocks_per_sm);
// Precision-form batch kernel over many jobs (per-job orbit32 in Params).
cudaError_t launch_f32_batch(const Params *jobs, const unsigned long long *starts, uint32_t njobs,
                             unsigned long long total, unsigned long long *queue, Counters *per_job, bool deriv,
                             bool bla, int sm_count, int cap, uint32_t defer, cudaStream_t st, int *blocks_per_sm);
}  // namespace fdk
