// Kernel launchers shared between the route's translation units.
#pragma once
#include <cuda_runtime.h>

namespace fdk {
struct Params;
// Precision-form kernel (perturb_f32.cu): orbit32 holds the 32-byte entries
// (zr, zi in f64; zr, zi in f32, NaN where |Z| < 2^-60; r^2 of the 2-step block at m).
cudaError_t launch_f32(const Params &p, const void *orbit32, bool deriv, bool bla, int sm_count, cudaStream_t st,
                       int *blocks_per_sm);
}  // namespace fdk
