// FP64 / FP32 ALU peak probe for the roofline of the perturbation kernels: independent
// multiply and add chains per thread on every SM, timed with CUDA events. Built with
// -fmad=false, so each multiply and each add is one instruction, the op mix the plain
// form is held to (it may not fuse, for parity with the reference).
#include <cuda_runtime.h>

#include <cstdint>

namespace {

template <class T, int CHAINS, int ITERS>
__global__ void __launch_bounds__(256) alu_chains(T *out, T a, T b) {
  T x[CHAINS];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
  for (int i = 0; i < ITERS; ++i) {
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) {
      x[c] = x[c] * a;
      x[c] = x[c] + b;
    }
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) s += x[c];
  if (s == (T)123.456) out[threadIdx.x] = s;  // keeps the chains live
}

template <class T>
double measure(int device) {
  constexpr int CHAINS = 8, ITERS = 4096;
  cudaDeviceProp prop;
  if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess) return -1;
  T *out = nullptr;
  if (cudaMalloc(&out, 256 * sizeof(T)) != cudaSuccess) return -1;
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, alu_chains<T, CHAINS, ITERS>, 256, 0);
  dim3 grid(prop.multiProcessorCount * (blocks > 0 ? blocks : 1)), block(256);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double best = 0;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    alu_chains<T, CHAINS, ITERS><<<grid, block>>>(out, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    double ops = 2.0 * CHAINS * ITERS * (double)grid.x * block.x;
    if (rep > 0 && ms > 0) best = best > ops / (ms * 1e-3) ? best : ops / (ms * 1e-3);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? best : -1;
}

}  // namespace

// Unfused FP64 and FP32 operations per second (multiplies + adds) on `device`, best of 5
// timed launches; negative on failure.
extern "C" int fdk_alu_peaks(int device, double *fp64_ops, double *fp32_ops) {
  *fp64_ops = measure<double>(device);
  *fp32_ops = measure<float>(device);
  return (*fp64_ops > 0 && *fp32_ops > 0) ? 0 : -1;
}
