// Allocation-free variant of the plain (FP64) perturbation kernel, for callers that
// cannot allocate device memory: a render service that owns all device memory through
// its own pool or arena (other allocations would fragment it or break its budget) and
// hands the library buffers carved from it. The caller passes the orbit and every
// output column as device pointers; the kernel's own scratch (work-queue head, counters
// and per-row iteration sums) lives in a file-scope device array of fixed size below,
// which every GPU that loads this library keeps until the process exits.
// Built with -fmad=false, like the other plain-form kernels: results are the same bits.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/fdcuda.h"
#include "perturb_f64.cuh"
#include "route_internal.hpp"

namespace {

constexpr unsigned long long SCRATCH_BYTES = FDC_NOALLOC_SCRATCH_BYTES;
constexpr unsigned long long HEADER_BYTES = 256;  // queue head, counters, deadline flag

// Layout: [0] queue head, [8..71] Counters, [72] timed-out flag, [256..] row sums (u64).
static __device__ __align__(256) unsigned char noalloc_scratch[SCRATCH_BYTES];

// Set-up per device: the array's device address, the SM count and the resident blocks
// per kernel variant. `ready` is published after the fields under g_setup, so concurrent
// first calls on one device do the set-up once and every caller sees it complete.
struct PerDevice {
  std::atomic<bool> ready{false};
  unsigned char *scratch = nullptr;
  int sm_count = 0;
  std::atomic<int> blocks_per_sm[4] = {};
};
PerDevice g_devices[64];
std::mutex g_setup;

// Puts the calling thread's current device back on every return.
struct CurrentDevice {
  int prev = -1;
  ~CurrentDevice() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// The checks fdc_open makes (a present sm_100 device), then the scratch array's device
// address with `device` current. Called under g_setup.
fdc_status setup_device(int device, PerDevice &pd, char *error, size_t cap);
// Copies a message into the caller's error buffer (if any) and returns the status.
fdc_status fail(fdc_status s, const std::string &m, char *error, size_t cap) {
  if (error && cap) {
    size_t n = m.size() < cap - 1 ? m.size() : cap - 1;
    std::memcpy(error, m.data(), n);
    error[n] = 0;
  }
  return s;
}

// The plain kernel's persistent loop, plus a per-row sum of the iterations spent.
template <bool EXT, bool D>
__global__ void __launch_bounds__(128) perturb_noalloc_kernel(fdk::Params p, unsigned long long *row_sums) {
  using namespace fdk;
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  State<EXT> s;
  Result res;
  bool active = false, exhausted = false;
  unsigned long long n_samples = 0, iters = 0;
  auto finish = [&](uint32_t idx, const Result &r) {
    put(p, idx, r);
    uint64_t spent = r.kind == 2 ? p.max_iter : r.n;
    iters += spent;
    n_samples += 1;
    atomicAdd(row_sums + (idx / p.nx - p.first_row), (unsigned long long)spent);
  };
  for (;;) {
    unsigned need = __ballot_sync(FULL, !active);
    while (need && !exhausted) {
      unsigned long long base = 0;
      int leader = __ffs((int)need) - 1;
      if ((int)lane == leader) base = atomicAdd(p.queue, (unsigned long long)__popc(need));
      base = __shfl_sync(FULL, base, leader);
      if (base >= p.total) {
        exhausted = true;
        break;
      }
      if (!active) {
        uint64_t slot = base + __popc(need & lt);
        if (slot < p.total) {
          int got = init<EXT, D, false>(p, slot, s, res);
          if (got == 1) active = true;
          else if (got == 2) finish(s.idx, res);
        }
      }
      need = __ballot_sync(FULL, !active);
    }
    if (!__any_sync(FULL, active)) break;
    if (active && step<EXT, D, false>(p, s, res)) {
      finish(s.idx, res);
      active = false;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    n_samples += __shfl_down_sync(FULL, n_samples, o);
    iters += __shfl_down_sync(FULL, iters, o);
  }
  if (lane == 0) {
    atomicAdd(&p.counters->samples, n_samples);
    atomicAdd(&p.counters->iterations, iters);
  }
}

void *noalloc_kernel(bool ext, bool d, int &variant) {
  variant = (ext ? 2 : 0) | (d ? 1 : 0);
  switch (variant) {
    case 0: return (void *)perturb_noalloc_kernel<false, false>;
    case 1: return (void *)perturb_noalloc_kernel<false, true>;
    case 2: return (void *)perturb_noalloc_kernel<true, false>;
    default: return (void *)perturb_noalloc_kernel<true, true>;
  }
}

fdc_status setup_device(int device, PerDevice &pd, char *error, size_t cap) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess)
    return fail(FDC_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e), error, cap);
  if (device >= count)
    return fail(FDC_NO_DEVICE, "no CUDA device " + std::to_string(device) + " (" + std::to_string(count) + " present)",
                error, cap);
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess)
    return fail(FDC_NO_DEVICE, std::string("device properties: ") + cudaGetErrorString(e), error, cap);
  if (prop.major != 10)
    return fail(FDC_NO_DEVICE, "device " + std::to_string(device) + " is sm_" + std::to_string(prop.major) +
                                   std::to_string(prop.minor) + ", not sm_100",
                error, cap);
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e), error, cap);
  void *ptr = nullptr;
  e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
  if (e != cudaSuccess)
    return fail(FDC_DEVICE_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e), error, cap);
  pd.scratch = (unsigned char *)ptr;
  pd.sm_count = prop.multiProcessorCount;
  pd.ready.store(true, std::memory_order_release);
  return FDC_OK;
}

// A device pointer the kernel reads or writes as `align`-byte words must be aligned to it.
bool misaligned(const void *ptr, uintptr_t align) { return ptr && ((uintptr_t)ptr & (align - 1)) != 0; }

}  // namespace

extern "C" fdc_status fdc_render_noalloc(int device, const double *orbit, uint64_t len, const fdc_job *job,
                                         const fdc_out *out, uint64_t *row_iterations, fdc_counters *counters,
                                         void *stream, char *error, size_t error_cap) {
  if (!job || !out || !orbit) return fail(FDC_INVALID, "null argument", error, error_cap);
  if (device < 0 || device >= 64) return fail(FDC_INVALID, "device index out of range", error, error_cap);
  const fdc_job &j = *job;
  if (j.flags & (FDC_BLA | FDC_F32 | FDC_SHIFT | FDC_SERIES))
    return fail(FDC_INVALID, "the allocation-free entry point renders the plain form without BLA or series only", error,
                error_cap);
  if (j.mask || j.offsets) return fail(FDC_INVALID, "the allocation-free entry point takes no mask or offsets", error, error_cap);
  if (len < 3 || len > (1ull << 20)) return fail(FDC_INVALID, "orbit length must be in [3, 2^20]", error, error_cap);
  if (j.nx == 0 || j.ny == 0 || j.ss == 0 || j.nx % j.ss || j.ny % j.ss)
    return fail(FDC_INVALID, "grid must be a non-empty whole number of pixels", error, error_cap);
  if ((uint64_t)j.nx * j.ny >= (1ull << 31)) return fail(FDC_INVALID, "grid larger than 2^31 samples", error, error_cap);
  if (j.tier < 0 || j.tier > 2) return fail(FDC_INVALID, "unknown tier", error, error_cap);
  if (j.max_iter >= (1ull << 32)) return fail(FDC_INVALID, "max_iter must be below 2^32", error, error_cap);
  if (!(j.escape_radius > 0.0) || !std::isfinite(j.escape_radius * j.escape_radius))
    return fail(FDC_INVALID, "escape radius must be positive and its square finite", error, error_cap);
  if (!(j.h_m >= 1.0 && j.h_m < 2.0)) return fail(FDC_INVALID, "h_m must lie in [1, 2)", error, error_cap);
  if (j.h_e < -(1ll << 30) || j.h_e > (1ll << 30))
    return fail(FDC_INVALID, "h_e must lie in [-2^30, 2^30]", error, error_cap);
  if (j.nucleus_period < -1 || j.nucleus_period >= (1ll << 31) - 1)
    return fail(FDC_INVALID, "nucleus_period must be -1 or in [0, 2^31 - 1)", error, error_cap);
  uint32_t first = j.first_row, rows = j.rows ? j.rows : j.ny - j.first_row;
  if (first >= j.ny || rows > j.ny - first) return fail(FDC_INVALID, "row range outside the grid", error, error_cap);
  const uint32_t cols = j.cols ? j.cols : j.nx - j.first_col;
  if (j.first_col >= j.nx || cols > j.nx - j.first_col)
    return fail(FDC_INVALID, "column range outside the grid", error, error_cap);
  if (HEADER_BYTES + 8ull * rows > SCRATCH_BYTES)
    return fail(FDC_INVALID, "job needs " + std::to_string(HEADER_BYTES + 8ull * rows) +
                                 " bytes of scratch; this entry point has " + std::to_string(SCRATCH_BYTES) +
                                 " (at most " + std::to_string((SCRATCH_BYTES - HEADER_BYTES) / 8) +
                                 " rows per call)",
                error, error_cap);
  // The kernel loads the orbit and stores z and dz as 16-byte words, the other columns
  // as words of their own size: a pointer off that boundary would fault on the GPU.
  if (misaligned(orbit, 16)) return fail(FDC_INVALID, "orbit must be 16-byte aligned", error, error_cap);
  const struct {
    const void *ptr;
    uintptr_t align;
    const char *name;
  } columns[] = {{out->z, 16, "z"},  {out->dz, 16, "dz"}, {out->nu, 8, "nu"},        {out->dexp, 8, "dexp"},
                 {out->n, 4, "n"},   {out->de, 4, "de"},  {out->normal, 2, "normal"}};
  for (const auto &c : columns)
    if (misaligned(c.ptr, c.align))
      return fail(FDC_INVALID, std::string("output column ") + c.name + " must be " + std::to_string(c.align) +
                                   "-byte aligned",
                  error, error_cap);
  CurrentDevice current;
  if (cudaGetDevice(&current.prev) != cudaSuccess) current.prev = -1;
  PerDevice &pd = g_devices[device];
  if (!pd.ready.load(std::memory_order_acquire)) {  // set-up, once per device
    std::lock_guard<std::mutex> lock(g_setup);
    if (!pd.ready.load(std::memory_order_relaxed)) {
      fdc_status st = setup_device(device, pd, error, error_cap);
      if (st != FDC_OK) return st;
    }
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("cudaSetDevice: ") + cudaGetErrorString(e), error, error_cap);
  cudaStream_t st = (cudaStream_t)stream;
  const bool ext = j.tier == FDC_TIER_SCALED, deriv = (j.flags & FDC_DERIVATIVE) != 0;
  fdk::Params p{};
  p.orbit = (const double2 *)orbit;
  p.last = (uint32_t)(len - 1);
  p.z0r = 0.0;
  p.z0i = 0.0;
  p.nx = j.nx;
  p.ny = j.ny;
  p.first_row = first;
  p.rows = rows;
  p.first_col = j.first_col;
  p.cols = cols;
  p.in_pitch = cols;
  p.out_pitch = j.nx;
  p.tile_shift = 3;  // 8x4-sample tiles in row-major order
  p.tile_order = nullptr;
  p.tiles_x = (cols + 7) / 8;
  p.tier = j.tier;
  p.flags = deriv ? fdk::F_DERIV : 0;
  p.c_re = j.c_re;
  p.c_im = j.c_im;
  p.h = j.h_m * fdroute::exp2i(j.h_e);
  p.h_m = j.h_m;
  p.h_e = j.h_e;
  p.cosr = j.cos_rot;
  p.sinr = j.sin_rot;
  p.half_x = (double)j.nx / 2.0;
  p.half_y = (double)j.ny / 2.0;
  p.max_iter = j.max_iter;
  p.r2 = j.escape_radius * j.escape_radius;
  p.nucleus = j.nucleus_period;
  p.px_m = j.h_m * (double)j.ss;
  p.px_e = j.h_e;
  const uint64_t b0 = (uint64_t)first * j.nx + j.first_col;  // the window's first sample
  p.cls = out->cls ? out->cls + b0 : nullptr;
  p.n_out = out->n ? out->n + b0 : nullptr;
  p.nu = out->nu ? out->nu + b0 : nullptr;
  p.de = out->de ? out->de + b0 : nullptr;
  p.normal = out->normal ? out->normal + b0 : nullptr;
  p.z_out = out->z ? (double2 *)out->z + b0 : nullptr;
  p.dz_out = out->dz ? (double2 *)out->dz + b0 : nullptr;
  p.dexp_out = out->dexp ? out->dexp + b0 : nullptr;
  p.status = out->status ? out->status + b0 : nullptr;
  p.total = (uint64_t)p.tiles_x * ((rows + 3) / 4) * 32;
  p.queue = (unsigned long long *)pd.scratch;
  p.counters = (fdk::Counters *)(pd.scratch + 8);
  p.timed_out = (uint32_t *)(pd.scratch + 72);
  unsigned long long *row_sums = (unsigned long long *)(pd.scratch + HEADER_BYTES);
  // Every call shares the scratch: clear the header and this call's row sums first.
  e = cudaMemsetAsync(pd.scratch, 0, HEADER_BYTES + 8ull * rows, st);
  if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e), error, error_cap);
  int variant = 0;
  void *fn = noalloc_kernel(ext, deriv, variant);
  int resident = pd.blocks_per_sm[variant].load(std::memory_order_relaxed);
  if (!resident) {  // the same value whichever thread computes it first
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, 128, 0);
    if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("occupancy: ") + cudaGetErrorString(e), error, error_cap);
    resident = b > 0 ? b : 1;
    pd.blocks_per_sm[variant].store(resident, std::memory_order_relaxed);
  }
  void *args[] = {&p, &row_sums};
  e = cudaLaunchKernel(fn, dim3(pd.sm_count * resident), dim3(128), args, 0, st);
  if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("launch: ") + cudaGetErrorString(e), error, error_cap);
  if (row_iterations || counters) {
    unsigned char head[HEADER_BYTES];
    e = cudaMemcpyAsync(head, pd.scratch, HEADER_BYTES, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && row_iterations)
      e = cudaMemcpyAsync(row_iterations, row_sums, 8ull * rows, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(FDC_DEVICE_ERROR, std::string("readback: ") + cudaGetErrorString(e), error, error_cap);
    if (counters) {
      fdk::Counters c;
      std::memcpy(&c, head + 8, sizeof c);
      std::memset(counters, 0, sizeof *counters);
      counters->samples = c.samples;
      counters->iterations = c.iterations;
      counters->launches = 1;
    }
  }
  return FDC_OK;
}
