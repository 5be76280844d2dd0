// C ABI of the CUDA perturbation route (include/fdcuda.h): contexts, orbit/BLA
// uploads, and fdc_render, which launches the persistent perturbation kernel.
// Built with -fmad=false (the plain form must round as the reference's Rust does).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/fdcuda.h"
#include "launch.hpp"
#include "bla_build.cuh"
#include "perturb_f64.cuh"
#include "route_internal.hpp"

namespace {

struct BlaDev {
  double *fused = nullptr;  // (zr, zi, r2 of the 2-step block at m, r2 of the 4-step block at m)
  double *r2 = nullptr;
  double2 *coef = nullptr;
  double2 *ab = nullptr;
  uint64_t points = 0, blocks = 0;  // sizes of the buffers above: fused 32 B per point; 8, 32, 16 B per block
  uint32_t levels = 0;
  uint32_t off[fdk::MAX_LEVELS] = {};
  uint32_t count[fdk::MAX_LEVELS] = {};
  double eps = 0, dc_max = 0;
  int64_t dc_exp = 0;
};

struct OrbitDev {
  double2 *z = nullptr;
  double *z32 = nullptr;  // precision-form entries, 4 doubles per point (launch.hpp)
  uint64_t len = 0;
  uint32_t bits = 0;
  double z0r = 0, z0i = 0;
  bool has_bla = false;
  BlaDev bla;
  // parameter-series start (fdc_upload_series): b_1..b_order in SERIES_SLOTS device entries
  bool has_series = false;
  uint32_t series_n = 0, series_order = 0;
  double series_rho = 0.0, series_inv = 0.0;
  double2 *series_b = nullptr;
  double *q = nullptr;  // error radii of the orbit's points (fdc_upload_error_radius), len entries
  uint32_t batch_refs = 0;  // live batches whose jobs read this orbit and its table
};

constexpr uint32_t SERIES_SLOTS = 64;  // SeriesConfig::default().max_order (series.rs:45)

// Device scratch of one context: work-queue head, counters, deadline flag.
struct Scratch {
  unsigned long long queue;
  unsigned long long pad[3];
  fdk::Counters counters;
  uint32_t timed_out;
  uint32_t bad;  // fdc_upload_bla's value checks
  uint32_t pad2[6];
};

class CopyPool;  // host threads of the staging copies (below)

}  // namespace

struct fdc_batch;

struct fdc_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Scratch *scratch = nullptr;
  std::map<int32_t, OrbitDev> orbits;
  int32_t next_orbit = 1;
  std::string err;
  // staging for host outputs / inputs, grown on demand
  void *stage = nullptr;
  size_t stage_bytes = 0;
  int blocks_per_sm[21] = {};
  int blocks_per_sm_f32[4] = {};
  int blocks_per_sm_batch[8] = {};
  int blocks_per_sm_batch_f32[4] = {};
  fdc_tuning tune{FDC_DEFAULT_DEFER, 0, 0, 0};
  // Device buffers of freed orbits and tables (and upload staging), kept by size for the
  // next upload of the same size: a film or a service re-uploading per frame allocates
  // once. Stream-ordered: every user runs on `stream`. Freed by fdc_close.
  std::multimap<size_t, void *> pool;
  // pinned staging for large host<->device copies: two chunk slots, each with the event
  // of the last transfer that used it
  char *pinned = nullptr;
  cudaEvent_t slot_ev[2] = {nullptr, nullptr};
  std::unique_ptr<CopyPool> copier;  // host threads of the staging copies
  // centre-first tile orders per window shape (tiles_x, tiles_y, tile_shift)
  std::map<std::tuple<uint32_t, uint32_t, uint32_t>, uint32_t *> orders;
};

// Persistent grid of a plain-form kernel: the occupancy limit, or fewer blocks per SM
// when the tuning asks for fewer.
// Lanes a warp gathers before applying BLA blocks (fdc_tuning.defer; 0: per variant).
static uint32_t defer_for(const fdc_ctx *ctx, bool ext) {
  if (ctx->tune.defer > 0) return ctx->tune.defer;
  return ext ? 12u : 8u;
}

// The tiles of a window, nearest to its centre first (squared distance of the tile's
// centre, ties in row-major order). Benchmark views and zoom films centre on a nucleus,
// whose surroundings hold the longest samples: handing those out first leaves the cheap
// border for the end of the launch, where warps run out of work.
static const uint32_t *centre_first(fdc_ctx *ctx, uint32_t tiles_x, uint32_t tiles_y, uint32_t shift) {
  auto key = std::make_tuple(tiles_x, tiles_y, shift);
  auto it = ctx->orders.find(key);
  if (it != ctx->orders.end()) return it->second;
  const uint64_t n = (uint64_t)tiles_x * tiles_y;
  const double tw = (double)(1u << shift), th = (double)(32u >> shift);
  std::vector<double> d(n);
  for (uint64_t t = 0; t < n; ++t) {
    const double x = ((double)(t % tiles_x) + 0.5) * tw - 0.5 * tiles_x * tw;
    const double y = ((double)(t / tiles_x) + 0.5) * th - 0.5 * tiles_y * th;
    d[t] = x * x + y * y;
  }
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return d[a] < d[b]; });
  uint32_t *dev = nullptr;
  if (cudaMalloc(&dev, n * sizeof(uint32_t)) != cudaSuccess) return nullptr;
  if (cudaMemcpy(dev, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(dev);
    return nullptr;
  }
  ctx->orders[key] = dev;
  return dev;
}

static int grid_blocks(const fdc_ctx *ctx, int occupancy) {
  int b = occupancy;
  if (ctx->tune.blocks_per_sm > 0 && (int)ctx->tune.blocks_per_sm < b) b = (int)ctx->tune.blocks_per_sm;
  return ctx->sm_count * b;
}

// A prepared batch (include/fdcuda.h): jobs grouped by kernel variant, each group's Params
// array and slot starts in device memory, per-job counters, and a CUDA graph of the
// whole run (clear queues and counters, one persistent launch per group).
struct fdc_batch {
  struct Group {
    bool f32, ext, deriv, bla;
    bool encode = false;      // BLA group with columns to encode after its kernel
    uint64_t max_window = 0;  // samples of its largest job window
    std::vector<uint32_t> order;  // original job index of each position
    fdk::Params *jobs = nullptr;
    unsigned long long *starts = nullptr;
    unsigned long long total = 0;
    uint32_t counter_base = 0;
  };
  std::vector<Group> groups;
  std::vector<int32_t> orbits;  // distinct orbit handles of the jobs, each holding a reference
  uint32_t njobs = 0;
  fdk::Counters *counters = nullptr;   // njobs, in group order
  unsigned long long *queues = nullptr;  // one per group
  void *raw = nullptr;  // raw-state scratch of BLA jobs the caller gave no z / dz / ... column
  size_t raw_bytes = 0;  // (from the context's pool, returned to it by fdc_batch_free)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

fdc_status fail(fdc_ctx *c, fdc_status s, const std::string &msg) {
  if (c) c->err = msg;
  return s;
}

// An f64 as Rust's Display prints the values a refusal message names: the shortest
// decimal that reads back to the same double, without a trailing ".0", NaN as "NaN".
std::string rust_f64(double x) {
  if (std::isnan(x)) return "NaN";
  if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
  char buf[64];
  for (int digits = 1; digits <= 17; ++digits) {
    std::snprintf(buf, sizeof buf, "%.*g", digits, x);
    if (std::strtod(buf, nullptr) == x) break;
  }
  return buf;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(ctx, FDC_DEVICE_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

void *pool_get(fdc_ctx *ctx, size_t bytes) {
  if (bytes == 0) return nullptr;
  auto it = ctx->pool.find(bytes);
  if (it != ctx->pool.end()) {
    void *p = it->second;
    ctx->pool.erase(it);
    return p;
  }
  void *p = nullptr;
  return cudaMalloc(&p, bytes) == cudaSuccess ? p : nullptr;
}

void pool_put(fdc_ctx *ctx, void *p, size_t bytes) {
  if (p && bytes) ctx->pool.emplace(bytes, p);
}

void free_bla(fdc_ctx *ctx, BlaDev &b) {
  pool_put(ctx, b.fused, 32 * b.points);
  pool_put(ctx, b.r2, 8 * b.blocks);
  pool_put(ctx, b.coef, 32 * b.blocks);
  pool_put(ctx, b.ab, 16 * b.blocks);
  b = BlaDev{};
}

void free_orbit_buffers(fdc_ctx *ctx, OrbitDev &o) {
  pool_put(ctx, o.z, 16 * o.len);
  pool_put(ctx, o.z32, 32 * o.len);
  free_bla(ctx, o.bla);
  pool_put(ctx, o.series_b, 16 * SERIES_SLOTS);
  pool_put(ctx, o.q, 8 * o.len);
  o.z = nullptr;
  o.z32 = nullptr;
  o.series_b = nullptr;
  o.has_series = false;
  o.q = nullptr;
}

// Orbit layouts built on the device from the caller's SoA (re[], im[]): interleaved
// double2 points, and the precision form's 32-byte entries (zr, zi f64; zr, zi f32 in one
// word, NaN where |Z| < 2^-60, whose steps take the exact path; r^2 of the 2-step block
// at m, -1 until a table is uploaded).
__global__ void pack_orbit(const double *__restrict__ re, const double *__restrict__ im, uint64_t len,
                           double2 *__restrict__ z, double *__restrict__ z32) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < len; k += (uint64_t)gridDim.x * blockDim.x) {
    const double x = re[k], y = im[k];
    z[k] = make_double2(x, y);
    float fr = __double2float_rn(x);
    const float fi = __double2float_rn(y);
    if (fmax(fabs(x), fabs(y)) < 0x1p-60) fr = __int_as_float(0x7fc00000);
    double *e = z32 + 4 * k;
    e[0] = x;
    e[1] = y;
    e[2] = __longlong_as_double((long long)(((unsigned long long)__float_as_uint(fi) << 32) | __float_as_uint(fr)));
    e[3] = -1.0;
  }
}

// Table of the export form ([f64; 7] per block: a.re, a.im, b.re, b.im, r, alpha, beta)
// split into r^2, (a, b) and (alpha, beta); bad |= 1 for a non-finite value, 2 for a
// negative radius (Bla::new's value checks, bla.rs:184-216).
__global__ void pack_bla(const double *__restrict__ b7, uint64_t total, double *__restrict__ r2,
                         double2 *__restrict__ coef, double2 *__restrict__ ab, unsigned *bad) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const double *v = b7 + 7 * k;
    double w[7];
    bool finite = true;
    for (int f = 0; f < 7; ++f) {
      w[f] = v[f];
      finite = finite && isfinite(w[f]);
    }
    if (!finite) atomicOr(bad, 1u);
    if (w[4] < 0.0) atomicOr(bad, 2u);
    r2[k] = w[4] * w[4];
    coef[2 * k] = make_double2(w[0], w[1]);
    coef[2 * k + 1] = make_double2(w[2], w[3]);
    ab[k] = make_double2(w[5], w[6]);
  }
}

// The fused stream: point m with the squared radii of the level-0 and level-1 blocks
// starting at Z_m (block t of level i starts at m = 1 + t 2^(i+1), bla.rs:131-135), -1
// where none starts; the level-0 radius also goes into the precision-form entries.
__global__ void fuse_bla(const double2 *__restrict__ z, uint64_t len, const double *__restrict__ r2, uint32_t levels,
                         uint64_t off0, uint64_t cnt0, uint64_t off1, uint64_t cnt1, double *__restrict__ fused,
                         double *__restrict__ z32) {
  for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < len; m += (uint64_t)gridDim.x * blockDim.x) {
    const double2 p = z[m];
    double a = -1.0, b = -1.0;
    if (m >= 1 && levels > 0 && ((m - 1) & 1) == 0 && ((m - 1) >> 1) < cnt0) a = r2[off0 + ((m - 1) >> 1)];
    if (m >= 1 && levels > 1 && ((m - 1) & 3) == 0 && ((m - 1) >> 2) < cnt1) b = r2[off1 + ((m - 1) >> 2)];
    double *f = fused + 4 * m;
    f[0] = p.x;
    f[1] = p.y;
    f[2] = a;
    f[3] = b;
    z32[4 * m + 3] = a;
  }
}

unsigned grid_for(uint64_t n) { return (unsigned)std::min<uint64_t>((n + 255) / 256, 148 * 16); }

template <bool EXT, bool D, bool L, bool S = false, bool B = false, bool T = false>
void *kernel_ptr() {
  return (void *)fdk::perturb_kernel<EXT, D, L, S, B, T>;
}

// series: a job starting from an admitted series (ordinary tiers only): variants 8-11;
// bounded: the bounded variant (ordinary tiers, derivative, no BLA or series): 12;
// stripe: the Stripe recorder (no series, not bounded): 13-20
void *pick_kernel(bool ext, bool d, bool l, bool series, bool bounded, int &variant, bool stripe = false) {
  if (bounded) {
    variant = 12;
    return kernel_ptr<false, true, false, false, true>();
  }
  if (stripe) {
    variant = 13 + ((ext ? 4 : 0) | (d ? 2 : 0) | (l ? 1 : 0));
    switch (variant - 13) {
      case 0: return kernel_ptr<false, false, false, false, false, true>();
      case 1: return kernel_ptr<false, false, true, false, false, true>();
      case 2: return kernel_ptr<false, true, false, false, false, true>();
      case 3: return kernel_ptr<false, true, true, false, false, true>();
      case 4: return kernel_ptr<true, false, false, false, false, true>();
      case 5: return kernel_ptr<true, false, true, false, false, true>();
      case 6: return kernel_ptr<true, true, false, false, false, true>();
      default: return kernel_ptr<true, true, true, false, false, true>();
    }
  }
  variant = (ext ? 4 : 0) | (d ? 2 : 0) | (l ? 1 : 0);
  if (series && !ext) {
    variant += 8;
    switch (variant) {
      case 8: return kernel_ptr<false, false, false, true>();
      case 9: return kernel_ptr<false, false, true, true>();
      case 10: return kernel_ptr<false, true, false, true>();
      default: return kernel_ptr<false, true, true, true>();
    }
  }
  switch (variant) {
    case 0: return kernel_ptr<false, false, false>();
    case 1: return kernel_ptr<false, false, true>();
    case 2: return kernel_ptr<false, true, false>();
    case 3: return kernel_ptr<false, true, true>();
    case 4: return kernel_ptr<true, false, false>();
    case 5: return kernel_ptr<true, false, true>();
    case 6: return kernel_ptr<true, true, false>();
    default: return kernel_ptr<true, true, true>();
  }
}

void *pick_batch_kernel(bool ext, bool d, bool l, int &variant) {
  variant = (ext ? 4 : 0) | (d ? 2 : 0) | (l ? 1 : 0);
  switch (variant) {
    case 0: return (void *)fdk::perturb_batch_kernel<false, false, false>;
    case 1: return (void *)fdk::perturb_batch_kernel<false, false, true>;
    case 2: return (void *)fdk::perturb_batch_kernel<false, true, false>;
    case 3: return (void *)fdk::perturb_batch_kernel<false, true, true>;
    case 4: return (void *)fdk::perturb_batch_kernel<true, false, false>;
    case 5: return (void *)fdk::perturb_batch_kernel<true, false, true>;
    case 6: return (void *)fdk::perturb_batch_kernel<true, true, false>;
    default: return (void *)fdk::perturb_batch_kernel<true, true, true>;
  }
}

void free_batch(fdc_batch *b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &g : b->groups) {
    cudaFree(g.jobs);
    cudaFree(g.starts);
  }
  cudaFree(b->counters);
  cudaFree(b->queues);
  cudaFree(b->raw);
  delete b;
}

fdc_status open_resources(fdc_ctx *ctx) {
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&ctx->ev0));
  CK(cudaEventCreate(&ctx->ev1));
  CK(cudaMalloc(&ctx->scratch, sizeof(Scratch)));
  CK(cudaEventCreateWithFlags(&ctx->slot_ev[0], cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&ctx->slot_ev[1], cudaEventDisableTiming));
  return FDC_OK;
}

// Large copies between the caller's (pageable) host arrays and the device go through two
// pinned chunk slots: the host side of chunk k is copied by several threads while the DMA
// of chunk k - 1 runs, and the DMA itself runs at pinned speed. Copies below STAGE_MIN go
// direct. A chunk is a quarter of the copy, between STAGE_MIN and CHUNK, so that even a
// mid-size array overlaps its two sides.
constexpr size_t CHUNK = 8u << 20;
constexpr size_t STAGE_MIN = 1u << 20;

size_t chunk_for(size_t bytes) {
  const size_t quarter = ((bytes / 4) + 65535) & ~(size_t)65535;
  return std::min(CHUNK, std::max(STAGE_MIN, quarter));
}

// Persistent host threads for the staging copies (created once per context instead of per
// chunk): a copy is cut into equal parts; the calling thread copies the last, the workers
// the others, and copy() returns when all are done.
class CopyPool {
 public:
  explicit CopyPool(unsigned workers) {
    try {
      for (unsigned i = 0; i < workers; ++i) threads_.emplace_back([this, i] { run(i); });
    } catch (...) {  // fewer threads than asked: the copies are cut into fewer parts
    }
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> l(m_);
      stop_ = true;
    }
    go_.notify_all();
    for (auto &t : threads_) t.join();
  }
  void copy(void *dst, const void *src, size_t bytes) {
    const size_t workers = threads_.size();
    if (workers == 0 || bytes < (256u << 10)) {
      std::memcpy(dst, src, bytes);
      return;
    }
    {
      std::lock_guard<std::mutex> l(m_);
      dst_ = (char *)dst;
      src_ = (const char *)src;
      bytes_ = bytes;
      part_ = ((bytes / (workers + 1)) + 63) & ~(size_t)63;
      pending_ = workers;
      ++gen_;
    }
    go_.notify_all();
    piece(workers);
    std::unique_lock<std::mutex> l(m_);
    done_.wait(l, [&] { return pending_ == 0; });
  }

 private:
  // part k of the current copy; its fields were set under the lock before the workers
  // were woken and stay until every part is done
  void piece(size_t k) {
    const size_t a = std::min(bytes_, k * part_), b = std::min(bytes_, a + part_);
    if (b > a) std::memcpy(dst_ + a, src_ + a, b - a);
  }
  void run(unsigned id) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> l(m_);
        go_.wait(l, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
      }
      piece(id);
      std::lock_guard<std::mutex> l(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex m_;
  std::condition_variable go_, done_;
  uint64_t gen_ = 0;
  size_t pending_ = 0;
  bool stop_ = false;
  char *dst_ = nullptr;
  const char *src_ = nullptr;
  size_t bytes_ = 0, part_ = 0;
};

cudaError_t ensure_pinned(fdc_ctx *ctx) {
  if (!ctx->copier) {
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    ctx->copier = std::make_unique<CopyPool>(hw - 1);
  }
  if (ctx->pinned) return cudaSuccess;
  return cudaHostAlloc((void **)&ctx->pinned, 2 * CHUNK, cudaHostAllocDefault);
}

cudaError_t upload(fdc_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (bytes < STAGE_MIN) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  cudaError_t e = ensure_pinned(ctx);
  const size_t chunk = chunk_for(bytes);
  int slot = 0;
  for (size_t off = 0; e == cudaSuccess && off < bytes; off += chunk, slot ^= 1) {
    const size_t n = std::min(chunk, bytes - off);
    char *stage = ctx->pinned + slot * CHUNK;
    e = cudaEventSynchronize(ctx->slot_ev[slot]);  // the DMA that last read this slot is done
    if (e != cudaSuccess) break;
    ctx->copier->copy(stage, (const char *)src + off, n);
    e = cudaMemcpyAsync((char *)dst + off, stage, n, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->slot_ev[slot], ctx->stream);
  }
  return e;
}

cudaError_t download(fdc_ctx *ctx, void *dst, const void *src, size_t bytes) {
  if (bytes < STAGE_MIN) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  cudaError_t e = ensure_pinned(ctx);
  const size_t chunk = chunk_for(bytes);
  const size_t chunks = (bytes + chunk - 1) / chunk;
  auto issue = [&](size_t k) {
    const size_t off = k * chunk, n = std::min(chunk, bytes - off);
    cudaError_t r = cudaMemcpyAsync(ctx->pinned + (k & 1) * CHUNK, (const char *)src + off, n,
                                    cudaMemcpyDeviceToHost, ctx->stream);
    return r == cudaSuccess ? cudaEventRecord(ctx->slot_ev[k & 1], ctx->stream) : r;
  };
  if (e == cudaSuccess) e = issue(0);
  for (size_t k = 0; e == cudaSuccess && k < chunks; ++k) {
    e = cudaEventSynchronize(ctx->slot_ev[k & 1]);  // chunk k has arrived
    if (e == cudaSuccess && k + 1 < chunks) e = issue(k + 1);  // the other slot is free: its copy-out is done
    if (e != cudaSuccess) break;
    const size_t off = k * chunk;
    ctx->copier->copy((char *)dst + off, ctx->pinned + (k & 1) * CHUNK, std::min(chunk, bytes - off));
  }
  return e;
}

// Validate a job against its orbit (the refusals of render_bla, grid.rs:378-413) and fill
// the per-job part of the kernel parameters (everything but outputs, queue, counters).
fdc_status prepare(fdc_ctx *ctx, const OrbitDev &o, const fdc_job &j, fdk::Params &p, uint32_t &first,
                   uint32_t &rows) {
  if (j.nx == 0 || j.ny == 0) return fail(ctx, FDC_INVALID, "empty sample grid");
  if (j.ss == 0 || j.nx % j.ss || j.ny % j.ss) return fail(ctx, FDC_INVALID, "grid must be a whole number of pixels");
  if ((uint64_t)j.nx * j.ny >= (1ull << 31)) return fail(ctx, FDC_INVALID, "grid larger than 2^31 samples");
  if (j.tier < 0 || j.tier > 2) return fail(ctx, FDC_INVALID, "unknown tier");
  if (j.max_iter >= (1ull << 32)) return fail(ctx, FDC_INVALID, "max_iter must be below 2^32");
  if (!(j.escape_radius > 0.0) || !std::isfinite(j.escape_radius * j.escape_radius))
    return fail(ctx, FDC_INVALID, "escape radius must be positive and its square finite");
  if (!(j.h_m >= 1.0 && j.h_m < 2.0)) return fail(ctx, FDC_INVALID, "h_m must lie in [1, 2)");
  if (j.h_e < -(1ll << 30) || j.h_e > (1ll << 30)) return fail(ctx, FDC_INVALID, "h_e must lie in [-2^30, 2^30]");
  if (j.nucleus_period < -1 || j.nucleus_period >= (1ll << 31) - 1)
    return fail(ctx, FDC_INVALID, "nucleus_period must be -1 or in [0, 2^31 - 1)");
  first = j.first_row;
  rows = j.rows ? j.rows : j.ny - j.first_row;
  if (first >= j.ny || rows > j.ny - first) return fail(ctx, FDC_INVALID, "row range outside the grid");
  const uint32_t cols = j.cols ? j.cols : j.nx - j.first_col;
  if (j.first_col >= j.nx || cols > j.nx - j.first_col) return fail(ctx, FDC_INVALID, "column range outside the grid");
  const bool ext = j.tier == FDC_TIER_SCALED;
  // The scaled tier's exact-range step from Z_0 continues at Z_1 (sample.rs:430-447),
  // which needs a next point after it.
  if (ext && o.len < 3) return fail(ctx, FDC_INVALID, "the scaled tier needs an orbit of at least 3 points");
  const bool bla = (j.flags & FDC_BLA) != 0;
  const bool deriv = (j.flags & FDC_DERIVATIVE) != 0;
  const bool series = (j.flags & FDC_SERIES) != 0;
  double h = j.h_m * fdroute::exp2i(j.h_e);
  // Largest unit offset: the grid's corner (grid.rs:428-444), or the supplied offsets'.
  auto largest_offset = [&]() {
    double half = std::hypot((double)j.nx / 2.0, (double)j.ny / 2.0);
    if (j.offsets) {
      half = 0.0;
      const uint64_t lo = 2ull * first * j.nx, hi = 2ull * (first + rows) * j.nx;
      for (uint64_t k = lo; k < hi; k += 2) half = std::max(half, std::hypot(j.offsets[k], j.offsets[k + 1]));
    }
    return half;
  };
  if (series) {  // Series::render_masked's refusals (grid.rs:341-366)
    if (!o.has_series) return fail(ctx, FDC_INVALID, "FDC_SERIES without an uploaded series");
    if (ext) return fail(ctx, FDC_INVALID, "a series start needs f64 deltas: not on the scaled tier");
    if (j.flags & FDC_F32) return fail(ctx, FDC_INVALID, "a series start runs on the plain form only");
    const double dc = h * largest_offset();
    if (std::isnan(dc) || dc > o.series_rho) return fail(ctx, FDC_INVALID, "view reaches |dc| beyond the series radius");
  }
  if (bla) {
    if (!o.has_bla) return fail(ctx, FDC_INVALID, "FDC_BLA without an uploaded BLA table");
    // grid.rs:392-411
    if (std::isnan(j.escape_radius) || j.escape_radius < 4.0)
      return fail(ctx, FDC_INVALID,
                  "escape radius " + rust_f64(j.escape_radius) +
                      " is below 4: BLA blocks may only skip iterates with |z| <= 2 (1 + 2 eps), which needs escape "
                      "radius >= 4");
    const double half = largest_offset();
    double dc = ext ? j.h_m * half : h * half;
    int64_t e = ext ? j.h_e : 0;
    bool over = e == o.bla.dc_exp ? dc > o.bla.dc_max
                                  : std::log2(dc) + (double)e > std::log2(o.bla.dc_max) + (double)o.bla.dc_exp;
    if (std::isnan(dc) || over) return fail(ctx, FDC_INVALID, "view reaches |dc| beyond the BLA table's dc_max");
  }
  p.orbit = o.z;
  p.last = (uint32_t)(o.len - 1);
  p.z0r = o.z0r;
  p.z0i = o.z0i;
  if (bla) {
    p.fused = (const double2 *)o.bla.fused;
    p.bla_r2 = o.bla.r2;
    p.bla_coef = o.bla.coef;
    p.bla_ab = o.bla.ab;
    p.bla_levels = o.bla.levels;
    std::memcpy(p.bla_off, o.bla.off, sizeof p.bla_off);
    std::memcpy(p.bla_count, o.bla.count, sizeof p.bla_count);
  }
  if (series && o.series_n > 0) {  // n = 0: no admitted prefix, the plain kernel (grid.rs:491)
    p.series_b = o.series_b;
    p.series_order = o.series_order;
    p.series_n = o.series_n;
    p.series_inv = o.series_inv;
  }
  p.nx = j.nx;
  p.ny = j.ny;
  p.first_row = first;
  p.rows = rows;
  p.tile_shift = ctx->tune.tile_w ? (uint32_t)__builtin_ctz(ctx->tune.tile_w) : 3u;
  p.first_col = j.first_col;
  p.cols = cols;
  p.in_pitch = cols;  // mask and offsets are staged as the window
  p.out_pitch = j.nx;
  p.tiles_x = (cols + (1u << p.tile_shift) - 1) >> p.tile_shift;
  p.tier = j.tier;
  p.flags = (deriv ? fdk::F_DERIV : 0) | (bla ? fdk::F_BLA : 0) | ((j.flags & FDC_SHIFT) ? fdk::F_SHIFT : 0);
  p.c_re = j.c_re;
  p.c_im = j.c_im;
  p.h = h;
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
  const uint32_t tile_h = 32u >> p.tile_shift;
  const uint32_t tiles_y = (rows + tile_h - 1) / tile_h;
  p.total = (uint64_t)p.tiles_x * tiles_y * 32;
  p.tile_order = nullptr;
  if (ctx->tune.order != FDC_ORDER_ROWS) {
    p.tile_order = centre_first(ctx, p.tiles_x, tiles_y, p.tile_shift);
    if (!p.tile_order) return fail(ctx, FDC_DEVICE_ERROR, "device memory for the tile order");
  }
  p.deadline_ns = j.deadline_ms > 0 ? (uint64_t)(j.deadline_ms * 1e6) : 0;
  p.defer = defer_for(ctx, p.tier == FDC_TIER_SCALED);

  p.orbit32 = o.z32;
  return FDC_OK;
}

}  // namespace

extern "C" {

int fdc_abi_version(void) { return FDC_ABI_VERSION; }

const char *fdc_last_error(const fdc_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

fdc_status fdc_open(int device, fdc_ctx **out) {
  if (!out) return FDC_INVALID;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return FDC_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return FDC_NO_DEVICE;
  fdc_ctx *ctx = new fdc_ctx;
  ctx->device = device;
  ctx->sm_count = prop.multiProcessorCount;
  fdc_status s = open_resources(ctx);
  if (s != FDC_OK) {
    fdc_close(ctx);
    return s;
  }
  *out = ctx;
  return FDC_OK;
}

void fdc_close(fdc_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &kv : ctx->orbits) free_orbit_buffers(ctx, kv.second);
  for (auto &kv : ctx->pool) cudaFree(kv.second);
  ctx->pool.clear();
  for (auto &kv : ctx->orders) cudaFree(kv.second);
  ctx->orders.clear();
  ctx->copier.reset();
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  for (auto &ev : ctx->slot_ev)
    if (ev) cudaEventDestroy(ev);
  cudaFree(ctx->scratch);
  cudaFree(ctx->stage);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

fdc_status fdc_upload_orbit(fdc_ctx *ctx, const double *re, const double *im, uint64_t len, uint32_t bits,
                            int32_t *orbit) {
  if (!ctx || !re || !im || !orbit) return fail(ctx, FDC_INVALID, "null argument");
  if (len < 2 || len > (1ull << 20)) return fail(ctx, FDC_INVALID, "orbit length must be in [2, 2^20]");
  if (re[0] != 0.0 || im[0] != 0.0)
    return fail(ctx, FDC_INVALID, "supplied reference orbit must start at Z_0 = 0");
  CK(cudaSetDevice(ctx->device));
  OrbitDev o;
  o.len = len;
  o.bits = bits;
  o.z0r = re[0];
  o.z0i = im[0];
  o.z = (double2 *)pool_get(ctx, 16 * len);
  o.z32 = (double *)pool_get(ctx, 32 * len);
  double *raw = (double *)pool_get(ctx, 16 * len);  // re[], im[] as the caller holds them
  if (!o.z || !o.z32 || !raw) {
    pool_put(ctx, raw, 16 * len);
    free_orbit_buffers(ctx, o);
    return fail(ctx, FDC_DEVICE_ERROR, "device memory for the orbit");
  }
  cudaError_t e = upload(ctx, raw, re, 8 * len);
  if (e == cudaSuccess) e = upload(ctx, raw + len, im, 8 * len);
  if (e == cudaSuccess) {
    pack_orbit<<<grid_for(len), 256, 0, ctx->stream>>>(raw, raw + len, len, o.z, o.z32);
    e = cudaGetLastError();
  }
  pool_put(ctx, raw, 16 * len);  // stream-ordered: the next user of it runs after the pack
  // the caller's arrays may be freed once this returns, pinned ones included
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    free_orbit_buffers(ctx, o);
    return fail(ctx, FDC_DEVICE_ERROR, std::string("orbit upload: ") + cudaGetErrorString(e));
  }
  int32_t id = ctx->next_orbit++;
  ctx->orbits[id] = o;
  *orbit = id;
  return FDC_OK;
}

fdc_status fdc_free_orbit(fdc_ctx *ctx, int32_t orbit) {
  if (!ctx) return FDC_INVALID;
  auto it = ctx->orbits.find(orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  if (it->second.batch_refs)
    return fail(ctx, FDC_INVALID, "orbit is read by a live batch: free the batch first");
  free_orbit_buffers(ctx, it->second);  // to the pool: later uploads reuse them in stream order
  ctx->orbits.erase(it);
  return FDC_OK;
}

fdc_status fdc_upload_bla(fdc_ctx *ctx, int32_t orbit, const double *blocks7, const uint64_t *level_offsets,
                          uint32_t levels, double eps, double dc_max, int64_t dc_exp) {
  if (!ctx) return FDC_INVALID;
  auto it = ctx->orbits.find(orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  OrbitDev &o = it->second;
  if (o.batch_refs) return fail(ctx, FDC_INVALID, "orbit is read by a live batch: free the batch first");
  // bla.rs:26-33 and Bla::new's shape/value checks (bla.rs:184-216)
  if (!(eps > 0.0 && eps <= 1.0 / (double)(1u << 24) && dc_max > 0.0 && std::isfinite(dc_max)))
    return fail(ctx, FDC_INVALID, "BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0");
  if (levels >= (uint32_t)fdk::MAX_LEVELS) return fail(ctx, FDC_INVALID, "too many BLA levels");
  if (levels > 0 && (!blocks7 || !level_offsets)) return fail(ctx, FDC_INVALID, "null BLA arrays");
  uint64_t steps = o.len >= 2 ? o.len - 2 : 0;
  uint64_t total = 0;
  for (uint32_t i = 0; i < levels; ++i) {
    if (level_offsets[i] != total)
      return fail(ctx, FDC_INVALID, "BLA level offsets must be contiguous and level-major");
    total += steps >> (i + 1);
  }
  CK(cudaSetDevice(ctx->device));
  BlaDev d;
  d.levels = levels;
  d.eps = eps;
  d.dc_max = dc_max;
  d.dc_exp = dc_exp;
  d.points = o.len;
  d.blocks = total;
  for (uint32_t i = 0; i < levels; ++i) {
    d.off[i] = (uint32_t)level_offsets[i];
    d.count[i] = (uint32_t)(steps >> (i + 1));
  }
  d.fused = (double *)pool_get(ctx, 32 * o.len);
  d.r2 = (double *)pool_get(ctx, 8 * total);
  d.coef = (double2 *)pool_get(ctx, 32 * total);
  d.ab = (double2 *)pool_get(ctx, 16 * total);
  double *raw = (double *)pool_get(ctx, 56 * total);  // the export form as the caller holds it
  if (!d.fused || (total && (!d.r2 || !d.coef || !d.ab || !raw))) {
    pool_put(ctx, raw, 56 * total);
    free_bla(ctx, d);
    return fail(ctx, FDC_DEVICE_ERROR, "device memory for the BLA table");
  }
  // split and check the table first; only a valid table touches the orbit's entries
  unsigned *bad = &ctx->scratch->bad;
  cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(unsigned), ctx->stream);
  if (e == cudaSuccess && total) e = upload(ctx, raw, blocks7, 56 * total);
  if (e == cudaSuccess && total) {
    pack_bla<<<grid_for(total), 256, 0, ctx->stream>>>(raw, total, d.r2, d.coef, d.ab, bad);
    e = cudaGetLastError();
  }
  pool_put(ctx, raw, 56 * total);
  unsigned flags = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&flags, bad, sizeof flags, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess || flags) {
    free_bla(ctx, d);
    if (e != cudaSuccess) return fail(ctx, FDC_DEVICE_ERROR, std::string("BLA upload: ") + cudaGetErrorString(e));
    return fail(ctx, FDC_INVALID, (flags & 1) ? "BLA level holds a non-finite value"
                                              : "BLA level holds a negative radius");
  }
  fuse_bla<<<grid_for(o.len), 256, 0, ctx->stream>>>(o.z, o.len, d.r2, levels, levels > 0 ? d.off[0] : 0,
                                                     levels > 0 ? d.count[0] : 0, levels > 1 ? d.off[1] : 0,
                                                     levels > 1 ? d.count[1] : 0, d.fused, o.z32);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    free_bla(ctx, d);
    return fail(ctx, FDC_DEVICE_ERROR, std::string("BLA upload: ") + cudaGetErrorString(e));
  }
  free_bla(ctx, o.bla);
  o.bla = d;
  o.has_bla = true;
  return FDC_OK;
}

// The table built on the device over the uploaded orbit (Bla::build_scaled, bla.rs:161-216):
// every possible level is queued at once (bla_level skips a level after one without a
// valid block), one read of the level flags gives the kept levels, and the table then takes
// the upload's path (pack_bla's value checks, fuse_bla). export7: optional host copy of
// the kept levels in the export form.
fdc_status fdc_build_bla(fdc_ctx *ctx, int32_t orbit, double eps, double dc_max, int64_t dc_exp, uint32_t *levels,
                         double *export7) {
  if (!ctx) return FDC_INVALID;
  auto it = ctx->orbits.find(orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  OrbitDev &o = it->second;
  if (o.batch_refs) return fail(ctx, FDC_INVALID, "orbit is read by a live batch: free the batch first");
  if (!(eps > 0.0 && eps <= 1.0 / (double)(1u << 24) && dc_max > 0.0 && std::isfinite(dc_max)))
    return fail(ctx, FDC_INVALID, "BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0");
  CK(cudaSetDevice(ctx->device));
  const uint64_t steps = o.len >= 2 ? o.len - 2 : 0;
  uint64_t size[fdk::MAX_LEVELS] = {}, at[fdk::MAX_LEVELS] = {}, room = 0;
  uint32_t built = 0;  // levels with at least one block (orbits of at most 2^20 points: <= 19)
  for (uint64_t n = steps / 2; n > 0 && built < (uint32_t)fdk::MAX_LEVELS; n /= 2) {
    at[built] = room;
    size[built++] = n;
    room += n;
  }
  const size_t flag_bytes = 256;
  char *buf = (char *)pool_get(ctx, flag_bytes + 56 * room);
  if (!buf) return fail(ctx, FDC_DEVICE_ERROR, "device memory for the BLA build");
  unsigned *valid = (unsigned *)buf;
  double *raw = (double *)(buf + flag_bytes);
  cudaError_t e = cudaMemsetAsync(valid, 0, flag_bytes, ctx->stream);
  for (uint32_t i = 0; e == cudaSuccess && i < built; ++i) {
    fdk::bla_level<<<grid_for(size[i]), 256, 0, ctx->stream>>>(
        o.z, i > 0 ? raw + 7 * at[i - 1] : nullptr, size[i], i, eps, dc_max, dc_exp, raw + 7 * at[i], valid);
    e = cudaGetLastError();
  }
  unsigned flags[fdk::MAX_LEVELS] = {};
  if (e == cudaSuccess) e = cudaMemcpyAsync(flags, valid, sizeof flags, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    pool_put(ctx, buf, flag_bytes + 56 * room);
    return fail(ctx, FDC_DEVICE_ERROR, std::string("BLA build: ") + cudaGetErrorString(e));
  }
  uint32_t kept = 0;
  while (kept < built && flags[kept]) ++kept;
  if (kept >= (uint32_t)fdk::MAX_LEVELS) {
    pool_put(ctx, buf, flag_bytes + 56 * room);
    return fail(ctx, FDC_INVALID, "too many BLA levels");
  }
  const uint64_t total = kept ? at[kept - 1] + size[kept - 1] : 0;
  BlaDev d;
  d.levels = kept;
  d.eps = eps;
  d.dc_max = dc_max;
  d.dc_exp = dc_exp;
  d.points = o.len;
  d.blocks = total;
  for (uint32_t i = 0; i < kept; ++i) {
    d.off[i] = (uint32_t)at[i];
    d.count[i] = (uint32_t)size[i];
  }
  d.fused = (double *)pool_get(ctx, 32 * o.len);
  d.r2 = (double *)pool_get(ctx, 8 * total);
  d.coef = (double2 *)pool_get(ctx, 32 * total);
  d.ab = (double2 *)pool_get(ctx, 16 * total);
  if (!d.fused || (total && (!d.r2 || !d.coef || !d.ab))) {
    pool_put(ctx, buf, flag_bytes + 56 * room);
    free_bla(ctx, d);
    return fail(ctx, FDC_DEVICE_ERROR, "device memory for the BLA table");
  }
  unsigned *bad = &ctx->scratch->bad;
  e = cudaMemsetAsync(bad, 0, sizeof(unsigned), ctx->stream);
  if (e == cudaSuccess && total) {
    pack_bla<<<grid_for(total), 256, 0, ctx->stream>>>(raw, total, d.r2, d.coef, d.ab, bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && export7 && total) e = download(ctx, export7, raw, 56 * total);
  unsigned badf = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&badf, bad, sizeof badf, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  pool_put(ctx, buf, flag_bytes + 56 * room);
  if (e != cudaSuccess || badf) {
    free_bla(ctx, d);
    if (e != cudaSuccess) return fail(ctx, FDC_DEVICE_ERROR, std::string("BLA build: ") + cudaGetErrorString(e));
    return fail(ctx, FDC_INVALID, (badf & 1) ? "BLA level holds a non-finite value"
                                             : "BLA level holds a negative radius");
  }
  fuse_bla<<<grid_for(o.len), 256, 0, ctx->stream>>>(o.z, o.len, d.r2, kept, kept > 0 ? d.off[0] : 0,
                                                     kept > 0 ? d.count[0] : 0, kept > 1 ? d.off[1] : 0,
                                                     kept > 1 ? d.count[1] : 0, d.fused, o.z32);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    free_bla(ctx, d);
    return fail(ctx, FDC_DEVICE_ERROR, std::string("BLA build: ") + cudaGetErrorString(e));
  }
  free_bla(ctx, o.bla);
  o.bla = d;
  o.has_bla = true;
  if (levels) *levels = kept;
  return FDC_OK;
}

fdc_status fdc_upload_series(fdc_ctx *ctx, int32_t orbit, uint64_t points, uint64_t n, double rho,
                             const double *coeffs, uint32_t order) {
  if (!ctx) return FDC_INVALID;
  auto it = ctx->orbits.find(orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  OrbitDev &o = it->second;
  if (points != o.len) return fail(ctx, FDC_INVALID, "series built over another orbit");  // grid.rs:353-355
  if (order > SERIES_SLOTS) return fail(ctx, FDC_INVALID, "series order above 64");
  if (n > 0) {
    if (n + 1 >= o.len) return fail(ctx, FDC_INVALID, "series start at or past the orbit's last point");
    if (order == 0 || !coeffs) return fail(ctx, FDC_INVALID, "series start without coefficients");
    if (!(rho > 0.0 && std::isfinite(rho))) return fail(ctx, FDC_INVALID, "series radius must be positive and finite");
  }
  CK(cudaSetDevice(ctx->device));
  if (!o.series_b) {
    o.series_b = (double2 *)pool_get(ctx, 16 * SERIES_SLOTS);
    if (!o.series_b) return fail(ctx, FDC_DEVICE_ERROR, "device memory for the series");
  }
  cudaError_t e = cudaSuccess;
  if (n > 0) e = cudaMemcpyAsync(o.series_b, coeffs, 16ull * order, cudaMemcpyHostToDevice, ctx->stream);
  // the caller's array may be freed once this returns
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return fail(ctx, FDC_DEVICE_ERROR, std::string("series upload: ") + cudaGetErrorString(e));
  o.has_series = true;
  o.series_n = (uint32_t)n;
  o.series_order = n > 0 ? order : 0;
  o.series_rho = rho;
  o.series_inv = 1.0 / rho;  // series.rs:250
  return FDC_OK;
}

}  // extern "C"

namespace {

// fdc_render, fdc_render_bounded and fdc_render_stripe: bout (the Bound column and raw
// radii) is null but for the second; with it, ordinary-tier jobs run the bounded variant
// (derivative on). stripe (with its column stripe_out) is null but for the third.
fdc_status render_impl(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, const fdc_bound_out *bout,
                       fdc_counters *counters, const fdc_stripe *stripe = nullptr, float *stripe_out = nullptr) {
  if (!ctx || !job || !out) return fail(ctx, FDC_INVALID, "null argument");
  auto it = ctx->orbits.find(job->orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  const OrbitDev &o = it->second;
  const fdc_job &j = *job;
  fdk::Params p{};
  uint32_t first = 0, rows = 0;
  fdc_status ps = prepare(ctx, o, j, p, first, rows);
  if (ps != FDC_OK) return ps;
  const bool ext = j.tier == FDC_TIER_SCALED;
  const bool bla = (j.flags & FDC_BLA) != 0;
  // Bounded renders (grid.rs:379-384, 588-593): every step certified, so no BLA blocks, no
  // series start and the plain form; the scaled tier has no radii and renders as usual
  // (Bound column 0, heuristic evidence).
  const bool bounded = bout != nullptr && !ext;
  if (bout) {
    if (bla) return fail(ctx, FDC_INVALID, "--columns bound certifies every step; BLA remainders are not certified (ACC-02)");
    if (j.flags & (FDC_SERIES | FDC_F32)) return fail(ctx, FDC_INVALID, "a bounded render runs the plain form from Z_0");
    if (bounded && !o.q) return fail(ctx, FDC_INVALID, "bounded render without uploaded error radii");
  }
  if (bounded) {
    p.q = o.q;
    p.flags |= fdk::F_DERIV;
  }
  if (stripe) {  // grid.rs:783-788; the route's own declines after
    if (stripe->window < 1 || stripe->window > 64 || !std::isfinite(stripe->freq))
      return fail(ctx, FDC_INVALID, "stripe window must be 1..=64 and the frequency finite");
    if (j.flags & (FDC_SERIES | FDC_F32))
      return fail(ctx, FDC_DECLINED, "the Stripe column renders on the plain form from Z_0 only");
    p.stripe_window = stripe->window;
    p.stripe_freq = stripe->freq;
  }
  const bool deriv = (j.flags & FDC_DERIVATIVE) != 0 || bounded;
  CK(cudaSetDevice(ctx->device));
  // the window: rows x cols samples; outputs and inputs of full frame rows (pitch nx),
  // staged as the window (pitch cols)
  const uint64_t n_rows = (uint64_t)rows * p.cols;
  const bool dev_out = (j.flags & FDC_DEVICE_OUT) != 0;
  const bool full = p.cols == j.nx;
  const uint64_t origin = (uint64_t)first * j.nx + p.first_col;
  auto window_copy = [&](void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                         cudaMemcpyKind kind) {
    if (full)
      return kind == cudaMemcpyHostToDevice ? upload(ctx, dst, src, width * rows) : download(ctx, dst, src, width * rows);
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, kind, ctx->stream);
  };

  // Device buffers: caller's (FDC_DEVICE_OUT) or staging for the rendered rows.
  constexpr int NCOL = 13;
  struct Col {
    void *host;
    size_t width;
  } cols[NCOL] = {{out->cls, 1}, {out->n, 4}, {out->nu, 8}, {out->de, 4}, {out->normal, 2},
                  {out->z, 16}, {out->dz, 16}, {out->dexp, 8}, {out->status, 1},
                  {bout ? bout->bound : nullptr, 4}, {bout ? bout->ez : nullptr, 8}, {bout ? bout->ed : nullptr, 8},
                  {stripe ? stripe_out : nullptr, 4}};
  // The BLA kernels of both forms outside the bounded and stripe variants store finished
  // samples' raw state and encode_kernel computes nu / de / normal from it afterwards:
  // class, count, status, z, dz/dc and its exponent must all exist, as scratch where the
  // caller asked for none (never copied back; at the outputs' pitch).
  const bool encode_later = !bounded && !stripe && bla;
  bool scratch[NCOL] = {};
  if (encode_later)
    for (int c : {0, 1, 5, 6, 7, 8}) scratch[c] = cols[c].host == nullptr;
  const uint64_t scratch_rows = (uint64_t)rows * (dev_out ? j.nx : p.cols);
  size_t need = 0;
  size_t offs[NCOL + 2];
  for (int c = 0; c < NCOL; ++c) {
    offs[c] = need;
    if (scratch[c]) need += (scratch_rows * cols[c].width + 255) & ~(size_t)255;
    else if (cols[c].host && !dev_out) need += (n_rows * cols[c].width + 255) & ~(size_t)255;
  }
  offs[NCOL] = need;  // mask
  if (j.mask) need += (n_rows + 255) & ~(size_t)255;
  offs[NCOL + 1] = need;  // offsets
  if (j.offsets) need += (n_rows * 16 + 255) & ~(size_t)255;
  if (need > ctx->stage_bytes) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    CK(cudaMalloc(&ctx->stage, need));
    ctx->stage_bytes = need;
  }
  char *stage = (char *)ctx->stage;
  void *dptr[NCOL];
  for (int c = 0; c < NCOL; ++c) {
    if (scratch[c]) dptr[c] = stage + offs[c];
    else if (!cols[c].host) dptr[c] = nullptr;
    else if (dev_out) dptr[c] = (char *)cols[c].host + origin * cols[c].width;
    else dptr[c] = stage + offs[c];
  }
  p.cls = (uint8_t *)dptr[0];
  p.n_out = (uint32_t *)dptr[1];
  p.nu = (double *)dptr[2];
  p.de = (float *)dptr[3];
  p.normal = (uint16_t *)dptr[4];
  p.z_out = (double2 *)dptr[5];
  p.dz_out = (double2 *)dptr[6];
  p.dexp_out = (int64_t *)dptr[7];
  p.status = (uint8_t *)dptr[8];
  p.bound_out = (float *)dptr[9];
  p.ez_out = (double *)dptr[10];
  p.ed_out = (double *)dptr[11];
  p.stripe_out = (float *)dptr[12];
  p.out_pitch = dev_out ? j.nx : p.cols;
  if (j.mask) {
    p.mask = (const uint8_t *)(stage + offs[NCOL]);
    CK(window_copy(stage + offs[NCOL], p.cols, j.mask + origin, j.nx, p.cols, cudaMemcpyHostToDevice));
  }
  if (j.offsets) {
    p.offsets = (const double2 *)(stage + offs[NCOL + 1]);
    CK(window_copy(stage + offs[NCOL + 1], p.cols * 16ull, j.offsets + 2 * origin, j.nx * 16ull, p.cols * 16ull,
                   cudaMemcpyHostToDevice));
  }
  // Samples that are never reached keep zeroed columns and status 0.
  for (int c = 0; c < NCOL; ++c) {
    if (!dptr[c]) continue;
    const size_t w = cols[c].width;
    if (scratch[c])
      CK(cudaMemsetAsync(dptr[c], 0, scratch_rows * w, ctx->stream));
    else if (!dev_out || full)
      CK(cudaMemsetAsync(dptr[c], 0, n_rows * w, ctx->stream));
    else
      CK(cudaMemset2DAsync(dptr[c], j.nx * w, 0, p.cols * w, rows, ctx->stream));
  }
  p.queue = &ctx->scratch->queue;
  p.counters = &ctx->scratch->counters;
  p.timed_out = &ctx->scratch->timed_out;
  CK(cudaMemsetAsync(ctx->scratch, 0, sizeof(Scratch), ctx->stream));

  uint32_t launches = 1;
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  if (j.flags & FDC_F32) {
    CK(fdk::launch_f32(p, o.z32, deriv, bla, ctx->sm_count, (int)ctx->tune.blocks_per_sm, ctx->stream,
                       ctx->blocks_per_sm_f32));
    if (encode_later && (p.nu || p.de || p.normal)) {
      fdk::encode_kernel<0><<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(p);
      CK(cudaGetLastError());
      launches += 1;
    }
  } else {
    int variant = 0;
    void *fn = pick_kernel(ext, deriv, bla, p.series_n > 0, bounded, variant, stripe != nullptr);
    if (!ctx->blocks_per_sm[variant]) {
      int b = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, 128, 0));
      ctx->blocks_per_sm[variant] = b > 0 ? b : 1;
    }
    dim3 grid(grid_blocks(ctx, ctx->blocks_per_sm[variant])), block(128);
    void *args[] = {&p};
    CK(cudaLaunchKernel(fn, grid, block, args, 0, ctx->stream));
    CK(cudaGetLastError());
    if (encode_later && (p.nu || p.de || p.normal)) {
      fdk::encode_kernel<0><<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(p);
      CK(cudaGetLastError());
      launches += 1;
    }
  }
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  if (!dev_out) {
    for (int c = 0; c < NCOL; ++c)
      if (cols[c].host) {
        const size_t w = cols[c].width;
        CK(window_copy((char *)cols[c].host + origin * w, j.nx * w, dptr[c], p.cols * w, p.cols * w,
                       cudaMemcpyDeviceToHost));
      }
  }
  Scratch sc;
  CK(cudaMemcpyAsync(&sc, ctx->scratch, sizeof sc, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (counters) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    counters->samples = sc.counters.samples;
    counters->iterations = sc.counters.iterations;
    counters->blocks = sc.counters.blocks;
    counters->skipped = sc.counters.skipped;
    counters->fallback_samples = sc.counters.fallback;
    counters->closed_form_samples = sc.counters.closed;
    double sh;
    std::memcpy(&sh, &sc.counters.shift_bits, 8);
    counters->shift = sh;
    counters->kernel_ms = ms;
    counters->launches = launches;
  }
  if (sc.timed_out) return fail(ctx, FDC_TIMEOUT, "deadline passed; unfinished samples have status 0");
  return FDC_OK;
}

}  // namespace

extern "C" {

fdc_status fdc_render(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, fdc_counters *counters) {
  return render_impl(ctx, job, out, nullptr, counters);
}

fdc_status fdc_render_bounded(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, const fdc_bound_out *bound,
                              fdc_counters *counters) {
  if (!bound) return fail(ctx, FDC_INVALID, "null argument");
  return render_impl(ctx, job, out, bound, counters);
}

fdc_status fdc_render_stripe(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, const fdc_stripe *stripe,
                             float *stripe_out, fdc_counters *counters) {
  if (!stripe || !stripe_out) return fail(ctx, FDC_INVALID, "null argument");
  return render_impl(ctx, job, out, nullptr, counters, stripe, stripe_out);
}

fdc_status fdc_upload_error_radius(fdc_ctx *ctx, int32_t orbit, const double *q, uint64_t len) {
  if (!ctx) return FDC_INVALID;
  auto it = ctx->orbits.find(orbit);
  if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "unknown orbit handle");
  OrbitDev &o = it->second;
  if (len != o.len || !q) return fail(ctx, FDC_INVALID, "error radii must cover the orbit's points");
  for (uint64_t m = 0; m < len; ++m)
    if (!(q[m] >= 0.0)) return fail(ctx, FDC_INVALID, "error radii must be non-negative");
  CK(cudaSetDevice(ctx->device));
  if (!o.q) {
    o.q = (double *)pool_get(ctx, 8 * o.len);
    if (!o.q) return fail(ctx, FDC_DEVICE_ERROR, "device memory for the error radii");
  }
  cudaError_t e = upload(ctx, o.q, q, 8 * len);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // the caller's array may go after return
  if (e != cudaSuccess) return fail(ctx, FDC_DEVICE_ERROR, std::string("error radii upload: ") + cudaGetErrorString(e));
  return FDC_OK;
}

fdc_status fdc_set_tuning(fdc_ctx *ctx, const fdc_tuning *t) {
  if (!ctx || !t) return fail(ctx, FDC_INVALID, "null argument");
  if (t->defer > 32) return fail(ctx, FDC_INVALID, "defer must be in [0, 32]");
  if (t->blocks_per_sm > 64) return fail(ctx, FDC_INVALID, "blocks_per_sm must be at most 64");
  if (t->tile_w > 32 || (t->tile_w & (t->tile_w - 1)))
    return fail(ctx, FDC_INVALID, "tile_w must be 0 or a power of two up to 32");
  if (t->order > FDC_ORDER_CENTRE) return fail(ctx, FDC_INVALID, "unknown tile order");
  ctx->tune = *t;
  return FDC_OK;
}

fdc_status fdc_get_tuning(const fdc_ctx *ctx, fdc_tuning *t) {
  if (!ctx || !t) return FDC_INVALID;
  *t = ctx->tune;
  return FDC_OK;
}

fdc_status fdc_batch_create(fdc_ctx *ctx, const fdc_job *jobs, const fdc_out *outs, uint32_t njobs,
                            fdc_batch **out) {
  if (!ctx || !jobs || !outs || !out || njobs == 0) return fail(ctx, FDC_INVALID, "null argument or empty batch");
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  std::vector<fdk::Params> params(njobs);
  std::vector<int> key(njobs);
  for (uint32_t k = 0; k < njobs; ++k) {
    const fdc_job &j = jobs[k];
    auto it = ctx->orbits.find(j.orbit);
    if (it == ctx->orbits.end()) return fail(ctx, FDC_INVALID, "job " + std::to_string(k) + ": unknown orbit handle");
    if (!(j.flags & FDC_DEVICE_OUT)) return fail(ctx, FDC_INVALID, "batch jobs write device outputs (FDC_DEVICE_OUT)");
    if (j.mask || j.offsets || j.deadline_ms > 0)
      return fail(ctx, FDC_INVALID, "batch jobs take no mask, offsets or deadline");
    if (j.flags & FDC_SERIES) return fail(ctx, FDC_INVALID, "batch jobs start at Z_0 (no FDC_SERIES)");
    uint32_t first = 0, rows = 0;
    fdc_status st = prepare(ctx, it->second, j, params[k], first, rows);
    if (st != FDC_OK) {
      ctx->err = "job " + std::to_string(k) + ": " + ctx->err;
      return st;
    }
    fdk::Params &p = params[k];
    const fdc_out &o = outs[k];
    const uint64_t b0 = (uint64_t)p.first_row * j.nx + p.first_col;  // the window's first sample
    p.cls = o.cls ? o.cls + b0 : nullptr;
    p.n_out = o.n ? o.n + b0 : nullptr;
    p.nu = o.nu ? o.nu + b0 : nullptr;
    p.de = o.de ? o.de + b0 : nullptr;
    p.normal = o.normal ? o.normal + b0 : nullptr;
    p.z_out = o.z ? (double2 *)o.z + b0 : nullptr;
    p.dz_out = o.dz ? (double2 *)o.dz + b0 : nullptr;
    p.dexp_out = o.dexp ? o.dexp + b0 : nullptr;
    p.status = o.status ? o.status + b0 : nullptr;
    key[k] = ((j.flags & FDC_F32) ? 8 : 0) | (j.tier == FDC_TIER_SCALED ? 4 : 0) |
             ((j.flags & FDC_DERIVATIVE) ? 2 : 0) | ((j.flags & FDC_BLA) ? 1 : 0);
  }
  fdc_batch *b = new fdc_batch;
  b->njobs = njobs;
  // The BLA kernels store a finished sample's raw state (class, count, status, z, dz/dc, its
  // exponent) and encode_jobs_kernel computes nu / de / normal afterwards: columns the caller
  // did not ask for get scratch at the job's output pitch (one allocation for the batch).
  {
    struct Need {
      uint32_t k;
      int col;
      size_t bytes;
    };
    std::vector<Need> need;
    size_t total_bytes = 0;
    for (uint32_t k = 0; k < njobs; ++k) {
      if (!(jobs[k].flags & FDC_BLA)) continue;
      const fdk::Params &p = params[k];
      if (p.rows == 0 || p.cols == 0) continue;
      const uint64_t span = (uint64_t)(p.rows - 1) * p.out_pitch + p.cols;
      const void *have[6] = {p.cls, p.n_out, p.status, p.z_out, p.dz_out, p.dexp_out};
      const size_t width[6] = {1, 4, 1, 16, 16, 8};
      for (int c = 0; c < 6; ++c)
        if (!have[c]) {
          need.push_back({k, c, (size_t)((span * width[c] + 255) & ~(uint64_t)255)});
          total_bytes += need.back().bytes;
        }
    }
    if (total_bytes) {
      // from the context's pool: a film or tile service creating a batch per step reuses it
      b->raw = pool_get(ctx, total_bytes);
      if (!b->raw) {
        free_batch(b);
        return fail(ctx, FDC_DEVICE_ERROR, "device memory for the batch's raw-state scratch");
      }
      b->raw_bytes = total_bytes;
      char *at = (char *)b->raw;
      for (const Need &n : need) {
        fdk::Params &p = params[n.k];
        switch (n.col) {
          case 0: p.cls = (uint8_t *)at; break;
          case 1: p.n_out = (uint32_t *)at; break;
          case 2: p.status = (uint8_t *)at; break;
          case 3: p.z_out = (double2 *)at; break;
          case 4: p.dz_out = (double2 *)at; break;
          default: p.dexp_out = (int64_t *)at; break;
        }
        at += n.bytes;
      }
    }
  }
  // group by kernel variant; within a group the deepest jobs first (their samples run
  // longest, so starting them first shortens the tail of the launch)
  std::map<int, std::vector<uint32_t>> by;
  for (uint32_t k = 0; k < njobs; ++k) by[key[k]].push_back(k);
  uint32_t base = 0;
  auto bail = [&](fdc_status st) {
    free_batch(b);
    return st;
  };
  for (auto &kv : by) {
    fdc_batch::Group g;
    g.f32 = kv.first & 8;
    g.ext = kv.first & 4;
    g.deriv = kv.first & 2;
    g.bla = kv.first & 1;
    g.order = kv.second;
    std::stable_sort(g.order.begin(), g.order.end(),
                     [&](uint32_t a, uint32_t c) { return jobs[a].h_e < jobs[c].h_e; });
    std::vector<fdk::Params> gp;
    std::vector<unsigned long long> starts;
    unsigned long long total = 0;
    for (uint32_t k : g.order) {
      starts.push_back(total);
      gp.push_back(params[k]);
      total += params[k].total;
      const fdk::Params &p = params[k];
      if (g.bla && (p.nu || p.de || p.normal)) g.encode = true;
      g.max_window = std::max<uint64_t>(g.max_window, (uint64_t)p.rows * p.cols);
    }
    starts.push_back(total);
    g.total = total;
    g.counter_base = base;
    base += (uint32_t)g.order.size();
    if (cudaMalloc(&g.jobs, gp.size() * sizeof(fdk::Params)) != cudaSuccess ||
        cudaMalloc(&g.starts, starts.size() * sizeof(unsigned long long)) != cudaSuccess) {
      b->groups.push_back(g);
      return bail(fail(ctx, FDC_DEVICE_ERROR, "cudaMalloc for batch jobs failed"));
    }
    b->groups.push_back(g);
    if (cudaMemcpy(g.jobs, gp.data(), gp.size() * sizeof(fdk::Params), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g.starts, starts.data(), starts.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice) !=
            cudaSuccess)
      return bail(fail(ctx, FDC_DEVICE_ERROR, "copying batch jobs failed"));
  }
  if (cudaMalloc(&b->counters, njobs * sizeof(fdk::Counters)) != cudaSuccess ||
      cudaMalloc(&b->queues, b->groups.size() * sizeof(unsigned long long)) != cudaSuccess)
    return bail(fail(ctx, FDC_DEVICE_ERROR, "cudaMalloc for batch scratch failed"));
  // occupancy outside the capture
  for (auto &g : b->groups) {
    if (g.f32) continue;
    int variant = 0;
    void *fn = pick_batch_kernel(g.ext, g.deriv, g.bla, variant);
    if (!ctx->blocks_per_sm_batch[variant]) {
      int occ = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0) != cudaSuccess)
        return bail(fail(ctx, FDC_DEVICE_ERROR, "occupancy query failed"));
      ctx->blocks_per_sm_batch[variant] = occ > 0 ? occ : 1;
    }
  }
  // capture one run: clear queues and counters, one persistent launch per group
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->counters, 0, njobs * sizeof(fdk::Counters), ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->queues, 0, b->groups.size() * sizeof(unsigned long long), ctx->stream);
  for (size_t gi = 0; gi < b->groups.size() && e == cudaSuccess; ++gi) {
    auto &g = b->groups[gi];
    unsigned long long *q = b->queues + gi;
    fdk::Counters *c = b->counters + g.counter_base;
    uint32_t n = (uint32_t)g.order.size();
    if (g.f32) {
      e = fdk::launch_f32_batch(g.jobs, g.starts, n, g.total, q, c, g.deriv, g.bla, ctx->sm_count,
                                (int)ctx->tune.blocks_per_sm, defer_for(ctx, g.ext), ctx->stream,
                                ctx->blocks_per_sm_batch_f32);
    } else {
      int variant = 0;
      void *fn = pick_batch_kernel(g.ext, g.deriv, g.bla, variant);
      uint32_t defer = defer_for(ctx, g.ext);
      void *args[] = {&g.jobs, &g.starts, &n, &g.total, &q, &c, &defer};
      e = cudaLaunchKernel(fn, dim3(grid_blocks(ctx, ctx->blocks_per_sm_batch[variant])), dim3(128), args, 0,
                           ctx->stream);
    }
    if (e == cudaSuccess && g.encode) {  // the group's columns from the raw state
      const unsigned per_job = std::max(1u, (unsigned)std::min<uint64_t>((g.max_window + 255) / 256, 64));
      for (uint32_t off = 0; off < n && e == cudaSuccess; off += 65535u) {  // grid.y <= 65535
        fdk::encode_jobs_kernel<0><<<dim3(per_job, std::min(n - off, 65535u)), 256, 0, ctx->stream>>>(g.jobs + off);
        e = cudaGetLastError();
      }
    }
  }
  cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &b->graph);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return bail(fail(ctx, FDC_DEVICE_ERROR, std::string("batch graph: ") + cudaGetErrorString(e)));
  // the jobs' orbits and tables stay put while the batch exists
  for (uint32_t k = 0; k < njobs; ++k) b->orbits.push_back(jobs[k].orbit);
  std::sort(b->orbits.begin(), b->orbits.end());
  b->orbits.erase(std::unique(b->orbits.begin(), b->orbits.end()), b->orbits.end());
  for (int32_t h : b->orbits) ++ctx->orbits.find(h)->second.batch_refs;  // each checked above
  *out = b;
  return FDC_OK;
}

fdc_status fdc_batch_run(fdc_ctx *ctx, fdc_batch *b, fdc_counters *total, fdc_counters *per_job) {
  if (!ctx || !b) return fail(ctx, FDC_INVALID, "null argument");
  CK(cudaSetDevice(ctx->device));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  CK(cudaGraphLaunch(b->exec, ctx->stream));
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  std::vector<fdk::Counters> c(b->njobs);
  CK(cudaMemcpyAsync(c.data(), b->counters, b->njobs * sizeof(fdk::Counters), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  fdc_counters sum{};
  for (auto &g : b->groups)
    for (size_t pos = 0; pos < g.order.size(); ++pos) {
      const fdk::Counters &k = c[g.counter_base + pos];
      fdc_counters one{};
      one.samples = k.samples;
      one.iterations = k.iterations;
      one.blocks = k.blocks;
      one.skipped = k.skipped;
      one.fallback_samples = k.fallback;
      one.closed_form_samples = k.closed;
      if (per_job) per_job[g.order[pos]] = one;
      sum.samples += one.samples;
      sum.iterations += one.iterations;
      sum.blocks += one.blocks;
      sum.skipped += one.skipped;
      sum.fallback_samples += one.fallback_samples;
      sum.closed_form_samples += one.closed_form_samples;
    }
  sum.kernel_ms = ms;
  sum.launches = 0;
  for (auto &g : b->groups)
    sum.launches += 1u + (g.encode ? ((uint32_t)g.order.size() + 65534u) / 65535u : 0u);
  if (total) *total = sum;
  return FDC_OK;
}

void fdc_batch_free(fdc_ctx *ctx, fdc_batch *b) {
  if (ctx) {
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    if (b) {
      for (int32_t h : b->orbits) {
        auto it = ctx->orbits.find(h);
        if (it != ctx->orbits.end() && it->second.batch_refs) --it->second.batch_refs;
      }
      pool_put(ctx, b->raw, b->raw_bytes);  // the stream is idle: the next user may take it
      b->raw = nullptr;
    }
  }
  free_batch(b);
}

}  // extern "C"
