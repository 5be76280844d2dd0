/*
 * fdcuda.h - C ABI of the B200 (sm_100a) perturbation route for fractodactyl.
 *
 * The route replaces the WGSL dispatch of junovhs/fractodactyl's existing GPU route
 * (crates/fd-cli/src/perturb_gpu/frame.rs:119-355, render_inner) with hand-written CUDA.
 * The caller keeps the reference's host side: it owns the Reference orbit
 * (crates/fd-kernel/src/reference.rs:7-10), the BLA table built by the CPU builder
 * (crates/fd-kernel/src/bla.rs:161-181) and the Samples columns
 * (crates/fd-samples/src/samples.rs:7-20). Every entry point takes plain pointers and
 * sizes, copies what it needs into device memory owned by the context, writes into
 * caller-owned buffers, and keeps no host pointer after it returns. No entry point
 * aborts or throws: failures come back as an fdc_status and fdc_last_error().
 *
 * Threading: a context is used by one thread at a time; it owns one CUDA stream.
 */
#ifndef FDCUDA_H
#define FDCUDA_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDC_ABI_VERSION 1

/* Status codes. On anything but FDC_OK the caller restarts the frame on the CPU from
 * n = 0, as restart_after_attempt does (frame.rs:357-368). */
typedef enum {
  FDC_OK = 0,
  FDC_DECLINED = 1,     /* the route does not take this job (caller renders on CPU) */
  FDC_INVALID = 2,      /* malformed input (sizes, handles, non-finite values) */
  FDC_DEVICE_ERROR = 3, /* a CUDA call failed; the context should be closed */
  FDC_TIMEOUT = 4,      /* the job's deadline passed; samples not finished keep status 0 */
  FDC_NO_DEVICE = 5     /* no usable sm_100 device */
} fdc_status;

/* Tiers (crates/fd-kernel/src/view.rs:7-14). */
enum { FDC_TIER_F64 = 0, FDC_TIER_FIXED = 1, FDC_TIER_SCALED = 2 };

/* Job flags. */
enum {
  FDC_DERIVATIVE = 1u << 0, /* track dz/dc (columns de/normal; sample.rs "D") */
  FDC_BLA = 1u << 1,        /* apply the uploaded BLA table (sample.rs "L") */
  FDC_SHIFT = 1u << 2,      /* accumulate the BLA first-order shift estimate (BlaStats.shift_px) */
  FDC_F32 = 1u << 3,        /* precision form: FP32-mantissa floatexp deltas (not bit-exact) */
  FDC_DEVICE_OUT = 1u << 4, /* fdc_out pointers are device pointers (no host copies) */
  FDC_SERIES = 1u << 5      /* start every sample from the orbit's uploaded series */
};

typedef struct fdc_ctx fdc_ctx;

/* One frame (or a sub-range of it). Geometry follows Plane (view.rs:42-128): sample
 * (i, j) has unit offset ux = cos x + sin y, uy = sin x - cos y with x = i + 0.5 - nx/2,
 * y = j + 0.5 - ny/2, and dc = (ux, uy) h_m 2^h_e. */
typedef struct {
  int32_t orbit;          /* handle from fdc_upload_orbit */
  int32_t tier;           /* FDC_TIER_* (the caller's resolved tier) */
  uint32_t nx, ny, ss;    /* sample grid; ss only scales the DE pixel */
  uint32_t flags;         /* FDC_* */
  double c_re, c_im;      /* centre rounded to f64 (F64 tier closed-form test) */
  double h_m;             /* spacing mantissa, 1 <= h_m < 2 */
  int64_t h_e;            /* spacing exponent */
  double cos_rot, sin_rot;
  uint64_t max_iter;      /* < 2^32 */
  double escape_radius;
  int64_t nucleus_period; /* Reference::nucleus_period (reference.rs:102-120); -1 = None */
  const uint8_t *mask;    /* optional, nx*ny host bytes: render only samples with mask != 0 */
  const double *offsets;  /* optional, 2*nx*ny host doubles: per-sample (ux, uy) instead of the grid */
  uint32_t first_row, rows; /* render rows [first_row, first_row + rows); rows 0 = all */
  double deadline_ms;     /* stop taking new samples after this long; 0 = none */
  uint32_t first_col, cols; /* and of those rows columns [first_col, first_col + cols); cols 0 = all.
                             * Outputs, mask and offsets still span whole rows of nx samples. */
} fdc_job;

/* Caller-owned outputs, nx*ny entries each (only rows rendered are written); any may be
 * NULL. With FDC_DEVICE_OUT they are device pointers. */
typedef struct {
  uint8_t *cls;      /* Class byte: Kind | Evidence << 2 (crates/fd-samples/src/class.rs) */
  uint32_t *n;       /* iterates (Escaped/Interior), max_iter for Unresolved */
  double *nu;        /* n + 1 - log2(log2 |z|) (store.rs:97-99), escaped only */
  float *de;         /* distance estimate in output pixels (store.rs:141-150) */
  uint16_t *normal;  /* screen normal angle, turns * 65536 (store.rs:107-111) */
  double *z;         /* 2 per sample: z at escape (raw state for the host encoder) */
  double *dz;        /* 2 per sample: dz/dc mantissa */
  int64_t *dexp;     /* dz/dc exponent */
  uint8_t *status;   /* 1 = finished, 0 = not computed (mask, deadline) */
} fdc_out;

/* Work counters of one fdc_render (Stats grid.rs:41-49 + BlaStats grid.rs:53-70). */
typedef struct {
  uint64_t samples;         /* samples finished */
  uint64_t iterations;      /* iterates, each applied block counted once */
  uint64_t blocks, skipped; /* BLA blocks applied and steps they replaced */
  uint64_t fallback_samples, closed_form_samples;
  double shift;             /* largest shift estimate in c units (FDC_SHIFT) */
  double kernel_ms;         /* device time of the render kernel(s) */
  uint32_t launches;        /* kernels launched */
} fdc_counters;

/* Library / device. */
int fdc_abi_version(void);
fdc_status fdc_open(int device, fdc_ctx **out);
void fdc_close(fdc_ctx *ctx);
const char *fdc_last_error(const fdc_ctx *ctx);

/* Upload a reference orbit Z_0..Z_{len-1} (SoA f64 as Reference keeps it) with the
 * precision it was computed at (53 = f64 tier). Replaces the wgpu orbit packing of
 * frame.rs:172-188. Z_0 must be 0; 2 <= len <= 2^20 (reference.rs:16). */
fdc_status fdc_upload_orbit(fdc_ctx *ctx, const double *re, const double *im, uint64_t len, uint32_t bits,
                            int32_t *orbit);
fdc_status fdc_free_orbit(fdc_ctx *ctx, int32_t orbit);

/* Upload the BLA table built over that orbit (Bla, bla.rs:137-151) in its export form:
 * level-major blocks of [f64; 7] = a.re, a.im, b.re, b.im, r, alpha, beta (bla.rs:52-57,
 * the fd-atlas chunk layout), level i (j = i + 1) at blocks7[7 * level_offsets[i]...],
 * (points - 2) >> (i + 1) blocks each. Replaces pack_bla (frame.rs:86-117). */
fdc_status fdc_upload_bla(fdc_ctx *ctx, int32_t orbit, const double *blocks7, const uint64_t *level_offsets,
                          uint32_t levels, double eps, double dc_max, int64_t dc_exp);

/* Build that table on the device from the uploaded orbit instead of uploading it:
 * Bla::build_scaled(reference, eps, dc_max, dc_exp) (bla.rs:161-216, which control.rs:359
 * and film.rs:1321 call before rendering), with the same blocks bit for bit and the same refusals
 * as fdc_upload_bla. *levels (optional) receives the kept level count; export7 (optional,
 * host memory for len - 3 blocks) receives the kept levels in the export form above,
 * level i at offset sum_{j<i} (len - 2) >> (j + 1). Replaces the host build and the
 * 56-byte-per-block upload. */
fdc_status fdc_build_bla(fdc_ctx *ctx, int32_t orbit, double eps, double dc_max, int64_t dc_exp, uint32_t *levels,
                         double *export7);

/* Upload a parameter-series start built over that orbit (Series, series.rs:57-84, e.g. by
 * fdh_series_build): jobs with FDC_SERIES start every sample at iterate n from delta =
 * sum_k b_k (dc / rho)^k, coeffs = b_1..b_order as (re, im) pairs (order <= 64), on the
 * F64 / Fixed tiers of the plain form, for views with |dc| <= rho; a sample whose series
 * start ends unresolved retries from zero (grid.rs:623-648). n = 0: no admitted prefix,
 * the plain kernel. Refused: points other than the orbit's length, n + 1 >= points.
 * Replaces the series arm of grid::run (render_series, grid.rs:213-226). */
fdc_status fdc_upload_series(fdc_ctx *ctx, int32_t orbit, uint64_t points, uint64_t n, double rho,
                             const double *coeffs, uint32_t order);

/* Render a job (replaces dispatch_batched, frame.rs:242-260, and the readback checks,
 * :271-286). Results are those of the CPU kernel (sample.rs:170-581) for the plain form:
 * class and n bit-exact, z and dz bit-exact, nu/de/normal within CUDA libm's ulps. */
fdc_status fdc_render(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, fdc_counters *counters);

/* Bounded renders (the Bound column; sample.rs's B variant, store.rs:88-106, grid.rs:
 * 379-384, 588-593). fdc_upload_error_radius attaches the orbit's error radii
 * q[m] >= |A_m - Z_m| (Reference::error_radius, reference.rs:122-148, e.g. from
 * fdh_error_radius; len = the orbit's points). fdc_render_bounded renders like fdc_render
 * and, on the F64 / Fixed tiers, tracks error radii on z and dz/dc every step (derivative
 * on): escaped samples whose radii prove escape get Bounded evidence (class byte
 * Escaped | 1 << 2), de scaled by the certified lower factor, and bound[] the nu error
 * bound (0 elsewhere); ez[] / ed[] receive each escaped sample's raw radii (the host
 * encoder's inputs). The scaled tier has no radii and renders as fdc_render (bound 0).
 * Refused: FDC_BLA (remainders are not certified), FDC_SERIES, FDC_F32. Any pointer of
 * fdc_bound_out may be NULL; they follow fdc_out's layout (FDC_DEVICE_OUT included). */
typedef struct {
  float *bound;   /* nu error bound of Bounded samples (store.rs:104-106) */
  double *ez;     /* error radius on z at escape */
  double *ed;     /* error radius on the dz/dc mantissa at escape */
} fdc_bound_out;
fdc_status fdc_upload_error_radius(fdc_ctx *ctx, int32_t orbit, const double *q, uint64_t len);
fdc_status fdc_render_bounded(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, const fdc_bound_out *bound,
                              fdc_counters *counters);

/* The Stripe column (crates/fd-kernel/src/stripe.rs; the column grid.rs:493-498, 772
 * writes, the refusal of grid.rs:783-788). fdc_render_stripe renders like fdc_render
 * and also records each sample's last 128 iterates and last 8 BLA block starts; an escape
 * whose window misses iterates replays them plainly from a kept block start, as the CPU
 * kernel does (sample.rs:231-236, 387-403), so every output of fdc_render is unchanged.
 * stripe_out receives the stripe average of escaped samples (0 elsewhere; f32, fdc_out's
 * layout, FDC_DEVICE_OUT included); the average's terms use CUDA's hypot / sin / atan2 /
 * log, so values are within a few ulps of the CPU's. FDC_INVALID: window outside 1..64 or
 * a frequency that is not finite. FDC_DECLINED (render on the CPU): FDC_SERIES, FDC_F32.
 * Each sample's recorder lives in local memory (~2.6 KB per resident lane). */
typedef struct {
  uint32_t window; /* iterates averaged before escape, 1..64 (StripeParams, stripe.rs:20-36) */
  double freq;     /* k of 0.5 + 0.5 sin(k arg z) */
} fdc_stripe;
fdc_status fdc_render_stripe(fdc_ctx *ctx, const fdc_job *job, fdc_out *out, const fdc_stripe *stripe,
                             float *stripe_out, fdc_counters *counters);

/* Launch tuning (no counterpart in the reference; the reference's shader has fixed
 * workgroups). defer: lanes of a warp whose next operation is a BLA block wait until
 * defer/32 of the warp's busy lanes wait, or no lane steps plainly, and then apply their
 * blocks together (1: at once; 0: the measured default of each kernel variant, 12 on
 * the floatexp tier and 8 elsewhere); results do not depend on it. blocks_per_sm:
 * resident 128-thread blocks per SM of the persistent launch, 0 for as many as fit.
 * tile_w: width of the warp-sized tiles of samples the work queue hands out (1, 2, 4, 8,
 * 16 or 32; the height is 32 / tile_w), 0 for 8. order: FDC_ORDER_CENTRE hands tiles out
 * nearest to the window's centre first (a nucleus-centred view's longest samples start
 * early instead of ending the launch), FDC_ORDER_ROWS in row-major order; 0 for
 * centre-first. Neither changes any result. A context starts with all four 0;
 * settings apply to later fdc_render calls and to batches created after them.
 * fractodactyl_b200.tune measures and picks them. */
#define FDC_DEFAULT_DEFER 0
#define FDC_ORDER_ROWS 1
#define FDC_ORDER_CENTRE 2
typedef struct fdc_tuning {
  uint32_t defer;
  uint32_t blocks_per_sm;
  uint32_t tile_w;
  uint32_t order;
} fdc_tuning;
fdc_status fdc_set_tuning(fdc_ctx *ctx, const fdc_tuning *tuning);
fdc_status fdc_get_tuning(const fdc_ctx *ctx, fdc_tuning *tuning);

/* Batches: many jobs (the frames of a zoom film, tiles of many locations, each job with
 * its own orbit handle, tier and device outputs) rendered by ONE persistent launch per
 * kernel variant from a single work queue over all jobs' tiles, deepest jobs first, the
 * whole run captured once in a CUDA graph and replayed by fdc_batch_run. Results equal
 * fdc_render's per job. Jobs need FDC_DEVICE_OUT, no mask/offsets/deadline/FDC_SERIES; orbits and
 * tables must stay uploaded while the batch exists: fdc_free_orbit, fdc_upload_bla and
 * fdc_build_bla refuse (FDC_INVALID) an orbit that a live batch reads, until fdc_batch_free.
 * Free batches before fdc_close. BLA jobs store each finished sample's raw state (class,
 * count, status, z, dz/dc, its exponent) and a second kernel per group encodes nu / de /
 * normal from it: the batch holds device scratch for those the job's fdc_out leaves null
 * (up to 46 bytes per sample of the window's rows at the output pitch). per_job (optional)
 * has njobs entries; counters->kernel_ms is the device time of the whole replay. */
typedef struct fdc_batch fdc_batch;
fdc_status fdc_batch_create(fdc_ctx *ctx, const fdc_job *jobs, const fdc_out *outs, uint32_t njobs,
                            fdc_batch **batch);
fdc_status fdc_batch_run(fdc_ctx *ctx, fdc_batch *batch, fdc_counters *counters, fdc_counters *per_job);
void fdc_batch_free(fdc_ctx *ctx, fdc_batch *batch);

/* Allocation-free rendering (no counterpart in the reference). For callers that cannot
 * allocate device memory: a render service that owns all device memory through its own
 * pool or arena (other allocations would fragment it or break its memory budget) and
 * hands the library buffers carved from it. It renders the plain form (FP64,
 * no BLA, series, mask or offsets) with no context, no cudaMalloc, no cudaFree and no
 * allocating library call: the caller passes the orbit (2*len doubles, interleaved
 * re/im, Z_0 = 0) and every output column of `out` as DEVICE pointers, and the kernel's
 * scratch (work-queue head, counters, per-row iteration sums) lives in one fixed device
 * array of FDC_NOALLOC_SCRATCH_BYTES, which every GPU that loads the library holds until
 * the process exits. That fixes the row limit: a job renders at most
 * (FDC_NOALLOC_SCRATCH_BYTES - 256) / 8 = 8160 rows per call (job->rows, or ny when 0);
 * larger jobs are refused with FDC_INVALID and a message naming the limit, and so are
 * an orbit or z / dz column off a 16-byte boundary and any other column off its element
 * size. The first call on a device checks it as fdc_open does (FDC_NO_DEVICE unless a
 * present sm_100 device) and looks up the array's device address (once per device, safe
 * under concurrent first calls); make that first call before any stream capture. The
 * calling thread's current device is the same after the call as before it. Every call
 * shares the array and clears what it
 * uses before its kernel runs: calls that overlap on the GPU (other streams, other host
 * threads) race on it, so serialise them. row_iterations (optional, host, `rows`
 * entries) receives the iterations spent per rendered row; counters (optional) the
 * sample and iteration totals. Both readbacks synchronise `stream` (NULL: the default
 * stream). Errors: the status, and a message in `error` (cap bytes, optional). */
#define FDC_NOALLOC_SCRATCH_BYTES 65536
fdc_status fdc_render_noalloc(int device, const double *orbit, uint64_t len, const fdc_job *job, const fdc_out *out,
                              uint64_t *row_iterations, fdc_counters *counters, void *stream, char *error,
                              size_t error_cap);

#ifdef __cplusplus
}
#endif
#endif
