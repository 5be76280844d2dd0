// The plain-form persistent kernels (fractodactyl_b200/csrc/perturb_f64.cuh: the frame
// kernel and the batch kernel) compiled for the host through cuda_host_shim.hpp and run on
// one thread as a single-lane warp over every sample, with their inputs packed as the
// route packs them on the device (pack_orbit / pack_bla / fuse_bla, prepare and
// fdc_batch_create in fdcuda.cu). The kernel-emulation tests compare their outputs with
// the oracle's on the CPU.
// TEST INFRASTRUCTURE ONLY.
// the standard headers first: the shim defines __noinline__, which libstdc++ uses
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "cuda_host_shim.hpp"

// The kernels' deadline clock (globaltimer): 1 us per read, from 0 at each launch, so a
// deadline of d ns lets a warp take about d / 1000 - 1 pickups.
namespace emu_clock {
inline uint64_t ticks = 0;
inline uint64_t now() { return ticks += 1000; }
}  // namespace emu_clock
#define FDK_HOST_TIMER() emu_clock::now()

#include "perturb_f32.cuh"
#include "bla_build.cuh"

extern "C" {

// The sample window and inputs of a job (fdc_job's first_row / rows / first_col / cols,
// mask and offsets over the whole frame, the tile width 2^tile_shift and the tile order)
// as fdc_render stages them: outputs keep their frame pitch, mask and offsets are copied
// to window pitch. tile_order: 0 row-major, 1 reversed (any permutation is legal).
// deadline_ns: fdc_job's deadline (0 none) on the emulated clock.
struct EmuWindow {
  uint32_t first_row, rows, first_col, cols, tile_shift, tile_order;
  const uint8_t *mask;
  const double *offsets;
  uint64_t deadline_ns;
};

// One job of a batch (fdc_job plus its orbit, BLA table and fdc_out): the orbit as re / im
// arrays, the BLA table in its export layout (or null), the frame, the row and column
// window (0 rows / cols: to the edge), whole-frame outputs (any null) and, returned, the
// job's counters (samples, iterations, blocks, skipped, fallback, closed-form).
struct EmuJob {
  const double *re, *im;
  uint64_t len;
  const double *blocks7;
  const uint64_t *level_offsets;
  uint32_t levels;
  int32_t tier;
  uint32_t flags;  // bit 0 derivative, bit 1 BLA, bit 2 the precision form
  uint32_t nx, ny, ss, max_iter;
  double c_re, c_im, h_m;
  int64_t h_e;
  double cos_rot, sin_rot, escape_radius;
  int64_t nucleus;
  uint32_t first_row, rows, first_col, cols;
  uint8_t *cls;
  uint32_t *n;
  double *nu;
  float *de;
  uint16_t *normal;
  double *z, *dz;
  int64_t *dexp;
  uint8_t *status;
  uint64_t counters[6];
};

}  // extern "C"

namespace {

// A job's Params and the staged arrays they point into.
struct Setup {
  std::vector<fdk::Entry32> z32;
  std::vector<double2> z, fused, coef, ab, offs;
  std::vector<double> r2;
  std::vector<uint8_t> mask;
  std::vector<uint32_t> order;
  fdk::Params p{};
  bool ext = false, deriv = false, bla = false;
  // raw-state scratch of a batch BLA job without those outputs (as fdc_batch_create gives)
  std::vector<uint8_t> raw_cls, raw_status;
  std::vector<uint32_t> raw_n;
  std::vector<double2> raw_z, raw_dz;
  std::vector<int64_t> raw_dexp;
};

template <bool EXT, bool D, bool L, bool S, bool B, bool T = false>
void launch(fdk::Params &p) {
  threadIdx.x = 0;
  blockIdx.x = 0;
  fdk::perturb_kernel<EXT, D, L, S, B, T>(p);
}

// The Stripe column of the next emu_render call that sets flag bit 5 (the stripe variant):
// its window, frequency and the whole-frame f32 output.
uint32_t g_stripe_window = 16;
double g_stripe_freq = 5.0;
float *g_stripe_out = nullptr;

template <bool D, bool L>
void launch_f32(fdk::Params &p, const fdk::Entry32 *orbit) {
  threadIdx.x = 0;
  blockIdx.x = 0;
  fdk::perturb_f32_kernel<D, L>(p, orbit);
}

template <bool EXT, bool D, bool L>
void launch_batch(const std::vector<fdk::Params> &jobs, const std::vector<unsigned long long> &starts,
                  fdk::Counters *per_job, uint32_t defer) {
  threadIdx.x = 0;
  blockIdx.x = 0;
  unsigned long long queue = 0;
  fdk::perturb_batch_kernel<EXT, D, L>(jobs.data(), starts.data(), (uint32_t)jobs.size(), starts.back(), &queue,
                                       per_job, defer);
}

template <bool D, bool L>
void launch_f32_batch(const std::vector<fdk::Params> &jobs, const std::vector<unsigned long long> &starts,
                      fdk::Counters *per_job, uint32_t defer) {
  threadIdx.x = 0;
  blockIdx.x = 0;
  unsigned long long queue = 0;
  fdk::perturb_f32_batch_kernel<D, L>(jobs.data(), starts.data(), (uint32_t)jobs.size(), starts.back(), &queue,
                                      per_job, defer);
}

// The orbit (pack_orbit) and BLA table (pack_bla, fuse_bla) of a job.
void stage_orbit(Setup &s, const double *re, const double *im, uint64_t len, const double *blocks7,
                 const uint64_t *level_offsets, uint32_t levels) {
  fdk::Params &p = s.p;
  s.z.resize(len);
  for (uint64_t m = 0; m < len; ++m) s.z[m] = make_double2(re[m], im[m]);
  p.orbit = s.z.data();
  // the precision form's entries (pack_orbit): f32 copies, NaN where |Z| < 2^-60
  s.z32.resize(len);
  for (uint64_t m = 0; m < len; ++m) {
    fdk::Entry32 &e = s.z32[m];
    e.zr = re[m];
    e.zi = im[m];
    e.zr32 = std::fmax(std::fabs(re[m]), std::fabs(im[m])) < 0x1p-60 ? __int_as_float(0x7fc00000) : (float)re[m];
    e.zi32 = (float)im[m];
    e.r2a = -1.0;
  }
  p.orbit32 = s.z32.data();
  p.last = (uint32_t)(len - 1);
  p.z0r = re[0];
  p.z0i = im[0];
  if (!s.bla) return;
  const uint64_t steps = len - 2, total = level_offsets[levels];
  s.r2.resize(total);
  s.coef.resize(2 * total);
  s.ab.resize(total);
  for (uint64_t k = 0; k < total; ++k) {
    const double *w = blocks7 + 7 * k;
    s.r2[k] = w[4] * w[4];
    s.coef[2 * k] = make_double2(w[0], w[1]);
    s.coef[2 * k + 1] = make_double2(w[2], w[3]);
    s.ab[k] = make_double2(w[5], w[6]);
  }
  p.bla_levels = levels;
  for (uint32_t i = 0; i < levels; ++i) {
    p.bla_off[i] = (uint32_t)level_offsets[i];
    p.bla_count[i] = (uint32_t)(steps >> (i + 1));
  }
  s.fused.resize(2 * len);
  for (uint64_t m = 0; m < len; ++m) {
    double a = -1.0, b = -1.0;
    if (m >= 1 && levels > 0 && ((m - 1) & 1) == 0 && ((m - 1) >> 1) < p.bla_count[0])
      a = s.r2[p.bla_off[0] + ((m - 1) >> 1)];
    if (m >= 1 && levels > 1 && ((m - 1) & 3) == 0 && ((m - 1) >> 2) < p.bla_count[1])
      b = s.r2[p.bla_off[1] + ((m - 1) >> 2)];
    s.fused[2 * m] = s.z[m];
    s.fused[2 * m + 1] = make_double2(a, b);
  }
  for (uint64_t m = 0; m < len; ++m) s.z32[m].r2a = s.fused[2 * m + 1].x;
  p.fused = s.fused.data();
  p.bla_r2 = s.r2.data();
  p.bla_coef = s.coef.data();
  p.bla_ab = s.ab.data();
}

// The frame, window, mask, offsets and tile order (prepare in fdcuda.cu); tiles of
// 2^shift x 32/2^shift samples. False when the window leaves the grid.
bool stage_frame(Setup &s, int32_t tier, uint32_t nx, uint32_t ny, uint32_t ss, double c_re, double c_im, double h_m,
                 int64_t h_e, double cos_rot, double sin_rot, uint32_t max_iter, double escape_radius, int64_t nucleus,
                 uint32_t first_row, uint32_t rows_in, uint32_t first_col, uint32_t cols_in, uint32_t shift,
                 const uint8_t *mask, const double *offsets, bool reversed) {
  fdk::Params &p = s.p;
  const uint32_t r0 = first_row, c0 = first_col;
  if (r0 >= ny || c0 >= nx || shift > 5) return false;
  const uint32_t rows = rows_in ? rows_in : ny - r0, cols = cols_in ? cols_in : nx - c0;
  if (rows > ny - r0 || cols > nx - c0) return false;
  p.nx = nx;
  p.ny = ny;
  p.first_row = r0;
  p.rows = rows;
  p.first_col = c0;
  p.cols = cols;
  p.tile_shift = shift;
  p.in_pitch = cols;
  p.out_pitch = nx;
  p.tiles_x = (cols + (1u << shift) - 1) >> shift;
  const uint64_t origin = (uint64_t)r0 * nx + c0;
  if (mask) {
    s.mask.resize((uint64_t)rows * cols);
    for (uint32_t j = 0; j < rows; ++j)
      for (uint32_t i = 0; i < cols; ++i) s.mask[(uint64_t)j * cols + i] = mask[origin + (uint64_t)j * nx + i];
    p.mask = s.mask.data();
  }
  if (offsets) {
    s.offs.resize((uint64_t)rows * cols);
    for (uint32_t j = 0; j < rows; ++j)
      for (uint32_t i = 0; i < cols; ++i) {
        const double *o = offsets + 2 * (origin + (uint64_t)j * nx + i);
        s.offs[(uint64_t)j * cols + i] = make_double2(o[0], o[1]);
      }
    p.offsets = s.offs.data();
  }
  p.tier = tier;
  p.flags = (s.deriv ? fdk::F_DERIV : 0) | (s.bla ? fdk::F_BLA : 0);
  p.c_re = c_re;
  p.c_im = c_im;
  p.h = h_m * fdk::exp2i(h_e);
  p.h_m = h_m;
  p.h_e = h_e;
  p.cosr = cos_rot;
  p.sinr = sin_rot;
  p.half_x = (double)nx / 2.0;
  p.half_y = (double)ny / 2.0;
  p.max_iter = max_iter;
  p.r2 = escape_radius * escape_radius;
  p.nucleus = nucleus;
  p.px_m = h_m * (double)ss;
  p.px_e = h_e;
  const uint32_t tile_h = 32u >> shift, tiles_y = (rows + tile_h - 1) / tile_h;
  const uint64_t ntiles = (uint64_t)p.tiles_x * tiles_y;
  p.total = ntiles * 32;
  p.tile_order = nullptr;
  if (reversed) {
    s.order.resize(ntiles);
    for (uint64_t t = 0; t < ntiles; ++t) s.order[t] = (uint32_t)(ntiles - 1 - t);
    p.tile_order = s.order.data();
  }
  p.deadline_ns = 0;
  p.defer = s.ext ? 12u : 8u;
  return true;
}

// Outputs address the window's first sample, rows nx apart.
void stage_outputs(fdk::Params &p, uint8_t *cls, uint32_t *n_out, double *nu, float *de, uint16_t *normal,
                   double *z_out, double *dz_out, int64_t *dexp_out, uint8_t *status) {
  const uint64_t origin = (uint64_t)p.first_row * p.nx + p.first_col;
  p.cls = cls ? cls + origin : nullptr;
  p.n_out = n_out ? n_out + origin : nullptr;
  p.nu = nu ? nu + origin : nullptr;
  p.de = de ? de + origin : nullptr;
  p.normal = normal ? normal + origin : nullptr;
  p.z_out = z_out ? (double2 *)z_out + origin : nullptr;
  p.dz_out = dz_out ? (double2 *)dz_out + origin : nullptr;
  p.dexp_out = dexp_out ? dexp_out + origin : nullptr;
  p.status = status ? status + origin : nullptr;
}

void copy_counters(const fdk::Counters &c, uint64_t *out) {
  out[0] = c.samples;
  out[1] = c.iterations;
  out[2] = c.blocks;
  out[3] = c.skipped;
  out[4] = c.fallback;
  out[5] = c.closed;
}

}  // namespace

extern "C" {

// One frame: tier 0 / 1 / 2, flags bit 0 derivative, bit 1 BLA, bit 2 series start, bit 3
// bounded, bit 4 the precision form (perturb_f32_kernel). blocks7 / level_offsets / levels: the BLA table in its export layout (or null);
// series_b (b_1..b_order as re, im), series_n, series_rho; q: error radii (bounded).
// Outputs (any null): class, n, nu, de, normal, z, dz, dexp, status, bound, ez, ed;
// counters[6] = samples, iterations, blocks, skipped, fallback, closed-form. win: the job's
// window and inputs, or null for the whole frame in row-major 8x4 tiles. Returns 0, 1 when
// the deadline passed (the kernel's timed_out flag), -1 for a refused job.
int emu_render_window(const double *re, const double *im, uint64_t len, const double *blocks7,
                      const uint64_t *level_offsets, uint32_t levels, const double *series_b, uint32_t series_order,
                      uint32_t series_n, double series_rho, const double *q, int32_t tier, uint32_t flags, uint32_t nx,
                      uint32_t ny, uint32_t ss, double c_re, double c_im, double h_m, int64_t h_e, double cos_rot,
                      double sin_rot, uint32_t max_iter, double escape_radius, int64_t nucleus, uint8_t *cls,
                      uint32_t *n_out, double *nu, float *de, uint16_t *normal, double *z_out, double *dz_out,
                      int64_t *dexp_out, uint8_t *status, float *bound, double *ez, double *ed, uint64_t *counters,
                      const EmuWindow *win) {
  const bool ext = tier == 2, deriv = flags & 1, bla = (flags & 2) != 0, series = (flags & 4) && series_n > 0,
             bounded = (flags & 8) && !ext, f32 = flags & 16, striped = (flags & 32) != 0;
  if (len < 3 || (bla && bounded) || (series && (ext || bounded)) || (f32 && (series || bounded)) ||
      (striped && (series || bounded || f32)))
    return -1;  // the route's refusals
  Setup s;
  s.ext = ext;
  s.deriv = deriv || bounded;
  s.bla = bla;
  stage_orbit(s, re, im, len, blocks7, level_offsets, levels);
  if (!stage_frame(s, tier, nx, ny, ss, c_re, c_im, h_m, h_e, cos_rot, sin_rot, max_iter, escape_radius, nucleus,
                   win ? win->first_row : 0, win ? win->rows : 0, win ? win->first_col : 0, win ? win->cols : 0,
                   win ? win->tile_shift : 3, win ? win->mask : nullptr, win ? win->offsets : nullptr,
                   win && win->tile_order))
    return -1;
  fdk::Params &p = s.p;
  stage_outputs(p, cls, n_out, nu, de, normal, z_out, dz_out, dexp_out, status);
  unsigned long long queue = 0;
  fdk::Counters cnt{};
  uint32_t timed_out = 0;
  p.queue = &queue;
  p.counters = &cnt;
  p.timed_out = &timed_out;
  p.deadline_ns = win ? win->deadline_ns : 0;
  emu_clock::ticks = 0;
  if (series) {
    p.series_b = (const double2 *)series_b;
    p.series_order = series_order;
    p.series_n = series_n;
    p.series_inv = 1.0 / series_rho;
  }
  if (bounded) {
    const uint64_t origin = (uint64_t)p.first_row * nx + p.first_col;
    p.q = q;
    p.bound_out = bound ? bound + origin : nullptr;
    p.ez_out = ez ? ez + origin : nullptr;
    p.ed_out = ed ? ed + origin : nullptr;
  }
  const bool d = s.deriv;
  if (striped) {
    p.stripe_out = g_stripe_out ? g_stripe_out + (uint64_t)p.first_row * nx + p.first_col : nullptr;
    p.stripe_window = g_stripe_window;
    p.stripe_freq = g_stripe_freq;
  }
  if (striped) {
    if (ext) {
      if (d) bla ? launch<true, true, true, false, false, true>(p) : launch<true, true, false, false, false, true>(p);
      else bla ? launch<true, false, true, false, false, true>(p) : launch<true, false, false, false, false, true>(p);
    } else {
      if (d) bla ? launch<false, true, true, false, false, true>(p) : launch<false, true, false, false, false, true>(p);
      else bla ? launch<false, false, true, false, false, true>(p) : launch<false, false, false, false, false, true>(p);
    }
  } else if (f32) {
    const fdk::Entry32 *o = s.z32.data();
    if (d) bla ? launch_f32<true, true>(p, o) : launch_f32<true, false>(p, o);
    else bla ? launch_f32<false, true>(p, o) : launch_f32<false, false>(p, o);
  } else if (bounded) launch<false, true, false, false, true>(p);
  else if (series) {
    if (d) bla ? launch<false, true, true, true, false>(p) : launch<false, true, false, true, false>(p);
    else bla ? launch<false, false, true, true, false>(p) : launch<false, false, false, true, false>(p);
  } else if (ext) {
    if (d) bla ? launch<true, true, true, false, false>(p) : launch<true, true, false, false, false>(p);
    else bla ? launch<true, false, true, false, false>(p) : launch<true, false, false, false, false>(p);
  } else {
    if (d) bla ? launch<false, true, true, false, false>(p) : launch<false, true, false, false, false>(p);
    else bla ? launch<false, false, true, false, false>(p) : launch<false, false, false, false, false>(p);
  }
  if (!bounded && !striped && bla) {  // the columns from the raw state, as fdc_render does
    threadIdx.x = 0;
    blockIdx.x = 0;
    fdk::encode_kernel<0>(p);
  }
  copy_counters(cnt, counters);
  return timed_out ? 1 : 0;
}

int emu_render(const double *re, const double *im, uint64_t len, const double *blocks7, const uint64_t *level_offsets,
               uint32_t levels, const double *series_b, uint32_t series_order, uint32_t series_n, double series_rho,
               const double *q, int32_t tier, uint32_t flags, uint32_t nx, uint32_t ny, uint32_t ss, double c_re,
               double c_im, double h_m, int64_t h_e, double cos_rot, double sin_rot, uint32_t max_iter,
               double escape_radius, int64_t nucleus, uint8_t *cls, uint32_t *n_out, double *nu, float *de,
               uint16_t *normal, double *z_out, double *dz_out, int64_t *dexp_out, uint8_t *status, float *bound,
               double *ez, double *ed, uint64_t *counters) {
  return emu_render_window(re, im, len, blocks7, level_offsets, levels, series_b, series_order, series_n, series_rho, q,
                           tier, flags, nx, ny, ss, c_re, c_im, h_m, h_e, cos_rot, sin_rot, max_iter, escape_radius,
                           nucleus, cls, n_out, nu, de, normal, z_out, dz_out, dexp_out, status, bound, ez, ed, counters,
                           nullptr);
}

// A batch as fdc_batch_create builds it and one replay of it: the jobs grouped by kernel
// variant (precision form, Scaled tier, derivative, BLA), each group's jobs deepest first (stable by h_e),
// their sample ranges laid end to end (starts), one batch-kernel run per group with a
// queue of its own and per-job counters returned in each job's own slot.
int emu_render_batch(EmuJob *jobs, uint32_t njobs) {
  std::vector<std::unique_ptr<Setup>> setups(njobs);
  std::map<int, std::vector<uint32_t>> by;
  for (uint32_t k = 0; k < njobs; ++k) {
    const EmuJob &j = jobs[k];
    if (j.len < 3 || j.tier < 0 || j.tier > 2) return -1;
    auto s = std::make_unique<Setup>();
    s->ext = j.tier == 2;
    s->deriv = j.flags & 1;
    s->bla = (j.flags & 2) != 0;
    stage_orbit(*s, j.re, j.im, j.len, j.blocks7, j.level_offsets, j.levels);
    if (!stage_frame(*s, j.tier, j.nx, j.ny, j.ss, j.c_re, j.c_im, j.h_m, j.h_e, j.cos_rot, j.sin_rot, j.max_iter,
                     j.escape_radius, j.nucleus, j.first_row, j.rows, j.first_col, j.cols, 3, nullptr, nullptr,
                     false))
      return -1;
    stage_outputs(s->p, j.cls, j.n, j.nu, j.de, j.normal, j.z, j.dz, j.dexp, j.status);
    if (s->bla && s->p.rows && s->p.cols) {  // the BLA batch kernels store raw state: scratch where absent
      fdk::Params &p = s->p;
      const size_t span = (size_t)(p.rows - 1) * p.out_pitch + p.cols;
      if (!p.cls) p.cls = (s->raw_cls.assign(span, 0), s->raw_cls.data());
      if (!p.status) p.status = (s->raw_status.assign(span, 0), s->raw_status.data());
      if (!p.n_out) p.n_out = (s->raw_n.assign(span, 0), s->raw_n.data());
      if (!p.z_out) p.z_out = (s->raw_z.assign(span, double2{0, 0}), s->raw_z.data());
      if (!p.dz_out) p.dz_out = (s->raw_dz.assign(span, double2{0, 0}), s->raw_dz.data());
      if (!p.dexp_out) p.dexp_out = (s->raw_dexp.assign(span, 0), s->raw_dexp.data());
    }
    by[((j.flags & 4) ? 8 : 0) | (s->ext ? 4 : 0) | (s->deriv ? 2 : 0) | (s->bla ? 1 : 0)].push_back(k);
    setups[k] = std::move(s);
  }
  for (auto &kv : by) {
    std::vector<uint32_t> order = kv.second;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return jobs[a].h_e < jobs[c].h_e; });
    std::vector<fdk::Params> gp;
    std::vector<unsigned long long> starts;
    unsigned long long total = 0;
    for (uint32_t k : order) {
      starts.push_back(total);
      gp.push_back(setups[k]->p);
      total += setups[k]->p.total;
    }
    starts.push_back(total);
    std::vector<fdk::Counters> cnt(order.size());
    const bool f32 = kv.first & 8, ext = kv.first & 4, d = kv.first & 2, l = kv.first & 1;
    const uint32_t defer = ext ? 12u : 8u;
    if (f32) {
      if (d) l ? launch_f32_batch<true, true>(gp, starts, cnt.data(), defer)
             : launch_f32_batch<true, false>(gp, starts, cnt.data(), defer);
      else l ? launch_f32_batch<false, true>(gp, starts, cnt.data(), defer)
             : launch_f32_batch<false, false>(gp, starts, cnt.data(), defer);
    } else if (ext) {
      if (d) l ? launch_batch<true, true, true>(gp, starts, cnt.data(), defer)
             : launch_batch<true, true, false>(gp, starts, cnt.data(), defer);
      else l ? launch_batch<true, false, true>(gp, starts, cnt.data(), defer)
             : launch_batch<true, false, false>(gp, starts, cnt.data(), defer);
    } else {
      if (d) l ? launch_batch<false, true, true>(gp, starts, cnt.data(), defer)
             : launch_batch<false, true, false>(gp, starts, cnt.data(), defer);
      else l ? launch_batch<false, false, true>(gp, starts, cnt.data(), defer)
             : launch_batch<false, false, false>(gp, starts, cnt.data(), defer);
    }
    if (l)  // the columns from the raw state, as fdc_batch_create's encode pass does
      for (const fdk::Params &p : gp)
        if (p.nu || p.de || p.normal) fdk::encode_window(p, 0, 1);
    for (size_t i = 0; i < order.size(); ++i) copy_counters(cnt[i], jobs[order[i]].counters);
  }
  return 0;
}

void emu_set_stripe(uint32_t window, double freq, float *out) {
  g_stripe_window = window;
  g_stripe_freq = freq;
  g_stripe_out = out;
}


// fdk::libm_hypot over n pairs against the host C library's hypot: how many differ (two
// NaN results count as equal).
uint64_t emu_hypot_check(const double *x, const double *y, uint64_t n) {
  uint64_t bad = 0;
  for (uint64_t k = 0; k < n; ++k) {
    const double a = fdk::libm_hypot(x[k], y[k]), b = std::hypot(x[k], y[k]);
    bad += !(std::memcmp(&a, &b, 8) == 0 || (std::isnan(a) && std::isnan(b)));
  }
  return bad;
}

// The device table builder (fdk::bla_level, one host thread per level) over an orbit, as
// fdc_build_bla queues it: every possible level, each skipped after a level without a
// valid block. out7: room for len - 3 blocks; the kept levels are written level-major.
// Returns the kept level count.
uint32_t emu_bla_build(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                       double *out7) {
  std::vector<double2> z(len);
  for (uint64_t k = 0; k < len; ++k) z[k] = make_double2(re[k], im[k]);
  const uint64_t steps = len >= 2 ? len - 2 : 0;
  std::vector<uint64_t> size, at;
  uint64_t room = 0;
  for (uint64_t n = steps / 2; n > 0 && size.size() < (size_t)fdk::MAX_LEVELS; n /= 2) {
    at.push_back(room);
    size.push_back(n);
    room += n;
  }
  std::vector<double> raw(7 * std::max<uint64_t>(room, 1));
  std::vector<unsigned> valid(fdk::MAX_LEVELS, 0);
  blockIdx.x = 0;
  threadIdx.x = 0;
  blockDim.x = 1;
  gridDim.x = 1;
  for (uint32_t i = 0; i < size.size(); ++i)
    fdk::bla_level(z.data(), i > 0 ? raw.data() + 7 * at[i - 1] : nullptr, size[i], i, eps, dc_max, dc_exp,
                   raw.data() + 7 * at[i], valid.data());
  uint32_t kept = 0;
  while (kept < size.size() && valid[kept]) ++kept;
  const uint64_t total = kept ? at[kept - 1] + size[kept - 1] : 0;
  std::copy(raw.begin(), raw.begin() + 7 * total, out7);
  return kept;
}

}  // extern "C"
