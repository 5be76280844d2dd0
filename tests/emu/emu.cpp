// The plain-form persistent kernel (fractodactyl_b200/csrc/perturb_f64.cuh) compiled for
// the host through cuda_host_shim.hpp and run on one thread as a single-lane warp over
// every sample of a frame, with its inputs packed as the route packs them on the device
// (pack_orbit / pack_bla / fuse_bla in fdcuda.cu). The kernel-emulation tests compare its
// outputs with the oracle's on the CPU.
// TEST INFRASTRUCTURE ONLY.
#include "cuda_host_shim.hpp"

#include <cmath>
#include <cstdint>
#include <vector>

#include "perturb_f64.cuh"

namespace {

struct Inputs {
  std::vector<double2> z, fused, coef, ab;
  std::vector<double> r2;
};

template <bool EXT, bool D, bool L, bool S, bool B>
void launch(fdk::Params &p) {
  threadIdx.x = 0;
  blockIdx.x = 0;
  fdk::perturb_kernel<EXT, D, L, S, B>(p);
}

}  // namespace

extern "C" {

// The sample window and inputs of a job (fdc_job's first_row / rows / first_col / cols,
// mask and offsets over the whole frame, the tile width 2^tile_shift and the tile order)
// as fdc_render stages them: outputs keep their frame pitch, mask and offsets are copied
// to window pitch. tile_order: 0 row-major, 1 reversed (any permutation is legal).
struct EmuWindow {
  uint32_t first_row, rows, first_col, cols, tile_shift, tile_order;
  const uint8_t *mask;
  const double *offsets;
};

// One frame: tier 0 / 1 / 2, flags bit 0 derivative, bit 1 BLA, bit 2 series start, bit 3
// bounded. blocks7 / level_offsets / levels: the BLA table in its export layout (or null);
// series_b (b_1..b_order as re, im), series_n, series_rho; q: error radii (bounded).
// Outputs (any null): class, n, nu, de, normal, z, dz, dexp, status, bound, ez, ed;
// counters[6] = samples, iterations, blocks, skipped, fallback, closed-form.
int emu_render_window(const double *re, const double *im, uint64_t len, const double *blocks7,
                      const uint64_t *level_offsets, uint32_t levels, const double *series_b, uint32_t series_order,
                      uint32_t series_n, double series_rho, const double *q, int32_t tier, uint32_t flags, uint32_t nx,
                      uint32_t ny, uint32_t ss, double c_re, double c_im, double h_m, int64_t h_e, double cos_rot,
                      double sin_rot, uint32_t max_iter, double escape_radius, int64_t nucleus, uint8_t *cls,
                      uint32_t *n_out, double *nu, float *de, uint16_t *normal, double *z_out, double *dz_out,
                      int64_t *dexp_out, uint8_t *status, float *bound, double *ez, double *ed, uint64_t *counters,
                      const EmuWindow *win);

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

int emu_render_window(const double *re, const double *im, uint64_t len, const double *blocks7,
                      const uint64_t *level_offsets, uint32_t levels, const double *series_b, uint32_t series_order,
                      uint32_t series_n, double series_rho, const double *q, int32_t tier, uint32_t flags, uint32_t nx,
                      uint32_t ny, uint32_t ss, double c_re, double c_im, double h_m, int64_t h_e, double cos_rot,
                      double sin_rot, uint32_t max_iter, double escape_radius, int64_t nucleus, uint8_t *cls,
                      uint32_t *n_out, double *nu, float *de, uint16_t *normal, double *z_out, double *dz_out,
                      int64_t *dexp_out, uint8_t *status, float *bound, double *ez, double *ed, uint64_t *counters,
                      const EmuWindow *win) {
  const bool ext = tier == 2, deriv = flags & 1, bla = (flags & 2) && levels > 0, series = (flags & 4) && series_n > 0,
             bounded = (flags & 8) && !ext;
  if (len < 3 || (bla && bounded) || (series && (ext || bounded))) return -1;  // the route's refusals
  Inputs in;
  in.z.resize(len);
  for (uint64_t m = 0; m < len; ++m) in.z[m] = make_double2(re[m], im[m]);
  fdk::Params p{};
  p.orbit = in.z.data();
  p.last = (uint32_t)(len - 1);
  p.z0r = re[0];
  p.z0i = im[0];
  if (bla) {  // pack_bla and fuse_bla
    const uint64_t steps = len - 2, total = level_offsets[levels];
    in.r2.resize(total);
    in.coef.resize(2 * total);
    in.ab.resize(total);
    for (uint64_t k = 0; k < total; ++k) {
      const double *w = blocks7 + 7 * k;
      in.r2[k] = w[4] * w[4];
      in.coef[2 * k] = make_double2(w[0], w[1]);
      in.coef[2 * k + 1] = make_double2(w[2], w[3]);
      in.ab[k] = make_double2(w[5], w[6]);
    }
    p.bla_levels = levels;
    for (uint32_t i = 0; i < levels; ++i) {
      p.bla_off[i] = (uint32_t)level_offsets[i];
      p.bla_count[i] = (uint32_t)(steps >> (i + 1));
    }
    in.fused.resize(2 * len);
    for (uint64_t m = 0; m < len; ++m) {
      double a = -1.0, b = -1.0;
      if (m >= 1 && levels > 0 && ((m - 1) & 1) == 0 && ((m - 1) >> 1) < p.bla_count[0])
        a = in.r2[p.bla_off[0] + ((m - 1) >> 1)];
      if (m >= 1 && levels > 1 && ((m - 1) & 3) == 0 && ((m - 1) >> 2) < p.bla_count[1])
        b = in.r2[p.bla_off[1] + ((m - 1) >> 2)];
      in.fused[2 * m] = in.z[m];
      in.fused[2 * m + 1] = make_double2(a, b);
    }
    p.fused = in.fused.data();
    p.bla_r2 = in.r2.data();
    p.bla_coef = in.coef.data();
    p.bla_ab = in.ab.data();
  }
  // the frame and window (prepare in fdcuda.cu); tiles of 2^shift x 32/2^shift samples
  const uint32_t r0 = win ? win->first_row : 0, rows = win && win->rows ? win->rows : ny - r0;
  const uint32_t c0 = win ? win->first_col : 0, cols = win && win->cols ? win->cols : nx - c0;
  const uint32_t shift = win ? win->tile_shift : 3;
  if (r0 >= ny || rows > ny - r0 || c0 >= nx || cols > nx - c0 || shift > 5) return -1;
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
  std::vector<uint8_t> mask;
  std::vector<double2> offs;
  if (win && win->mask) {
    mask.resize((uint64_t)rows * cols);
    for (uint32_t j = 0; j < rows; ++j)
      for (uint32_t i = 0; i < cols; ++i) mask[(uint64_t)j * cols + i] = win->mask[origin + (uint64_t)j * nx + i];
    p.mask = mask.data();
  }
  if (win && win->offsets) {
    offs.resize((uint64_t)rows * cols);
    for (uint32_t j = 0; j < rows; ++j)
      for (uint32_t i = 0; i < cols; ++i) {
        const double *o = win->offsets + 2 * (origin + (uint64_t)j * nx + i);
        offs[(uint64_t)j * cols + i] = make_double2(o[0], o[1]);
      }
    p.offsets = offs.data();
  }
  p.tier = tier;
  p.flags = (deriv || bounded ? fdk::F_DERIV : 0) | (bla ? fdk::F_BLA : 0);
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
  // outputs address the window's first sample, rows nx apart
  p.cls = cls ? cls + origin : nullptr;
  p.n_out = n_out ? n_out + origin : nullptr;
  p.nu = nu ? nu + origin : nullptr;
  p.de = de ? de + origin : nullptr;
  p.normal = normal ? normal + origin : nullptr;
  p.z_out = z_out ? (double2 *)z_out + origin : nullptr;
  p.dz_out = dz_out ? (double2 *)dz_out + origin : nullptr;
  p.dexp_out = dexp_out ? dexp_out + origin : nullptr;
  p.status = status ? status + origin : nullptr;
  unsigned long long queue = 0;
  fdk::Counters cnt{};
  uint32_t timed_out = 0;
  p.queue = &queue;
  p.counters = &cnt;
  const uint32_t tile_h = 32u >> shift, tiles_y = (rows + tile_h - 1) / tile_h;
  const uint64_t ntiles = (uint64_t)p.tiles_x * tiles_y;
  p.total = ntiles * 32;
  std::vector<uint32_t> order;
  p.tile_order = nullptr;
  if (win && win->tile_order) {
    order.resize(ntiles);
    for (uint64_t t = 0; t < ntiles; ++t) order[t] = (uint32_t)(ntiles - 1 - t);
    p.tile_order = order.data();
  }
  p.deadline_ns = 0;
  p.timed_out = &timed_out;
  p.defer = ext ? 12u : 8u;
  if (series) {
    p.series_b = (const double2 *)series_b;
    p.series_order = series_order;
    p.series_n = series_n;
    p.series_inv = 1.0 / series_rho;
  }
  if (bounded) {
    p.q = q;
    p.bound_out = bound ? bound + origin : nullptr;
    p.ez_out = ez ? ez + origin : nullptr;
    p.ed_out = ed ? ed + origin : nullptr;
  }
  const bool d = deriv || bounded;
  if (bounded) launch<false, true, false, false, true>(p);
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
  counters[0] = cnt.samples;
  counters[1] = cnt.iterations;
  counters[2] = cnt.blocks;
  counters[3] = cnt.skipped;
  counters[4] = cnt.fallback;
  counters[5] = cnt.closed;
  return 0;
}

}  // extern "C"
