/*
 * fdhost.h - host-side set-up of the B200 perturbation route, in C++.
 *
 * These are the parts of junovhs/fractodactyl's path that stay on the CPU because they
 * are serial or cheap (reference orbit in fixed point, the view's plane, the BLA table
 * built by the CPU builder, the nucleus gate), offered behind a C ABI for callers that
 * do not bring their own (the reference's Rust side computes them itself and calls only
 * fdcuda.h). Results equal the reference's bit for bit: orbit points are exact integer
 * arithmetic rounded by the same rule, BLA blocks use the same operation order.
 * Errors: negative return, message in fdh_last_error() (per thread).
 */
#ifndef FDHOST_H
#define FDHOST_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char *fdh_last_error(void);

/* Plane::new (crates/fd-kernel/src/view.rs:42-87): sample spacing h = h_m 2^h_e, the
 * cheapest valid tier (0 F64, 1 Fixed, 2 Scaled), fixed-point bits, centre as f64,
 * rotation cos/sin. */
typedef struct {
  double c_re, c_im, h_m;
  int64_t h_e;
  int32_t tier;
  uint64_t bits;
  double cos_rot, sin_rot;
} fdh_plane;
int fdh_plane_new(const char *center_re, const char *center_im, const char *width, double rotation, uint32_t nx,
                  uint32_t ny, fdh_plane *out);

/* Reference orbits (crates/fd-kernel/src/reference.rs). The orbit is written into
 * caller arrays of capacity cap (>= min(max_iter, 2^20 - 1) + 1); returns its length.
 *   fdh_orbit_fixed: Reference::from_fixed over fd_fixed::orbit (reference.rs:85-96,
 *                    crates/fd-fixed/src/orbit.rs:14-43) at the exact decimal centre.
 *   fdh_orbit_fixed_threads: the same orbit, bit for bit; threads >= 3 splits each
 *                    step's three squarings over three threads when the orbit has at
 *                    least 28 limbs (~1,700 bits), 1 keeps it serial, 0 picks 3 when the
 *                    host has 4 or more hardware threads (no counterpart: the
 *                    reference's orbit is serial).
 *   fdh_orbit_f64:   Reference::new (reference.rs:21-48). */
int64_t fdh_orbit_fixed(const char *center_re, const char *center_im, uint64_t bits, uint64_t max_iter, double *re,
                        double *im, uint64_t cap);
int64_t fdh_orbit_fixed_threads(const char *center_re, const char *center_im, uint64_t bits, uint64_t max_iter,
                                double *re, double *im, uint64_t cap, int threads);
int64_t fdh_orbit_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius, double *re, double *im,
                      uint64_t cap);

/* Reference::nucleus_period (reference.rs:102-120); -1 for None. */
int64_t fdh_nucleus_period(const double *re, const double *im, uint64_t len);

/* Bla::build_scaled (crates/fd-kernel/src/bla.rs:161-181) over an orbit, in the export
 * layout fdc_upload_bla takes: level-major [f64; 7] blocks. First call with blocks7 =
 * NULL to learn the level count and block count; level_offsets has levels + 1 entries.
 * threads <= 0: all cores. */
int fdh_bla_build(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                  int threads, double *blocks7, uint64_t *level_offsets, uint32_t *levels, uint64_t *blocks);

/* The same table built once into caller buffers of cap_blocks blocks and cap_levels + 1
 * offsets (len - 2 blocks and 64 levels always suffice); levels and blocks receive the
 * sizes. With cap_blocks >= len - 2 the levels are merged in place in blocks7, whose
 * entries past the table's are then scratch. Returns -1 if the table does not fit (the
 * offsets untouched). */
int fdh_bla_build_into(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                       int threads, double *blocks7, uint64_t cap_blocks, uint64_t *level_offsets, uint32_t cap_levels,
                       uint32_t *levels, uint64_t *blocks);

/* GuardedBla::build (crates/fd-kernel/src/bla/guarded.rs:110-134): the BLA blocks with
 * the affine uncertainty envelopes that the reference's approximate GPU route admits its
 * results by, over the orbit and its reference radii q[len] (Reference::error_radius):
 * level-major [f64; 9] blocks (a.re, a.im, b.re, b.im, r, alpha, beta, derivative alpha,
 * derivative beta), level i at blocks9[9 * level_offsets[i]...], levels + 1 offsets. The
 * CUDA route runs the reference's algorithm exactly and needs no admission; this serves
 * callers that keep the reference's guarded route. Refusals: bla.rs:27-33, a radius that
 * is negative or not finite. */
int fdh_guarded_bla_build(const double *re, const double *im, const double *q, uint64_t len, double eps,
                          double dc_max, double *blocks9, uint64_t cap_blocks, uint64_t *level_offsets,
                          uint32_t cap_levels, uint32_t *levels, uint64_t *blocks);

/* external_escape_ok (crates/fd-kernel/src/store.rs:152-198): 1 when an externally
 * computed escaped state (n, z, dz/dc = (dr, di) 2^dexp) with error radii ez on z and ed on
 * the derivative mantissa encodes within half the comparison budget for the output pixel
 * px_m 2^px_e (host libm, as the reference's Rust); 0 otherwise. */
int fdh_external_escape_ok(uint64_t n, double zr, double zi, double dr, double di, int64_t dexp, double ez, double ed,
                           double px_m, int64_t px_e);

/* Reference::error_radius (crates/fd-kernel/src/reference.rs:122-148) into q (len
 * entries): bounds on each orbit point's distance from the exact orbit of the exact centre,
 * for the Bound column (fdc_upload_error_radius). bits >= 0: a fixed-point orbit of that
 * many fraction bits; bits < 0: an f64 orbit from the correctly rounded centre (c_re, c_im). */
int fdh_error_radius(const double *re, const double *im, uint64_t len, int64_t bits, double c_re, double c_im,
                     double *q);

/* Series::build (crates/fd-kernel/src/series.rs:86-245) with SeriesConfig::default()
 * (series.rs:43-55) over an orbit, for samples with |dc| <= rho and output pixels of
 * `pixel` in c: the parameter-series start every sample of a frame may take (n iterates
 * skipped; n = 0: none admitted). stalled_steps bounds consecutive rejections (32 in
 * Series::build, 0 unbounded). coeffs receives b_1..b_order as (re, im) pairs (room for
 * cap_order pairs; 64 always suffice). */
typedef struct fdh_series {
  uint64_t n, points, built_steps, coefficient_pairs;
  uint32_t order, growth_count;
  double rho, state_bound, derivative_bound, shift_px;
  char stop[16];
} fdh_series;
int fdh_series_build(const double *re, const double *im, uint64_t len, double rho, double pixel, uint64_t max_iter,
                     uint64_t stalled_steps, fdh_series *out, double *coeffs, uint32_t cap_order);

/* grid.rs:418-444: bound m 2^e on |dc| over a view's samples for a tier. */
void fdh_dc_bound(const fdh_plane *plane, int32_t tier, uint32_t nx, uint32_t ny, double *dc, int64_t *e);

/* Store::put for the escaped samples of a render (crates/fd-kernel/src/store.rs:66-112,
 * Bound column absent): nu = n + 1 - log2(0.5 log2 |z|^2), de in output pixels
 * (store.rs:141-150) and the screen normal (samples.rs:45-48) from the raw state the
 * device returns (z, dz/dc = (dr, di) 2^dexp), evaluated with the host's libm as the
 * reference's Rust is, so the columns are the CPU route's bytes. Samples whose class byte
 * is not escaped (0) are left untouched; any output may be NULL. threads <= 0: all cores. */
void fdh_encode(const fdh_plane *plane, uint32_t ss, uint64_t count, const uint8_t *cls, const uint32_t *n,
                const double *z, const double *dz, const int64_t *dexp, double *nu, float *de, uint16_t *normal,
                int threads);

/* Location recipe of the benchmark frames (no reference API; the construction of
 * tools/research/twolevel/ref.py:31-117 around a Misiurewicz point):
 *   1. the repelling Misiurewicz point M(q, r), q <= 60, r <= 4, nearest the start (Newton
 *      on z_{q+r}(c) = z_q(c) from it, ref.py:31-43);
 *   2. the lowest-period nucleus in the disc of radius R around M + 0.345 R e^{i theta}
 *      (ball period, ref.py:46-52; Newton clamped to R/4, :54-67), with log10 R bisected
 *      (14 steps) until the nucleus's size estimate (:69-74) is about width/30.
 * Fixed point at `bits` fraction bits. Writes the nucleus as decimal strings (caller
 * buffers of cap bytes), its period and log10(size / width); returns 0 on success. */
int fdh_location(const char *start_re, const char *start_im, double theta, double log10_width, uint64_t bits,
                 uint64_t max_period, char *re_out, char *im_out, size_t cap, uint64_t *period,
                 double *log10_size_over_width);

#ifdef __cplusplus
}
#endif
#endif
