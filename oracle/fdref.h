/*
 * fdref — CPU oracle for the perturbation hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is a plain C++ restatement of the
 * reference CPU kernel (crates/fd-kernel, crates/fd-fixed, crates/fd-samples of
 * junovhs/fractodactyl). It is the parity checker for the CUDA route and the timed
 * CPU baseline. Nothing in the product (the fractodactyl_b200 package and its
 * CUDA library) links, loads or calls it; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg do.
 *
 * Parity pins (checked by tests/test_oracle_golden.py):
 *   - FNV-1a hashes of four 8x4 .fds renders (crates/fd-kernel/src/sample.rs:715-752)
 *   - exact escape counts of the reference's sample tests (sample.rs:965-1340)
 *   - the frozen mpmath truth pack bench/truth/v1 (5 cases x 1024 observations)
 *   - per-frame digests of crates/fd-kernel/fixtures/KERN-05.bundle (minor-0 frames)
 *
 * Build: oracle/Makefile (g++ -O2 -ffp-contract=off; no FMA contraction, as Rust).
 */
#ifndef FDREF_H
#define FDREF_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Column bits, as fd-samples Column (crates/fd-samples/src/column.rs:7-24). */
enum {
  FDREF_COL_CLASS = 1,
  FDREF_COL_NU = 2,
  FDREF_COL_DE = 4,
  FDREF_COL_NORMAL = 8,
  FDREF_COL_BOUND = 16,
  FDREF_COL_STRIPE = 32
};

/* Tier (crates/fd-kernel/src/view.rs:7-14); -1 = cheapest valid. */
enum { FDREF_TIER_AUTO = -1, FDREF_TIER_F64 = 0, FDREF_TIER_FIXED = 1, FDREF_TIER_SCALED = 2 };

/* View + Params (crates/fd-samples/src/header.rs:14-27, crates/fd-kernel/src/grid.rs:17-38). */
typedef struct {
  const char *center_re;
  const char *center_im;
  const char *width;
  double rotation;
  uint32_t nx, ny, ss;
  uint64_t max_iter;
  double escape_radius;
  uint32_t columns; /* FDREF_COL_* bits; CLASS implied */
  int32_t threads;
  int32_t tier;
  uint32_t row_first, row_step; /* render rows row_first, +row_step, ... (0, 0 = all) */
  uint32_t stripe_window;       /* Stripe column: iterates averaged (grid.rs:36-37; 0 = 16) */
  double stripe_freq;           /* Stripe column: k of sin(k arg z) (0 = 5) */
} fdref_job;

typedef struct fdref_ref fdref_ref; /* Reference orbit (reference.rs:7-10) + bits */
typedef struct fdref_bla fdref_bla; /* Bla table (bla.rs:137-151) */

/* Outcome of one sample (sample.rs:21-40): kind 0 escaped, 1 interior, 2 unresolved. */
typedef struct {
  int32_t kind;
  uint64_t n;
  double zr, zi, dr, di;
  int64_t dexp;
  uint64_t blocks, skipped;
  double shift;
  double ez, ed; /* error radii of an escaped bounded sample (infinite otherwise) */
} fdref_outcome;

/* Work counters: Stats (grid.rs:41-49) + BlaStats (grid.rs:53-70). */
typedef struct {
  uint64_t reference_len;
  uint64_t iterations;
  uint64_t blocks, skipped, fallback_samples, closed_form_samples;
  double shift_px; /* NaN when untracked */
} fdref_stats;

const char *fdref_last_error(void);

/* Plane::new (view.rs:42-87): spacing h = h_m 2^h_e, tier, bits, centre as f64. */
int fdref_plane(const fdref_job *job, double *h_m, int64_t *h_e, int32_t *tier,
                uint64_t *bits, double *c_re, double *c_im);

/* grid::reference (grid.rs:87-90) for the job, or an orbit from arrays. */
fdref_ref *fdref_reference(const fdref_job *job);
fdref_ref *fdref_reference_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius);
fdref_ref *fdref_reference_fixed(const char *re, const char *im, uint64_t bits, uint64_t max_iter);
fdref_ref *fdref_reference_arrays(const double *re, const double *im, uint64_t len, uint32_t bits);
uint64_t fdref_ref_len(const fdref_ref *r);
uint32_t fdref_ref_bits(const fdref_ref *r);
void fdref_ref_copy(const fdref_ref *r, double *re, double *im);
int64_t fdref_ref_nucleus_period(const fdref_ref *r); /* -1 for None */
void fdref_ref_free(fdref_ref *r);

/* Bla::build_scaled (bla.rs:161-181). NULL + error on refusal. */
fdref_bla *fdref_bla_build(const fdref_ref *r, double eps, double dc_max, int64_t dc_exp);
uint32_t fdref_bla_levels(const fdref_bla *t);
/* Export level-major [f64;7] blocks (a.re,a.im,b.re,b.im,r,alpha,beta), bla.rs:52-57. */
uint64_t fdref_bla_block_count(const fdref_bla *t);
void fdref_bla_export(const fdref_bla *t, double *blocks7, uint64_t *level_offsets);
/* Bla::find (bla.rs:234-249): returns the step count (0 for None) and the block index. */
uint64_t fdref_bla_find(const fdref_bla *t, uint64_t m, double d2, uint64_t budget,
                        uint64_t *level, uint64_t *index);
void fdref_bla_free(fdref_bla *t);
/* grid::bla_dc_bound (grid.rs:418-427). */
int fdref_bla_dc_bound(const fdref_job *job, double *dc, int64_t *e);

/* sample::iterate (sample.rs:170-581) for one sample. extended: Binary64Exponent.
 * has_c: absolute c for the closed-form test. nucleus: -2 = take r.nucleus_period(),
 * -1 = None, else the period. */
int fdref_iterate(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative,
                  int has_c, double cr, double ci, double ar, double ai, int64_t offset_exp,
                  uint64_t max_iter, double r2, int64_t nucleus, fdref_outcome *out);

/* render_with / render_bla (grid.rs:106-208, run :446-535). Caller-owned outputs of
 * nx*ny entries; any may be NULL. ref NULL: computed (grid.rs:802-815). bla NULL: plain. */
int fdref_render(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla,
                 uint8_t *cls, double *nu, float *de, uint16_t *normal, uint64_t *n_out,
                 double *z_out, double *dz_out, int64_t *dexp_out, fdref_stats *stats,
                 char *kernel, size_t kernel_cap);

/* sample::iterate from a supplied state (Start, sample.rs:69-80, 186-228): start_n
 * iterates done, delta (start_xr, start_xi) and dz/dc (start_dr, start_di); start_n 0 is
 * fdref_iterate. Refused on the extended tier and at or past the orbit's last point. */
/* sample::iterate with the Stripe recorder (stripe.rs; window, freq: StripeParams) for one
 * sample from Z_0: the outcome and the sample's stripe value (0 unless escaped). */
int fdref_iterate_stripe(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative, double ar,
                         double ai, int64_t offset_exp, uint64_t max_iter, double r2, int64_t nucleus,
                         uint32_t window, double freq, fdref_outcome *out, float *value);
int fdref_iterate_from(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative,
                       int has_c, double cr, double ci, double ar, double ai, int64_t offset_exp,
                       uint64_t max_iter, double r2, int64_t nucleus, uint64_t start_n,
                       double start_xr, double start_xi, double start_dr, double start_di,
                       fdref_outcome *out);
/* Series (crates/fd-kernel/src/series.rs): Series::build with SeriesConfig::default()
 * (series.rs:43-55) and build_stalled's bound (32 in Series::build; 0 = unbounded). */
typedef struct fdref_series fdref_series;
typedef struct {
  uint64_t n, points, built_steps, coefficient_pairs, order, growth_count;
  double rho, state_bound, derivative_bound, shift_px;
  char stop[16];
} fdref_series_info;
fdref_series *fdref_series_build(const fdref_ref *r, double rho, double pixel, uint64_t max_iter,
                                 uint64_t stalled_steps);
/* info, and the coefficients b[1..order] as (re, im) pairs when coeffs != NULL */
void fdref_series_get(const fdref_series *s, fdref_series_info *info, double *coeffs);
/* a copy whose admitted prefix is n (n = 0: the plain kernel) */
fdref_series *fdref_series_with_n(const fdref_series *s, uint64_t n);
/* Series::eval (series.rs:247-271): out4 = delta re, im, dz/dc re, im (0 without derivative) */
void fdref_series_eval(const fdref_series *s, int derivative, double ar, double ai, double *out4);
void fdref_series_free(fdref_series *s);
/* render_series / Series::render_masked (grid.rs:213-226, 341-373): fdref_render with every
 * sample started from the series; mask (nx*ny bytes, NULL = all) renders only samples
 * with mask != 0, leaving the others' outputs untouched. */
int fdref_render_series(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla,
                        const fdref_series *series, const uint8_t *mask, uint8_t *cls, double *nu,
                        float *de, uint16_t *normal, uint64_t *n_out, double *z_out, double *dz_out,
                        int64_t *dexp_out, fdref_stats *stats, char *kernel, size_t kernel_cap);
/* Reference::error_radius (reference.rs:122-148) into q (len entries): bits >= 0 for a
 * fixed-point orbit of that many fraction bits, -1 for an f64 orbit from (c_re, c_im). */
int fdref_error_radius(const fdref_ref *r, int64_t bits, double c_re, double c_im, double *q);
/* sample::iterate's bounded variant (B, sample.rs:221-229, 338-350, 373-377, 419-421) on
 * an ordinary tier: the orbit's error radii from (bits, c_re, c_im) as above; out->ez,
 * out->ed receive the escaped sample's radii. */
int fdref_iterate_bounded(const fdref_ref *r, int derivative, int has_c, double cr, double ci, double ar,
                          double ai, uint64_t max_iter, double r2, int64_t bits, double c_re, double c_im,
                          fdref_outcome *out);
/* All outputs of a render, any NULL: the fdref_render columns plus the Bound column
 * (FDREF_COL_BOUND: f32 nu error bound, store.rs:104-106) and the raw error radii of
 * escaped samples. */
typedef struct {
  uint8_t *cls;
  double *nu;
  float *de;
  uint16_t *normal;
  float *bound;
  uint64_t *n;
  double *z, *dz;
  int64_t *dexp;
  double *ez, *ed;
  float *stripe; /* FDREF_COL_STRIPE: the stripe average of escaped samples (stripe.rs) */
} fdref_columns;
/* Precision experiment, not the reference's algorithm: bits in [1, 52] rounds every
 * delta the kernel writes to that many mantissa bits (24: an ideal FP32-mantissa delta)
 * when the write leaves the iteration count n in [from_n, to_n); round_orbit also rounds
 * the orbit point a plain step multiplies the delta by (an FP32 copy of Z); bits 0
 * restores the reference's binary64 kernel. Process-wide; -1 for arguments out of range. */
int fdref_set_delta_bits(int bits, uint64_t from_n, uint64_t to_n, int round_orbit);

/* fdref_render / fdref_render_series with every output: series and mask may be NULL. */
int fdref_render_columns(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla,
                         const fdref_series *series, const uint8_t *mask, const fdref_columns *out,
                         fdref_stats *stats, char *kernel, size_t kernel_cap);
/* Encode one escaped state's columns exactly as Store::put (store.rs:66-112). */
void fdref_store_escaped(double h_m, int64_t h_e, uint32_t ss, double rotation, uint64_t n,
                         double zr, double zi, double dr, double di, int64_t dexp,
                         double *nu, float *de, uint16_t *normal);

/* The .fds v1 bytes of a render (fd_samples::write, crates/fd-samples/src/write.rs:8-53).
 * Returns the byte count; writes at most cap bytes (call with cap 0 to size). */
int64_t fdref_render_fds(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla,
                         uint8_t *buf, uint64_t cap);

/* fd-fixed direct iteration at one sample's exact c = centre + (ar, ai) 2^oe: the escape
 * count (0 if none within max_iter) and z there; ~0 on a parse error. */
uint64_t fdref_direct(const char *cre, const char *cim, double ar, double ai, int64_t oe, uint64_t bits,
                      uint64_t max_iter, double escape_radius, double *zr, double *zi);

#ifdef __cplusplus
}
#endif
#endif
