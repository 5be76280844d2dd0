// The plain (FP64) perturbation kernel: one lane per sample, persistent warps that
// refill finished lanes from an atomic tile queue. The per-sample state machine is
// iterate() of crates/fd-kernel/src/sample.rs:170-581 (Binary64 and Binary64Exponent,
// number.rs:92-124) with the reference's operation order: one loop iteration is
// find_block, then apply_block or plain_update, then post; warp_step runs it for a
// warp (with BLA deferral), step for one lane. Compile with -fmad=false.
#pragma once
#include <cstdint>

#include "fd_device.cuh"

namespace fdk {

constexpr int MAX_LEVELS = 40;

// Resident 128-thread blocks per SM each kernel variant is compiled for (caps registers
// at 65536 / (128 * blocks)): floatexp-tier variants (EXT) and ordinary-tier variants;
// chosen by measurement (5 floatexp blocks at 96 registers: the 1920x1080 frame at a 1e-100
// nucleus, 10^6 iterations, 37.95 -> 37.53 ms).
#ifndef FDK_MIN_BLOCKS_EXT
#define FDK_MIN_BLOCKS_EXT 5
#endif
#ifndef FDK_MIN_BLOCKS_FIX
#define FDK_MIN_BLOCKS_FIX 4
#endif
template <bool EXT>
struct Occupancy {
  static constexpr int blocks = EXT ? FDK_MIN_BLOCKS_EXT : FDK_MIN_BLOCKS_FIX;
};

struct Counters {
  unsigned long long samples, iterations, blocks, skipped, fallback, closed;
  unsigned long long shift_bits;  // max of the non-negative shift estimates, as bits
  unsigned long long pad;
};

// Everything one launch needs; passed by value (kernel parameter space).
struct Params {
  const double2 *__restrict__ orbit;  // Z_0..Z_last, interleaved re/im
  // With BLA: Z_m fused with the squared radii of the level-1 and level-2 blocks (j = 1, 2)
  // starting at m, or -1 where none starts there: 32-byte entries (zr, zi, r2a, r2b), so the
  // first two levels of Bla::find come with the orbit point each step loads anyway.
  const double2 *__restrict__ fused;
  const void *orbit32;  // precision-form entries (perturb_f32.cuh), per job in batches
  uint32_t last;
  double z0r, z0i;
  // BLA, level-major: r2[off + t], coef[2 (off + t)] = (a.re, a.im), (b.re, b.im), ab = (alpha, beta)
  const double *__restrict__ bla_r2;
  const double2 *__restrict__ bla_coef;
  const double2 *__restrict__ bla_ab;
  uint32_t bla_levels;
  uint32_t bla_off[MAX_LEVELS];
  uint32_t bla_count[MAX_LEVELS];
  // frame
  uint32_t nx, ny, first_row, rows, tiles_x;
  uint32_t first_col, cols;        // rendered window: columns [first_col, first_col + cols) of those rows
  uint32_t in_pitch, out_pitch;    // row pitch (samples) of the mask/offsets inputs and of the outputs,
                                   // whose pointers address the window's first sample
  uint32_t tile_shift;  // tiles are 2^tile_shift samples wide and 32 / 2^tile_shift rows high
  const uint32_t *tile_order;  // order the queue hands tiles out in (row-major tile indices), or null
  int32_t tier;
  uint32_t flags;
  double c_re, c_im, h, h_m;
  int64_t h_e;
  double cosr, sinr, half_x, half_y;
  uint32_t max_iter;  // < 2^32 (checked by the route)
  double r2;
  int64_t nucleus;
  double px_m;  // DE output pixel h_m * ss (store.rs:57-63)
  int64_t px_e;
  const uint8_t *__restrict__ mask;
  const double2 *__restrict__ offsets;
  // outputs (device)
  uint8_t *cls;
  uint32_t *n_out;
  double *nu;
  float *de;
  uint16_t *normal;
  double2 *z_out, *dz_out;
  int64_t *dexp_out;
  uint8_t *status;
  // scratch: work queue and counters
  unsigned long long *queue;
  Counters *counters;
  uint64_t total;        // queue slots (tiles * 32)
  uint64_t deadline_ns;  // 0 = none
  uint32_t *timed_out;
  uint32_t defer;     // BLA lanes a warp gathers before it applies their blocks (warp_step)
  // Parameter-series start (series.rs:57-84, ordinary tiers): every sample starts at
  // iterate series_n from delta = sum_k b_k x^k, x = dc / rho; series_n = 0: none.
  const double2 *__restrict__ series_b;  // b_1..b_order as (re, im)
  uint32_t series_order, series_n;
  double series_inv;  // 1 / rho
  // Bounded variant (B, ordinary tiers): the orbit's error radii q[m] >= |A_m - Z_m|
  // (reference.rs:122-148) and the outputs it adds: the Bound column and the raw radii
  const double *__restrict__ q;
  float *bound_out;
  double *ez_out, *ed_out;
  // Stripe variant (T): the column (stripe.rs) and its settings (window 1..64, frequency)
  float *stripe_out;
  uint32_t stripe_window;
  double stripe_freq;
};

constexpr double SAFE = 1.0 + 8.0 * U;  // sample.rs:56

enum : uint32_t { F_DERIV = 1u, F_BLA = 2u, F_SHIFT = 4u };

// Per-lane sample state (sample.rs:187-236).
template <bool EXT>
struct State {
  double xr, xi, dr, di;
  double fr, fi;  // z = Z[m] + delta (carried between steps on the ordinary tier)
  double Zr, Zi;  // Z[m]
  double r2a, r2b;  // radii^2 of the blocks of 2 and 4 steps starting at m (BLA kernels)
  double ar, ai;  // sample offset (mantissa on the extended tier)
  double dc_r, dc_i, scale, inverse;
  double sr, si, qr, qi, qstep;
  double near;  // save_point(): the near-return bound of the save point (sr, si)
  Multiplier mu;
  Contraction ct;
  double adc, shift;
  double e, ed, rc;  // B: error radii on z and dz/dc, the offset's own error (sample.rs:221-225)
  int32_t offset_exp, delta_exp;  // |h_e| <= 2^30 (checked by the route): deltas stay within 32 bits
  int64_t derivative_exp;
  int32_t nucleus;               // < 2^31 - 1 (checked by the route)
  uint32_t n, chk, sn, hold, blocks, skipped;  // n < max_iter < 2^32; chk saturates at 2^32 - 1
  uint32_t lim;  // relimit()
  uint32_t m, idx;
  int returns;
  bool pending, predicted;
  bool replaying;  // T: re-walking a stripe window plainly (sample.rs:231-236) ...
  uint32_t limit;  // ... up to this iterate
};

// Result of a finished sample (sample.rs:21-40): kind 0 escaped, 1 interior, 2 unresolved.
struct Result {
  int kind;
  uint64_t n;
  double zr, zi, dr, di;
  int64_t dexp;
  double ez, ed;  // B: error radii of an escaped sample (sample.rs:373-377)
};

// The loop state at the start of a BLA block, from which a stripe replay restarts
// (stripe.rs:39-52).
struct StripeSnap {
  uint32_t m, n;
  double xr, xi;
  int32_t delta_exp;
  double scale, dc_r, dc_i;
  uint64_t valid;  // first iterate of the recorded run that reached n
};

// The Stripe column's recorder for one lane (stripe.rs:12-241): the last 128 iterates, the
// last 8 block starts, and the escape the blocks found while a replay re-walks its window.
// Only the stripe variants (T) hold one; it lives in local memory (~2.6 KB per lane).
struct StripeTrace {
  static constexpr uint32_t RING = 128, SNAPS = 8;
  double2 ring[RING];
  StripeSnap snaps[SNAPS];
  Result first;
  double first_r, first_i;
  uint64_t first_at;
  uint64_t valid;
  uint32_t count;
  float value;

  __device__ __forceinline__ void begin() {  // stripe.rs:164-168
    valid = ~0ull;
    count = 0;
    value = 0.0f;
  }
  __device__ __forceinline__ void start(uint64_t n) { valid = n + 1; }
  __device__ __forceinline__ void record(uint64_t n, double zr, double zi) { ring[n % RING] = make_double2(zr, zi); }
  __device__ __forceinline__ void snap(StripeSnap s, uint64_t landed) {  // stripe.rs:180-187
    s.valid = valid;
    snaps[count % SNAPS] = s;
    count += 1;
    valid = landed;
  }
  // stripe.rs:157-160 and 189-204: a kept block start to replay from when the windows
  // ending at z_n miss iterates (the latest at or before n - window, else the oldest)
  __device__ bool rewind(uint64_t n, uint32_t window, StripeSnap &out) {
    const uint64_t need = n > window ? n - window : 0;
    if (count == 0 || valid <= (need > 1 ? need : 1)) return false;
    const uint32_t kept = count < SNAPS ? count : SNAPS;
    int pick = -1;
    for (uint32_t j = 0; j < kept && pick < 0; ++j) {
      const uint32_t k = (count - 1 - j) % SNAPS;
      if (snaps[k].n <= need) pick = (int)k;
    }
    if (pick < 0) {
      for (uint32_t j = 0; j < kept; ++j) {
        const uint32_t k = (count - 1 - j) % SNAPS;
        if (pick < 0 || snaps[k].n < snaps[pick].n) pick = (int)k;
      }
    }
    valid = snaps[pick].valid;
    out = snaps[pick];
    return true;
  }
  // stripe.rs:132-152: 0.5 + 0.5 sin(k arg z); a whole k up to 16 as the sign of k times
  // Im (z / |z|)^|k|
  __device__ static double term(double zr, double zi, double k) {
    double s;
    if (k == trunc(k) && fabs(k) <= 16.0) {
      const double h = hypot(zr, zi);
      const double ur = zr / h, ui = zi / h;
      double pr = 1.0, pi = 0.0;
      const int reps = (int)fabs(k);
      for (int q = 0; q < reps; ++q) {
        const double nr = pr * ur - pi * ui, ni = pr * ui + pi * ur;
        pr = nr;
        pi = ni;
      }
      s = k < 0.0 ? -pi : pi;
    } else {
      s = sin(k * atan2(zi, zr));
    }
    return 0.5 + 0.5 * s;
  }
  // stripe.rs:206-240: the windows ending at z_n and z_{n-1}, interpolated by how far
  // past the escape radius z_n landed
  __device__ void finish(uint64_t n, double zr, double zi, double r2, uint32_t window, double k) {
    const uint64_t lo = n > window ? n - window : 0;
    const uint64_t first_i = lo > 1 ? lo : 1;
    double now = 0.0, before = 0.0;
    uint32_t cn = 0, cb = 0;
    for (uint64_t i = first_i; i <= n; ++i) {
      if (i < valid) continue;
      const double2 z = ring[i % RING];
      const double t = term(z.x, z.y, k);
      if (i > first_i || (first_i == 1 && n <= window)) {
        now += t;
        cn += 1;
      }
      if (i < n) {
        before += t;
        cb += 1;
      }
    }
    if (cn == 0) {
      value = 0.0f;
      return;
    }
    now /= (double)cn;
    before = cb > 0 ? before / (double)cb : now;
    double frac = 1.0 - log2(log(zr * zr + zi * zi) / log(r2));
    if (frac < 0.0) frac = 0.0;  // f64::clamp keeps NaN
    if (frac > 1.0) frac = 1.0;
    value = (float)(before * (1.0 - frac) + now * frac);
  }
};

// A periodicity save point (sample.rs:488-491, 522-575): the point and the bound that a
// later z's distance from it is compared with, fabs(sr) + fabs(si) scaled as each tier's
// near-return test scales it. The reference evaluates the bound every iteration from the
// same two values, so evaluating it once here gives the same double.
template <bool EXT>
__device__ __forceinline__ void save_point(State<EXT> &s, double r, double i) {
  s.sr = r;
  s.si = i;
  const double size = fabs(r) + fabs(i);
  s.near = EXT ? 1e-13 * size + 1e-300 : 1e-3 * size;
}

// The iteration limit behind Bla::find's budget (sample.rs:246-263) with n left out:
// min(max_iter, the next periodicity save point, nucleus + 1), kept in the state and
// recomputed whenever one of its inputs (hold, sn, pending, chk, nucleus) changes, so an
// iteration only subtracts n. The reference's n == 0 case (a budget of 1) never reaches
// the search: with a nucleus gate, m == 0 skips the BLA. lim <= max_iter < 2^32.
template <bool EXT>
__device__ __forceinline__ void relimit(const Params &p, State<EXT> &s) {
  uint64_t cap = s.hold > 0 ? (uint64_t)s.sn + s.hold : (s.pending ? ~0ull : (uint64_t)s.chk);
  uint64_t b = p.max_iter < cap ? p.max_iter : cap;
  if (s.nucleus >= 0 && (uint64_t)s.nucleus + 1 < b) b = (uint64_t)s.nucleus + 1;
  s.lim = (uint32_t)b;
}

// Bla::find (bla.rs:234-249) at the top of an iteration: the level of the longest valid
// block starting at m that fits the budget, or -1, with its index in that level in `at`.
// The radii of the first two levels come with the orbit entry (r2a, r2b); those of the
// next PRE levels are loaded together before the comparisons that would stop at them.
template <bool EXT>
__device__ __forceinline__ double block_d2(const State<EXT> &s) {
  return EXT ? (s.xr * s.xr + s.xi * s.xi) * s.scale * s.scale : s.xr * s.xr + s.xi * s.xi;
}

// Whether Bla::find finds any block at m: one test for the nucleus gate, the budget and
// the level-1 block (r2a is -1 unless a block starts at m); every operand is evaluated,
// which costs fewer branches than returning at the first that fails.
template <bool EXT>
__device__ __forceinline__ bool block_starts(const State<EXT> &s) {
  const uint32_t budget = s.lim > s.n ? s.lim - s.n : 0u;
  return (s.nucleus < 0 || s.m != 0) & (budget >= 2) & (block_d2(s) < s.r2a);
}

// The rest of Bla::find once block_starts holds: the level of the longest valid block.
template <bool EXT>
__device__ __forceinline__ int block_level(const Params &p, const State<EXT> &s, uint32_t &at) {
  const uint32_t budget = s.lim > s.n ? s.lim - s.n : 0u;
  const double d2 = block_d2(s);
  const uint32_t k = s.m - 1u;     // m = 0 wraps: odd, no block
  at = k >> 1;
  if (budget < 4 || !(d2 < s.r2b)) return 0;
  at = k >> 2;
  const uint32_t tz = k == 0 ? 32u : (uint32_t)(__ffs((int)k) - 1);
  const uint32_t top = tz < p.bla_levels ? tz : p.bla_levels;
  constexpr uint32_t PRE = 4;  // levels 2..5
  double r[PRE];
  bool ok[PRE];
#pragma unroll
  for (uint32_t q = 0; q < PRE; ++q) {
    const uint32_t i = 2 + q, a = k >> (i + 1);
    ok[q] = i < top && (2u << i) <= budget && a < p.bla_count[i];
    r[q] = ok[q] ? __ldg(p.bla_r2 + p.bla_off[i] + a) : -1.0;
  }
  // the prefetched levels that pass, as bits; the block is the last level of the passing
  // run from level 2 up (the same level and index as testing them in order)
  uint32_t pass = 0;
#pragma unroll
  for (uint32_t q = 0; q < PRE; ++q) pass |= (uint32_t)(ok[q] && d2 < r[q]) << q;
  const uint32_t run = (uint32_t)__ffs((int)~pass) - 1u;  // bit PRE of ~pass is set: run <= PRE
  if (run > 0) at = k >> (2 + run);
  if (run < PRE) return (int)(1 + run);
  int lv = (int)(1 + PRE);
  for (uint32_t i = 2 + PRE; i < top; ++i) {
    if ((2ull << i) > budget) break;
    const uint32_t a = k >> (i + 1);
    if (a >= p.bla_count[i]) break;
    if (!(d2 < __ldg(p.bla_r2 + p.bla_off[i] + a))) break;
    lv = (int)i;
    at = a;
  }
  return lv;
}

template <bool EXT>
__device__ __forceinline__ int find_block(const Params &p, const State<EXT> &s, uint32_t &at) {
  return block_starts(s) ? block_level(p, s, at) : -1;
}

// A BLA block application (sample.rs:264-315): delta' = A delta + B dc, dz' = A dz + B.
template <bool EXT, bool D>
__device__ __forceinline__ void apply_block(const Params &p, State<EXT> &s, int lv, uint32_t at) {
  const uint32_t b = p.bla_off[lv] + at;
  const double2 A = __ldg(p.bla_coef + 2 * b), B = __ldg(p.bla_coef + 2 * b + 1);
  const uint32_t len = 2u << lv;
  if (s.nucleus >= 0 && s.n >= 1) s.ct.multiply(A.x, A.y);
  if (!EXT && s.hold > 0) s.mu.multiply(A.x, A.y);
  if (EXT) {
    normalise(s.xr, s.xi, s.delta_exp, 0);
    if (D) {
      normalise(s.dr, s.di, s.derivative_exp, INT64_MAX / 4);
      s.inverse = exp2i(-s.derivative_exp);
    }
    s.scale = exp2i(s.delta_exp);
    double factor = exp2i(s.offset_exp - s.delta_exp);
    s.dc_r = s.ar * factor;
    s.dc_i = s.ai * factor;
  }
  if (D) {
    double t = A.x * s.dr - A.y * s.di + B.x * s.inverse;
    s.di = A.x * s.di + A.y * s.dr + B.y * s.inverse;
    s.dr = t;
    if (!EXT && (p.flags & F_SHIFT)) {
      double2 ab = __ldg(p.bla_ab + b);
      s.shift += (ab.x * sqrt(s.xr * s.xr + s.xi * s.xi) + ab.y * s.adc) / sqrt(s.dr * s.dr + s.di * s.di);
    }
  }
  double t = A.x * s.xr - A.y * s.xi + B.x * s.dc_r - B.y * s.dc_i;
  s.xi = A.x * s.xi + A.y * s.xr + B.x * s.dc_i + B.y * s.dc_r;
  s.xr = t;
  if (EXT) {
    normalise(s.xr, s.xi, s.delta_exp, 0);
    if (D) {
      normalise(s.dr, s.di, s.derivative_exp, INT64_MAX / 4);
      s.inverse = exp2i(-s.derivative_exp);
    }
    s.scale = exp2i(s.delta_exp);
    double factor = exp2i(s.offset_exp - s.delta_exp);
    s.dc_r = s.ar * factor;
    s.dc_i = s.ai * factor;
  }
  s.m += len;
  s.n += len;
  s.blocks += 1;
  s.skipped += len;
}

// One ordinary step (sample.rs:331-380; number.rs:92-124): z = Z[m] + delta is carried
// from the end of the previous iteration in (fr, fi).
template <bool EXT, bool D, bool B = false>
__device__ __forceinline__ void plain_update(State<EXT> &s, const double *__restrict__ q = nullptr) {
  const double fr = s.fr, fi = s.fi;
  if (s.nucleus >= 0 && s.n >= 1) s.ct.multiply(2.0 * fr, 2.0 * fi);
  if (!EXT && s.hold > 0) s.mu.multiply(2.0 * fr, 2.0 * fi);
  if (B) {  // sample.rs:338-350: the radii through this step, from the state before it
    const double qm = __ldg(q + s.m);
    const double af = sqrt(fr * fr + fi * fi) * (1.0 + 4.0 * U) + 1e-150;  // >= |f|
    const double ef = s.e + qm + 2.0 * U * af;                              // >= |z_exact - f|
    const double ad = fabs(s.dr) + fabs(s.di);
    s.ed = (2.0 * (af + ef) * s.ed + 2.0 * ef * ad + 8.0 * U * (2.0 * af * ad + 1.0)) * SAFE;
    const double aw = fabs(s.Zr) + fabs(s.Zi), ax = fabs(s.xr) + fabs(s.xi);
    // the delta step's defect against 2 A delta + delta^2 + dc_exact
    const double rho = 8.0 * U * (2.0 * aw * ax + ax * ax + fabs(s.ar) + fabs(s.ai)) + 2.0 * qm * ax + s.rc;
    const double w = af + qm + 2.0 * U * af;  // >= |A_m + delta|
    s.e = (s.e * (2.0 * w + s.e) + rho) * SAFE;
  }
  if (D) {
    double t = 2.0 * (fr * s.dr - fi * s.di) + s.inverse;
    s.di = 2.0 * (fr * s.di + fi * s.dr);
    s.dr = t;
    if (EXT && rmax(fabs(s.dr), fabs(s.di)) > HI) {
      s.dr = s.dr * LO;
      s.di = s.di * LO;
      s.derivative_exp += 32;
      s.inverse = exp2i(-s.derivative_exp);
    }
  }
  const double wr = s.xr, wi = s.xi, zr = s.Zr, zi = s.Zi;
  if (EXT) {  // number.rs:109-124
    s.xr = 2.0 * (zr * wr - zi * wi) + s.scale * (wr * wr - wi * wi) + s.dc_r;
    s.xi = 2.0 * (zr * wi + zi * wr) + s.scale * (2.0 * wr * wi) + s.dc_i;
  } else {  // number.rs:92-107
    s.xr = 2.0 * (zr * wr - zi * wi) + wr * wr - wi * wi + s.dc_r;
    s.xi = 2.0 * (zr * wi + zi * wr + wr * wi) + s.dc_i;
  }
  s.m += 1;
  s.n += 1;
}

// The rest of the iteration after the update (sample.rs:381-575): the next orbit point,
// bailout, nucleus gate, rebase, rescaling and periodicity. Zn/Rn hold the prefetched
// entry m + 1 of the iteration's start, right after a plain step; after a block (took)
// the entry at the new m is loaded here. Returns true when the sample has an outcome.
// T: the Stripe recorder tr records the iterate, and an escape whose window misses
// iterates replays them from a kept block start (sample.rs:369-403).
template <bool EXT, bool D, bool L, bool B = false, bool T = false>
__device__ __forceinline__ bool post(const Params &p, State<EXT> &s, Result &res, bool took, double2 Zn,
                                     double2 Rn, StripeTrace *tr = nullptr) {
  double2 Z = Zn;
  if (L) {
    if (took) {  // a block moved m by its length
      Z = __ldg(p.fused + 2 * s.m);
      Rn = __ldg(p.fused + 2 * s.m + 1);
    }
    s.r2a = Rn.x;
    s.r2b = Rn.y;
  }
  s.Zr = Z.x;
  s.Zi = Z.y;
  double pr = EXT ? s.scale * s.xr : s.xr, pi = EXT ? s.scale * s.xi : s.xi;
  double fr = Z.x + pr, fi = Z.y + pi;
  double f2 = fr * fr + fi * fi;
  if (T) tr->record(s.n, fr, fi);
  const bool replaying = T && s.replaying;  // no nucleus gate or periodicity while replaying
  {
    // The common iterations leave through a short path: no escape, nucleus gate or
    // near-return (the full sequence below handles those), and at most a rebase onto Z_0
    // whose delta keeps binary64's range (f2 > SQUARE_OK on the extended tier), a +-32
    // rescaling of the extended tier's delta, or a Brent save point of the extended tier.
    // Each of those is the full sequence's own expressions in its own order, so the state
    // after either path is the same; the divergent work per lane is a few instructions.
    const double delta2 = pr * pr + pi * pi;
    const bool rebase = EXT ? f2 <= delta2 : f2 < delta2;
    const bool reb = rebase || s.m == p.last;
    bool common = !(f2 > p.r2) && !(!replaying && s.nucleus >= 0 && s.n == (uint32_t)s.nucleus + 1u);
    if (B || (EXT && !(f2 > SQUARE_OK))) common = common && !reb;  // bounded radii; sum2 rebase
    // the judge reads the delta after a rebase on the ordinary tiers (it is then z itself)
    const double check_r = EXT ? pr : (reb ? fr : s.xr), check_i = EXT ? pi : (reb ? fi : s.xi);
    bool judge = check_r * check_r + check_i * check_i > RES2 * f2;
    if (EXT) judge = judge && s.returns < 4;
    const double dist = fabs(fr - s.sr) + fabs(fi - s.si);
    if (replaying) {
    } else if (EXT) {
      common = common && !(judge && dist < s.near);
    } else {
      const bool held = s.hold > 0 && s.n - s.sn < s.hold;  // sn <= n while hold > 0
      common = common && (judge ? !(dist < s.near) && (s.hold > 0 ? held : !(s.pending || s.n >= s.chk))
                                : (s.hold > 0 ? held : s.n < s.chk));
    }
    if (__builtin_expect(common, 1)) {
      bool moved = false;
      if (__builtin_expect(reb, 0)) {  // sample.rs:418-452 without sum2 or TINY (scale is 1)
        moved = true;
        s.xr = fr;
        s.xi = fi;
        s.m = 0;
        s.Zr = p.z0r;
        s.Zi = p.z0i;
        s.r2a = -1.0;  // no block starts at Z_0 (bla.rs:235-236)
        s.r2b = -1.0;
        if (EXT) {
          s.delta_exp = 0;
          s.scale = exp2i(s.delta_exp);
          double factor = exp2i(s.offset_exp - s.delta_exp);
          s.dc_r = s.ar * factor;
          s.dc_i = s.ai * factor;
        }
      } else if (EXT) {  // sample.rs:453-467
        const double magnitude = rmax(fabs(s.xr), fabs(s.xi));
        int32_t k = 0;
        if (magnitude > HI && s.delta_exp < 0)
          k = -s.delta_exp < 32 ? -s.delta_exp : 32;
        else if (magnitude < LO && magnitude != 0.0)
          k = -32;
        if (__builtin_expect(k != 0, 0)) {
          moved = true;
          double factor = exp2i(-k);
          s.xr = s.xr * factor;
          s.xi = s.xi * factor;
          s.delta_exp = s.delta_exp + k;
          s.scale = exp2i(s.delta_exp);
          double f = exp2i(s.offset_exp - s.delta_exp);
          s.dc_r = s.ar * f;
          s.dc_i = s.ai * f;
        }
      }
      if (moved) {  // the next iteration's z (sample.rs:331; number.rs:113 on the extended tier)
        s.fr = EXT ? s.Zr + s.scale * s.xr : s.Zr + s.xr;
        s.fi = EXT ? s.Zi + s.scale * s.xi : s.Zi + s.xi;
      } else {
        s.fr = fr;
        s.fi = fi;
      }
      if (EXT && !replaying && __builtin_expect(s.n >= s.chk, 0)) {  // sample.rs:488-491 / :571-574
        save_point(s, fr, fi);
        s.sn = s.n;
        s.chk = s.chk >= 0x80000000u ? 0xffffffffu : s.chk * 2;
        relimit(p, s);
      }
      return false;
    }
  }
  if (__builtin_expect(f2 > p.r2, 0)) {
    res.kind = 0;
    res.n = s.n;
    res.zr = fr;
    res.zi = fi;
    res.dr = s.dr;
    res.di = s.di;
    res.dexp = s.derivative_exp;
    if (B) {  // sample.rs:373-377
      res.ez = s.e + __ldg(p.q + s.m) + 4.0 * U * sqrt(f2);
      res.ed = s.ed;
    }
    if (T) {  // sample.rs:387-403
      if (replaying) {  // the replay reached an escape: the blocks' outcome, this window
        tr->finish(s.n, fr, fi, p.r2, p.stripe_window, p.stripe_freq);
        res = tr->first;
        return true;
      }
      StripeSnap sn;
      if (tr->rewind(s.n, p.stripe_window, sn)) {
        tr->first = res;
        tr->first_at = s.n;
        tr->first_r = fr;
        tr->first_i = fi;
        s.replaying = true;
        const uint64_t give_up = (uint64_t)s.n + 64;  // sample.rs:397
        s.limit = (uint32_t)(give_up < p.max_iter ? give_up : p.max_iter);
        s.m = sn.m;
        s.n = sn.n;
        s.xr = sn.xr;
        s.xi = sn.xi;
        s.delta_exp = sn.delta_exp;
        s.scale = sn.scale;
        s.dc_r = sn.dc_r;
        s.dc_i = sn.dc_i;
        const double2 Zm = __ldg(p.orbit + s.m);  // z of the replay's first step
        s.Zr = Zm.x;
        s.Zi = Zm.y;
        s.fr = EXT ? s.Zr + s.scale * s.xr : s.Zr + s.xr;
        s.fi = EXT ? s.Zi + s.scale * s.xi : s.Zi + s.xi;
        return false;
      }
      tr->finish(s.n, fr, fi, p.r2, p.stripe_window, p.stripe_freq);
    }
    return true;
  }
  if (!replaying && __builtin_expect(s.nucleus >= 0, 0) && s.n == (uint32_t)s.nucleus + 1u) {
    if (s.ct.small()) {
      res.kind = 1;
      res.n = s.n;
      return true;
    }
    s.nucleus = -1;
    relimit(p, s);
  }
  double delta2 = pr * pr + pi * pi;
  bool rebase = EXT ? f2 <= delta2 : f2 < delta2;
  // z of the next iteration, Z[m] + delta with the final m and delta: (fr, fi) unless the
  // delta or its scale changes below
  bool moved = false;
  if (__builtin_expect(rebase || s.m == p.last, 0)) {
    moved = true;
    if (B) s.e += __ldg(p.q + s.m) + 4.0 * U * sqrt(f2) + 1e-300;  // sample.rs:419-421: delta := f
    if (EXT) {
      if (f2 > SQUARE_OK) {
        s.xr = fr;
        s.xi = fi;
        s.delta_exp = 0;
      } else {
        Cx3 t = sum2(Cx3{Z.x, Z.y, 0}, Cx3{s.xr, s.xi, s.delta_exp}, s.delta_exp);
        s.xr = t.re;
        s.xi = t.im;
        s.delta_exp = (int32_t)t.e;
      }
      s.scale = exp2i(s.delta_exp);
      s.m = 0;
      s.Zr = p.z0r;
      s.Zi = p.z0i;
      s.r2a = -1.0;  // no block starts at Z_0 (bla.rs:235-236)
      s.r2b = -1.0;
      if (s.scale < 1.0 / 1e270) {  // TINY, sample.rs:17
        s.nucleus = -1;
        relimit(p, s);
        if (D) {
          Cx3 v = zero_step_dz(Cx3{s.xr, s.xi, s.delta_exp}, Cx3{s.dr, s.di, s.derivative_exp});
          s.dr = v.re;
          s.di = v.im;
          s.derivative_exp = v.e;
          s.inverse = exp2i(-s.derivative_exp);
        }
        Cx3 w = zero_step(Cx3{s.xr, s.xi, s.delta_exp}, Cx3{s.ar, s.ai, s.offset_exp});
        s.xr = w.re;
        s.xi = w.im;
        s.delta_exp = (int32_t)w.e;
        s.scale = exp2i(s.delta_exp);
        s.m = 1;
        s.n = s.n + 1;
        if (T) tr->start(s.n);  // this step's iterate is not recorded (sample.rs:444-446)
        double2 Z1 = __ldg(p.orbit + 1);
        s.Zr = Z1.x;
        s.Zi = Z1.y;
        if (L) {
          double2 rr = __ldg(p.fused + 3);
          s.r2a = rr.x;
          s.r2b = rr.y;
        }
      }
      double factor = exp2i(s.offset_exp - s.delta_exp);
      s.dc_r = s.ar * factor;
      s.dc_i = s.ai * factor;
    } else {
      s.xr = fr;
      s.xi = fi;
      s.m = 0;
      s.Zr = p.z0r;
      s.Zi = p.z0i;
      s.r2a = -1.0;
      s.r2b = -1.0;
    }
  } else if (EXT) {
    double magnitude = rmax(fabs(s.xr), fabs(s.xi));
    int32_t k = 0;
    if (magnitude > HI && s.delta_exp < 0)
      k = -s.delta_exp < 32 ? -s.delta_exp : 32;
    else if (magnitude < LO && magnitude != 0.0)
      k = -32;
    if (__builtin_expect(k != 0, 0)) {
      moved = true;
      double factor = exp2i(-k);
      s.xr = s.xr * factor;
      s.xi = s.xi * factor;
      s.delta_exp = s.delta_exp + k;
      s.scale = exp2i(s.delta_exp);
      double f = exp2i(s.offset_exp - s.delta_exp);
      s.dc_r = s.ar * f;
      s.dc_i = s.ai * f;
    }
  }
  if (moved) {  // the next iteration's z (sample.rs:331; number.rs:113 on the extended tier)
    s.fr = EXT ? s.Zr + s.scale * s.xr : s.Zr + s.xr;
    s.fi = EXT ? s.Zi + s.scale * s.xi : s.Zi + s.xi;
  } else {  // the same expressions on the same values
    s.fr = fr;
    s.fi = fi;
  }
  if (replaying) return false;  // sample.rs:470-472: the replay only re-walks iterates
  double check_r = EXT ? pr : s.xr, check_i = EXT ? pi : s.xi;
  bool judge = check_r * check_r + check_i * check_i > RES2 * f2;
  if (EXT) judge = judge && s.returns < 4;
  if (!judge) {
    if (EXT) {
      if (s.n >= s.chk) {
        save_point(s, fr, fi);
        s.sn = s.n;
        s.chk = s.chk >= 0x80000000u ? 0xffffffffu : s.chk * 2;
        relimit(p, s);
      }
    } else if (s.hold > 0) {
      if (s.n - s.sn >= s.hold) {  // sn <= n while hold > 0
        s.hold = 0;
        s.predicted = false;
        s.pending = true;
        relimit(p, s);
      }
    } else if (s.n >= s.chk) {
      s.pending = true;
      relimit(p, s);
    }
    return false;
  }
  double dist = fabs(fr - s.sr) + fabs(fi - s.si);
  if (EXT) {
    if (s.returns < 4 && dist < s.near) {
      if (contracting(p.orbit, p.last, s.m, check_r, check_i, s.ar * exp2i(s.offset_exp),
                      s.ai * exp2i(s.offset_exp), (uint64_t)(s.n - s.sn))) {
        res.kind = 2;
        return true;
      }
      s.returns += 1;
    }
    if (s.n >= s.chk) {
      save_point(s, fr, fi);
      s.sn = s.n;
      s.chk = s.chk >= 0x80000000u ? 0xffffffffu : s.chk * 2;
      relimit(p, s);
    }
    return false;
  }
  if (dist < s.near) {
    uint32_t period = s.n - s.sn;
    if (s.hold == period && s.mu.below_one()) {
      double mr, mi;
      s.mu.value(mr, mi);
      double gr = fr - s.sr, gi = fi - s.si;
      double er = mr - 1.0, ei = mi;
      double den = er * er + ei * ei;
      double qpr = s.sr - (gr * er + gi * ei) / den;
      double qpi = s.si - (gi * er - gr * ei) / den;
      double tol = rmin(0.1 * sqrt(den), 1e-2) * s.qstep + 16.0 * U * (fabs(s.sr) + fabs(s.si));
      if (s.predicted && fabs(qpr - s.qr) + fabs(qpi - s.qi) <= tol) {
        res.kind = 1;
        res.n = s.n;
        return true;
      }
      s.qr = qpr;
      s.qi = qpi;
      s.qstep = (fabs(gr) + fabs(gi)) / sqrt(den);
      s.predicted = true;
    } else {
      s.predicted = false;
    }
    s.hold = period;
    save_point(s, fr, fi);
    s.sn = s.n;
    s.pending = false;
    s.mu.reset();
    relimit(p, s);
    return false;
  }
  if (s.hold > 0) {
    if (s.n - s.sn < s.hold) return false;
    s.hold = 0;
    s.predicted = false;
    s.pending = true;
  }
  if (s.pending || s.n >= s.chk) {
    uint64_t np = next_pow2((uint64_t)s.n + 1);
    uint32_t np32 = np > 0xffffffffull ? 0xffffffffu : (uint32_t)np;
    s.chk = s.chk > np32 ? s.chk : np32;
    save_point(s, fr, fi);
    s.sn = s.n;
    s.pending = false;
  }
  relimit(p, s);
  return false;
}

// One iteration of the while loop of sample.rs:237-575 for one lane (the allocation-free
// kernel's form). Returns true when the sample has an outcome (written to res).
template <bool EXT, bool D, bool L>
__device__ __forceinline__ bool step(const Params &p, State<EXT> &s, Result &res) {
  if (s.n >= p.max_iter) {
    res.kind = 2;
    return true;
  }
  // next orbit point, loaded before the step's arithmetic so its latency overlaps it
  // (m < last here: a sample that reaches the last point rebases to Z_0)
  double2 Zn, Rn = make_double2(-1.0, -1.0);
  if (L) {
    Zn = __ldg(p.fused + 2 * (s.m + 1));
    Rn = __ldg(p.fused + 2 * (s.m + 1) + 1);
  } else {
    Zn = __ldg(p.orbit + s.m + 1);
  }
  uint32_t at = 0;
  const int lv = L ? find_block(p, s, at) : -1;
  if (lv >= 0)
    apply_block<EXT, D>(p, s, lv, at);
  else
    plain_update<EXT, D>(s);
  return post<EXT, D, L>(p, s, res, lv >= 0, Zn, Rn);
}

// A lane's BLA block found but not yet applied.
struct Waiting {
  bool on;
  int lv;
  uint32_t at;
};

// A warp's reserved queue slots [base, end): one atomic on the queue head takes 32
// consecutive slots (one tile), which the warp then hands to its idle lanes in order, so
// one round trip to the head serves a tile instead of each lane as it finishes, and
// neighbouring samples share a warp. Held slots start only as the warp's own lanes finish,
// so over the last eighth of the queue a warp takes just the slots its idle lanes need:
// there a long sample left waiting behind busy lanes would lengthen the launch's tail.
// Every lane holds the same copy.
struct Reservation {
  unsigned long long base = 0, end = 0;
  bool tail = false;  // within the last eighth of the queue
  // Slots for the `need` idle lanes (warp-uniform): false when the queue is spent;
  // otherwise the lanes of need with rank < count take first + rank.
  __device__ __forceinline__ bool take(unsigned long long *queue, unsigned long long total, unsigned need,
                                       unsigned lane, unsigned long long &first, unsigned &count) {
    if (base >= end) {
      const unsigned long long grab = tail ? (unsigned long long)__popc(need) : 32ull;
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(queue, grab);
      b = __shfl_sync(0xffffffffu, b, 0);
      if (b >= total) return false;
      base = b;
      end = b + grab < total ? b + grab : total;
      tail = total - b <= total / 8;
    }
    const unsigned long long left = end - base, want = (unsigned long long)__popc(need);
    count = (unsigned)(want < left ? want : left);
    first = base;
    base += count;
    return true;
  }
};

// One iteration for the active lanes of a warp (every lane of the warp calls it). A lane
// whose next operation is a BLA block waits until at least defer/32 of the warp's busy
// lanes wait or no lane steps plainly; the waiting lanes then apply their blocks together. The warp
// runs the block path for many lanes at a time instead of for one or two lanes on
// nearly every iteration, and each lane's own sequence of operations is unchanged.
template <bool EXT, bool D, bool L, bool B = false, bool T = false>
__device__ __forceinline__ bool warp_step(const Params &p, State<EXT> &s, Result &res, bool active, Waiting &w,
                                          uint32_t defer, StripeTrace *tr = nullptr) {
  bool upd = false, took = false, done = false;
  double2 Zn = make_double2(0.0, 0.0), Rn = make_double2(-1.0, -1.0);
  if (active && !w.on) {
    if (s.n >= (T ? s.limit : p.max_iter)) {
      if (T && s.replaying) {  // sample.rs:576-579: the replay gave up; from what was recorded
        tr->finish(tr->first_at, tr->first_r, tr->first_i, p.r2, p.stripe_window, p.stripe_freq);
        res = tr->first;
      } else {
        res.kind = 2;
      }
      done = true;
    } else {
      if (L) {
        Zn = __ldg(p.fused + 2 * (s.m + 1));
        Rn = __ldg(p.fused + 2 * (s.m + 1) + 1);
      } else {
        Zn = __ldg(p.orbit + s.m + 1);
      }
      // a lane that finds a block waits; its level is searched when the waiting lanes
      // apply their blocks together (nothing the search reads changes while it waits)
      if (L && !(T && s.replaying) && block_starts(s)) {
        w.on = true;
      } else {
        plain_update<EXT, D, B>(s, p.q);
        upd = true;
      }
    }
  }
  if (L) {
    const unsigned FULL = 0xffffffffu;
    const unsigned waiting = __ballot_sync(FULL, w.on);
    const unsigned stepping = __ballot_sync(FULL, upd);
    // the threshold is `defer` of 32 lanes, scaled to the lanes still busy (waiting or
    // stepping): once the queue runs dry and lanes go idle, a fixed threshold would hold
    // every waiting lane until the last plain-stepping lane finds a block
    const uint32_t busy = (uint32_t)__popc(waiting | stepping);
    const uint32_t thr = max(1u, (busy * defer) >> 5);
    if (waiting && ((uint32_t)__popc(waiting) >= thr || !stepping) && w.on) {
      w.lv = block_level(p, s, w.at);
      if (T)  // sample.rs:267-281: the block start, for a later replay
        tr->snap(StripeSnap{s.m, s.n, s.xr, s.xi, s.delta_exp, s.scale, s.dc_r, s.dc_i, 0}, s.n + (2u << w.lv));
      apply_block<EXT, D>(p, s, w.lv, w.at);
      w.on = false;
      upd = took = true;
    }
  }
  if (upd) done = post<EXT, D, L, B, T>(p, s, res, took, Zn, Rn, tr);
  return done;
}

// Series::eval (series.rs:247-271): Horner on x = dc / rho for p = sum b_k x^(k-1) and
// q = p'; delta = x p and, with D, dz/dc = (p + x q) / rho.
template <bool D>
__device__ __forceinline__ void series_start(const Params &p, double ar, double ai, double &xr, double &xi,
                                             double &dr, double &di) {
  const double sc = p.series_inv;
  const double ur = ar * sc, ui = ai * sc;
  double pr = 0.0, pi = 0.0, qr = 0.0, qi = 0.0;
  for (int k = (int)p.series_order - 1; k >= 0; --k) {
    const double2 c = __ldg(p.series_b + k);
    if (D) {
      const double nr = qr * ur - qi * ui + pr, ni = qr * ui + qi * ur + pi;
      qr = nr;
      qi = ni;
    }
    const double nr = pr * ur - pi * ui + c.x, ni = pr * ui + pi * ur + c.y;
    pr = nr;
    pi = ni;
  }
  xr = pr * ur - pi * ui;
  xi = pr * ui + pi * ur;
  if (D) {
    dr = (pr + qr * ur - qi * ui) * sc;
    di = (pi + qr * ui + qi * ur) * sc;
  } else {
    dr = 0.0;
    di = 0.0;
  }
}

// Start sample `slot` of the tile queue (one warp-sized tile per 32 slots, tiles in
// row-major order; 8x4 samples unless tuned). Returns
// false when the slot holds no sample to iterate (outside the grid, masked, or settled
// by the closed-form main-component test, whose result is written here).
template <bool EXT, bool D, bool L, bool B = false>
__device__ __forceinline__ void start_sample(const Params &p, State<EXT> &s, bool use_series, bool keep_counts);

template <bool EXT, bool D, bool L, bool S = false, bool B = false>
__device__ __forceinline__ int init(const Params &p, uint64_t slot, State<EXT> &s, Result &res) {
  uint64_t tile = slot >> 5;
  if (p.tile_order) tile = __ldg(p.tile_order + tile);  // queue position -> row-major tile
  uint32_t w = (uint32_t)slot & 31u;
  uint32_t tx = (uint32_t)(tile % p.tiles_x), ty = (uint32_t)(tile / p.tiles_x);
  uint32_t ii = (tx << p.tile_shift) + (w & ((1u << p.tile_shift) - 1u));
  uint32_t jj = ty * (32u >> p.tile_shift) + (w >> p.tile_shift);
  if (ii >= p.cols || jj >= p.rows) return 0;
  uint32_t i = p.first_col + ii, j = p.first_row + jj;
  uint32_t idx = j * p.nx + i;
  const uint64_t in = (uint64_t)jj * p.in_pitch + ii;  // inputs hold the window only
  if (p.mask && !p.mask[in]) return 0;
  s.idx = idx;
  double ux, uy;
  if (p.offsets) {
    double2 o = p.offsets[in];
    ux = o.x;
    uy = o.y;
  } else {  // view.rs:118-122
    double x = (double)i + 0.5 - p.half_x;
    double y = (double)j + 0.5 - p.half_y;
    ux = p.cosr * x + p.sinr * y;
    uy = p.sinr * x - p.cosr * y;
  }
  if (EXT) {  // grid.rs:709-723
    s.ar = ux * p.h_m;
    s.ai = uy * p.h_m;
    s.offset_exp = (int32_t)p.h_e;
  } else {
    s.ar = ux * p.h;
    s.ai = uy * p.h;
    s.offset_exp = 0;
    if (p.tier == 0 && in_main_components(p.c_re + s.ar, p.c_im + s.ai)) {  // sample.rs:187-189
      res.kind = 1;
      res.n = 0;
      return 2;
    }
  }
  start_sample<EXT, D, L, B>(p, s, S, false);
  return 1;
}

// The iteration state of a sample whose offset (ar, ai, offset_exp) and index are set:
// the ordinary start at Z_0, or the series start when one is given and use_series.
// keep_counts keeps the block counters (a retry from zero after a series start counts
// both runs, grid.rs:623-648).
template <bool EXT, bool D, bool L, bool B>
__device__ __forceinline__ void start_sample(const Params &p, State<EXT> &s, bool use_series, bool keep_counts) {
  s.xr = 0.0;
  s.xi = 0.0;
  s.delta_exp = EXT ? s.offset_exp : 0;
  s.scale = EXT ? exp2i(s.delta_exp) : 1.0;
  s.dc_r = s.ar;
  s.dc_i = s.ai;
  s.dr = 0.0;
  s.di = 0.0;
  s.derivative_exp = 0;
  s.inverse = 1.0;
  s.m = 0;
  s.n = 0;
  s.Zr = p.z0r;
  s.Zi = p.z0i;
  s.r2a = -1.0;
  s.r2b = -1.0;
  s.fr = EXT ? p.z0r + s.scale * 0.0 : p.z0r + 0.0;  // z of the first iteration
  s.fi = EXT ? p.z0i + s.scale * 0.0 : p.z0i + 0.0;
  save_point(s, 0.0, 0.0);
  s.chk = 16;
  s.replaying = false;
  s.limit = (uint32_t)p.max_iter;
  s.sn = EXT ? 0 : 8;
  s.returns = 0;
  s.pending = false;
  s.mu.reset();
  s.hold = 0;
  s.predicted = false;
  s.qr = 0.0;
  s.qi = 0.0;
  s.qstep = 0.0;
  s.adc = L ? sqrt(s.ar * s.ar + s.ai * s.ai) : 0.0;
  s.nucleus = (int32_t)p.nucleus;
  s.ct.reset();
  if (!keep_counts) {
    s.blocks = 0;
    s.skipped = 0;
    s.shift = 0.0;
  }
  if (!EXT && use_series && p.series_n > 0) {
    // sample.rs:191-228 from the series' state: n = m = series_n, the state is the first
    // Brent save (saves resume at the next power of two), no nucleus contraction
    series_start<D>(p, s.ar, s.ai, s.xr, s.xi, s.dr, s.di);
    const uint32_t m = p.series_n;
    s.m = m;
    s.n = m;
    if (L) {
      const double2 Z = __ldg(p.fused + 2 * m), R = __ldg(p.fused + 2 * m + 1);
      s.Zr = Z.x;
      s.Zi = Z.y;
      s.r2a = R.x;
      s.r2b = R.y;
    } else {
      const double2 Z = __ldg(p.orbit + m);
      s.Zr = Z.x;
      s.Zi = Z.y;
    }
    s.fr = s.Zr + s.xr;
    s.fi = s.Zi + s.xi;
    save_point(s, s.Zr + s.xr, s.Zi + s.xi);
    s.sn = m;
    const uint64_t np = next_pow2((uint64_t)m + 1);
    s.chk = np > 16 ? (uint32_t)np : 16u;
    s.nucleus = -1;
  }
  if (B) {  // sample.rs:221-229: radii from zero; a bounded render has no nucleus heuristic
    s.e = 0.0;
    s.ed = 0.0;
    s.rc = 16.0 * U * (fabs(s.ar) + fabs(s.ai)) + 1e-300;
    s.nucleus = -1;
  }
  relimit(p, s);
}

// Column encoder (store.rs:66-112, Bound absent) and raw state.
// store.rs:115-151 (B): Bounded evidence for an escaped sample with |z| = az, |dz/dc| = ad
// and radii ez, ed: the lower DE factor and the nu bound, or false unless the radii prove
// escape (|z| - ez > 2) and ed < ad / 2. CUDA's log / log1p / exp / exp2 (the columns
// within their ulps of the host's; byte-exact columns come from the raw radii).
__device__ __forceinline__ bool bounds(uint64_t n, double az, double ez, double ad, double ed, double &de_lo,
                                       double &bound) {
  const double lo = az - ez;
  if (!(lo > 2.0 && ed < 0.5 * ad)) return false;
  const double lnz = log(az), llo = log(lo), lhi = log(az + ez);
  const double nu = log1p(-log1p(-ez / az) / llo) / LN_2 + 8.0 * U * ((double)n + 8.0);
  const double g = lhi * exp2(-(double)n);
  de_lo = (lo * llo) / (az * lnz) * ad / (ad + ed) * exp(-g) * (1.0 - 4.0 / (lo * lo)) * (1.0 - 1e-6);
  const double de_hi = ((az + ez) * lhi) / (az * lnz) * ad / (ad - ed) * (1.0 + 1e-6);
  bound = nu * de_hi / de_lo * (1.0 + 1e-6);
  return true;
}

// nu, de and normal of an escaped sample (store.rs:66-112, 145-150; samples.rs:45-48):
// the Bounded evidence's lower DE factor de_lo scales de when bounded.
__device__ __forceinline__ void encode_columns(const Params &p, uint64_t idx, const Result &r, double z2,
                                               double log2z, bool bounded, double de_lo) {
  if (p.nu) p.nu[idx] = (double)r.n + 1.0 - log2(log2z);
  if (p.de) {  // store.rs:145-150
    double lnz = log2z * LN_2;
    double base = 2.0 * sqrt(z2) * lnz / (hypot(r.dr, r.di) * p.px_m);
    int64_t k = -(r.dexp + p.px_e);
    k = k < -4000 ? -4000 : (k > 4000 ? 4000 : k);
    const float d = (float)(base * exp2i(k / 2) * exp2i(k - k / 2));
    p.de[idx] = bounded ? (float)((double)d * de_lo) : d;
  }
  if (p.normal) {  // samples.rs:45-48 through view.rs:132-134
    double re = r.zr * r.dr + r.zi * r.di, im = r.zi * r.dr - r.zr * r.di;
    double x = p.cosr * re + p.sinr * im, y = p.sinr * re - p.cosr * im;
    double t = atan2(y, x) * (65536.0 / TAU);
    p.normal[idx] = (uint16_t)(int64_t)round(t);
  }
}

// A finished sample's outputs. R: only the raw state (status, count, class, z, dz/dc and
// its exponent, every pointer present) is stored here, and encode_kernel computes the
// columns of escaped samples afterwards from it, with all threads of a warp busy instead of
// the one lane that finishes.
template <bool B = false, bool T = false, bool R = false>
__device__ __forceinline__ void put(const Params &p, uint32_t sample, const Result &r, float stripe = 0.0f) {
  const uint32_t j = sample / p.nx, i = sample - j * p.nx;
  const uint64_t idx = (uint64_t)(j - p.first_row) * p.out_pitch + (i - p.first_col);
  if (p.status) p.status[idx] = 1;
  if (T && p.stripe_out) p.stripe_out[idx] = stripe;  // grid.rs:772: 0 unless escaped
  if (p.n_out) p.n_out[idx] = (uint32_t)(r.kind == 2 ? p.max_iter : r.n);
  if (r.kind != 0) {
    if (p.cls) p.cls[idx] = (uint8_t)(r.kind == 2 ? 2 : 1);
    return;
  }
  if (p.z_out) p.z_out[idx] = make_double2(r.zr, r.zi);
  if (p.dz_out) p.dz_out[idx] = make_double2(r.dr, r.di);
  if (p.dexp_out) p.dexp_out[idx] = r.dexp;
  if (R) {
    p.cls[idx] = 0;  // Escaped, heuristic evidence
    return;
  }
  double z2 = r.zr * r.zr + r.zi * r.zi;
  double log2z = 0.5 * log2(z2);
  double de_lo = 0.0, bnd = 0.0;
  bool bounded = false;
  if (B) {  // store.rs:88-106
    bounded = bounds(r.n, sqrt(z2), r.ez, hypot(r.dr, r.di), r.ed, de_lo, bnd);
    if (p.bound_out) p.bound_out[idx] = bounded ? (float)bnd : 0.0f;
    if (p.ez_out) p.ez_out[idx] = r.ez;
    if (p.ed_out) p.ed_out[idx] = r.ed;
  }
  if (p.cls) p.cls[idx] = bounded ? 4 : 0;  // Escaped | Bounded << 2
  encode_columns(p, idx, r, z2, log2z, bounded, de_lo);
}

// The columns of the escaped samples of a window whose persistent kernel stored only their
// raw state (put with R), samples t = start, start + stride, ... of the window: the same
// expressions as put.
__device__ __forceinline__ void encode_window(const Params &p, uint64_t start, uint64_t stride) {
  const uint64_t total = (uint64_t)p.rows * p.cols;
  for (uint64_t t = start; t < total; t += stride) {
    const uint64_t jj = t / p.cols, ii = t - jj * p.cols;
    const uint64_t idx = jj * p.out_pitch + ii;
    if (!p.status[idx] || p.cls[idx] != 0) continue;
    Result r;
    r.kind = 0;
    r.n = p.n_out[idx];
    const double2 z = p.z_out[idx], dz = p.dz_out[idx];
    r.zr = z.x;
    r.zi = z.y;
    r.dr = dz.x;
    r.di = dz.y;
    r.dexp = p.dexp_out[idx];
    const double z2 = r.zr * r.zr + r.zi * r.zi;
    encode_columns(p, idx, r, z2, 0.5 * log2(z2), false, 0.0);
  }
}

// One thread per sample of a frame job's window. (Templates, so that every translation unit
// including this header may hold them.)
template <int V = 0>
__global__ void encode_kernel(Params p) {
  encode_window(p, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

// The same for the jobs of a batch group after its persistent kernel: job blockIdx.y.
template <int V = 0>
__global__ void encode_jobs_kernel(const Params *__restrict__ jobs) {
  const Params &p = jobs[blockIdx.y];
  if (!(p.nu || p.de || p.normal)) return;
  encode_window(p, (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, (uint64_t)gridDim.x * blockDim.x);
}

// S: the series-start variant (ordinary tiers, jobs with an admitted series); the others
// compile without the series start and its retry.
// B: the bounded variant (ordinary tiers, derivative on, no BLA or series): error radii,
// Bounded evidence and the Bound column.
// T: the stripe variant: every lane holds a Stripe recorder and writes the Stripe column.
template <bool T>
struct TraceSlot {
  __device__ __forceinline__ StripeTrace *get() { return nullptr; }
};
template <>
struct TraceSlot<true> {
  StripeTrace t;
  __device__ __forceinline__ StripeTrace *get() { return &t; }
};

// The BLA variants outside B and T store finished samples' raw state only (put's R: every
// raw pointer present) and encode_kernel fills nu, de and normal afterwards (measured on the
// 1920x1080 frame at a 1e-100 nucleus: 40.1 -> 39.2 ms, its fixed-tier variant 35.7 -> 33.8
// ms; without BLA the 480x270 1e-12 frame ran 3% slower, so those variants encode as they
// finish).
template <bool EXT, bool D, bool L, bool S = false, bool B = false, bool T = false>
__global__ void __launch_bounds__(128, Occupancy<EXT>::blocks) perturb_kernel(Params p) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  State<EXT> s;
  Result res;
  Waiting w{false, -1, 0};
  bool active = false, exhausted = false;
  Reservation slots;
  TraceSlot<T> trace;
  StripeTrace *tr = trace.get();
  uint64_t t0 = p.deadline_ns ? globaltimer() : 0;
  unsigned long long n_samples = 0, iters = 0, blocks = 0, skipped = 0, fallback = 0, closed = 0;
  double shift = 0.0;
  // Series start (grid.rs:623-648): the iterations a sample's count leaves out. The prefix
  // on a first run from the series (> 0); after an unresolved first run retried from zero,
  // prefix - max_iter, so that the first run counts max_iter - prefix.
  int64_t bias = 0;
  auto finish = [&](uint32_t idx, const Result &r, uint64_t nblocks, uint64_t nskipped, double sh) {
    put<B, T, L && !B && !T>(p, idx, r, T && r.kind == 0 ? tr->value : 0.0f);
    uint64_t spent = (uint64_t)((int64_t)(r.kind == 2 ? p.max_iter : r.n) - bias);
    bias = 0;
    if (L) {
      spent = spent - nskipped + nblocks;
      blocks += nblocks;
      skipped += nskipped;
      bool cf = r.kind == 1 && r.n == 0;
      closed += cf;
      fallback += (nblocks == 0 && !cf);
      shift = fmax(shift, sh);
    }
    iters += spent;
    n_samples += 1;
  };
  for (;;) {
    unsigned need = __ballot_sync(FULL, !active);
    while (need && !exhausted) {
      if (p.deadline_ns) {
        uint64_t now = 0;
        if (lane == 0) now = globaltimer();
        now = __shfl_sync(FULL, now, 0);
        if (now - t0 > p.deadline_ns) {
          exhausted = true;
          if (lane == 0) atomicExch(p.timed_out, 1u);
          break;
        }
      }
      unsigned long long base = 0;
      unsigned take = 0;
      if (!slots.take(p.queue, p.total, need, lane, base, take)) {
        exhausted = true;
        break;
      }
      if (!active) {
        const unsigned rank = __popc(need & lt);
        const uint64_t slot = base + rank;
        if (rank < take) {
          int got = init<EXT, D, L, S, B>(p, slot, s, res);
          if (got == 1) {
            active = true;
            if (S) bias = p.series_n;
            if (T) {  // Job::one (grid.rs:630) and the loop's start (sample.rs:235)
              tr->begin();
              tr->start(s.n);
            }
          } else if (got == 2) {
            finish(s.idx, res, 0, 0, 0.0);
          }
        }
      }
      need = __ballot_sync(FULL, !active);
    }
    if (!__any_sync(FULL, active)) break;
    if (warp_step<EXT, D, L, B, T>(p, s, res, active, w, p.defer, tr)) {
      if (S && bias > 0 && res.kind == 2) {
        // an unresolved series start retries from zero, keeping the nucleus heuristic
        // (grid.rs:637-642); its count and blocks carry over
        bias -= (int64_t)p.max_iter;
        start_sample<EXT, D, L, B>(p, s, false, true);
        if (T) {  // grid.rs:638
          tr->begin();
          tr->start(s.n);
        }
      } else {
        finish(s.idx, res, s.blocks, s.skipped, s.shift);
        active = false;
      }
    }
  }
  // warp reduction of the counters, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) {
    n_samples += __shfl_down_sync(FULL, n_samples, o);
    iters += __shfl_down_sync(FULL, iters, o);
    blocks += __shfl_down_sync(FULL, blocks, o);
    skipped += __shfl_down_sync(FULL, skipped, o);
    fallback += __shfl_down_sync(FULL, fallback, o);
    closed += __shfl_down_sync(FULL, closed, o);
    shift = fmax(shift, __shfl_down_sync(FULL, shift, o));
  }
  if (lane == 0) {
    atomicAdd(&p.counters->samples, n_samples);
    atomicAdd(&p.counters->iterations, iters);
    if (L) {
      atomicAdd(&p.counters->blocks, blocks);
      atomicAdd(&p.counters->skipped, skipped);
      atomicAdd(&p.counters->fallback, fallback);
      atomicAdd(&p.counters->closed, closed);
      if (shift > 0.0 && !isnan(shift)) atomicMax(&p.counters->shift_bits, (unsigned long long)__double_as_longlong(shift));
    }
  }
}

}  // namespace fdk

namespace fdk {

// Batches: many jobs (frames, tiles, locations) in one persistent launch. Job j owns
// queue slots [starts[j], starts[j+1]); a lane takes a slot, finds its job by binary
// search, and runs the same init/step/put as the single-job kernel on that job's Params
// (read from global memory), so results equal fdc_render's bit for bit. Counters are
// kept per job, flushed with atomics when a lane moves to another job.
__device__ __forceinline__ uint32_t job_of(const unsigned long long *__restrict__ starts, uint32_t njobs,
                                           unsigned long long slot) {
  uint32_t lo = 0, hi = njobs;  // starts[lo] <= slot < starts[hi]
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (__ldg(starts + mid) <= slot) lo = mid;
    else hi = mid;
  }
  return lo;
}

struct LaneCounters {
  unsigned long long samples, iterations, blocks, skipped, fallback, closed;
  __device__ __forceinline__ void clear() { samples = iterations = blocks = skipped = fallback = closed = 0; }
  __device__ __forceinline__ void flush(Counters *c) {
    if (samples) atomicAdd(&c->samples, samples);
    if (iterations) atomicAdd(&c->iterations, iterations);
    if (blocks) atomicAdd(&c->blocks, blocks);
    if (skipped) atomicAdd(&c->skipped, skipped);
    if (fallback) atomicAdd(&c->fallback, fallback);
    if (closed) atomicAdd(&c->closed, closed);
    clear();
  }
};

template <bool EXT, bool D, bool L>
__global__ void __launch_bounds__(128, Occupancy<EXT>::blocks)
    perturb_batch_kernel(const Params *__restrict__ jobs, const unsigned long long *__restrict__ starts,
                         uint32_t njobs, unsigned long long total, unsigned long long *queue, Counters *per_job,
                         uint32_t defer) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  State<EXT> s;
  Result res;
  Waiting w{false, -1, 0};
  bool active = false, exhausted = false;
  uint32_t job = 0, counted = 0xffffffffu;
  Reservation slots;
  LaneCounters lc;
  lc.clear();
  // the BLA variants store a finished sample's raw state; encode_jobs_kernel computes the
  // columns afterwards (every raw pointer present: fdc_batch_create provides scratch)
  auto finish = [&](const Params &p, uint32_t idx, const Result &r, uint64_t nblocks, uint64_t nskipped) {
    put<false, false, L>(p, idx, r);
    if (counted != job) {
      if (counted != 0xffffffffu) lc.flush(per_job + counted);
      counted = job;
    }
    uint64_t spent = r.kind == 2 ? p.max_iter : r.n;
    if (L) {
      spent = spent - nskipped + nblocks;
      lc.blocks += nblocks;
      lc.skipped += nskipped;
      bool cf = r.kind == 1 && r.n == 0;
      lc.closed += cf;
      lc.fallback += (nblocks == 0 && !cf);
    }
    lc.iterations += spent;
    lc.samples += 1;
  };
  for (;;) {
    unsigned need = __ballot_sync(FULL, !active);
    while (need && !exhausted) {
      unsigned long long base = 0;
      unsigned take = 0;
      if (!slots.take(queue, total, need, lane, base, take)) {
        exhausted = true;
        break;
      }
      if (!active) {
        const unsigned rank = __popc(need & lt);
        const unsigned long long slot = base + rank;
        if (rank < take) {
          job = job_of(starts, njobs, slot);
          const Params &p = jobs[job];
          int got = init<EXT, D, L>(p, slot - __ldg(starts + job), s, res);
          if (got == 1) active = true;
          else if (got == 2) finish(p, s.idx, res, 0, 0);
        }
      }
      need = __ballot_sync(FULL, !active);
    }
    if (!__any_sync(FULL, active)) break;
    const Params &p = jobs[job];
    if (warp_step<EXT, D, L>(p, s, res, active, w, defer)) {
      finish(p, s.idx, res, s.blocks, s.skipped);
      active = false;
    }
  }
  if (counted != 0xffffffffu) lc.flush(per_job + counted);
}

}  // namespace fdk
