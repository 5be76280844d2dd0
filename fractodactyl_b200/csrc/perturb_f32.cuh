// The precision form of the perturbation kernel: the delta recurrence runs on FP32
// mantissas with one int exponent per sample (delta = w 2^e, rescaled by 2^32 only when
// the mantissa leaves [2^-32, 2^32]); FP64 stays on exactly four steps:
//   1. the rebase test |Z + delta| <= |delta| (sample.rs:412-418, extended-tier rule),
//   2. the bailout |Z + delta|^2 > R^2 and the smooth iteration's log-log (store.rs:86-99),
//   3. the BLA validity radius comparisons |delta|^2 < r^2 (bla.rs:234-249),
//   4. the derivative dz/dc for distance estimates (sample.rs:352-360).
// Periodicity, the nucleus contraction and Newton's cycle prediction run in FP32.
// Steps from an orbit point whose FP32 copy is not exact enough (|Z| < 2^-60: Z_0 and a
// nucleus's returns) and BLA block applications use wide-exponent FP64 arithmetic.
// Compiled with fused multiply-adds (this form is not bit-exact by design).
#pragma once
#include <cstdint>

#include "perturb_f64.cuh"

namespace fdk {

// Resident 128-thread blocks per SM the precision-form kernels are compiled for. The loop
// body carries both arithmetics, and instruction fetch bounded it: the rare paths below
// (delta renormalisation, wide-exponent sums, multiplier rescaling, the block's derivative
// renormalisation, Newton's cycle prediction) are out-of-line functions, one copy each
// instead of one per call site, which leaves 126 registers without spills at 4 blocks.
#ifndef FDK_MIN_BLOCKS_F32
#define FDK_MIN_BLOCKS_F32 4
#endif

// 32-byte orbit entry of the precision form: Z in f64, Z in f32 (NaN where |Z| < 2^-60),
// the squared radius of the 2-step block starting at m (or -1).
struct __align__(16) Entry32 {
  double zr, zi;
  float zr32, zi32;
  double r2a;
};

__device__ __forceinline__ float exp2f_int(int e) {  // 2^e as f32, 0 below the normal range
  return e < -126 ? 0.0f : (e > 127 ? __int_as_float(0x7f800000) : __int_as_float((e + 127) << 23));
}

// Multiplier / Contraction of sample.rs:600-698 on f32 mantissas with an int exponent.
struct MulF {
  float re, im;
  int exp;
  __device__ __forceinline__ void reset(float r = 1.0f) {
    re = r;
    im = 0.0f;
    exp = 0;
  }
  __device__ __forceinline__ void multiply(float r, float i) {
    float nr = re * r - im * i, ni = re * i + im * r;
    re = nr;
    im = ni;
    float a = fmaxf(fabsf(re), fabsf(im));
    if (!(a > 1e-18f && a < 1e18f) && a > 0.0f && isfinite(a)) *this = renorm(*this, a);
  }
  static __device__ __noinline__ MulF renorm(MulF m, float a) {
    int e = ilogbf(a);
    m.re = scalbnf(m.re, -e);
    m.im = scalbnf(m.im, -e);
    m.exp += e;
    return m;
  }
  // The same for an FP64 factor of any size (a BLA block's multiplier A can exceed f32's
  // range): scaled by a power of two into [1, 2) before the f32 product, the power carried
  // in the exponent, as Contraction::multiply scales its factors (sample.rs:672-681).
  __device__ __forceinline__ void multiply_wide(double r, double i) { *this = times_wide(*this, r, i); }
  static __device__ __noinline__ MulF times_wide(MulF m, double r, double i) {
    const double a = fmax(fabs(r), fabs(i));
    if (a == 0.0 || !isfinite(a)) {
      m.multiply((float)r, (float)i);
      return m;
    }
    const int k = floor_log2(a);
    const double h = exp2i(-(k / 2)), l = exp2i(-(k - k / 2));
    m.multiply((float)(r * h * l), (float)(i * h * l));
    m.exp += k;
    return m;
  }
  __device__ __forceinline__ bool below(float lim) const {  // |v|^2 < lim
    return isfinite(re) && isfinite(im) &&
           (exp < -64 || (exp <= 64 && ((double)re * re + (double)im * im) * exp2i(2 * exp) < lim));
  }
};

struct StateF {
  float wr, wi;        // delta mantissa
  float s32;           // 2^e (0 below f32's normal range)
  float dcr, dci;      // dc 2^-e
  float zr32, zi32;    // Z_m in f32 (NaN: take the exact step)
  float sr, si, qr, qi, qstep;
  int e;
  double s64;          // 2^e in f64
  double ar, ai;       // dc = a 2^oe
  int oe;
  double d2;           // |delta|^2 in f64 (physical), from the end of the previous iteration
  double fr, fi;       // z = Z_m + delta in f64
  double Zr, Zi, r2a;
  double dr, di, inverse;
  int64_t dexp;
  MulF mu, ct;
  bool ct_started;
  uint32_t n, chk, sn, hold, m, idx, blocks, skipped;
  uint32_t lim;  // relimit_f32()
  int nucleus;
  bool pending, predicted;
};

// delta = (re, im) 2^k (f64 mantissas, any k) into the f32 form, the exponent kept at or
// above oe - 64 so that dc 2^-e stays representable.
// The delta's f32 form as set_delta stores it (an out-of-line function: set_delta has
// several call sites, all rare).
struct DeltaF {
  float wr, wi, s32, dcr, dci;
  int e;
  double s64;
};

static __device__ __noinline__ DeltaF make_delta(double re, double im, int64_t k, int oe, double ar, double ai) {
  double a = fmax(fabs(re), fabs(im));
  int64_t e = k;
  if (a != 0.0 && isfinite(a)) e = k + ilogb(a);
  if (e < (int64_t)oe - 64) e = (int64_t)oe - 64;
  int64_t sh = k - e;  // re 2^k = (re 2^sh) 2^e, 2^sh applied in two factors
  double f1 = exp2i(sh / 2), f2 = exp2i(sh - sh / 2);
  DeltaF d;
  d.wr = (float)(re * f1 * f2);
  d.wi = (float)(im * f1 * f2);
  d.e = (int)e;
  d.s32 = exp2f_int(d.e);
  d.s64 = exp2i(d.e);
  double g = exp2i((int64_t)oe - d.e);
  d.dcr = (float)(ar * g);
  d.dci = (float)(ai * g);
  return d;
}

__device__ __forceinline__ void set_delta(StateF &s, double re, double im, int64_t k) {
  const DeltaF d = make_delta(re, im, k, s.oe, s.ar, s.ai);
  s.wr = d.wr;
  s.wi = d.wi;
  s.e = d.e;
  s.s32 = d.s32;
  s.s64 = d.s64;
  s.dcr = d.dcr;
  s.dci = d.dci;
}

// Sum of two wide-exponent complex terms (as sum2, sample.rs:1094-1114), with a zero
// term passed over: sum2 scales every term by 2^(e - top), and a zero term whose
// exponent lies more than 2046 above the other's (an orbit point that is 0 in f64 next
// to a delta far below f64's range) would give 0 * inf.
static __device__ __noinline__ Cx3 add3(Cx3 a, Cx3 b) {
  if (a.re == 0.0 && a.im == 0.0) return b;
  if (b.re == 0.0 && b.im == 0.0) return a;
  return sum2(a, b, a.e);
}

// delta = w 2^e as f64 (the physical delta of the FP64 steps): the f32 bits moved into
// an f64 with the exponent e added, exact; subnormal, zero and non-finite w, and results
// outside f64's normal range, take the conversion and a multiply by s64 = 2^e.
__device__ __forceinline__ double phys(float w, int e, double s64) {
  const uint32_t b = __float_as_uint(w);
  const uint32_t ef = (b >> 23) & 0xffu;
  const int E = (int)ef - 127 + e + 1023;
  if (ef - 1u < 254u && E >= 1 && E <= 2046) {
    const uint32_t hi = (b & 0x80000000u) | ((uint32_t)E << 20) | ((b & 0x7fffffu) >> 3);
    return __hiloint2double((int)hi, (int)(b << 29));
  }
  return (double)w * s64;
}

// Bla::find's iteration limit with n left out (relimit of the plain form).
// Views whose deltas can fall below f64's range (spacing under 2^-960): save points
// advance as the extended tier's do and a pending save never lifts the budget (blocks
// stop at the next power-of-two save point, sample.rs:246-263). Shallower views keep
// the ordinary tier's rule, whose longer blocks are faster.
__device__ __forceinline__ bool below_f64(const Params &p) { return p.h_e < -960; }

__device__ __forceinline__ void relimit_f32(const Params &p, StateF &s) {
  const bool open = s.pending && !below_f64(p);
  uint64_t cap = s.hold > 0 ? (uint64_t)s.sn + s.hold : (open ? ~0ull : (uint64_t)s.chk);
  uint64_t b = p.max_iter < cap ? p.max_iter : cap;
  if (s.nucleus >= 0 && (uint64_t)s.nucleus + 1 < b) b = (uint64_t)s.nucleus + 1;
  s.lim = (uint32_t)b;
}

// Whether Bla::find (on the FP64 |delta|^2 of the iteration's start, s.d2) finds a block.
__device__ __forceinline__ bool block_starts_f32(const StateF &s) {
  const uint32_t budget = s.lim > s.n ? s.lim - s.n : 0u;
  return (s.nucleus < 0 || s.m != 0) & (budget >= 2) & (s.d2 < s.r2a);
}

// The rest of Bla::find once block_starts_f32 holds: the level of the longest valid block.
__device__ __forceinline__ int block_level_f32(const Params &p, const StateF &s, uint32_t &at) {
  const uint32_t budget = s.lim > s.n ? s.lim - s.n : 0u;
  const double d2 = s.d2;
  const uint32_t k = s.m - 1u;
  at = k >> 1;
  const uint32_t tz = k == 0 ? 32u : (uint32_t)(__ffs((int)k) - 1);
  const uint32_t top = tz < p.bla_levels ? tz : p.bla_levels;
  constexpr uint32_t PRE = 4;  // levels 1..4
  double r[PRE];
  bool ok[PRE];
#pragma unroll
  for (uint32_t q = 0; q < PRE; ++q) {
    const uint32_t i = 1 + q, a = k >> (i + 1);
    ok[q] = i < top && (2u << i) <= budget && a < p.bla_count[i];
    r[q] = ok[q] ? __ldg(p.bla_r2 + p.bla_off[i] + a) : -1.0;
  }
  // the prefetched levels that pass, as bits; the block is the last level of the passing
  // run from level 1 up (the same level and index as testing them in order)
  uint32_t pass = 0;
#pragma unroll
  for (uint32_t q = 0; q < PRE; ++q) pass |= (uint32_t)(ok[q] && d2 < r[q]) << q;
  const uint32_t run = (uint32_t)__ffs((int)~pass) - 1u;  // bit PRE of ~pass is set: run <= PRE
  if (run > 0) at = k >> (1 + run);
  if (run < PRE) return (int)run;
  int lv = (int)PRE;
  for (uint32_t i = 1 + PRE; i < top; ++i) {
    if ((2ull << i) > budget) break;
    const uint32_t a = k >> (i + 1);
    if (a >= p.bla_count[i]) break;
    if (!(d2 < __ldg(p.bla_r2 + p.bla_off[i] + a))) break;
    lv = (int)i;
    at = a;
  }
  return lv;
}

// dz' = A dz + B with the renormalisations around it (sample.rs:296-323), out of line.
struct DzF {
  double dr, di, inverse;
  int64_t dexp;
};

static __device__ __noinline__ DzF block_dz(double dr, double di, int64_t dexp, double2 A, double2 B) {
  normalise(dr, di, dexp, INT64_MAX / 4);
  double inverse = exp2i(-dexp);
  double t = A.x * dr - A.y * di + B.x * inverse;
  di = A.x * di + A.y * dr + B.y * inverse;
  dr = t;
  normalise(dr, di, dexp, INT64_MAX / 4);
  return DzF{dr, di, exp2i(-dexp), dexp};
}

// delta' = A delta + B dc with wide exponents, dz' = A dz + B in FP64.
template <bool D>
__device__ __forceinline__ void apply_block_f32(const Params &p, StateF &s, int lv, uint32_t at) {
  const uint32_t b = p.bla_off[lv] + at;
  const double2 A = __ldg(p.bla_coef + 2 * b), B = __ldg(p.bla_coef + 2 * b + 1);
  const uint32_t len = 2u << lv;
  if (s.nucleus >= 0 && s.n >= 1) {
    s.ct.multiply_wide(A.x, A.y);
    s.ct_started = true;
  }
  if (s.hold > 0) s.mu.multiply_wide(A.x, A.y);
  if (D) {
    DzF z = block_dz(s.dr, s.di, s.dexp, A, B);
    s.dr = z.dr;
    s.di = z.di;
    s.dexp = z.dexp;
    s.inverse = z.inverse;
  }
  const double wr = s.wr, wi = s.wi;
  Cx3 ad{A.x * wr - A.y * wi, A.x * wi + A.y * wr, s.e};
  Cx3 bd{B.x * s.ar - B.y * s.ai, B.x * s.ai + B.y * s.ar, s.oe};
  Cx3 d = add3(ad, bd);
  set_delta(s, d.re, d.im, d.e);
  s.m += len;
  s.n += len;
  s.blocks += 1;
  s.skipped += len;
}

// One ordinary step: FP64 derivative on z = Z_m + delta (carried in fr, fi), FP32 delta.
template <bool D>
__device__ __forceinline__ void plain_update_f32(StateF &s) {
  if (s.nucleus >= 0 && s.n >= 1) {
    s.ct.multiply((float)(2.0 * s.fr), (float)(2.0 * s.fi));
    s.ct_started = true;
  }
  if (s.hold > 0) s.mu.multiply((float)(2.0 * s.fr), (float)(2.0 * s.fi));
  if (D) {  // FP64 derivative (sample.rs:352-360)
    double t = 2.0 * (s.fr * s.dr - s.fi * s.di) + s.inverse;
    s.di = 2.0 * (s.fr * s.di + s.fi * s.dr);
    s.dr = t;
    if (fmax(fabs(s.dr), fabs(s.di)) > HI) {
      s.dr = s.dr * LO;
      s.di = s.di * LO;
      s.dexp += 32;
      s.inverse = exp2i(-s.dexp);
    }
  }
  if (!isnan(s.zr32)) {
    // FP32: w' = 2 Z w + 2^e w^2 + dc 2^-e
    const float wr = s.wr, wi = s.wi;
    const float zwr = s.zr32 * wr - s.zi32 * wi, zwi = s.zr32 * wi + s.zi32 * wr;
    const float nwr = 2.0f * zwr + s.s32 * (wr * wr - wi * wi) + s.dcr;
    const float nwi = 2.0f * zwi + s.s32 * (2.0f * wr * wi) + s.dci;
    s.wr = nwr;
    s.wi = nwi;
    const float mag = fmaxf(fabsf(nwr), fabsf(nwi));
    if (mag > 4294967296.0f || (mag < 2.3283064e-10f && s.e > s.oe - 64)) set_delta(s, nwr, nwi, s.e);
  } else {
    // exact step at a tiny Z_m: 2 Z delta + delta^2 + dc with wide exponents
    const double wr = s.wr, wi = s.wi;
    Cx3 zd{2.0 * (s.Zr * wr - s.Zi * wi), 2.0 * (s.Zr * wi + s.Zi * wr), s.e};
    Cx3 dd{wr * wr - wi * wi, 2.0 * wr * wi, 2 * (int64_t)s.e};
    Cx3 a{s.ar, s.ai, s.oe};
    Cx3 t = add3(add3(zd, dd), a);
    set_delta(s, t.re, t.im, t.e);
  }
  s.m += 1;
  s.n += 1;
}

// Newton's prediction of the cycle's point from a near return (sample.rs:524-552 in FP32),
// out of line: the prediction, its step, and whether it lands within tolerance of the last.
struct Newton {
  float qr, qi, qstep;
  bool hit;
};

static __device__ __noinline__ Newton newton(MulF mu, float gr, float gi, float sr, float si, float oqr, float oqi,
                                             float oqstep, float size) {
  float sc = mu.exp < -60 ? 0.0f : exp2f_int(mu.exp < 60 ? mu.exp : 60);
  float mr = mu.re * sc, mi = mu.im * sc;
  float hr = gr - sr, hi = gi - si;
  float er = mr - 1.0f, ei = mi;
  float den = er * er + ei * ei;
  float qpr = sr - (hr * er + hi * ei) / den;
  float qpi = si - (hi * er - hr * ei) / den;
  float tol = fminf(0.1f * sqrtf(den), 1e-2f) * oqstep + 16.0f * 5.96e-8f * size;
  Newton n;
  n.hit = fabsf(qpr - oqr) + fabsf(qpi - oqi) <= tol;
  n.qr = qpr;
  n.qi = qpi;
  n.qstep = (fabsf(hr) + fabsf(hi)) / sqrtf(den);
  return n;
}

// After the update: next entry, FP64 bailout and rebase test, FP32 periodicity. nz/nr
// hold the entry m + 1 prefetched at the iteration's start (after a plain step); after a
// block (took) the entry at the new m is loaded here.
template <bool D, bool L>
__device__ __forceinline__ bool post_f32(const Params &p, const Entry32 *__restrict__ orbit, StateF &s,
                                         Result &res, bool took, double2 nz, double2 nr) {
  double2 Z = nz;
  if (took) {
    const double2 *e3 = reinterpret_cast<const double2 *>(orbit + s.m);
    Z = __ldg(e3);
    nr = __ldg(e3 + 1);
  }
  s.Zr = Z.x;
  s.Zi = Z.y;
  s.zr32 = __int_as_float((int)(__double_as_longlong(nr.x) & 0xffffffffll));
  s.zi32 = __int_as_float((int)(__double_as_longlong(nr.x) >> 32));
  s.r2a = nr.y;
  // FP64: the physical delta, z, the bailout and the rebase test
  const double pr = phys(s.wr, s.e, s.s64), pi = phys(s.wi, s.e, s.s64);
  const double fr = Z.x + pr, fi = Z.y + pi;
  const double f2 = fr * fr + fi * fi;
  if (f2 > p.r2) {
    res.kind = 0;
    res.n = s.n;
    res.zr = fr;
    res.zi = fi;
    res.dr = s.dr;
    res.di = s.di;
    res.dexp = s.dexp;
    return true;
  }
  if (s.nucleus >= 0 && s.n == (uint32_t)s.nucleus + 1) {
    if (s.ct_started && s.ct.below(1e-6f)) {
      res.kind = 1;
      res.n = s.n;
      return true;
    }
    s.nucleus = -1;
    relimit_f32(p, s);
  }
  const double delta2 = pr * pr + pi * pi;
  if (f2 <= delta2 || s.m == p.last) {  // rebase onto Z_0 (extended-tier rule)
    if (f2 > SQUARE_OK) {
      set_delta(s, fr, fi, 0);
    } else {  // z below f64's reach: Z + delta with wide exponents (sample.rs:421-429)
      const Cx3 t = add3(Cx3{Z.x, Z.y, 0}, Cx3{(double)s.wr, (double)s.wi, s.e});
      set_delta(s, t.re, t.im, t.e);
    }
    s.m = 0;
    s.Zr = p.z0r;
    s.Zi = p.z0i;
    s.zr32 = __int_as_float(0x7fc00000);  // Z_0 = 0: exact step
    s.zi32 = 0.0f;
    s.r2a = -1.0;
    const double xr = phys(s.wr, s.e, s.s64), xi = phys(s.wi, s.e, s.s64);
    s.d2 = xr * xr + xi * xi;
    s.fr = s.Zr + xr;
    s.fi = s.Zi + xi;
  } else {
    s.d2 = delta2;
    s.fr = fr;
    s.fi = fi;
  }
  // periodicity in FP32 (ordinary-tier rule, sample.rs:473-574) on the rebased delta
  const bool judge = s.d2 > RES2 * f2;
  if (!judge) {
    if (below_f64(p)) {
      // An unjudged save point advances as the extended tier's does (sample.rs:479-486).
      // Below f64's range no iterate is ever judged; an unlimited budget would then let
      // blocks run each sample to the orbit's last point, whose rebase onto z = Z_last
      // (delta below f64) would put every sample on the reference orbit.
      if (s.n >= s.chk) {
        s.sr = (float)fr;
        s.si = (float)fi;
        s.sn = s.n;
        s.chk = s.chk >= 0x80000000u ? 0xffffffffu : s.chk * 2;
        relimit_f32(p, s);
      }
    } else if (s.hold > 0) {
      if (s.n >= s.sn + s.hold) {
        s.hold = 0;
        s.predicted = false;
        s.pending = true;
        relimit_f32(p, s);
      }
    } else if (s.n >= s.chk) {
      s.pending = true;
      relimit_f32(p, s);
    }
    return false;
  }
  const float gr = (float)fr, gi = (float)fi;
  const float dist = fabsf(gr - s.sr) + fabsf(gi - s.si);
  const float size = fabsf(s.sr) + fabsf(s.si);
  if (dist < 1e-3f * size) {
    uint32_t period = s.n - s.sn;
    if (s.hold == period && s.mu.below(1.0f)) {
      const Newton nw = newton(s.mu, gr, gi, s.sr, s.si, s.qr, s.qi, s.qstep, size);
      if (s.predicted && nw.hit) {
        res.kind = 1;
        res.n = s.n;
        return true;
      }
      s.qr = nw.qr;
      s.qi = nw.qi;
      s.qstep = nw.qstep;
      s.predicted = true;
    } else {
      s.predicted = false;
    }
    s.hold = period;
    s.sr = gr;
    s.si = gi;
    s.sn = s.n;
    s.pending = false;
    s.mu.reset();
    relimit_f32(p, s);
    return false;
  }
  if (s.hold > 0) {
    if (s.n < s.sn + s.hold) return false;
    s.hold = 0;
    s.predicted = false;
    s.pending = true;
  }
  if (s.pending || s.n >= s.chk) {
    uint32_t np = (uint32_t)next_pow2((uint64_t)s.n + 1);
    s.chk = s.chk > np ? s.chk : np;
    s.sr = gr;
    s.si = gi;
    s.sn = s.n;
    s.pending = false;
  }
  relimit_f32(p, s);
  return false;
}

// One iteration of the precision form for the active lanes of a warp, with the block
// deferral of warp_step.
template <bool D, bool L>
__device__ __forceinline__ bool warp_step_f32(const Params &p, const Entry32 *__restrict__ orbit, StateF &s,
                                              Result &res, bool active, Waiting &w, uint32_t defer) {
  bool upd = false, took = false, done = false;
  double2 nz = make_double2(0.0, 0.0), nr = make_double2(0.0, -1.0);
  if (active && !w.on) {
    if (s.n >= p.max_iter) {
      res.kind = 2;
      done = true;
    } else {
      // speculative load of the next entry (m < last at the top of every iteration)
      const double2 *e2 = reinterpret_cast<const double2 *>(orbit + s.m + 1);
      nz = __ldg(e2);
      nr = __ldg(e2 + 1);
      // a lane that finds a block waits; its level is searched when the waiting lanes
      // apply their blocks together (nothing the search reads changes while it waits)
      if (L && block_starts_f32(s)) {
        w.on = true;
      } else {
        plain_update_f32<D>(s);
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
      w.lv = block_level_f32(p, s, w.at);
      apply_block_f32<D>(p, s, w.lv, w.at);
      w.on = false;
      upd = took = true;
    }
  }
  if (upd) done = post_f32<D, L>(p, orbit, s, res, took, nz, nr);
  return done;
}

template <bool D, bool L>
__device__ __forceinline__ int init_f32(const Params &p, uint64_t slot, StateF &s, Result &res) {
  uint64_t tile = slot >> 5;
  if (p.tile_order) tile = __ldg(p.tile_order + tile);  // queue position -> row-major tile
  uint32_t w = (uint32_t)slot & 31u;
  uint32_t tx = (uint32_t)(tile % p.tiles_x), ty = (uint32_t)(tile / p.tiles_x);
  uint32_t ii = (tx << p.tile_shift) + (w & ((1u << p.tile_shift) - 1u));
  uint32_t jj = ty * (32u >> p.tile_shift) + (w >> p.tile_shift);
  if (ii >= p.cols || jj >= p.rows) return 0;
  uint32_t i = p.first_col + ii, j = p.first_row + jj;
  uint32_t idx = j * p.nx + i;
  const uint64_t in = (uint64_t)jj * p.in_pitch + ii;
  if (p.mask && !p.mask[in]) return 0;
  s.idx = idx;
  double ux, uy;
  if (p.offsets) {
    double2 o = p.offsets[in];
    ux = o.x;
    uy = o.y;
  } else {
    double x = (double)i + 0.5 - p.half_x;
    double y = (double)j + 0.5 - p.half_y;
    ux = p.cosr * x + p.sinr * y;
    uy = p.sinr * x - p.cosr * y;
  }
  // dc = (ux, uy) h_m 2^h_e on every tier: the same value as the ordinary tiers' ux h
  // (scaling by 2^h_e is exact), kept as mantissa and exponent so that dc 2^-e stays in
  // f32's range however deep the view
  if (p.tier == 0 && in_main_components(p.c_re + ux * p.h, p.c_im + uy * p.h)) {
    res.kind = 1;
    res.n = 0;
    return 2;
  }
  s.ar = ux * p.h_m;
  s.ai = uy * p.h_m;
  s.oe = (int)p.h_e;
  set_delta(s, 0.0, 0.0, s.oe);
  s.d2 = 0.0;
  s.Zr = p.z0r;
  s.Zi = p.z0i;
  s.fr = s.Zr;
  s.fi = s.Zi;
  s.zr32 = __int_as_float(0x7fc00000);
  s.zi32 = 0.0f;
  s.r2a = -1.0;
  s.dr = s.di = 0.0;
  s.dexp = 0;
  s.inverse = 1.0;
  s.m = 0;
  s.n = 0;
  s.sr = s.si = 0.0f;
  s.chk = 16;
  s.sn = 8;
  s.pending = false;
  s.mu.reset();
  s.hold = 0;
  s.predicted = false;
  s.qr = s.qi = s.qstep = 0.0f;
  s.nucleus = (int)p.nucleus;
  s.ct.reset();
  s.ct_started = false;
  s.blocks = 0;
  s.skipped = 0;
  relimit_f32(p, s);
  return 1;
}

template <bool D, bool L>
__global__ void __launch_bounds__(128, FDK_MIN_BLOCKS_F32) perturb_f32_kernel(Params p, const Entry32 *__restrict__ orbit) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  StateF s;
  Result res;
  Waiting w{false, -1, 0};
  bool active = false, exhausted = false;
  uint64_t t0 = p.deadline_ns ? globaltimer() : 0;
  unsigned long long n_samples = 0, iters = 0, blocks = 0, skipped = 0, fallback = 0, closed = 0;
  // the BLA variants store a finished sample's raw state; encode_kernel computes its nu, de
  // and normal afterwards with full warps (the column code stays out of this loop)
  auto finish = [&](uint32_t idx, const Result &r, uint64_t nblocks, uint64_t nskipped) {
    put<false, false, L>(p, idx, r);
    uint64_t spent = r.kind == 2 ? p.max_iter : r.n;
    if (L) {
      spent = spent - nskipped + nblocks;
      blocks += nblocks;
      skipped += nskipped;
      bool cf = r.kind == 1 && r.n == 0;
      closed += cf;
      fallback += (nblocks == 0 && !cf);
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
          int got = init_f32<D, L>(p, slot, s, res);
          if (got == 1) active = true;
          else if (got == 2) finish(s.idx, res, 0, 0);
        }
      }
      need = __ballot_sync(FULL, !active);
    }
    if (!__any_sync(FULL, active)) break;
    if (warp_step_f32<D, L>(p, orbit, s, res, active, w, p.defer)) {
      finish(s.idx, res, s.blocks, s.skipped);
      active = false;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    n_samples += __shfl_down_sync(FULL, n_samples, o);
    iters += __shfl_down_sync(FULL, iters, o);
    blocks += __shfl_down_sync(FULL, blocks, o);
    skipped += __shfl_down_sync(FULL, skipped, o);
    fallback += __shfl_down_sync(FULL, fallback, o);
    closed += __shfl_down_sync(FULL, closed, o);
  }
  if (lane == 0) {
    atomicAdd(&p.counters->samples, n_samples);
    atomicAdd(&p.counters->iterations, iters);
    if (L) {
      atomicAdd(&p.counters->blocks, blocks);
      atomicAdd(&p.counters->skipped, skipped);
      atomicAdd(&p.counters->fallback, fallback);
      atomicAdd(&p.counters->closed, closed);
    }
  }
}

}  // namespace fdk

namespace fdk {

// Batch form of the precision kernel (see perturb_batch_kernel).
template <bool D, bool L>
__global__ void __launch_bounds__(128, FDK_MIN_BLOCKS_F32)
    perturb_f32_batch_kernel(const Params *__restrict__ jobs, const unsigned long long *__restrict__ starts,
                             uint32_t njobs, unsigned long long total, unsigned long long *queue, Counters *per_job,
                             uint32_t defer) {
  const unsigned FULL = 0xffffffffu;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  StateF s;
  Result res;
  Waiting w{false, -1, 0};
  bool active = false, exhausted = false;
  uint32_t job = 0, counted = 0xffffffffu;
  LaneCounters lc;
  lc.clear();
  // as the plain batch kernel: the BLA variants store raw state for encode_jobs_kernel
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
      int leader = __ffs((int)need) - 1;
      if ((int)lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(need));
      base = __shfl_sync(FULL, base, leader);
      if (base >= total) {
        exhausted = true;
        break;
      }
      if (!active) {
        unsigned long long slot = base + __popc(need & lt);
        if (slot < total) {
          job = job_of(starts, njobs, slot);
          const Params &p = jobs[job];
          int got = init_f32<D, L>(p, slot - __ldg(starts + job), s, res);
          if (got == 1) active = true;
          else if (got == 2) finish(p, s.idx, res, 0, 0);
        }
      }
      need = __ballot_sync(FULL, !active);
    }
    if (!__any_sync(FULL, active)) break;
    const Params &p = jobs[job];
    if (warp_step_f32<D, L>(p, (const Entry32 *)p.orbit32, s, res, active, w, defer)) {
      finish(p, s.idx, res, s.blocks, s.skipped);
      active = false;
    }
  }
  if (counted != 0xffffffffu) lc.flush(per_job + counted);
}

}  // namespace fdk
