// Host-side set-up of the perturbation route (include/fdhost.h): exact decimal centres,
// the fixed-point reference orbit, the view plane, the nucleus gate, the BLA table and
// the benchmark locations' nucleus recipe. Compiled with -ffp-contract=off so every f64
// result rounds as the reference's Rust does.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fdhost.h"
#include "route_internal.hpp"

using fdroute::exp2i;
using fdroute::exponent_field;

namespace {

thread_local std::string g_err;

typedef unsigned __int128 u128;

// ------------------------------------------------------------------------------------
// Exact decimals. Grammar of fd_fixed::Decimal::parse (crates/fd-fixed/src/decimal.rs:
// 20-49): [+-]digits[.digits][(e|E)[+-]digits], surrounding whitespace ignored.
struct Dec {
  bool neg = false;
  std::string digits;  // '0'..'9', most significant first
  int64_t exp10 = 0;
};

Dec parse_decimal(const char *text) {
  std::string s(text ? text : "");
  const std::string bad = "not a decimal number: \"" + s + "\"";
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) ++a;
  while (b > a && isspace((unsigned char)s[b - 1])) --b;
  Dec d;
  if (a < b && (s[a] == '-' || s[a] == '+')) d.neg = s[a++] == '-';
  size_t e = s.find_first_of("eE", a);
  size_t mant_end = e == std::string::npos || e >= b ? b : e;
  int64_t ex = 0;
  if (mant_end < b) {
    size_t i = mant_end + 1;
    bool eneg = false;
    if (i < b && (s[i] == '+' || s[i] == '-')) eneg = s[i++] == '-';
    if (i >= b) throw std::runtime_error(bad);
    u128 v = 0;
    for (; i < b; ++i) {
      if (s[i] < '0' || s[i] > '9') throw std::runtime_error(bad);
      v = v * 10 + (unsigned)(s[i] - '0');
      if (v > (u128)INT64_MAX + 1) throw std::runtime_error(bad);
    }
    if (!eneg && v > (u128)INT64_MAX) throw std::runtime_error(bad);
    ex = eneg ? (int64_t)(0 - (uint64_t)v) : (int64_t)v;
  }
  size_t frac_len = 0;
  bool seen_dot = false;
  for (size_t i = a; i < mant_end; ++i) {
    char c = s[i];
    if (c == '.' && !seen_dot) {
      seen_dot = true;
      continue;
    }
    if (c < '0' || c > '9') throw std::runtime_error(bad);
    d.digits.push_back(c);
    if (seen_dot) ++frac_len;
  }
  if (d.digits.empty()) throw std::runtime_error(bad);
  if ((__int128)ex - (__int128)frac_len < INT64_MIN) throw std::runtime_error(bad);
  d.exp10 = ex - (int64_t)frac_len;
  if (d.digits.find_first_not_of('0') == std::string::npos) d.neg = false;
  return d;
}

// log2 |d| to ~1e-15 (decimal.rs:52-59).
double log2_abs(const Dec &d) {
  size_t first = d.digits.find_first_not_of('0');
  if (first == std::string::npos) return -INFINITY;
  size_t n = d.digits.size() - first;
  double head = 0.0;
  for (size_t i = 0; i < n && i < 17; ++i) head = head * 10.0 + (double)(d.digits[first + i] - '0');
  double rest = n > 17 ? (double)(n - 17) : 0.0;
  return (std::log10(head) + rest + (double)d.exp10) * 3.321928094887362347870319429489390175864831393;
}

// ------------------------------------------------------------------------------------
// Sign-magnitude fixed point: L little-endian u64 limbs, the top one the integer part.
struct Fix {
  bool neg = false;
  std::vector<uint64_t> mag;
};

size_t limbs_for(uint64_t bits) { return 1 + (size_t)((bits + 63) / 64); }

// floor(|d| 2^(64 (L-1))) (decimal.rs:62-96): the digits as a big integer, scaled by
// 10^exp10 with the result's integer part required to fit one limb.
Fix to_fix(const Dec &d, size_t L) {
  std::vector<uint64_t> big{0};
  auto mul_add = [&](uint64_t m, uint64_t add) {
    u128 carry = add;
    for (auto &x : big) {
      u128 t = (u128)x * m + carry;
      x = (uint64_t)t;
      carry = t >> 64;
    }
    if (carry) big.push_back((uint64_t)carry);
  };
  static const uint64_t P10[20] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull, 10000000ull,
                                   100000000ull, 1000000000ull, 10000000000ull, 100000000000ull,
                                   1000000000000ull, 10000000000000ull, 100000000000000ull,
                                   1000000000000000ull, 10000000000000000ull, 100000000000000000ull,
                                   1000000000000000000ull, 10000000000000000000ull};
  for (size_t at = 0; at < d.digits.size(); at += 19) {
    size_t len = std::min<size_t>(19, d.digits.size() - at);
    uint64_t chunk = 0;
    for (size_t i = 0; i < len; ++i) chunk = chunk * 10 + (uint64_t)(d.digits[at + i] - '0');
    mul_add(P10[len], chunk);
  }
  int64_t e = d.exp10;
  while (e > 0) {
    int k = (int)std::min<int64_t>(e, 19);
    mul_add(P10[k], 0);
    e -= k;
    if (big.size() > 1) throw std::runtime_error("value too large for fixed point");
  }
  std::vector<uint64_t> v(L - 1, 0);
  v.insert(v.end(), big.begin(), big.end());
  while (e < 0) {
    int k = (int)std::min<int64_t>(-e, 19);
    u128 r = 0;
    for (size_t i = v.size(); i-- > 0;) {
      u128 cur = (r << 64) | v[i];
      v[i] = (uint64_t)(cur / P10[k]);
      r = cur % P10[k];
    }
    e += k;
    if (std::all_of(v.begin(), v.end(), [](uint64_t x) { return x == 0; })) break;
  }
  for (size_t i = L; i < v.size(); ++i)
    if (v[i]) throw std::runtime_error("value too large for fixed point");
  v.resize(L);
  Fix f;
  f.mag = v;
  f.neg = d.neg && std::any_of(v.begin(), v.end(), [](uint64_t x) { return x != 0; });
  return f;
}

// (m, e) with v = m 2^e from the top three limbs, rounded as fd_fixed::frexp does
// (crates/fd-fixed/src/lib.rs:75-83): top + next 2^-64 + third 2^-128 in f64, in that order.
bool frexp_fix(bool neg, const uint64_t *mag, size_t L, double &m, int64_t &e) {
  size_t k = L;
  while (k > 0 && mag[k - 1] == 0) --k;
  if (k == 0) return false;
  --k;
  double v = (double)mag[k] + (k >= 1 ? (double)mag[k - 1] : 0.0) * exp2i(-64) +
             (k >= 2 ? (double)mag[k - 2] : 0.0) * exp2i(-128);
  int64_t ve = exponent_field(v);
  double mm = v * exp2i(-ve);
  m = neg ? -mm : mm;
  e = ve + 64 * ((int64_t)k - ((int64_t)L - 1));
  return true;
}

// crates/fd-fixed/src/lib.rs:86-93
double fix_to_f64(bool neg, const uint64_t *mag, size_t L) {
  double m;
  int64_t e;
  if (!frexp_fix(neg, mag, L, m, e)) return 0.0;
  if (e < -1000) return m * exp2i(e + 100) * exp2i(-100);
  return m * exp2i(e);
}

// Magnitude arithmetic on L limbs.
inline int mag_cmp(const uint64_t *a, const uint64_t *b, size_t L) {
  for (size_t i = L; i-- > 0;)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}
inline void mag_add(const uint64_t *a, const uint64_t *b, uint64_t *o, size_t L) {
  u128 c = 0;
  for (size_t i = 0; i < L; ++i) {
    c += (u128)a[i] + b[i];
    o[i] = (uint64_t)c;
    c >>= 64;
  }
}
inline void mag_sub(const uint64_t *a, const uint64_t *b, uint64_t *o, size_t L) {
  uint64_t borrow = 0;
  for (size_t i = 0; i < L; ++i) {
    u128 t = (u128)a[i] - b[i] - borrow;
    o[i] = (uint64_t)t;
    borrow = (uint64_t)(t >> 64) & 1;
  }
}
inline bool nonzero(const uint64_t *a, size_t L) {
  for (size_t i = 0; i < L; ++i)
    if (a[i]) return true;
  return false;
}
// Signed sum; zero is never negative. Returns the sign of o.
inline bool sadd(bool an, const uint64_t *a, bool bn, const uint64_t *b, uint64_t *o, size_t L) {
  if (an == bn) {
    mag_add(a, b, o, L);
    return an && nonzero(o, L);
  }
  if (mag_cmp(a, b, L) < 0) {
    mag_sub(b, a, o, L);
    return bn;
  }
  mag_sub(a, b, o, L);
  return an && nonzero(o, L);
}

// o = floor(a^2 / 2^(64 (L-1))), from the full 2L-limb square in prod. The products
// a_i a_j with i < j are summed row by row (operand scanning: one 64-bit carry per row,
// so the multiplies of a row do not wait on each other's additions), doubled by a one-bit
// shift, and the squares a_i^2 added on the diagonal. Exact.
void square_trunc(const uint64_t *a, uint64_t *o, size_t L, uint64_t *prod) {
  uint64_t *r = prod;
  for (size_t k = 0; k < 2 * L; ++k) r[k] = 0;
  for (size_t i = 0; i + 1 < L; ++i) {
    const uint64_t ai = a[i];
    uint64_t c = 0;
    for (size_t j = i + 1; j < L; ++j) {
      const u128 t = (u128)ai * a[j] + r[i + j] + c;  // < 2^128: (2^64-1)^2 + 2 (2^64-1)
      r[i + j] = (uint64_t)t;
      c = (uint64_t)(t >> 64);
    }
    r[i + L] = c;
  }
  uint64_t top = 0;
  for (size_t k = 0; k < 2 * L; ++k) {
    const uint64_t v = r[k];
    r[k] = (v << 1) | top;
    top = v >> 63;
  }
  u128 c = 0;
  for (size_t i = 0; i < L; ++i) {
    const u128 p = (u128)a[i] * a[i];
    c += (u128)r[2 * i] + (uint64_t)p;
    r[2 * i] = (uint64_t)c;
    c >>= 64;
    c += (u128)r[2 * i + 1] + (uint64_t)(p >> 64);
    r[2 * i + 1] = (uint64_t)c;
    c >>= 64;
  }
  std::memcpy(o, r + (L - 1), L * sizeof(uint64_t));
}

// Spin on `ready` (a short pause per try), then yield: the thread being waited for is
// always making progress, so the wait ends.
template <class P>
void spin_until(P ready) {
  for (unsigned i = 0; !ready(); ++i) {
    if (i < 4096) {
#if defined(__x86_64__) || defined(__i386__)
      __builtin_ia32_pause();
#endif
    } else {
      std::this_thread::yield();
    }
  }
}

// Two helper threads for the squarings of a wide orbit step: the caller squares x while
// one helper squares y and the other x + y. The caller publishes a step's inputs by
// bumping `go`; each helper reports its square by storing that generation in its own
// `done`. The arithmetic is that of the serial step, so every orbit point is the same.
class SquareCrew {
 public:
  explicit SquareCrew(size_t L) : L_(L) {}
  ~SquareCrew() { stop(); }
  // Starts the helpers on (y -> y2) and (s -> s2); false (and no helper) if a thread
  // cannot be created.
  bool start(const uint64_t *y, uint64_t *y2, const uint64_t *s, uint64_t *s2) {
    try {
      threads_.emplace_back([this, y, y2] { run(0, y, y2); });
      threads_.emplace_back([this, s, s2] { run(1, s, s2); });
    } catch (...) {
      stop();
      return false;
    }
    return true;
  }
  void round() { go_.fetch_add(1, std::memory_order_release); }
  void wait() {
    const uint64_t g = go_.load(std::memory_order_relaxed);
    for (auto &d : done_) spin_until([&] { return d.v.load(std::memory_order_acquire) == g; });
  }
  void stop() {
    if (threads_.empty()) return;
    stop_.store(true, std::memory_order_relaxed);
    go_.fetch_add(1, std::memory_order_release);
    for (auto &t : threads_) t.join();
    threads_.clear();
  }

 private:
  void run(int k, const uint64_t *in, uint64_t *out) {
    std::vector<uint64_t> prod(2 * L_);
    uint64_t seen = 0;
    for (;;) {
      uint64_t g = 0;
      spin_until([&] { return (g = go_.load(std::memory_order_acquire)) != seen; });
      if (stop_.load(std::memory_order_relaxed)) return;
      seen = g;
      square_trunc(in, out, L_, prod.data());
      done_[k].v.store(g, std::memory_order_release);
    }
  }
  struct alignas(64) Counter {
    std::atomic<uint64_t> v{0};
  };
  size_t L_;
  std::vector<std::thread> threads_;
  alignas(64) std::atomic<uint64_t> go_{0};
  Counter done_[2];
  std::atomic<bool> stop_{false};
};

// Orbits of at least this many limbs (~1,700 bits) split each step's squarings over
// three threads when asked to (threads >= 3); below it two barrier crossings per step
// cost more than the squarings they share.
constexpr size_t CREW_MIN_LIMBS = 28;

// Z_{n+1} = Z_n^2 + C from Z_0 = 0 in L-limb fixed point with three squarings per step
// (x' = x^2 - y^2 + cr, y' = (x + y)^2 - x^2 - y^2 + ci, crates/fd-fixed/src/orbit.rs:
// 14-43), each point rounded to f64 by fix_to_f64; stops after `steps` points or at the
// first point with |Z|^2 > escape2. threads >= 3 runs the three squarings of a step in
// parallel on wide orbits.
uint64_t fixed_orbit(const Fix &cr, const Fix &ci, uint64_t steps, double escape2, double *re, double *im,
                     int threads) {
  const size_t L = cr.mag.size();
  // each array on cache lines of its own (the crew's threads write y2 and s2)
  const size_t W = (L + 7) & ~(size_t)7;
  std::vector<uint64_t> buf(7 * W + 8, 0);
  uint64_t *x = buf.data() + ((8 - ((uintptr_t)buf.data() / 8) % 8) % 8);
  uint64_t *y = x + W, *x2 = y + W, *y2 = x2 + W, *s = y2 + W, *s2 = s + W, *t = s2 + W;
  std::vector<uint64_t> prod(2 * L);
  bool xn = false, yn = false;
  SquareCrew crew(L);
  const bool par = threads >= 3 && L >= CREW_MIN_LIMBS && steps > 1 && crew.start(y, y2, s, s2);
  uint64_t n = 0;
  for (; n < steps;) {
    if (par) {
      sadd(xn, x, yn, y, s, L);
      crew.round();
      square_trunc(x, x2, L, prod.data());
      crew.wait();
    } else {
      square_trunc(x, x2, L, prod.data());
      square_trunc(y, y2, L, prod.data());
      sadd(xn, x, yn, y, s, L);
      square_trunc(s, s2, L, prod.data());
    }
    bool tn = sadd(false, x2, true, y2, t, L);
    xn = sadd(tn, t, cr.neg, cr.mag.data(), x, L);
    mag_add(x2, y2, s, L);
    tn = sadd(false, s2, true, s, t, L);
    yn = sadd(tn, t, ci.neg, ci.mag.data(), y, L);
    double fx = fix_to_f64(xn, x, L), fy = fix_to_f64(yn, y, L);
    re[n] = fx;
    im[n] = fy;
    ++n;
    if (fx * fx + fy * fy > escape2) break;
  }
  return n;
}

// ------------------------------------------------------------------------------------
// BLA blocks (crates/fd-kernel/src/bla.rs:35-129), stored as [f64; 7].
struct Blk {
  double ar, ai, br, bi, r, alpha, beta;
};

inline Blk blk_single(double zr, double zi, double eps) {  // bla.rs:72-85
  double az = std::hypot(zr, zi);
  double r = 2.0 * eps * az;
  if (!(r > 0.0 && az <= 2.0)) return Blk{0, 0, 0, 0, 0, 0, 0};
  return Blk{2.0 * zr + 0.0, 2.0 * zi + 0.0, 1.0, 0.0, r, r, 0.0};
}

inline double times_exp2(double v, int64_t e) {  // bla.rs:115-121
  return e >= -1022 ? v * exp2i(e) : v * exp2i(-1022) * exp2i(e + 1022);
}

inline double fmin_rust(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }

inline Blk blk_merge(const Blk &x, const Blk &y, double c, int64_t ce) {  // bla.rs:91-112
  if (x.r == 0.0 || y.r == 0.0) return Blk{0, 0, 0, 0, 0, 0, 0};
  double ax = std::hypot(x.ar, x.ai), ay = std::hypot(y.ar, y.ai);
  double ahat = ax + x.alpha;
  double bhat = std::hypot(x.br, x.bi) + x.beta;
  double r = fmin_rust(x.r, (y.r - times_exp2(bhat * c, ce)) / ahat);
  Blk z;
  z.ar = y.ar * x.ar - y.ai * x.ai + 0.0 + 0.0;
  z.ai = y.ar * x.ai + y.ai * x.ar + 0.0 + 0.0;
  z.br = y.ar * x.br - y.ai * x.bi + y.br + 0.0;
  z.bi = y.ar * x.bi + y.ai * x.br + y.bi + 0.0;
  z.r = r;
  z.alpha = ay * x.alpha + y.alpha * ahat;
  z.beta = ay * x.beta + y.alpha * bhat + y.beta;
  bool fin = std::isfinite(z.ar) && std::isfinite(z.ai) && std::isfinite(z.br) && std::isfinite(z.bi) &&
             std::isfinite(z.r) && std::isfinite(z.alpha) && std::isfinite(z.beta);
  if (r > 0.0 && fin) return z;
  return Blk{0, 0, 0, 0, 0, 0, 0};
}

template <class F>
void parallel_for(uint64_t n, int threads, F f) {
  if (threads <= 1 || n < 4096) {
    f(0, n);
    return;
  }
  std::vector<std::thread> pool;
  uint64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    uint64_t a = t * chunk, b = std::min<uint64_t>(n, a + chunk);
    if (a >= b) break;
    pool.emplace_back([=] { f(a, b); });
  }
  for (auto &th : pool) th.join();
}

template <class F>
bool parallel_any(uint64_t n, int threads, F f) {  // parallel_for whose parts return a flag: their OR
  if (threads <= 1 || n < 4096) return f(0, n);
  std::vector<std::thread> pool;
  std::vector<char> hit(threads, 0);
  uint64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    uint64_t a = t * chunk, b = std::min<uint64_t>(n, a + chunk);
    if (a >= b) break;
    pool.emplace_back([=, &hit] { hit[t] = f(a, b); });
  }
  for (auto &th : pool) th.join();
  return std::find(hit.begin(), hit.end(), 1) != hit.end();
}

inline void put_blk(double *dst, const Blk &b) { std::memcpy(dst, &b, sizeof(Blk)); }
inline Blk get_blk(const double *src) {
  Blk b;
  std::memcpy(&b, src, sizeof(Blk));
  return b;
}

// bla.rs:161-216: singles over Z_1..Z_steps, pairwise merges level by level, stopping
// before the first level without a valid block. The levels are written level-major into
// `out` ([f64; 7] blocks) as they are merged, each level from the one before it in place;
// the level that stops the build is written after the kept ones, so `out` needs room for
// steps - 1 blocks (the sum of steps >> i over i >= 1), steps = len - 2. False (with the
// error set) on invalid eps / dc_max.
bool bla_levels(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                       int threads, double *out, uint32_t &levels, uint64_t &total) {
  if (!(eps > 0.0 && eps <= 1.0 / (double)(1u << 24) && dc_max > 0.0 && std::isfinite(dc_max))) {
    g_err = "BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0";
    return false;
  }
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  const uint64_t steps = len >= 2 ? len - 2 : 0;
  uint64_t n = steps / 2, off = 0;
  // level 1 directly from pairs of singles
  bool valid = parallel_any(n, threads, [&](uint64_t a, uint64_t b) {
    bool any = false;
    for (uint64_t t = a; t < b; ++t) {
      const Blk z = blk_merge(blk_single(re[2 * t + 1], im[2 * t + 1], eps),
                              blk_single(re[2 * t + 2], im[2 * t + 2], eps), dc_max, dc_exp);
      put_blk(out + 7 * t, z);
      any |= z.r > 0.0;
    }
    return any;
  });
  levels = 0;
  total = 0;
  while (valid) {  // keep this level; merge the next from it
    levels += 1;
    total += n;
    const uint64_t m = n / 2, at = off + n;
    valid = parallel_any(m, threads, [&](uint64_t a, uint64_t b) {
      bool any = false;
      for (uint64_t t = a; t < b; ++t) {
        const Blk z = blk_merge(get_blk(out + 7 * (off + 2 * t)), get_blk(out + 7 * (off + 2 * t + 1)), dc_max, dc_exp);
        put_blk(out + 7 * (at + t), z);
        any |= z.r > 0.0;
      }
      return any;
    });
    off = at;
    n = m;
  }
  return true;
}

// Level offsets of a table built by bla_levels: level i starts after levels 0..i-1, each
// half the one before.
void bla_offsets(uint64_t len, uint32_t levels, uint64_t *level_offsets) {
  const uint64_t steps = len >= 2 ? len - 2 : 0;
  uint64_t at = 0, n = steps / 2;
  for (uint32_t i = 0; i < levels; ++i, n /= 2) {
    level_offsets[i] = at;
    at += n;
  }
  level_offsets[levels] = at;
}

// Fixed-point to decimal string with `digits` fraction digits (truncated).
std::string fix_to_string(const Fix &f, size_t digits) {
  const size_t L = f.mag.size();
  std::string out = f.neg ? "-" : "";
  out += std::to_string(f.mag[L - 1]);
  out += '.';
  std::vector<uint64_t> frac(f.mag.begin(), f.mag.end() - 1);
  while (digits > 0) {
    int k = (int)std::min<size_t>(digits, 19);
    uint64_t m = 1;
    for (int i = 0; i < k; ++i) m *= 10;
    u128 carry = 0;
    for (auto &x : frac) {
      u128 t = (u128)x * m + carry;
      x = (uint64_t)t;
      carry = t >> 64;
    }
    std::string part = std::to_string((uint64_t)carry);
    out += std::string(k - part.size(), '0') + part;
    digits -= k;
  }
  return out;
}

// Floating value m 2^e (|m| in [1, 2)) with a wide exponent, for derivatives that leave
// f64's range.
struct Fec {
  double re = 0, im = 0;
  int64_t e = 0;
};
inline Fec fec_norm(double re, double im, int64_t e) {
  double a = std::max(std::fabs(re), std::fabs(im));
  if (a == 0.0) return Fec{0, 0, 0};
  int k = std::ilogb(a);
  return Fec{std::scalbn(re, -k), std::scalbn(im, -k), e + k};
}

// v as a fixed-point magnitude with F = 64 (L-1) fraction bits (|v| = m 2^e < 2^63).
Fix fe_to_fix(double m, int64_t e, size_t L) {
  Fix f;
  f.mag.assign(L, 0);
  if (m == 0.0) return f;
  f.neg = m < 0;
  int k;
  double mm = std::frexp(std::fabs(m), &k);  // mm in [0.5, 1)
  uint64_t bits53 = (uint64_t)std::ldexp(mm, 53);
  int64_t shift = e + k - 53 + 64 * (int64_t)(L - 1);  // value = bits53 2^shift in units of 2^-F
  for (int b = 0; b < 53; ++b) {
    if (!((bits53 >> b) & 1)) continue;
    int64_t pos = shift + b;
    if (pos < 0 || pos >= (int64_t)(64 * L)) continue;
    f.mag[pos / 64] |= 1ull << (pos % 64);
  }
  return f;
}

}  // namespace

// ------------------------------------------------------------------------------------
// Guarded BLA (crates/fd-kernel/src/bla/guarded.rs:1-134): the BLA blocks with the
// affine uncertainty envelopes of the approximate GPU route's admission (alpha / beta on
// the state, derivative alpha / beta on dz/dc), built over the same reference with the
// reference's radii q[k]. Stored as [f64; 9]: the block's seven fields, then the two
// derivative envelopes.
struct GBlk {
  Blk b;
  double da, db;
};

inline double l1(double re, double im) { return std::fabs(re) + std::fabs(im); }  // guarded.rs:8-10
inline double up(double x) {  // guarded.rs:11-13
  return x * (1.0 + 64.0 * std::numeric_limits<double>::epsilon()) + std::numeric_limits<double>::min();
}

inline GBlk gblk_single(double zr, double zi, double q, double eps) {  // guarded.rs:35-50
  Blk b = blk_single(zr, zi, eps);
  if (b.r == 0.0 || !std::isfinite(q) || q < 0.0 || l1(zr, zi) + q > 2.0) return GBlk{};
  const double da = up(2.0 * b.r + 2.0 * q);
  b.alpha = up(b.r + 2.0 * q);
  return GBlk{b, da, 0.0};
}

inline GBlk gblk_merge(const GBlk &gx, const GBlk &gy, double c) {  // guarded.rs:51-98
  const Blk &x = gx.b, &y = gy.b;
  if (x.r == 0.0 || y.r == 0.0) return GBlk{};
  const double eps64 = std::numeric_limits<double>::epsilon();
  const double ax = l1(x.ar, x.ai), ay = l1(y.ar, y.ai), bx = l1(x.br, x.bi);
  const double r = fmin_rust(x.r, (y.r - up((bx + x.beta) * c)) / up(ax + x.alpha)) * (1.0 - 64.0 * eps64);
  GBlk z;
  z.b.ar = y.ar * x.ar - y.ai * x.ai + 0.0 + 0.0;  // affine(x.a, y.a, 0) (bla.rs:124-129)
  z.b.ai = y.ar * x.ai + y.ai * x.ar + 0.0 + 0.0;
  z.b.br = y.ar * x.br - y.ai * x.bi + y.br + 0.0;  // affine(x.b, y.a, y.b)
  z.b.bi = y.ar * x.bi + y.ai * x.br + y.bi + 0.0;
  z.b.r = r;
  const double ra = up(32.0 * eps64 * ay * ax);
  const double rb = up(32.0 * eps64 * (ay * bx + l1(y.br, y.bi)));
  // remainder(ay, ax, bx, xa, xb, ya, yb) (guarded.rs:14-19) for the state and derivative
  auto rem_a = [&](double xa, double ya) { return up(ay * xa + ya * (ax + xa)); };
  auto rem_b = [&](double xb, double ya, double yb) { return up(ay * xb + ya * (bx + xb) + yb); };
  z.b.alpha = up(rem_a(x.alpha, y.alpha) + ra);
  z.b.beta = up(rem_b(x.beta, y.alpha, y.beta) + rb);
  z.da = up(rem_a(gx.da, gy.da) + ra);
  z.db = up(rem_b(gx.db, gy.da, gy.db) + rb);
  const double v[9] = {z.b.ar, z.b.ai, z.b.br, z.b.bi, z.b.r, z.b.alpha, z.b.beta, z.da, z.db};
  bool fin = true;
  for (double t : v) fin = fin && std::isfinite(t);
  return (r > 0.0 && fin) ? z : GBlk{};
}

extern "C" {

const char *fdh_last_error(void) { return g_err.c_str(); }

int fdh_plane_new(const char *center_re, const char *center_im, const char *width, double rotation, uint32_t nx,
                  uint32_t ny, fdh_plane *out) {
  try {
    // crates/fd-kernel/src/view.rs:42-87
    if (nx == 0 || ny == 0) throw std::runtime_error("empty sample grid");
    Dec w = parse_decimal(width);
    double lw = log2_abs(w);
    if (w.neg || !std::isfinite(lw)) throw std::runtime_error("view width must be positive");
    double need = std::ceil(std::max(64.0 - lw, 64.0));
    Fix wf = to_fix(w, limbs_for((uint64_t)need));
    double wm;
    int64_t we;
    if (!frexp_fix(wf.neg, wf.mag.data(), wf.mag.size(), wm, we)) throw std::runtime_error("view width underflowed");
    double q = wm / (double)nx;
    int64_t qe = exponent_field(q);
    out->h_m = q * exp2i(-qe);
    out->h_e = we + qe;
    auto num = [](const char *s) {
      parse_decimal(s);
      return std::strtod(s, nullptr);
    };
    out->c_re = num(center_re);
    out->c_im = num(center_im);
    if (!(std::isfinite(out->c_re) && std::isfinite(out->c_im))) throw std::runtime_error("view centre out of range");
    double c_mag = std::max(std::max(std::fabs(out->c_re), std::fabs(out->c_im)), exp2i(-1022));
    bool f64_ok = std::log2(c_mag) - 52.0 <= (double)out->h_e - 10.0 && out->h_e > -1000;
    out->tier = f64_ok ? 0 : (out->h_e >= -900 ? 1 : 2);
    out->bits = (uint64_t)std::max<int64_t>(128 - out->h_e, 128);
    out->sin_rot = std::sin(rotation);
    out->cos_rot = std::cos(rotation);
    return 0;
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

int64_t fdh_orbit_fixed(const char *center_re, const char *center_im, uint64_t bits, uint64_t max_iter, double *re,
                        double *im, uint64_t cap) {
  return fdh_orbit_fixed_threads(center_re, center_im, bits, max_iter, re, im, cap, 1);
}

int64_t fdh_orbit_fixed_threads(const char *center_re, const char *center_im, uint64_t bits, uint64_t max_iter,
                                double *re, double *im, uint64_t cap, int threads) {
  try {
    uint64_t steps = std::min<uint64_t>(max_iter, (1ull << 20) - 1);
    if (cap < steps + 1) throw std::runtime_error("orbit buffers too small");
    size_t L = limbs_for(bits);
    Fix cr = to_fix(parse_decimal(center_re), L), ci = to_fix(parse_decimal(center_im), L);
    re[0] = 0.0;
    im[0] = 0.0;
    if (threads == 0) threads = std::thread::hardware_concurrency() >= 4 ? 3 : 1;
    return (int64_t)(1 + fixed_orbit(cr, ci, steps, 4294967296.0, re + 1, im + 1, threads));
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

int64_t fdh_orbit_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius, double *re, double *im,
                      uint64_t cap) {
  uint64_t steps = std::min<uint64_t>(max_iter, (1ull << 20) - 1);
  if (cap < steps + 1) {
    g_err = "orbit buffers too small";
    return -1;
  }
  // reference.rs:21-48
  double x = 0.0, y = 0.0, lim = escape_radius * escape_radius;
  re[0] = 0.0;
  im[0] = 0.0;
  uint64_t n = 1;
  for (uint64_t s = 0; s < steps; ++s) {
    double t = x * x - y * y + c_re;
    y = 2.0 * x * y + c_im;
    x = t;
    re[n] = x;
    im[n] = y;
    ++n;
    if (x * x + y * y > lim) break;
  }
  return (int64_t)n;
}

int64_t fdh_nucleus_period(const double *re, const double *im, uint64_t len) {
  // reference.rs:102-120
  if (len < 2) return -1;
  double record = std::hypot(re[1], im[1]);
  double log_beta = 0.0;
  for (uint64_t p = 2; p < len / 2; ++p) {
    double previous = std::hypot(re[p - 1], im[p - 1]);
    log_beta += 1.0 + std::log2(previous);
    double radius = std::hypot(re[p], im[p]);
    if (radius > 1e-140 && radius < 1e-24 && radius < record * 1e-12 && 1.0 + log_beta + std::log2(radius) < -40.0 &&
        std::hypot(re[2 * p], im[2 * p]) <= 2.0 * radius)
      return (int64_t)p;
    record = fmin_rust(record, radius);
  }
  return -1;
}

int fdh_bla_build(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                  int threads, double *blocks7, uint64_t *level_offsets, uint32_t *levels, uint64_t *blocks) {
  const uint64_t steps = len >= 2 ? len - 2 : 0;
  std::vector<double> buf(7 * std::max<uint64_t>(steps, 1));
  if (!bla_levels(re, im, len, eps, dc_max, dc_exp, threads, buf.data(), *levels, *blocks)) return -1;
  if (blocks7) {
    std::memcpy(blocks7, buf.data(), *blocks * sizeof(Blk));
    if (level_offsets) bla_offsets(len, *levels, level_offsets);
  }
  return 0;
}

int fdh_bla_build_into(const double *re, const double *im, uint64_t len, double eps, double dc_max, int64_t dc_exp,
                       int threads, double *blocks7, uint64_t cap_blocks, uint64_t *level_offsets, uint32_t cap_levels,
                       uint32_t *levels, uint64_t *blocks) {
  const uint64_t steps = len >= 2 ? len - 2 : 0;
  if (!level_offsets || (steps >= 2 && !blocks7)) {
    g_err = "null BLA buffers";
    return -1;
  }
  uint32_t lv = 0;
  uint64_t total = 0;
  if (cap_blocks >= steps) {  // room for every level the build writes: build in place
    if (!bla_levels(re, im, len, eps, dc_max, dc_exp, threads, blocks7, lv, total)) return -1;
  } else {
    std::vector<double> buf(7 * std::max<uint64_t>(steps, 1));
    if (!bla_levels(re, im, len, eps, dc_max, dc_exp, threads, buf.data(), lv, total)) return -1;
    if (total <= cap_blocks && lv <= cap_levels) std::memcpy(blocks7, buf.data(), total * sizeof(Blk));
  }
  *levels = lv;
  *blocks = total;
  if (total > cap_blocks || lv > cap_levels) {
    g_err = "BLA table larger than the buffers given";
    return -1;
  }
  bla_offsets(len, lv, level_offsets);
  return 0;
}

// GuardedBla::build (guarded.rs:110-134): singles over Z_1..Z_{len-2} with their radii
// q, pairwise merges level by level, the levels kept up to the first without a valid block;
// level-major [f64; 9] blocks (level i: (len - 2) >> (i + 1) of them).
int fdh_guarded_bla_build(const double *re, const double *im, const double *q, uint64_t len, double eps,
                          double dc_max, double *blocks9, uint64_t cap_blocks, uint64_t *level_offsets,
                          uint32_t cap_levels, uint32_t *levels, uint64_t *blocks) {
  if (!(eps > 0.0 && eps <= 1.0 / (double)(1u << 24) && dc_max > 0.0 && std::isfinite(dc_max))) {
    g_err = "BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0";
    return -1;
  }
  if (!re || !im || !q || !levels || !blocks || !level_offsets) {
    g_err = "null guarded BLA argument";
    return -1;
  }
  for (uint64_t k = 0; k < len; ++k)
    if (!std::isfinite(q[k]) || q[k] < 0.0) {
      g_err = "guarded BLA needs one finite nonnegative reference radius per point";
      return -1;
    }
  std::vector<GBlk> next;
  for (uint64_t k = 1; k + 1 < len; ++k) next.push_back(gblk_single(re[k], im[k], q[k], eps));
  uint32_t lv = 0;
  uint64_t total = 0;
  std::vector<GBlk> kept;
  std::vector<uint64_t> offs;
  for (;;) {
    std::vector<GBlk> merged(next.size() / 2);
    bool any = false;
    for (size_t t = 0; t < merged.size(); ++t) {
      merged[t] = gblk_merge(next[2 * t], next[2 * t + 1], dc_max);
      any = any || merged[t].b.r > 0.0;
    }
    next.swap(merged);
    if (!any) break;
    offs.push_back(total);
    kept.insert(kept.end(), next.begin(), next.end());
    total += next.size();
    ++lv;
  }
  *levels = lv;
  *blocks = total;
  if (total > cap_blocks || lv + 1 > cap_levels || (total && !blocks9)) {
    g_err = "guarded BLA table larger than the buffers given";
    return -1;
  }
  for (uint64_t t = 0; t < total; ++t) {
    const GBlk &g = kept[t];
    const double v[9] = {g.b.ar, g.b.ai, g.b.br, g.b.bi, g.b.r, g.b.alpha, g.b.beta, g.da, g.db};
    std::memcpy(blocks9 + 9 * t, v, sizeof v);
  }
  for (uint32_t i = 0; i < lv; ++i) level_offsets[i] = offs[i];
  level_offsets[lv] = total;
  return 0;
}

// external_escape_ok (crates/fd-kernel/src/store.rs:152-198): whether an externally
// computed escaped state (n, z, dz/dc = (dr, di) 2^dexp) with error radii ez (z units)
// and ed (derivative-mantissa units) encodes within half the comparison budget (1e-3 px,
// 0.2% DE, 0.2 degrees) for the output pixel px_m 2^px_e; the Bounded evidence of
// store.rs:115-151 and de_px of store.rs:153-160, with the host's libm. 1 or 0.
int fdh_external_escape_ok(uint64_t n, double zr, double zi, double dr, double di, int64_t dexp, double ez, double ed,
                           double px_m, int64_t px_e) {
  const double U = std::numeric_limits<double>::epsilon() / 2.0;
  const double LN_2 = 0.693147180559945309417232121458176568;
  const double TAU = 6.28318530717958647692528676655900577;
  const double az = std::hypot(zr, zi), ad = std::hypot(dr, di);
  if (!(ez >= 0.0 && ed >= 0.0 && std::isfinite(ez) && std::isfinite(ed) && std::isfinite(az) && std::isfinite(ad)))
    return 0;
  // bounds (store.rs:115-151)
  const double lo = az - ez;
  if (!(lo > 2.0 && ed < 0.5 * ad)) return 0;
  const double lnz = std::log(az), llo = std::log(lo), lhi = std::log(az + ez);
  const double nu = std::log1p(-std::log1p(-ez / az) / llo) / LN_2 + 8.0 * U * ((double)n + 8.0);
  const double g = lhi * std::exp2(-(double)n);
  const double de_lo0 = (lo * llo) / (az * lnz) * ad / (ad + ed) * std::exp(-g) * (1.0 - 4.0 / (lo * lo)) * (1.0 - 1e-6);
  const double de_hi0 = ((az + ez) * lhi) / (az * lnz) * ad / (ad - ed) * (1.0 + 1e-6);
  const double blo = de_lo0, bound = nu * de_hi0 / de_lo0 * (1.0 + 1e-6);
  // de_px (store.rs:153-160) at log2 |z|
  const double lnz2 = std::log2(az) * LN_2;
  const double base0 = 2.0 * az * lnz2 / (std::hypot(dr, di) * px_m);
  int64_t kk = -(dexp + px_e);
  kk = std::max<int64_t>(-4000, std::min<int64_t>(4000, kk));
  const double de = (double)(float)(base0 * exp2i(kk / 2) * exp2i(kk - kk / 2));
  const double displacement = bound * de * blo * LN_2 / 2.0;
  const double base = az * std::log(az);
  const double de_hi = (az + ez) * std::log(az + ez) / base * ad / (ad - ed);
  const double de_lo = (az - ez) * std::log(az - ez) / base * ad / (ad + ed);
  const double angle = std::asin(ez / az) + std::asin(ed / ad);
  const double f32eps = (double)std::numeric_limits<float>::epsilon();
  return std::isfinite(displacement) && displacement <= 5e-4 && std::isfinite(de) && de_hi - 1.0 + f32eps <= 1e-3 &&
         1.0 - de_lo + f32eps <= 1e-3 && angle + TAU / 65536.0 <= 0.1 * (TAU / 360.0);
}

// Reference::error_radius (crates/fd-kernel/src/reference.rs:122-148): bounds
// q[m] >= |A_m - Z_m| on each stored point's distance from the exact orbit A of the exact
// centre. A fixed-point orbit (bits >= 0) carries its three truncated squares and the
// centre's truncation, each under 2^-bits, plus the rounding to f64; an f64 orbit
// (bits < 0) from the correctly rounded centre (c_re, c_im) carries the roundings of
// x^2 - y^2 + c and 2xy + c and of the centre.
int fdh_error_radius(const double *re, const double *im, uint64_t len, int64_t bits, double c_re, double c_im,
                     double *q) {
  const double U = 1.1102230246251565e-16, MIN_POSITIVE = 2.2250738585072014e-308;
  if (len && (!re || !im || !q)) {
    g_err = "null orbit or output";
    return -1;
  }
  const double c1 = std::fabs(c_re) + std::fabs(c_im);
  const bool fixed = bits >= 0;
  double unit = fixed ? exp2i(4 - bits) : 0.0;
  if (fixed && !(unit > MIN_POSITIVE)) unit = MIN_POSITIVE;
  double a = 0.0;  // |A_m - F_m|, F the orbit as computed before its rounding to f64
  for (uint64_t m = 0; m < len; ++m) {
    const double s = std::sqrt(re[m] * re[m] + im[m] * im[m]) * (1.0 + 4.0 * U);
    const double round = fixed ? 2.0 * U * s + MIN_POSITIVE : 0.0;
    const double defect = fixed ? unit : 8.0 * U * (s * s + c1) + 2.0 * U * c1 + MIN_POSITIVE;
    q[m] = a + round;
    a = (a * (2.0 * (s + round) + a) + defect) * (1.0 + 8.0 * U);
  }
  return 0;
}

// Series::build (crates/fd-kernel/src/series.rs:86-245) with SeriesConfig::default()
// (series.rs:43-55): the coefficients b_k of delta_n(x) = sum b_k x^k, x = dc / rho, are
// stepped with the orbit (b_1' = 2 Z b_1 + rho, b_k' = 2 Z b_k + sum_{i+j=k} b_i b_j) over
// the first `active` orders, with majorants E (state) and F (its x-derivative) of what the
// truncation omits; the last step whose error maps to at most shift_px output pixels is
// admitted, then orders whose norms fit in half the remaining slack are trimmed. Every
// expression is the reference's, in its order (the start decides each sample's outcome).
int fdh_series_build(const double *re, const double *im, uint64_t len, double rho, double pixel, uint64_t max_iter,
                     uint64_t stalled_steps, fdh_series *out, double *coeffs, uint32_t cap_order) {
  const size_t start_order = 8, max_order = 64;
  const double grow_at = 1e-4, shift_px = 1e-8, derivative_rel = 1e-6;
  try {
    std::memset(out, 0, sizeof(*out));
    out->rho = rho;
    out->points = len;
    std::strncpy(out->stop, "reference", sizeof(out->stop) - 1);
    const size_t k_max = max_order;
    size_t active = start_order;
    std::vector<double> br(k_max + 1, 0.0), bi(k_max + 1, 0.0), sq_r(2 * k_max + 1, 0.0), sq_i(2 * k_max + 1, 0.0);
    std::vector<double> keep_r, keep_i;  // the admitted step's b_1..b_active
    double e = 0.0, f = 0.0;
    bool have = false;
    uint64_t best_n = 0;
    double best_e = 0, best_f = 0, best_budget_e = 0, best_budget_f = 0, best_dmin = 0;
    const uint64_t limit = std::min(len >= 2 ? len - 2 : 0, max_iter >= 1 ? max_iter - 1 : 0);
    auto set_stop = [&](const char *why) { std::strncpy(out->stop, why, sizeof(out->stop) - 1); };
    if (!(rho > 0.0 && std::isfinite(rho) && pixel > 0.0)) {
      set_stop("radius");
      return 0;
    }
    const double cap_e = shift_px * pixel * 2.0 / rho, cap_f = derivative_rel * 2.0;
    for (uint64_t n = 0; n < limit; ++n) {
      const double zr = re[n], zi = im[n];
      const double az = std::hypot(zr, zi);
      std::fill(sq_r.begin(), sq_r.begin() + 2 * active + 1, 0.0);
      std::fill(sq_i.begin(), sq_i.begin() + 2 * active + 1, 0.0);
      for (size_t i = 1; i <= active; ++i) {  // the square of the active polynomial
        const double ar = br[i], ai = bi[i];
        if (ar == 0.0 && ai == 0.0) continue;
        sq_r[2 * i] += ar * ar - ai * ai;
        sq_i[2 * i] += 2.0 * ar * ai;
        const double tr = 2.0 * ar, ti = 2.0 * ai;
        for (size_t j = i + 1; j <= active; ++j) {
          sq_r[i + j] += tr * br[j] - ti * bi[j];
          sq_i[i + j] += tr * bi[j] + ti * br[j];
        }
      }
      out->coefficient_pairs += (uint64_t)(active * (active + 1) / 2);
      double mag = 0.0, dmag = 0.0, omit = 0.0, domit = 0.0;
      for (size_t k = 1; k <= active; ++k) {
        const double a = std::hypot(br[k], bi[k]);
        mag += a;
        dmag += (double)k * a;
      }
      for (size_t k = active + 1; k <= 2 * active; ++k) {  // the square's omitted orders
        const double a = std::hypot(sq_r[k], sq_i[k]);
        omit += a;
        domit += (double)k * a;
      }
      const double e_next = 2.0 * (az + mag) * e + e * e + omit;
      f = 2.0 * (az + mag + e) * f + 2.0 * e * dmag + domit;
      e = e_next;
      for (size_t k = 1; k <= active; ++k) {
        const double xr = br[k], xi = bi[k];
        br[k] = 2.0 * (zr * xr - zi * xi) + sq_r[k];
        bi[k] = 2.0 * (zr * xi + zi * xr) + sq_i[k];
      }
      br[1] += rho;
      const uint64_t step = n + 1;  // the state after step n + 1
      out->built_steps = step;
      double m1 = 0.0, tail_d = 0.0;
      for (size_t k = 1; k <= active; ++k) {
        const double a = std::hypot(br[k], bi[k]);
        m1 += a;
        if (k >= 2) tail_d += (double)k * a;
      }
      if (!(std::isfinite(e) && std::isfinite(f))) {
        set_stop("non-finite");
        break;
      }
      if (std::hypot(re[step], im[step]) + m1 + e >= 2.0) {
        set_stop("escape");
        break;
      }
      const double dmin = std::hypot(br[1], bi[1]) - tail_d - f;
      const double budget = dmin > 0.0 ? shift_px * pixel * dmin / rho : 0.0;
      if (dmin > 0.0 && e <= budget && f <= derivative_rel * dmin) {
        have = true;
        best_n = step;
        keep_r.assign(br.begin() + 1, br.begin() + 1 + active);
        keep_i.assign(bi.begin() + 1, bi.begin() + 1 + active);
        best_e = e;
        best_f = f;
        best_budget_e = budget;
        best_budget_f = derivative_rel * dmin;
        best_dmin = dmin;
      } else if (e > cap_e || f > cap_f) {
        set_stop("budget");
        break;
      }
      if (active < k_max && e > grow_at * budget) {
        active = std::min(2 * active, k_max);
        out->growth_count += 1;
      }
      if (stalled_steps > 0 && have && step - best_n >= stalled_steps) {
        set_stop("stall");
        break;
      }
    }
    if (have) {
      const double slack_e = best_budget_e - best_e, slack_f = best_budget_f - best_f;
      double te = 0.0, tf = 0.0;
      size_t order = keep_r.size();
      while (order > 1) {
        const double a = std::hypot(keep_r[order - 1], keep_i[order - 1]);
        if (te + a > 0.5 * slack_e || tf + (double)order * a > 0.5 * slack_f) break;
        te += a;
        tf += (double)order * a;
        order -= 1;
      }
      if (order > cap_order || !coeffs) throw std::runtime_error("series coefficients larger than the buffer given");
      out->n = best_n;
      out->order = (uint32_t)order;
      out->state_bound = best_e + te;
      out->derivative_bound = best_f + tf;
      out->shift_px = out->state_bound * rho / (best_dmin * pixel);
      for (size_t k = 0; k < order; ++k) {
        coeffs[2 * k] = keep_r[k];
        coeffs[2 * k + 1] = keep_i[k];
      }
    }
    return 0;
  } catch (std::exception &ex) {
    g_err = ex.what();
    return -1;
  }
}

void fdh_encode(const fdh_plane *plane, uint32_t ss, uint64_t count, const uint8_t *cls, const uint32_t *n,
                const double *z, const double *dz, const int64_t *dexp, double *nu, float *de, uint16_t *normal,
                int threads) {
  const double LN_2 = 0.693147180559945309417232121458176568;
  const double TAU = 6.28318530717958647692528676655900577;
  const double px_m = plane->h_m * (double)ss;
  const int64_t px_e = plane->h_e;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  parallel_for(count, threads, [&](uint64_t a, uint64_t b) {
    for (uint64_t k = a; k < b; ++k) {
      if (cls[k] & 3) continue;  // escaped samples only (store.rs:67-85)
      double zr = z[2 * k], zi = z[2 * k + 1], dr = dz[2 * k], di = dz[2 * k + 1];
      double z2 = zr * zr + zi * zi;
      double log2z = 0.5 * std::log2(z2);
      if (nu) nu[k] = (double)n[k] + 1.0 - std::log2(log2z);
      if (de) {
        double lnz = log2z * LN_2;
        double base = 2.0 * std::sqrt(z2) * lnz / (std::hypot(dr, di) * px_m);
        int64_t kk = -(dexp[k] + px_e);
        kk = std::max<int64_t>(-4000, std::min<int64_t>(4000, kk));
        de[k] = (float)(base * exp2i(kk / 2) * exp2i(kk - kk / 2));
      }
      if (normal) {
        double re = zr * dr + zi * di, im = zi * dr - zr * di;
        double x = plane->cos_rot * re + plane->sin_rot * im, y = plane->sin_rot * re - plane->cos_rot * im;
        double t = std::round(std::atan2(y, x) * (65536.0 / TAU));
        int64_t v = std::isnan(t) ? 0 : (int64_t)t;
        normal[k] = (uint16_t)(uint64_t)v;
      }
    }
  });
}

void fdh_dc_bound(const fdh_plane *plane, int32_t tier, uint32_t nx, uint32_t ny, double *dc, int64_t *e) {
  // grid.rs:428-444
  double half = std::hypot((double)nx / 2.0, (double)ny / 2.0);
  if (tier == 2) {
    *dc = plane->h_m * half;
    *e = plane->h_e;
  } else {
    *dc = plane->h_m * exp2i(plane->h_e) * half;
    *e = 0;
  }
}

namespace {

// Orbit machinery of the location recipe: z in L-limb fixed point (exact z^2 + c),
// derivatives and multipliers in wide-exponent complex floating point.
struct Walker {
  size_t L;
  std::vector<uint64_t> buf, prod;
  uint64_t *x, *y, *x2, *y2, *s, *s2, *t;
  bool xn = false, yn = false;
  explicit Walker(size_t l) : L(l), buf(8 * l), prod(2 * l) {
    x = buf.data();
    y = x + L;
    x2 = y + L;
    y2 = x2 + L;
    s = y2 + L;
    s2 = s + L;
    t = s2 + L;
  }
  void reset() {
    std::fill(buf.begin(), buf.end(), 0);
    xn = yn = false;
  }
  Fec z() const {
    double mr = 0, mi = 0;
    int64_t er = 0, ei = 0;
    bool hr = frexp_fix(xn, x, L, mr, er), hi = frexp_fix(yn, y, L, mi, ei);
    if (!hr && !hi) return Fec{0, 0, 0};
    int64_t e = !hr ? ei : (!hi ? er : std::max(er, ei));
    double a = hr ? std::ldexp(mr, (int)std::max<int64_t>(er - e, -2000)) : 0.0;
    double b = hi ? std::ldexp(mi, (int)std::max<int64_t>(ei - e, -2000)) : 0.0;
    return fec_norm(a, b, e);
  }
  // z' = z^2 + c (three squarings); false once |z|^2 > 4e8 (escaped: the recipe's
  // iterates never need more).
  bool step(const Fix &a, const Fix &b) {
    square_trunc(x, x2, L, prod.data());
    square_trunc(y, y2, L, prod.data());
    sadd(xn, x, yn, y, s, L);
    square_trunc(s, s2, L, prod.data());
    bool tn = sadd(false, x2, true, y2, t, L);
    xn = sadd(tn, t, a.neg, a.mag.data(), x, L);
    mag_add(x2, y2, s, L);
    tn = sadd(false, s2, true, s, t, L);
    yn = sadd(tn, t, b.neg, b.mag.data(), y, L);
    double fx = fix_to_f64(xn, x, L), fy = fix_to_f64(yn, y, L);
    return fx * fx + fy * fy <= 4.0e8;
  }
};

inline double lg2(const Fec &v) {
  if (v.re == 0 && v.im == 0) return -(double)INFINITY;
  return 0.5 * std::log2(v.re * v.re + v.im * v.im) + (double)v.e;
}
inline Fec fmul(const Fec &a, const Fec &b) {
  return fec_norm(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re, a.e + b.e);
}
inline Fec fdiv(const Fec &a, const Fec &b) {
  double d = b.re * b.re + b.im * b.im;
  return fec_norm((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d, a.e - b.e);
}
inline Fec fadd(const Fec &a, const Fec &b) {
  if (a.re == 0 && a.im == 0) return b;
  if (b.re == 0 && b.im == 0) return a;
  int64_t e = std::max(a.e, b.e);
  double sa = std::ldexp(1.0, (int)std::max<int64_t>(a.e - e, -2000));
  double sb = std::ldexp(1.0, (int)std::max<int64_t>(b.e - e, -2000));
  return fec_norm(a.re * sa + b.re * sb, a.im * sa + b.im * sb, e);
}
// dz' = 2 z dz + 1
inline Fec dz_step(const Fec &z, const Fec &dz) { return fadd(fmul(fec_norm(2 * z.re, 2 * z.im, z.e), dz), Fec{1, 0, 0}); }

Fix fec_part_to_fix(double m, int64_t e, size_t L) { return fe_to_fix(m, e, L); }

// c -= step (fixed point)
void fix_sub_step(Fix &cr, Fix &ci, const Fec &st, size_t L) {
  Fix dr = fe_to_fix(st.re, st.e, L), di = fe_to_fix(st.im, st.e, L);
  Fix nr, ni;
  nr.mag.assign(L, 0);
  ni.mag.assign(L, 0);
  nr.neg = sadd(cr.neg, cr.mag.data(), !dr.neg, dr.mag.data(), nr.mag.data(), L);
  ni.neg = sadd(ci.neg, ci.mag.data(), !di.neg, di.mag.data(), ni.mag.data(), L);
  cr = nr;
  ci = ni;
}

Fec fix_diff(const Fix &ar, const Fix &ai, const Fix &br, const Fix &bi, size_t L) {
  std::vector<uint64_t> dr(L), di(L);
  bool nr = sadd(ar.neg, ar.mag.data(), !br.neg, br.mag.data(), dr.data(), L);
  bool ni = sadd(ai.neg, ai.mag.data(), !bi.neg, bi.mag.data(), di.data(), L);
  double mr = 0, mi = 0;
  int64_t er = 0, ei = 0;
  bool hr = frexp_fix(nr, dr.data(), L, mr, er), hi = frexp_fix(ni, di.data(), L, mi, ei);
  if (!hr && !hi) return Fec{0, 0, 0};
  int64_t e = !hr ? ei : (!hi ? er : std::max(er, ei));
  return fec_norm(hr ? std::ldexp(mr, (int)std::max<int64_t>(er - e, -2000)) : 0.0,
                  hi ? std::ldexp(mi, (int)std::max<int64_t>(ei - e, -2000)) : 0.0, e);
}

// Newton on z_{q+r}(c) = z_q(c) (ref.py:31-43), steps clamped to 1e-3. Converged, repelling
// (|prod 2 z_k| > 1.01 over one cycle) and not a centre (no |z_k| ~ 0) only.
bool misiurewicz(Fix &cr, Fix &ci, int q, int r, size_t L) {
  Walker w(L);
  const double tol = -(double)(64 * (L - 1)) + 24;
  for (int it = 0; it < 80; ++it) {
    w.reset();
    Fec dz{0, 0, 0}, dzq{0, 0, 0};
    Fix zqr, zqi;
    for (int n = 1; n <= q + r; ++n) {
      dz = dz_step(w.z(), dz);
      if (!w.step(cr, ci)) return false;
      if (n == q) {
        dzq = dz;
        zqr = Fix{w.xn, std::vector<uint64_t>(w.x, w.x + L)};
        zqi = Fix{w.yn, std::vector<uint64_t>(w.y, w.y + L)};
      }
    }
    Fix zr{w.xn, std::vector<uint64_t>(w.x, w.x + L)}, zi{w.yn, std::vector<uint64_t>(w.y, w.y + L)};
    Fec f = fix_diff(zr, zi, zqr, zqi, L);
    Fec df = fadd(dz, fec_norm(-dzq.re, -dzq.im, dzq.e));
    if (df.re == 0 && df.im == 0) return false;
    if (f.re == 0 && f.im == 0) break;
    Fec st = fdiv(f, df);
    double l = lg2(st);
    if (l > std::log2(1e-3)) {
      double k = std::exp2(std::log2(1e-3) - l);
      st = fec_norm(st.re * k, st.im * k, st.e);
    }
    fix_sub_step(cr, ci, st, L);
    if (l < tol) break;
    if (it == 79) return false;
  }
  // verify on one more pass
  w.reset();
  Fec rho{1, 0, 0};
  double zmin = INFINITY;
  Fix zqr, zqi;
  for (int n = 1; n <= q + r; ++n) {
    if (!w.step(cr, ci)) return false;
    Fec z = w.z();
    zmin = std::min(zmin, lg2(z));
    if (n == q) {
      zqr = Fix{w.xn, std::vector<uint64_t>(w.x, w.x + L)};
      zqi = Fix{w.yn, std::vector<uint64_t>(w.y, w.y + L)};
    }
    if (n >= q && n < q + r) rho = fmul(rho, fec_norm(2 * z.re, 2 * z.im, z.e));
  }
  Fix zr{w.xn, std::vector<uint64_t>(w.x, w.x + L)}, zi{w.yn, std::vector<uint64_t>(w.y, w.y + L)};
  double res = lg2(fix_diff(zr, zi, zqr, zqi, L));
  return res < -(double)(64 * (L - 1)) / 2 && lg2(rho) > std::log2(1.01) && zmin > -100.0;
}

// Ball period (ref.py:46-52): first p <= max_period with |z_p| < R |dz_p|; 0 if none.
uint64_t ball_period(const Fix &cr, const Fix &ci, double log2_R, uint64_t max_period, size_t L) {
  Walker w(L);
  Fec dz{0, 0, 0};
  for (uint64_t k = 1; k <= max_period; ++k) {
    dz = dz_step(w.z(), dz);
    if (!w.step(cr, ci)) return 0;
    if (lg2(w.z()) < log2_R + lg2(dz)) return k;
  }
  return 0;
}

// Newton on z_p(c) = 0 with steps clamped to 2^log2_max (ref.py:54-67).
bool nucleus_newton(Fix &cr, Fix &ci, uint64_t p, double log2_max, size_t L) {
  Walker w(L);
  const double tol = -(double)(64 * (L - 1)) + 16;
  for (int it = 0; it < 200; ++it) {
    w.reset();
    Fec dz{0, 0, 0};
    for (uint64_t k = 0; k < p; ++k) {
      dz = dz_step(w.z(), dz);
      if (!w.step(cr, ci)) return false;
    }
    Fec z = w.z();
    if (z.re == 0 && z.im == 0) return true;
    Fec st = fdiv(z, dz);
    double l = lg2(st);
    if (l > log2_max) {
      double k = std::exp2(log2_max - l);
      st = fec_norm(st.re * k, st.im * k, st.e);
    }
    fix_sub_step(cr, ci, st, L);
    if (l < tol) return true;
  }
  return false;
}

// log2 of the size estimate |1 / (beta lambda^2)| of the period-p nucleus (ref.py:69-74).
double log2_size(const Fix &cr, const Fix &ci, uint64_t p, size_t L) {
  Walker w(L);
  Fec l{1, 0, 0}, b{1, 0, 0};
  for (uint64_t k = 1; k < p; ++k) {
    w.step(cr, ci);
    Fec z = w.z();
    l = fmul(fec_norm(2 * z.re, 2 * z.im, z.e), l);
    b = fadd(b, fdiv(Fec{1, 0, 0}, l));
  }
  return -lg2(fmul(b, fmul(l, l)));
}

}  // namespace

extern "C" int fdh_location(const char *start_re, const char *start_im, double theta, double log10_width,
                            uint64_t bits, uint64_t max_period, char *re_out, char *im_out, size_t cap,
                            uint64_t *period, double *log10_size_over_width) {
  try {
    const size_t L = limbs_for(bits);
    const double LOG2_10 = 3.321928094887362;
    const Fix sr = to_fix(parse_decimal(start_re), L), si = to_fix(parse_decimal(start_im), L);
    // 1. the nearest repelling Misiurewicz point of low order
    const size_t Lm = limbs_for(192);
    Fix s0r = to_fix(parse_decimal(start_re), Lm), s0i = to_fix(parse_decimal(start_im), Lm);
    double best = INFINITY;
    int bq = 0, br = 0;
    for (int q = 3; q <= 60; ++q)
      for (int r = 1; r <= 4; ++r) {
        Fix mr = s0r, mi = s0i;
        if (!misiurewicz(mr, mi, q, r, Lm)) continue;
        double d = lg2(fix_diff(mr, mi, s0r, s0i, Lm));
        if (d < best - 1e-9) {
          best = d;
          bq = q;
          br = r;
        }
      }
    if (!bq) throw std::runtime_error("no repelling Misiurewicz point near the start");
    Fix mr = sr, mi = si;
    if (!misiurewicz(mr, mi, bq, br, L)) throw std::runtime_error("Misiurewicz refinement failed");
    // 2. ladder nucleus near M with size ~ width / 30, bisecting log10 R (ref.py:95-117)
    double lo = log10_width * 0.5 - 1.0, hi = log10_width * 0.95;
    bool have = false;
    Fix bestr, besti;
    uint64_t bestp = 0;
    double bests = 0;
    for (int it = 0; it < 14; ++it) {
      double mid = 0.5 * (lo + hi);
      double log2_R = mid * LOG2_10;
      // c0 = M + 0.345 R e^{i theta}
      Fec off = fec_norm(0.345 * std::cos(theta), 0.345 * std::sin(theta), 0);
      off.e += (int64_t)std::floor(log2_R);
      double frac = std::exp2(log2_R - std::floor(log2_R));
      off = fec_norm(off.re * frac, off.im * frac, off.e);
      Fix cr = mr, ci = mi;
      fix_sub_step(cr, ci, fec_norm(-off.re, -off.im, off.e), L);
      uint64_t p = ball_period(cr, ci, log2_R, max_period, L);
      if (!p || !nucleus_newton(cr, ci, p, log2_R - 2.0, L)) {
        hi = mid;
        continue;
      }
      double rel = (log2_size(cr, ci, p, L) / LOG2_10) - log10_width;  // log10 (size / W)
      if (!have || std::fabs(rel + std::log10(30.0)) < std::fabs(bests + std::log10(30.0))) {
        have = true;
        bestr = cr;
        besti = ci;
        bestp = p;
        bests = rel;
      }
      if (rel > -std::log10(30.0)) lo = mid;
      else hi = mid;
      if (std::fabs(rel + std::log10(30.0)) < 0.3) break;
    }
    if (!have) throw std::runtime_error("no nucleus found near the Misiurewicz point");
    size_t digits = (size_t)std::ceil(64.0 * (double)(L - 1) * 0.30102999566398120) + 2;
    std::string sre = fix_to_string(bestr, digits), sim = fix_to_string(besti, digits);
    if (sre.size() + 1 > cap || sim.size() + 1 > cap) throw std::runtime_error("output buffer too small");
    std::memcpy(re_out, sre.c_str(), sre.size() + 1);
    std::memcpy(im_out, sim.c_str(), sim.size() + 1);
    *period = bestp;
    *log10_size_over_width = bests;
    return 0;
  } catch (std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

}  // extern "C"
