// Oracle part 2: fd-kernel's CPU perturbation path restated in C++17 with the
// reference's operation order (no FP contraction: build with -ffp-contract=off).
// TEST INFRASTRUCTURE ONLY (see fdref.h). Each function cites the file:line of
// junovhs/fractodactyl it follows.
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <thread>

#include "fdref_internal.hpp"

namespace fdref {

static const double HI = 4294967296.0;  // sample.rs:14
static const double LO = 1.0 / HI;      // sample.rs:15
static const double SQUARE_OK = 1e-290; // sample.rs:16
static const double TINY = 1.0 / 1e270; // sample.rs:17
static const double U = 1.1102230246251565e-16;  // sample.rs:54 (EPSILON / 2)
static const double SAFE = 1.0 + 8.0 * U;         // sample.rs:56
static const double RESOLVABLE = 1e-12;          // sample.rs:702
static const double LN_2 = 0.693147180559945309417232121458176568;
static const double TAU = 6.28318530717958647692528676655900577;

// Rust f64::max / f64::min: NaN-ignoring.
static inline double rmax(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
static inline double rmin(double a, double b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
static inline int64_t floor_log2(double a) { return f2i(std::floor(std::log2(a))); }

// ---------------------------------------------------------------- view.rs
// view.rs:39
static const int64_t SCALED_BELOW = -900;

// view.rs:42-87
Plane Plane::make(const View &v, uint32_t nx, uint32_t ny) {
  if (nx == 0 || ny == 0) throw std::runtime_error("empty sample grid");
  Decimal width = Decimal::parse(v.width);
  double lw = width.log2_abs();
  if (width.neg || !std::isfinite(lw)) throw std::runtime_error("view width must be positive");
  double need = std::ceil(rmax(64.0 - lw, 64.0));
  Fixed wfix = width.to_fixed(limbs_for((uint64_t)need));
  double wm;
  int64_t we;
  if (!frexp_limbs(wfix.neg, wfix.mag.data(), wfix.mag.size(), wm, we))
    throw std::runtime_error("view width underflowed");
  double q = wm / (double)nx;
  int64_t qe = biased_exp(q);
  Plane p;
  p.h_m = q * exp2i(-qe);
  p.h_e = we + qe;
  auto num = [](const std::string &s) {
    Decimal::parse(s);
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    std::string t = s.substr(a, b - a);
    return std::strtod(t.c_str(), nullptr);
  };
  p.c_re = num(v.center_re);
  p.c_im = num(v.center_im);
  if (!(std::isfinite(p.c_re) && std::isfinite(p.c_im))) throw std::runtime_error("view centre out of range");
  double c_mag = rmax(rmax(std::fabs(p.c_re), std::fabs(p.c_im)), exp2i(-1022));
  bool f64_ok = std::log2(c_mag) - 52.0 <= (double)p.h_e - 10.0 && p.h_e > -1000;
  p.tier = f64_ok ? Tier::F64 : (p.h_e >= SCALED_BELOW ? Tier::Fixed : Tier::Scaled);
  p.bits = (uint64_t)std::max<int64_t>(128 - p.h_e, 128);
  p.sin = std::sin(v.rotation);
  p.cos = std::cos(v.rotation);
  p.half_x = (double)nx / 2.0;
  p.half_y = (double)ny / 2.0;
  return p;
}

// view.rs:90-96
std::string Plane::kernel(Tier t) const {
  switch (t) {
    case Tier::F64: return "pert-f64/1";
    case Tier::Fixed: return "pert-fx/1 bits=" + std::to_string(bits);
    default: return "pert-fx-scaled/1 bits=" + std::to_string(bits);
  }
}
// view.rs:99-105
bool Plane::allows(Tier t) const {
  if (t == Tier::F64) return tier == Tier::F64;
  if (t == Tier::Fixed) return tier != Tier::Scaled;
  return true;
}
// view.rs:118-122
void Plane::unit_offset(size_t i, size_t j, double &ux, double &uy) const {
  double x = (double)i + 0.5 - half_x;
  double y = (double)j + 0.5 - half_y;
  ux = cos * x + sin * y;
  uy = sin * x - cos * y;
}
// view.rs:126-128
double Plane::h() const { return h_m * exp2i(h_e); }
// view.rs:132-134
void Plane::to_screen(double re, double im, double &x, double &y) const {
  x = cos * re + sin * im;
  y = sin * re - cos * im;
}

// ---------------------------------------------------------------- reference.rs
// reference.rs:21-48
Reference Reference::make_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius) {
  Reference r;
  uint64_t steps = std::min<uint64_t>(max_iter, MAX_LEN - 1);
  r.re.push_back(0.0);
  r.im.push_back(0.0);
  double x = 0.0, y = 0.0;
  for (uint64_t s = 0; s < steps; ++s) {
    double t = x * x - y * y + c_re;
    y = 2.0 * x * y + c_im;
    x = t;
    r.re.push_back(x);
    r.im.push_back(y);
    if (x * x + y * y > escape_radius * escape_radius) break;
  }
  r.bits = 53;
  return r;
}

// reference.rs:85-96
Reference Reference::from_fixed(const Fixed &cr, const Fixed &ci, uint64_t max_iter) {
  Reference r;
  uint64_t steps = std::min<uint64_t>(max_iter, MAX_LEN - 1);
  r.re.push_back(0.0);
  r.im.push_back(0.0);
  orbit(cr, ci, steps, 4294967296.0, [&](double a, double b) {
    r.re.push_back(a);
    r.im.push_back(b);
  });
  return r;
}

// reference.rs:102-120
std::optional<size_t> Reference::nucleus_period() const {
  if (len() < 2) return std::nullopt;
  double record = std::hypot(re[1], im[1]);
  double log_beta = 0.0;
  for (size_t p = 2; p < len() / 2; ++p) {
    double previous = std::hypot(re[p - 1], im[p - 1]);
    log_beta += 1.0 + std::log2(previous);
    double radius = std::hypot(re[p], im[p]);
    if (radius > 1e-140 && radius < 1e-24 && radius < record * 1e-12 &&
        1.0 + log_beta + std::log2(radius) < -40.0 && std::hypot(re[2 * p], im[2 * p]) <= 2.0 * radius)
      return p;
    record = rmin(record, radius);
  }
  return std::nullopt;
}

// reference.rs:122-148
std::vector<double> Reference::error_radius(std::optional<uint64_t> bits, double c_re, double c_im) const {
  const double MIN_POSITIVE = 2.2250738585072014e-308;
  const double c1 = std::fabs(c_re) + std::fabs(c_im);
  // fixed point: three truncated squares per component plus the centre's own truncation,
  // each under one unit of 2^-bits
  const bool fixed = bits.has_value();
  const double d = fixed ? rmax(exp2i(4 - (int64_t)*bits), MIN_POSITIVE) : 0.0;
  std::vector<double> q;
  q.reserve(len());
  double a = 0.0;  // |A_m - F_m|, F the orbit as computed before rounding to f64
  for (size_t m = 0; m < len(); ++m) {
    const double s = std::sqrt(re[m] * re[m] + im[m] * im[m]) * (1.0 + 4.0 * U);
    double round, defect;
    if (fixed) {
      round = 2.0 * U * s + MIN_POSITIVE;
      defect = d;
    } else {  // f64: rounding of x^2 - y^2 + c and 2xy + c, plus the centre's rounding
      round = 0.0;
      defect = 8.0 * U * (s * s + c1) + 2.0 * U * c1 + MIN_POSITIVE;
    }
    q.push_back(a + round);
    a = (a * (2.0 * (s + round) + a) + defect) * (1.0 + 8.0 * U);
  }
  return q;
}

// ---------------------------------------------------------------- bla.rs
// bla.rs:17,24
static const double EPS_LIMIT = 1.0 / (double)(1ull << 24);

bool Block::finite() const {
  return std::isfinite(ar) && std::isfinite(ai) && std::isfinite(br) && std::isfinite(bi) &&
         std::isfinite(r) && std::isfinite(alpha) && std::isfinite(beta);
}

// bla.rs:27-33
static void check(double eps, double dc_max) {
  if (!(eps > 0.0 && eps <= EPS_LIMIT && dc_max > 0.0 && std::isfinite(dc_max)))
    throw std::runtime_error("BLA needs 0 < eps <= 2^-24 and a finite dc_max > 0");
}

// bla.rs:72-85
static Block single(double zr, double zi, double eps) {
  double az = std::hypot(zr, zi);
  double r = 2.0 * eps * az;
  if (!(r > 0.0 && az <= 2.0)) return Block{};
  Block b;
  b.ar = 2.0 * zr + 0.0;
  b.ai = 2.0 * zi + 0.0;
  b.br = 1.0;
  b.bi = 0.0;
  b.r = r;
  b.alpha = r;
  b.beta = 0.0;
  return b;
}

// bla.rs:115-121
static double times_exp2(double v, int64_t e) {
  if (e >= -1022) return v * exp2i(e);
  return v * exp2i(-1022) * exp2i(e + 1022);
}

// bla.rs:91-112 (affine at bla.rs:124-129)
static Block merge(const Block &x, const Block &y, double c, int64_t ce) {
  if (x.r == 0.0 || y.r == 0.0) return Block{};
  double ax = std::hypot(x.ar, x.ai), ay = std::hypot(y.ar, y.ai);
  double ahat = ax + x.alpha;
  double bhat = std::hypot(x.br, x.bi) + x.beta;
  double r = rmin(x.r, (y.r - times_exp2(bhat * c, ce)) / ahat);
  Block z;
  z.ar = y.ar * x.ar - y.ai * x.ai + 0.0 + 0.0;
  z.ai = y.ar * x.ai + y.ai * x.ar + 0.0 + 0.0;
  z.br = y.ar * x.br - y.ai * x.bi + y.br + 0.0;
  z.bi = y.ar * x.bi + y.ai * x.br + y.bi + 0.0;
  z.r = r;
  z.alpha = ay * x.alpha + y.alpha * ahat;
  z.beta = ay * x.beta + y.alpha * bhat + y.beta;
  if (r > 0.0 && z.finite()) return z;
  return Block{};
}

// bla.rs:161-181 + Bla::new bla.rs:184-216
Bla Bla::build_scaled(const Reference &r, double eps, double dc_max, int64_t dc_exp) {
  check(eps, dc_max);
  size_t steps = r.len() >= 2 ? r.len() - 2 : 0;
  auto merge_all = [&](const std::vector<Block> &l) {
    std::vector<Block> out(l.size() / 2);
    for (size_t i = 0; i < l.size() / 2; ++i) out[i] = merge(l[2 * i], l[2 * i + 1], dc_max, dc_exp);
    return out;
  };
  std::vector<Block> singles(steps);
  for (size_t k = 1; k <= steps; ++k) singles[k - 1] = single(r.re[k], r.im[k], eps);
  Bla t;
  std::vector<Block> next = merge_all(singles);
  auto any_valid = [](const std::vector<Block> &l) {
    for (auto &b : l)
      if (b.r > 0.0) return true;
    return false;
  };
  while (any_valid(next)) {
    std::vector<Block> up = merge_all(next);
    t.levels.push_back(std::move(next));
    next = std::move(up);
  }
  t.eps = eps;
  t.dc_max = dc_max;
  t.points = r.len();
  for (size_t i = 0; i < t.levels.size(); ++i) {
    if (i + 1 >= 64 || t.levels[i].size() != (steps >> (i + 1)))
      throw std::runtime_error("BLA level shape mismatch");
    std::vector<double> r2;
    r2.reserve(t.levels[i].size());
    for (auto &b : t.levels[i]) r2.push_back(b.r * b.r);
    t.r2.push_back(std::move(r2));
  }
  t.dc_exp = dc_exp;
  return t;
}

// bla.rs:234-249
const Block *Bla::find(size_t m, double d2, uint64_t budget, size_t &len, size_t *level, size_t *index) const {
  size_t k = m - 1;  // wrapping
  size_t tz = k == 0 ? 64 : (size_t)__builtin_ctzll((unsigned long long)k);
  size_t top = std::min(tz, levels.size());
  auto ok = [&](size_t i) {
    if (!((2ull << i) <= budget)) return false;
    size_t at = k >> (i + 1);
    return at < r2[i].size() && d2 < r2[i][at];
  };
  if (top == 0 || !ok(0)) return nullptr;
  size_t i = 0;
  while (i + 1 < top && ok(i + 1)) ++i;
  len = (size_t)2 << i;
  if (level) *level = i;
  if (index) *index = k >> (i + 1);
  return &levels[i][k >> (i + 1)];
}

// ---------------------------------------------------------------- interior.rs
// interior.rs:6-10
bool in_main_components(double cr, double ci) {
  double y2 = ci * ci;
  double q = (cr - 0.25) * (cr - 0.25) + y2;
  return q * (q + (cr - 0.25)) <= 0.25 * y2 || (cr + 1.0) * (cr + 1.0) + y2 <= 0.0625;
}

// interior.rs:16-47, 55-65
static bool contracting(const Reference &r, size_t m0, double x0r, double x0i, double ar, double ai,
                        uint64_t period) {
  const double *zr = r.re.data(), *zi = r.im.data();
  size_t last = r.len() - 1;
  size_t m = m0;
  double xr = x0r, xi = x0i, dr = 1.0, di = 0.0;
  for (uint64_t s = 0; s < period; ++s) {
    double fr = zr[m] + xr, fi = zi[m] + xi;
    double t = 2.0 * (fr * dr - fi * di);
    di = 2.0 * (fr * di + fi * dr);
    dr = t;
    t = 2.0 * (zr[m] * xr - zi[m] * xi) + xr * xr - xi * xi + ar;
    xi = 2.0 * (zr[m] * xi + zi[m] * xr + xr * xi) + ai;
    xr = t;
    m += 1;
    fr = zr[m] + xr;
    fi = zi[m] + xi;
    double f2 = fr * fr + fi * fi;
    if (f2 > 4.0) return false;
    if (f2 < xr * xr + xi * xi || m == last) {
      xr = fr;
      xi = fi;
      m = 0;
    }
  }
  return dr * dr + di * di < 1.0;
}

// ---------------------------------------------------------------- sample.rs helpers
// sample.rs:586-595
static inline void normalise(double &re, double &im, int64_t &e, int64_t max_e) {
  double a = rmax(std::fabs(re), std::fabs(im));
  if (a == 0.0 || !std::isfinite(a)) return;
  __int128 diff = (__int128)max_e - (__int128)e;  // i64::saturating_sub
  int64_t sat = diff > INT64_MAX ? INT64_MAX : (diff < INT64_MIN ? INT64_MIN : (int64_t)diff);
  int64_t k = std::min<int64_t>(floor_log2(a), sat);
  double h = exp2i(-(k / 2)), l = exp2i(-(k - k / 2));
  re = re * h * l;
  im = im * h * l;
  e = e + k;
}

// sample.rs:600-652
struct Multiplier {
  double re = 1.0, im = 0.0;
  int64_t exp = 0;
  inline void multiply(double r, double i) {
    double nr = re * r - im * i, ni = re * i + im * r;
    re = nr;
    im = ni;
    double a = rmax(std::fabs(re), std::fabs(im));
    if (!(a > 1e-120 && a < 1e120)) renormalise(a);
  }
  void renormalise(double a) {
    if (a > 0.0 && std::isfinite(a)) {
      int64_t e = floor_log2(a);
      double s = exp2i(-e);
      re = re * s;
      im = im * s;
      exp = exp + e;
    }
  }
  void value(double &r, double &i) const {
    double s = exp < -1000 ? 0.0 : exp2i(std::min<int64_t>(exp, 1000));
    r = re * s;
    i = im * s;
  }
  bool below_one() const {
    return std::isfinite(re) && std::isfinite(im) &&
           (exp < -64 || (exp <= 64 && (re * re + im * im) * exp2i(2 * exp) < 1.0));
  }
};

// sample.rs:658-698
struct Contraction {
  double re = 0.0, im = 0.0;
  int64_t exp = 0;
  bool started = false;
  inline void multiply(double r, double i, int64_t e) {
    if (!started) {
      re = 1.0;
      started = true;
    }
    double a = rmax(std::fabs(r), std::fabs(i));
    if (a != 0.0 && !(LO <= a && a <= HI)) {
      int64_t k = floor_log2(a);
      double s = exp2i(-k);
      r *= s;
      i *= s;
      e += k;
    }
    double nr = re * r - im * i, ni = re * i + im * r;
    re = nr;
    im = ni;
    exp += e;
    a = rmax(std::fabs(re), std::fabs(im));
    if (a != 0.0 && !(LO <= a && a <= HI)) {
      int64_t k = floor_log2(a);
      double s = exp2i(-k);
      re *= s;
      im *= s;
      exp += k;
    }
  }
  bool small() const {
    return started && std::isfinite(re) && std::isfinite(im) &&
           (exp < -64 || (exp <= 64 && (re * re + im * im) * exp2i(2 * exp) < 1e-6));
  }
};

// sample.rs:706-708
static inline bool resolvable(double xr, double xi, double f2) {
  return xr * xr + xi * xi > RESOLVABLE * RESOLVABLE * f2;
}

struct Term {
  double re, im;
  int64_t e;
};

// sample.rs:1094-1114
static Term sum2(const Term *t, size_t n, int64_t zero_e) {
  bool have = false;
  int64_t top = 0;
  for (size_t i = 0; i < n; ++i) {
    double a = rmax(std::fabs(t[i].re), std::fabs(t[i].im));
    if (a != 0.0) {
      int64_t v = floor_log2(a) + t[i].e;
      if (!have || v > top) top = v;
      have = true;
    }
  }
  if (!have) return Term{0.0, 0.0, zero_e};
  auto sc = [](double x, int64_t k) {
    if (k < -2046) return 0.0;
    return x * exp2i(k / 2) * exp2i(k - k / 2);
  };
  double re = 0.0, im = 0.0;
  for (size_t i = 0; i < n; ++i) {
    re = re + sc(t[i].re, t[i].e - top);
    im = im + sc(t[i].im, t[i].e - top);
  }
  return Term{re, im, top};
}

// sample.rs:1119-1122
static Term zero_step(Term w, Term a) {
  Term t[2] = {{w.re * w.re - w.im * w.im, 2.0 * w.re * w.im, 2 * w.e}, a};
  return sum2(t, 2, w.e);
}

// sample.rs:1127-1134
static Term zero_step_dz(Term w, Term v) {
  Term t[2] = {{2.0 * (w.re * v.re - w.im * v.im), 2.0 * (w.re * v.im + w.im * v.re), w.e + v.e},
               {1.0, 0.0, 0}};
  return sum2(t, 2, v.e);
}

static inline uint64_t next_pow2(uint64_t x) {
  if (x <= 1) return 1;
  return 1ull << (64 - __builtin_clzll(x - 1));
}

// ---------------------------------------------------------------- stripe.rs
// stripe.rs:164-168
void Stripe::begin() {
  valid = UINT64_MAX;
  count = 0;
  value = 0.0f;
}

// stripe.rs:180-187: keep the block start with the run it continues, the run restarts
// at the iterate the block lands on
void Stripe::snap(StripeSnap s, uint64_t landed) {
  s.valid = valid;
  snaps[count % SNAPS] = s;
  count += 1;
  valid = landed;
}

// stripe.rs:157-160: both windows ending at z_n recorded
bool Stripe::complete(uint64_t n) const {
  const uint64_t a = n > window ? n - window : 0;
  return valid <= (a > 1 ? a : 1);
}

// stripe.rs:189-204: the latest kept block start at or before n - window, else the
// oldest kept one; the replay records from its n + 1 on
bool Stripe::rewind(uint64_t n, StripeSnap &out) {
  if (count == 0 || complete(n)) return false;
  const uint64_t need = n > window ? n - window : 0;
  const size_t kept = count < SNAPS ? count : SNAPS;
  const StripeSnap *pick = nullptr;
  for (size_t j = 0; j < kept && !pick; ++j) {
    const StripeSnap &c = snaps[(count - 1 - j) % SNAPS];
    if (c.n <= need) pick = &c;
  }
  if (!pick) {  // the first of the equally oldest, in most-recent-first order
    for (size_t j = 0; j < kept; ++j) {
      const StripeSnap &c = snaps[(count - 1 - j) % SNAPS];
      if (!pick || c.n < pick->n) pick = &c;
    }
  }
  valid = pick->valid;
  out = *pick;
  return true;
}

// stripe.rs:132-152: 0.5 + 0.5 sin(k arg z); a whole k up to 16 as the sign of k times
// Im (z / |z|)^|k|
double Stripe::term(double zr, double zi) const {
  const double k = freq;
  double s;
  if (k == std::trunc(k) && std::fabs(k) <= 16.0) {
    const double h = std::hypot(zr, zi);
    const double ur = zr / h, ui = zi / h;
    double pr = 1.0, pi = 0.0;
    const int reps = (int)std::fabs(k);
    for (int q = 0; q < reps; ++q) {
      const double nr = pr * ur - pi * ui, ni = pr * ui + pi * ur;
      pr = nr;
      pi = ni;
    }
    s = k < 0.0 ? -pi : pi;
  } else {
    s = std::sin(k * std::atan2(zi, zr));
  }
  return 0.5 + 0.5 * s;
}

// stripe.rs:206-240: the windows ending at z_n and z_{n-1}, interpolated by how far past
// the escape radius z_n landed
void Stripe::finish(uint64_t n, double zr, double zi, double r2) {
  const uint64_t lo = n > window ? n - window : 0;
  const uint64_t first = lo > 1 ? lo : 1;
  double now = 0.0, before = 0.0;
  uint32_t count_now = 0, count_before = 0;
  for (uint64_t i = first; i <= n; ++i) {
    if (i < valid) continue;
    const double t = term(ring_r[i % RING], ring_i[i % RING]);
    if (i > first || (first == 1 && n <= window)) {
      now += t;
      count_now += 1;
    }
    if (i < n) {
      before += t;
      count_before += 1;
    }
  }
  if (count_now == 0) {
    value = 0.0f;
    return;
  }
  now /= (double)count_now;
  before = count_before > 0 ? before / (double)count_before : now;
  double frac = 1.0 - std::log2(std::log(zr * zr + zi * zi) / std::log(r2));
  if (frac < 0.0) frac = 0.0;  // f64::clamp: NaN stays NaN
  if (frac > 1.0) frac = 1.0;
  value = (float)(before * (1.0 - frac) + now * frac);
}

// Precision experiment (not the reference's algorithm): with g_delta_bits in [1, 52],
// the delta is rounded to that many mantissa bits (round half to even) after every update
// that writes it (plain step, block, rebase), everything else staying binary64. 24 bits
// is an ideal FP32-mantissa delta: the accuracy ceiling of any FP32-delta kernel, free of
// that kernel's own shortcuts. 0 (the default) leaves the reference's algorithm as it is.
static std::atomic<int> g_delta_bits{0};
// ... applied only to updates that leave the iteration count in [g_round_from, g_round_to)
static std::atomic<uint64_t> g_round_from{0}, g_round_to{UINT64_MAX};
// ... and, when set, the orbit point a plain step multiplies the delta by is rounded to
// the same width (an FP32 copy of Z, as any FP32 recurrence holds it)
static std::atomic<bool> g_round_orbit{false};

static inline double round_bits(double x, int bits) {
  if (x == 0.0 || !std::isfinite(x)) return x;
  int e;
  const double m = std::frexp(x, &e);  // x = m 2^e, 0.5 <= |m| < 1
  return std::ldexp(std::nearbyint(std::ldexp(m, bits)), e - bits);
}

// ---------------------------------------------------------------- sample.rs:170-581
// The B (bounded) variant and the Stripe recorder (T) are template arguments, so the
// plain kernel compiles without them. A series start (Start, sample.rs:69-80) is supported.
// T: the Stripe column's recorder is on (sample.rs:231-236): each iterate is recorded,
// each block start kept, and an escape whose window misses iterates replays them plainly
// from a kept block start, the outcome staying the first escape's.
template <bool EXT, bool D, bool L, bool B, bool T = false>
static Outcome iterate_t(const Reference &r, const Bla *bla, Skip &skip,
                         std::optional<std::pair<double, double>> c, double ar, double ai,
                         int64_t offset_exp, uint64_t max_iter, double r2,
                         std::optional<size_t> nucleus, const Start &start, const double *q,
                         Stripe *trace = nullptr) {
  Outcome o;
  if (c && in_main_components(c->first, c->second)) {
    o.kind = Kind::Interior;
    o.n = 0;
    return o;
  }
  const double *zr = r.re.data(), *zi = r.im.data();
  size_t last = r.len() - 1;
  // sample.rs:186: a supplied start is an ordinary-tier state below the last point
  if (start.n > 0 && (EXT || start.n >= (uint64_t)last)) throw std::runtime_error("invalid start state");
  double xr = start.xr, xi = start.xi;
  int64_t delta_exp = EXT ? offset_exp : 0;
  double scale = EXT ? exp2i(delta_exp) : 1.0;
  double dc_r = ar, dc_i = ai;
  double dr = start.dr, di = start.di;
  int64_t derivative_exp = 0;
  double inverse = 1.0;
  size_t m = (size_t)start.n;
  uint64_t n = start.n;
  double sr = 0.0, si = 0.0;
  uint64_t chk = 16, sn = EXT ? 0 : 8;
  if (n > 0) {  // sample.rs:205-213: the supplied state is the first save
    sr = zr[m] + xr;
    si = zi[m] + xi;
    sn = n;
    chk = std::max<uint64_t>(next_pow2(n + 1), 16);
  }
  int returns = 0;
  bool pending = false;
  Multiplier mu;
  uint64_t hold = 0;
  bool predicted = false;
  double qr = 0.0, qi = 0.0, qstep = 0.0;
  double adc = L ? std::sqrt(ar * ar + ai * ai) : 0.0;
  // sample.rs:221-225 (B): error radii e >= |z_exact - (A_m + delta)|, ed on dz/dc; rc:
  // the f64 offset's distance from the exact sample position
  double e = 0.0, ed = 0.0;
  const double rc = 16.0 * U * (std::fabs(ar) + std::fabs(ai)) + 1e-300;
  Contraction contraction;
  const int delta_bits = g_delta_bits.load(std::memory_order_relaxed);
  const uint64_t round_from = g_round_from.load(std::memory_order_relaxed);
  const uint64_t round_to = g_round_to.load(std::memory_order_relaxed);
  const bool round_orbit = g_round_orbit.load(std::memory_order_relaxed);
  auto rounded = [&]() {
    if (delta_bits > 0 && n >= round_from && n < round_to) {
      xr = round_bits(xr, delta_bits);
      xi = round_bits(xi, delta_bits);
    }
  };
  uint64_t limit = max_iter;
  bool replaying = false;
  Outcome first;  // the escape the blocks found, while a replay re-walks its window
  uint64_t first_at = 0;
  double first_r = 0.0, first_i = 0.0;
  if (T) trace->start(n);
  while (n < limit) {
    const Block *b = nullptr;
    size_t len = 0;
    if (L && bla && !replaying && (!nucleus || m != 0)) {
      double d2 = EXT ? (xr * xr + xi * xi) * scale * scale : xr * xr + xi * xi;
      uint64_t cap = hold > 0 ? sn + hold : (pending ? UINT64_MAX : chk);
      uint64_t budget = std::min(max_iter, cap);
      budget = std::min(budget, nucleus ? (n == 0 ? (uint64_t)1 : (uint64_t)*nucleus + 1) : UINT64_MAX);
      budget = budget > n ? budget - n : 0;
      b = bla->find(m, d2, budget, len);
    }
    if (b) {
      if (T) trace->snap(StripeSnap{m, n, xr, xi, delta_exp, scale, dc_r, dc_i, 0}, n + len);
      double a_r = b->ar, a_i = b->ai, b_r = b->br, b_i = b->bi;
      if (nucleus && n >= 1) contraction.multiply(a_r, a_i, 0);
      if (!EXT && hold > 0) mu.multiply(a_r, a_i);
      if (EXT) {
        normalise(xr, xi, delta_exp, 0);
        if (D) {
          normalise(dr, di, derivative_exp, INT64_MAX / 4);
          inverse = exp2i(-derivative_exp);
        }
        scale = exp2i(delta_exp);
        double factor = exp2i(offset_exp - delta_exp);
        dc_r = ar * factor;
        dc_i = ai * factor;
      }
      if (D) {
        double t = a_r * dr - a_i * di + b_r * inverse;
        di = a_r * di + a_i * dr + b_i * inverse;
        dr = t;
        if (!EXT) skip.shift += (b->alpha * std::sqrt(xr * xr + xi * xi) + b->beta * adc) / std::sqrt(dr * dr + di * di);
      }
      double t = a_r * xr - a_i * xi + b_r * dc_r - b_i * dc_i;
      xi = a_r * xi + a_i * xr + b_r * dc_i + b_i * dc_r;
      xr = t;
      if (EXT) {
        normalise(xr, xi, delta_exp, 0);
        if (D) {
          normalise(dr, di, derivative_exp, INT64_MAX / 4);
          inverse = exp2i(-derivative_exp);
        }
        scale = exp2i(delta_exp);
        double factor = exp2i(offset_exp - delta_exp);
        dc_r = ar * factor;
        dc_i = ai * factor;
      }
      m += len;
      n += len;
      skip.blocks += 1;
      skip.skipped += len;
      rounded();
    } else {
      double fr = zr[m] + scale * xr, fi = zi[m] + scale * xi;
      if (nucleus && n >= 1) contraction.multiply(2.0 * fr, 2.0 * fi, 0);
      if (!EXT && hold > 0) mu.multiply(2.0 * fr, 2.0 * fi);
      if (B) {  // sample.rs:338-350
        const double af = std::sqrt(fr * fr + fi * fi) * (1.0 + 4.0 * U) + 1e-150;  // >= |f|
        const double ef = e + q[m] + 2.0 * U * af;                                   // >= |z_exact - f|
        const double ad = std::fabs(dr) + std::fabs(di);
        ed = (2.0 * (af + ef) * ed + 2.0 * ef * ad + 8.0 * U * (2.0 * af * ad + 1.0)) * SAFE;
        const double aw = std::fabs(zr[m]) + std::fabs(zi[m]), ax = std::fabs(xr) + std::fabs(xi);
        // the delta step's defect against 2 A delta + delta^2 + dc_exact
        const double rho = 8.0 * U * (2.0 * aw * ax + ax * ax + std::fabs(ar) + std::fabs(ai)) + 2.0 * q[m] * ax + rc;
        const double w = af + q[m] + 2.0 * U * af;  // >= |A_m + delta|
        e = (e * (2.0 * w + e) + rho) * SAFE;
      }
      if (D) {
        double t = 2.0 * (fr * dr - fi * di) + inverse;
        di = 2.0 * (fr * di + fi * dr);
        dr = t;
        if (EXT && rmax(std::fabs(dr), std::fabs(di)) > HI) {
          dr = dr * LO;
          di = di * LO;
          derivative_exp += 32;
          inverse = exp2i(-derivative_exp);
        }
      }
      double Zr = zr[m], Zi = zi[m];
      if (round_orbit && delta_bits > 0 && n >= round_from && n < round_to) {
        Zr = round_bits(Zr, delta_bits);
        Zi = round_bits(Zi, delta_bits);
      }
      double nr, ni;
      if (EXT) {  // number.rs:109-124
        nr = 2.0 * (Zr * xr - Zi * xi) + scale * (xr * xr - xi * xi) + dc_r;
        ni = 2.0 * (Zr * xi + Zi * xr) + scale * (2.0 * xr * xi) + dc_i;
      } else {  // number.rs:92-107
        nr = 2.0 * (Zr * xr - Zi * xi) + xr * xr - xi * xi + dc_r;
        ni = 2.0 * (Zr * xi + Zi * xr + xr * xi) + dc_i;
      }
      xr = nr;
      xi = ni;
      m += 1;
      n += 1;
      rounded();
    }
    double physical_r = scale * xr, physical_i = scale * xi;
    double fr = zr[m] + physical_r, fi = zi[m] + physical_i;
    double f2 = fr * fr + fi * fi;
    if (T) trace->record(n, fr, fi);
    if (f2 > r2) {
      o.kind = Kind::Escaped;
      o.n = n;
      o.zr = fr;
      o.zi = fi;
      o.dr = dr;
      o.di = di;
      o.dexp = derivative_exp;
      if (B) {  // sample.rs:373-377
        o.ez = e + q[m] + 4.0 * U * std::sqrt(f2);
        o.ed = ed;
      }
      if (T) {  // sample.rs:387-403
        if (replaying) {
          trace->finish(n, fr, fi, r2);
          return first;
        }
        StripeSnap sn;
        if (trace->rewind(n, sn)) {
          first = o;
          first_at = n;
          first_r = fr;
          first_i = fi;
          replaying = true;
          limit = std::min<uint64_t>(max_iter, n + 64);
          m = sn.m;
          n = sn.n;
          xr = sn.xr;
          xi = sn.xi;
          delta_exp = sn.delta_exp;
          scale = sn.scale;
          dc_r = sn.dc_r;
          dc_i = sn.dc_i;
          continue;
        }
        trace->finish(n, fr, fi, r2);
      }
      return o;
    }
    if (!replaying && nucleus && n == (uint64_t)*nucleus + 1) {
      if (contraction.small()) {
        o.kind = Kind::Interior;
        o.n = n;
        return o;
      }
      nucleus.reset();
    }
    double delta2 = physical_r * physical_r + physical_i * physical_i;
    bool rebase = EXT ? f2 <= delta2 : f2 < delta2;
    if (rebase || m == last) {
      if (B) e += q[m] + 4.0 * U * std::sqrt(f2) + 1e-300;  // sample.rs:419-421: delta := f
      if (EXT) {
        if (f2 > SQUARE_OK) {
          xr = fr;
          xi = fi;
          delta_exp = 0;
        } else {
          Term t[2] = {{zr[m], zi[m], 0}, {xr, xi, delta_exp}};
          Term s = sum2(t, 2, delta_exp);
          xr = s.re;
          xi = s.im;
          delta_exp = s.e;
        }
        scale = exp2i(delta_exp);
        m = 0;
        if (scale < TINY) {
          nucleus.reset();
          if (D) {
            Term v = zero_step_dz(Term{xr, xi, delta_exp}, Term{dr, di, derivative_exp});
            dr = v.re;
            di = v.im;
            derivative_exp = v.e;
            inverse = exp2i(-derivative_exp);
          }
          Term w = zero_step(Term{xr, xi, delta_exp}, Term{ar, ai, offset_exp});
          xr = w.re;
          xi = w.im;
          delta_exp = w.e;
          scale = exp2i(delta_exp);
          m = 1;
          n = n + 1;
          if (T) trace->start(n);  // this step's iterate is not recorded
        }
        rounded();
        double factor = exp2i(offset_exp - delta_exp);
        dc_r = ar * factor;
        dc_i = ai * factor;
      } else {
        xr = fr;
        xi = fi;
        m = 0;
        rounded();
      }
    } else if (EXT) {
      double magnitude = rmax(std::fabs(xr), std::fabs(xi));
      int64_t k = 0;
      if (magnitude > HI && delta_exp < 0)
        k = std::min<int64_t>(32, -delta_exp);
      else if (magnitude < LO && magnitude != 0.0)
        k = -32;
      if (k != 0) {
        double factor = exp2i(-k);
        xr = xr * factor;
        xi = xi * factor;
        delta_exp = delta_exp + k;
        scale = exp2i(delta_exp);
        double f = exp2i(offset_exp - delta_exp);
        dc_r = ar * f;
        dc_i = ai * f;
      }
    }
    if (T && replaying) continue;  // sample.rs:470-472: the replay only re-walks iterates
    double check_r = EXT ? physical_r : xr, check_i = EXT ? physical_i : xi;
    bool judge = EXT ? (returns < 4 && resolvable(check_r, check_i, f2)) : resolvable(check_r, check_i, f2);
    if (!judge) {
      if (EXT) {
        if (n >= chk) {
          sr = fr;
          si = fi;
          sn = n;
          chk = chk * 2;
        }
      } else if (hold > 0) {
        if (n >= sn + hold) {
          hold = 0;
          predicted = false;
          pending = true;
        }
      } else if (n >= chk) {
        pending = true;
      }
      continue;
    }
    double dist = std::fabs(fr - sr) + std::fabs(fi - si);
    double size = std::fabs(sr) + std::fabs(si);
    if (EXT && returns < 4 && dist < 1e-13 * size + 1e-300) {
      if (contracting(r, m, check_r, check_i, ar * exp2i(offset_exp), ai * exp2i(offset_exp), n - sn)) {
        o.kind = Kind::Unresolved;
        return o;
      }
      returns += 1;
    }
    if (!EXT) {
      if (dist < 1e-3 * size) {
        uint64_t period = n - sn;
        if (hold == period && mu.below_one()) {
          double mr, mi;
          mu.value(mr, mi);
          double gr = fr - sr, gi = fi - si;
          double er = mr - 1.0, ei = mi;
          double den = er * er + ei * ei;
          double pr = sr - (gr * er + gi * ei) / den;
          double pi = si - (gi * er - gr * ei) / den;
          double tol = rmin(0.1 * std::sqrt(den), 1e-2) * qstep + 16.0 * U * size;
          if (predicted && std::fabs(pr - qr) + std::fabs(pi - qi) <= tol) {
            o.kind = Kind::Interior;
            o.n = n;
            return o;
          }
          qr = pr;
          qi = pi;
          qstep = (std::fabs(gr) + std::fabs(gi)) / std::sqrt(den);
          predicted = true;
        } else {
          predicted = false;
        }
        hold = period;
        sr = fr;
        si = fi;
        sn = n;
        pending = false;
        mu = Multiplier();
        continue;
      }
      if (hold > 0) {
        if (n < sn + hold) continue;
        hold = 0;
        predicted = false;
        pending = true;
      }
      if (pending || n >= chk) {
        chk = std::max(chk, next_pow2(n + 1));
        sr = fr;
        si = fi;
        sn = n;
        pending = false;
      }
      continue;
    }
    if (n == chk || (EXT && n > chk)) {
      sr = fr;
      si = fi;
      sn = n;
      chk = chk * 2;
    }
  }
  if (T && replaying) {  // sample.rs:576-579: the replay gave up; from what was recorded
    trace->finish(first_at, first_r, first_i, r2);
    return first;
  }
  o.kind = Kind::Unresolved;
  return o;
}

// GCC flags the copy of a disengaged std::optional into iterate_t's parameter as a read
// of its (unused) payload; the payload is only read when engaged.
#pragma GCC diagnostic push
#pragma GCC diagnostic ignored "-Wmaybe-uninitialized"
Outcome iterate(bool extended, bool D, bool L, const Reference &r, const Bla *bla, Skip &skip,
                std::optional<std::pair<double, double>> c, double ar, double ai, int64_t offset_exp,
                uint64_t max_iter, double r2, std::optional<size_t> nucleus, const Start &start,
                const double *q, Stripe *trace) {
  // sample.rs:226-229: a supplied state skipped the contraction's products, and a
  // bounded render has no proof for the heuristic, so both decline it
  if (start.n > 0 || q) nucleus = std::nullopt;
  if (q) {  // sample.rs:185-186, 246: the bounded variant is ordinary-tier, unblocked, from Z_0
    if (extended || start.n > 0) throw std::runtime_error("bounded iteration needs an ordinary tier and no series start");
    if (trace)
      return D ? iterate_t<false, true, false, true, true>(r, nullptr, skip, c, ar, ai, 0, max_iter, r2, nucleus,
                                                           start, q, trace)
               : iterate_t<false, false, false, true, true>(r, nullptr, skip, c, ar, ai, 0, max_iter, r2, nucleus,
                                                            start, q, trace);
    return D ? iterate_t<false, true, false, true>(r, nullptr, skip, c, ar, ai, 0, max_iter, r2, nucleus, start, q)
             : iterate_t<false, false, false, true>(r, nullptr, skip, c, ar, ai, 0, max_iter, r2, nucleus, start, q);
  }
#define FDREF_IT(E, DD, LL)                                                                                     \
  (trace ? iterate_t<E, DD, LL, false, true>(r, bla, skip, c, ar, ai, offset_exp, max_iter, r2, nucleus, start, \
                                             nullptr, trace)                                                    \
         : iterate_t<E, DD, LL, false>(r, bla, skip, c, ar, ai, offset_exp, max_iter, r2, nucleus, start, nullptr))
  if (extended) {
    if (D) return L ? FDREF_IT(true, true, true) : FDREF_IT(true, true, false);
    return L ? FDREF_IT(true, false, true) : FDREF_IT(true, false, false);
  }
  if (D) return L ? FDREF_IT(false, true, true) : FDREF_IT(false, true, false);
  return L ? FDREF_IT(false, false, true) : FDREF_IT(false, false, false);
#undef FDREF_IT
}
#pragma GCC diagnostic pop

}  // namespace fdref

extern "C" int fdref_set_delta_bits(int bits, uint64_t from_n, uint64_t to_n, int round_orbit) {
  if (bits < 0 || bits > 52 || from_n > to_n) return -1;
  fdref::g_round_orbit.store(round_orbit != 0);
  fdref::g_delta_bits.store(bits);
  fdref::g_round_from.store(from_n);
  fdref::g_round_to.store(to_n);
  return 0;
}
