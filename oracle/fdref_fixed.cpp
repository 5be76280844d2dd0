// Oracle part 1: fd-fixed restated (exact decimal parse, sign-magnitude fixed point,
// the three-squaring reference orbit, exp2i/frexp/to_f64). TEST INFRASTRUCTURE ONLY.
// Every routine here is exact integer arithmetic or a fixed rounding sequence, so the
// f64 values it emits equal the reference's bit for bit.
#include "fdref_internal.hpp"

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

namespace fdref {

// crates/fd-fixed/src/lib.rs:32-42
double exp2i(int64_t k) {
  if (k > 1023) return INFINITY;
  if (k >= -1022) {
    uint64_t b = (uint64_t)(k + 1023) << 52;
    double d;
    std::memcpy(&d, &b, 8);
    return d;
  }
  if (k >= -1074) {
    uint64_t b = 1ull << (k + 1074);
    double d;
    std::memcpy(&d, &b, 8);
    return d;
  }
  return 0.0;
}

// Rust `f as i64`: saturating, NaN -> 0.
int64_t f2i(double f) {
  if (std::isnan(f)) return 0;
  if (f >= 9223372036854775807.0) return INT64_MAX;
  if (f <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)f;
}

int64_t biased_exp(double q) {
  uint64_t b;
  std::memcpy(&b, &q, 8);
  return (int64_t)((b >> 52) & 0x7ff) - 1023;
}

// ---- limbs (crates/fd-fixed/src/limbs.rs) ----
namespace limbs {
// limbs.rs:5-14
int cmp(const uint64_t *a, const uint64_t *b, size_t l) {
  for (size_t i = l; i-- > 0;) {
    if (a[i] < b[i]) return -1;
    if (a[i] > b[i]) return 1;
  }
  return 0;
}
// limbs.rs:17-27
void add(const uint64_t *a, const uint64_t *b, uint64_t *out, size_t l) {
  unsigned c = 0;
  for (size_t i = 0; i < l; ++i) {
    uint64_t s = a[i] + b[i];
    unsigned c1 = s < a[i];
    uint64_t s2 = s + c;
    unsigned c2 = s2 < s;
    out[i] = s2;
    c = c1 | c2;
  }
}
// limbs.rs:30-40
void sub(const uint64_t *a, const uint64_t *b, uint64_t *out, size_t l) {
  unsigned br = 0;
  for (size_t i = 0; i < l; ++i) {
    uint64_t d = a[i] - b[i];
    unsigned b1 = a[i] < b[i];
    uint64_t d2 = d - br;
    unsigned b2 = d < (uint64_t)br;
    out[i] = d2;
    br = b1 | b2;
  }
}
static bool any(const uint64_t *v, size_t l) {
  for (size_t i = 0; i < l; ++i)
    if (v[i]) return true;
  return false;
}
// limbs.rs:43-60
bool add_signed(bool an, const uint64_t *a, bool bn, const uint64_t *b, uint64_t *out, size_t l) {
  if (an == bn) {
    add(a, b, out, l);
    return an && any(out, l);
  }
  if (cmp(a, b, l) < 0) {
    sub(b, a, out, l);
    return bn;
  }
  sub(a, b, out, l);
  return an && any(out, l);
}
// limbs.rs:64-100: out = floor(a^2 / 2^(64(L-1))), prod scratch of 2L.
void sqr(const uint64_t *a, uint64_t *prod, uint64_t *out, size_t l) {
  std::memset(prod, 0, 2 * l * 8);
  for (size_t i = 0; i < l; ++i) {
    unsigned __int128 ai = a[i];
    if (ai == 0) continue;
    uint64_t c = 0;
    for (size_t j = i + 1; j < l; ++j) {
      unsigned __int128 t = ai * a[j] + (unsigned __int128)prod[i + j] + c;
      prod[i + j] = (uint64_t)t;
      c = (uint64_t)(t >> 64);
    }
    prod[i + l] = c;
  }
  uint64_t top = 0;
  for (size_t k = 0; k < 2 * l; ++k) {
    uint64_t next = prod[k] >> 63;
    prod[k] = (prod[k] << 1) | top;
    top = next;
  }
  uint64_t c = 0;
  for (size_t i = 0; i < l; ++i) {
    unsigned __int128 sq = (unsigned __int128)a[i] * a[i];
    unsigned __int128 t = (unsigned __int128)prod[2 * i] + (uint64_t)sq + c;
    prod[2 * i] = (uint64_t)t;
    unsigned __int128 t2 = (unsigned __int128)prod[2 * i + 1] + (sq >> 64) + (t >> 64);
    prod[2 * i + 1] = (uint64_t)t2;
    c = (uint64_t)(t2 >> 64);
  }
  std::memcpy(out, prod + (l - 1), l * 8);
}
// limbs.rs:103-114
void mul_small(std::vector<uint64_t> &v, uint64_t m) {
  uint64_t c = 0;
  for (auto &x : v) {
    unsigned __int128 t = (unsigned __int128)x * m + c;
    x = (uint64_t)t;
    c = (uint64_t)(t >> 64);
  }
  if (c) v.push_back(c);
}
// limbs.rs:116-129
void add_small(std::vector<uint64_t> &v, uint64_t a) {
  uint64_t c = a;
  for (auto &x : v) {
    uint64_t s = x + c;
    c = s < x;
    x = s;
    if (!c) return;
  }
  if (c) v.push_back(c);
}
// limbs.rs:132-139
void div_small(std::vector<uint64_t> &v, uint64_t d) {
  unsigned __int128 r = 0;
  for (size_t i = v.size(); i-- > 0;) {
    unsigned __int128 cur = (r << 64) | v[i];
    v[i] = (uint64_t)(cur / d);
    r = cur % d;
  }
}
}  // namespace limbs

// ---- Decimal (crates/fd-fixed/src/decimal.rs) ----
static std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// Rust `str::parse::<i64>`: optional sign, at least one digit, no overflow.
static bool parse_i64(const std::string &s, int64_t &out) {
  size_t i = 0;
  bool neg = false;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) neg = s[i++] == '-';
  if (i >= s.size()) return false;
  __int128 v = 0;
  for (; i < s.size(); ++i) {
    if (s[i] < '0' || s[i] > '9') return false;
    v = v * 10 + (s[i] - '0');
    if (v > (__int128)INT64_MAX + 1) return false;
  }
  if (neg) v = -v;
  if (v > INT64_MAX || v < INT64_MIN) return false;
  out = (int64_t)v;
  return true;
}

// decimal.rs:20-49
Decimal Decimal::parse(const std::string &s) {
  std::string bad = "not a decimal number: \"" + s + "\"";
  std::string t = trim(s);
  bool neg = false;
  if (!t.empty() && t[0] == '-') {
    neg = true;
    t = t.substr(1);
  } else if (!t.empty() && t[0] == '+') {
    t = t.substr(1);
  }
  std::string mant = t;
  int64_t exp = 0;
  size_t e = t.find_first_of("eE");
  if (e != std::string::npos) {
    mant = t.substr(0, e);
    if (!parse_i64(t.substr(e + 1), exp)) throw std::runtime_error(bad);
  }
  std::string ip = mant, fp;
  size_t dot = mant.find('.');
  if (dot != std::string::npos) {
    ip = mant.substr(0, dot);
    fp = mant.substr(dot + 1);
  }
  Decimal d;
  for (char c : ip + fp) d.digits.push_back((uint8_t)((unsigned char)c - '0'));
  if (d.digits.empty()) throw std::runtime_error(bad);
  for (uint8_t x : d.digits)
    if (x > 9) throw std::runtime_error(bad);
  __int128 e10 = (__int128)exp - (__int128)fp.size();
  if (e10 < INT64_MIN) throw std::runtime_error(bad);
  d.exp10 = (int64_t)e10;
  bool zero = true;
  for (uint8_t x : d.digits)
    if (x) zero = false;
  d.neg = neg && !zero;
  return d;
}

// decimal.rs:52-59
double Decimal::log2_abs() const {
  size_t first = 0;
  while (first < digits.size() && digits[first] == 0) ++first;
  if (first == digits.size()) return -INFINITY;
  double head = 0.0;
  size_t n = digits.size() - first;
  for (size_t i = 0; i < n && i < 17; ++i) head = head * 10.0 + (double)digits[first + i];
  double rest = n > 17 ? (double)(n - 17) : 0.0;
  const double LOG2_10 = 3.321928094887362347870319429489390175864831393;
  return (std::log10(head) + rest + (double)exp10) * LOG2_10;
}

// decimal.rs:62-96
Fixed Decimal::to_fixed(size_t nlimbs) const {
  static const uint64_t TEN19 = 10000000000000000000ull;
  auto pow10 = [](uint32_t k) {
    uint64_t p = 1;
    for (uint32_t i = 0; i < k; ++i) p *= 10;
    return p;
  };
  std::vector<uint64_t> n{0};
  for (size_t at = 0; at < digits.size(); at += 19) {
    size_t len = std::min<size_t>(19, digits.size() - at);
    limbs::mul_small(n, pow10((uint32_t)len));
    uint64_t v = 0;
    for (size_t i = 0; i < len; ++i) v = v * 10 + digits[at + i];
    limbs::add_small(n, v);
  }
  int64_t e = exp10;
  while (e > 0) {
    uint32_t k = (uint32_t)std::min<int64_t>(e, 19);
    limbs::mul_small(n, pow10(k));
    e -= k;
    if (n.size() > 1) throw std::runtime_error("value too large for fixed point");
  }
  std::vector<uint64_t> v(nlimbs - 1, 0);
  v.insert(v.end(), n.begin(), n.end());
  while (e < 0) {
    uint32_t k = (uint32_t)std::min<int64_t>(-e, 19);
    limbs::div_small(v, k == 19 ? TEN19 : pow10(k));
    e += k;
    bool all0 = true;
    for (auto x : v)
      if (x) all0 = false;
    if (all0) break;
  }
  for (size_t i = nlimbs; i < v.size(); ++i)
    if (v[i]) throw std::runtime_error("value too large for fixed point");
  v.resize(nlimbs);
  Fixed f;
  bool nz = false;
  for (auto x : v)
    if (x) nz = true;
  f.neg = neg && nz;
  f.mag = v;
  return f;
}

size_t limbs_for(uint64_t bits) { return 1 + (size_t)((bits + 63) / 64); }

Fixed Fixed::parse(const std::string &s, size_t nlimbs) { return Decimal::parse(s).to_fixed(nlimbs); }

// lib.rs:75-83
bool frexp_limbs(bool neg, const uint64_t *mag, size_t l, double &m, int64_t &e) {
  ptrdiff_t k = -1;
  for (size_t i = l; i-- > 0;)
    if (mag[i]) {
      k = (ptrdiff_t)i;
      break;
    }
  if (k < 0) return false;
  auto below = [&](ptrdiff_t d) -> double { return k - d >= 0 ? (double)mag[k - d] : 0.0; };
  double v = (double)mag[k] + below(1) * exp2i(-64) + below(2) * exp2i(-128);
  int64_t ve = biased_exp(v);
  double mm = v * exp2i(-ve);
  int64_t scale = 64 * ((int64_t)k - ((int64_t)l - 1));
  m = neg ? -mm : mm;
  e = ve + scale;
  return true;
}

// lib.rs:86-93
double to_f64_limbs(bool neg, const uint64_t *mag, size_t l) {
  double m;
  int64_t e;
  if (!frexp_limbs(neg, mag, l, m, e)) return 0.0;
  if (e < -1000) return m * exp2i(e + 100) * exp2i(-100);
  return m * exp2i(e);
}

// orbit.rs:14-43: Z_{n+1} = Z_n^2 + C with x' = x^2 - y^2 + cr, y' = (x+y)^2 - x^2 - y^2 + ci.
void orbit(const Fixed &cr, const Fixed &ci, uint64_t steps, double escape2,
           const std::function<void(double, double)> &emit) {
  size_t l = cr.mag.size();
  if (l != ci.mag.size()) throw std::runtime_error("orbit: coordinates need equal precision");
  std::vector<uint64_t> x(l), y(l), x2(l), y2(l), s(l), s2(l), t(l), prod(2 * l);
  bool xn = false, yn = false;
  for (uint64_t it = 0; it < steps; ++it) {
    limbs::sqr(x.data(), prod.data(), x2.data(), l);
    limbs::sqr(y.data(), prod.data(), y2.data(), l);
    limbs::add_signed(xn, x.data(), yn, y.data(), s.data(), l);
    limbs::sqr(s.data(), prod.data(), s2.data(), l);
    bool tn = limbs::add_signed(false, x2.data(), true, y2.data(), t.data(), l);
    xn = limbs::add_signed(tn, t.data(), cr.neg, cr.mag.data(), x.data(), l);
    limbs::add(x2.data(), y2.data(), s.data(), l);
    tn = limbs::add_signed(false, s2.data(), true, s.data(), t.data(), l);
    yn = limbs::add_signed(tn, t.data(), ci.neg, ci.mag.data(), y.data(), l);
    double fx = to_f64_limbs(xn, x.data(), l), fy = to_f64_limbs(yn, y.data(), l);
    emit(fx, fy);
    if (fx * fx + fy * fy > escape2) break;
  }
}

}  // namespace fdref

namespace fdref {

// Exact fixed-point value of m 2^e (m a finite double) with L limbs, truncated toward zero.
Fixed fixed_from_double(double m, int64_t e, size_t L) {
  Fixed f;
  f.mag.assign(L, 0);
  if (m == 0.0) return f;
  f.neg = m < 0;
  int k;
  double mm = std::frexp(std::fabs(m), &k);  // |m| = mm 2^k, mm in [0.5, 1)
  uint64_t bits53 = (uint64_t)std::ldexp(mm, 53);
  int64_t shift = e + k - 53 + 64 * (int64_t)(L - 1);
  for (int b = 0; b < 53; ++b) {
    if (!((bits53 >> b) & 1)) continue;
    int64_t pos = shift + b;
    if (pos < 0 || pos >= (int64_t)(64 * L)) continue;
    f.mag[pos / 64] |= 1ull << (pos % 64);
  }
  return f;
}

// Direct iteration z <- z^2 + c from z = 0 at c = centre + (ar, ai) 2^oe in L-limb fixed
// point (the fd-fixed orbit step, orbit.rs:14-43, at the sample's own c), until
// |z|^2 > 2^32; the last steps to the escape radius in f64 (z is then far from 0, so f64
// carries it to 1e-16 relative). Returns the escape count (0: none within max_iter).
uint64_t direct_escape(const std::string &cre, const std::string &cim, double ar, double ai, int64_t oe,
                       uint64_t bits, uint64_t max_iter, double r2, double &zr_out, double &zi_out) {
  size_t L = limbs_for(bits);
  Fixed c0r = Fixed::parse(cre, L), c0i = Fixed::parse(cim, L);
  Fixed dr = fixed_from_double(ar, oe, L), di = fixed_from_double(ai, oe, L);
  Fixed cr, ci;
  cr.mag.assign(L, 0);
  ci.mag.assign(L, 0);
  cr.neg = limbs::add_signed(c0r.neg, c0r.mag.data(), dr.neg, dr.mag.data(), cr.mag.data(), L);
  ci.neg = limbs::add_signed(c0i.neg, c0i.mag.data(), di.neg, di.mag.data(), ci.mag.data(), L);
  uint64_t n = 0;
  double fx = 0, fy = 0;
  bool out = false;
  const double stop = r2 < 4294967296.0 ? r2 : 4294967296.0;
  orbit(cr, ci, max_iter, stop, [&](double a, double b) {
    ++n;
    fx = a;
    fy = b;
    if (a * a + b * b > stop) out = true;
  });
  if (!out) {
    if (fx * fx + fy * fy > r2) {
      zr_out = fx;
      zi_out = fy;
      return n;
    }
    return 0;
  }
  double x = fx, y = fy, c_r = to_f64_limbs(cr.neg, cr.mag.data(), L), c_i = to_f64_limbs(ci.neg, ci.mag.data(), L);
  // the orbit stopped at the first point past 2^16 in modulus: check it, then continue
  while (!(x * x + y * y > r2)) {
    if (n >= max_iter) return 0;
    double t = x * x - y * y + c_r;
    y = 2.0 * x * y + c_i;
    x = t;
    ++n;
  }
  zr_out = x;
  zi_out = y;
  return n;
}

}  // namespace fdref

extern "C" uint64_t fdref_direct(const char *cre, const char *cim, double ar, double ai, int64_t oe, uint64_t bits,
                                 uint64_t max_iter, double escape_radius, double *zr, double *zi) {
  try {
    return fdref::direct_escape(cre, cim, ar, ai, oe, bits, max_iter, escape_radius * escape_radius, *zr, *zi);
  } catch (...) {
    return ~0ull;
  }
}
