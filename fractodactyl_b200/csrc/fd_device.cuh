// Device helpers shared by the perturbation kernels (sm_100a).
//
// Bit-exactness rules for the plain (FP64) form: the translation units that include
// this header for that form are compiled with -fmad=false, so every a*b+c below rounds
// twice exactly as the reference's Rust (which never contracts); division and sqrt of
// doubles are IEEE round-to-nearest on the device. The only libm call that reaches a
// class or count decision in the reference is floor(log2(a)) (sample.rs:591, :629,
// :673, :1097); floor_log2 below computes floor(RN(log2 a)) exactly.
#pragma once
#include <cstdint>

namespace fdk {

constexpr double HI = 4294967296.0;           // sample.rs:14
constexpr double LO = 1.0 / 4294967296.0;     // sample.rs:15
constexpr double SQUARE_OK = 1e-290;          // sample.rs:16
constexpr double U = 1.1102230246251565e-16;  // sample.rs:54
constexpr double RES2 = 1e-12 * 1e-12;        // RESOLVABLE^2, sample.rs:702-708
constexpr double LN_2 = 0.6931471805599453;
constexpr double TAU = 6.283185307179586;

// crates/fd-fixed/src/lib.rs:32-42: 2^k as f64, exact where representable.
__device__ __forceinline__ double exp2i(int64_t k) {
  if (k > 1023) return __longlong_as_double(0x7ff0000000000000ll);
  if (k >= -1022) return __longlong_as_double((long long)((uint64_t)(k + 1023) << 52));
  if (k >= -1074) return __longlong_as_double((long long)(1ull << (k + 1074)));
  return 0.0;
}

// The same for 32-bit exponents: one range test on the common path.
__device__ __forceinline__ double exp2i(int k) {
  if ((unsigned)(k + 1022) <= 2045u) return __hiloint2double((k + 1023) << 20, 0);
  return exp2i((int64_t)k);
}

// Rust f64::max / f64::min ignore a NaN operand, as fmax/fmin do.
__device__ __forceinline__ double rmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double rmin(double a, double b) { return fmin(a, b); }

// floor(RN(log2 a)) for a > 0 finite: the exponent e of a, plus one when log2(a) lies
// so close below e + 1 that round-to-nearest gives e + 1 (a just below a power of two
// with |e + 1| > 1). d = e + 1 - log2(a) = -log2(1 - t/2), t = 2 - m, to ~1e-24.
__device__ __noinline__ static int64_t floor_log2_slow(double a) {
  int e = ilogb(a);
  double m = scalbn(a, -e);
  if (m < 2.0 - 0x1p-40) return e;
  double t = 2.0 - m;  // exact
  double d = t * 0.72134752044448170368 * (1.0 + 0.25 * t);  // t / (2 ln 2) (1 + t/4)
  int T = e + 1;
  if (T == 0) return e;
  int aT = T < 0 ? -T : T;
  int be = 31 - __clz(aT);  // ilogb(|T|)
  bool pow2 = (aT & (aT - 1)) == 0;
  // spacing of doubles on the side of T the value lies (below T for T > 0)
  double s = (T > 0 && pow2) ? scalbn(1.0, be - 53) : scalbn(1.0, be - 52);
  return d <= 0.5 * s ? T : e;
}

// The same for the common case from the bits: a normal double whose mantissa is below
// 2 - 2^-40 (not all of its top 40 fraction bits set) has floor(RN(log2 a)) = its
// exponent field - 1023. Tested on the two 32-bit halves.
__device__ __forceinline__ int floor_log2(double a) {
  const unsigned hi = (unsigned)__double2hiint(a), lo = (unsigned)__double2loint(a);
  const int ef = (int)((hi >> 20) & 0x7ffu);
  const bool top40 = (hi & 0xfffffu) == 0xfffffu && (lo & 0xfffff000u) == 0xfffff000u;
  if (ef != 0 && !top40) return ef - 1023;
  return (int)floor_log2_slow(a);
}

// Rust `f as i64` for the finite values floor_log2's callers pass.
struct Cx3 {
  double re, im;
  int64_t e;
};

// sample.rs:586-595, for a 64-bit exponent (the derivative's) or a 32-bit one (the
// delta's, whose range the route bounds far inside 32 bits).
template <typename E>
__device__ __forceinline__ void normalise(double &re, double &im, E &e, E max_e) {
  double a = rmax(fabs(re), fabs(im));
  if (a == 0.0 || !isfinite(a)) return;
  // i64::saturating_sub; max_e is 0 or i64::MAX/4 and |e| stays far below 2^62. The
  // shift is min(floor(log2 a), max_e - e): |floor(log2 a)| <= 1075 and max_e - e stays
  // above -2^31 for both callers' exponents, so it fits 32 bits.
  int k = floor_log2(a);
  const E lim = max_e - e;
  if (lim < (E)k) k = (int)lim;
  double h = exp2i(-(k / 2)), l = exp2i(-(k - k / 2));
  re = re * h * l;
  im = im * h * l;
  e = e + (E)k;
}

// sample.rs:600-652
struct Multiplier {
  double re, im;
  int64_t exp;
  __device__ __forceinline__ void reset() {
    re = 1.0;
    im = 0.0;
    exp = 0;
  }
  __device__ __forceinline__ void multiply(double r, double i) {
    double nr = re * r - im * i, ni = re * i + im * r;
    re = nr;
    im = ni;
    double a = rmax(fabs(re), fabs(im));
    if (!(a > 1e-120 && a < 1e120)) {
      if (a > 0.0 && isfinite(a)) {
        int64_t e = floor_log2(a);
        double s = exp2i(-e);
        re = re * s;
        im = im * s;
        exp = exp + e;
      }
    }
  }
  __device__ __forceinline__ void value(double &r, double &i) const {
    double s = exp < -1000 ? 0.0 : exp2i(exp < 1000 ? exp : 1000);
    r = re * s;
    i = im * s;
  }
  __device__ __forceinline__ bool below_one() const {
    return isfinite(re) && isfinite(im) && (exp < -64 || (exp <= 64 && (re * re + im * im) * exp2i(2 * exp) < 1.0));
  }
};

// sample.rs:658-698
struct Contraction {
  double re, im;
  int64_t exp;
  bool started;
  __device__ __forceinline__ void reset() {
    re = 0.0;
    im = 0.0;
    exp = 0;
    started = false;
  }
  // (r, i) 2^-k with k = floor(log2 max(|r|, |i|)) (0 for a non-finite a), and k: the
  // rescaling of multiply, out of line (one copy for its two uses and their call sites)
  static __device__ __noinline__ Cx3 scaled(double r, double i, double a) {
    int64_t k = isfinite(a) ? floor_log2(a) : 0;
    double s = exp2i(-k);
    return Cx3{r * s, i * s, k};
  }
  __device__ __forceinline__ void multiply(double r, double i) {
    if (!started) {
      re = 1.0;
      started = true;
    }
    int64_t e = 0;
    double a = rmax(fabs(r), fabs(i));
    if (a != 0.0 && !(LO <= a && a <= HI)) {
      const Cx3 t = scaled(r, i, a);
      r = t.re;
      i = t.im;
      e += t.e;
    }
    double nr = re * r - im * i, ni = re * i + im * r;
    re = nr;
    im = ni;
    exp += e;
    a = rmax(fabs(re), fabs(im));
    if (a != 0.0 && !(LO <= a && a <= HI)) {
      const Cx3 t = scaled(re, im, a);
      re = t.re;
      im = t.im;
      exp += t.e;
    }
  }
  __device__ __forceinline__ bool small() const {
    return started && isfinite(re) && isfinite(im) &&
           (exp < -64 || (exp <= 64 && (re * re + im * im) * exp2i(2 * exp) < 1e-6));
  }
};

// sample.rs:1094-1114 for two terms.
static __device__ __noinline__ Cx3 sum2(Cx3 a, Cx3 b, int64_t zero_e) {
  bool have = false;
  int64_t top = 0;
  double aa = rmax(fabs(a.re), fabs(a.im));
  if (aa != 0.0) {
    top = (isfinite(aa) ? floor_log2(aa) : 0) + a.e;
    have = true;
  }
  double ab = rmax(fabs(b.re), fabs(b.im));
  if (ab != 0.0) {
    int64_t v = (isfinite(ab) ? floor_log2(ab) : 0) + b.e;
    if (!have || v > top) top = v;
    have = true;
  }
  if (!have) return Cx3{0.0, 0.0, zero_e};
  auto sc = [](double x, int64_t k) { return k < -2046 ? 0.0 : x * exp2i(k / 2) * exp2i(k - k / 2); };
  double re = 0.0, im = 0.0;
  re = re + sc(a.re, a.e - top);
  im = im + sc(a.im, a.e - top);
  re = re + sc(b.re, b.e - top);
  im = im + sc(b.im, b.e - top);
  return Cx3{re, im, top};
}

// sample.rs:1119-1122
__device__ __forceinline__ Cx3 zero_step(Cx3 w, Cx3 a) {
  return sum2(Cx3{w.re * w.re - w.im * w.im, 2.0 * w.re * w.im, 2 * w.e}, a, w.e);
}
// sample.rs:1127-1134
__device__ __forceinline__ Cx3 zero_step_dz(Cx3 w, Cx3 v) {
  return sum2(Cx3{2.0 * (w.re * v.re - w.im * v.im), 2.0 * (w.re * v.im + w.im * v.re), w.e + v.e},
              Cx3{1.0, 0.0, 0}, v.e);
}

// interior.rs:6-10
__device__ __forceinline__ bool in_main_components(double cr, double ci) {
  double y2 = ci * ci;
  double q = (cr - 0.25) * (cr - 0.25) + y2;
  return q * (q + (cr - 0.25)) <= 0.25 * y2 || (cr + 1.0) * (cr + 1.0) + y2 <= 0.0625;
}

// interior.rs:16-65: does the period-step map from phase m0, delta x0, contract?
static __device__ __noinline__ bool contracting(const double2 *__restrict__ orbit, uint32_t last, uint32_t m0, double x0r,
                                         double x0i, double ar, double ai, uint64_t period) {
  uint32_t m = m0;
  double xr = x0r, xi = x0i, dr = 1.0, di = 0.0;
  for (uint64_t s = 0; s < period; ++s) {
    double2 Z = __ldg(orbit + m);
    double fr = Z.x + xr, fi = Z.y + xi;
    double t = 2.0 * (fr * dr - fi * di);
    di = 2.0 * (fr * di + fi * dr);
    dr = t;
    t = 2.0 * (Z.x * xr - Z.y * xi) + xr * xr - xi * xi + ar;
    xi = 2.0 * (Z.x * xi + Z.y * xr + xr * xi) + ai;
    xr = t;
    m += 1;
    double2 Z1 = __ldg(orbit + m);
    fr = Z1.x + xr;
    fi = Z1.y + xi;
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

__device__ __forceinline__ uint64_t next_pow2(uint64_t x) { return x <= 1 ? 1 : 1ull << (64 - __clzll(x - 1)); }

__device__ __forceinline__ uint64_t globaltimer() {
#if defined(__CUDA_ARCH__)
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
#elif defined(FDK_HOST_TIMER)
  return FDK_HOST_TIMER();  // a host build that supplies its own clock (nanoseconds)
#else
  return 0;  // host builds of this header (no device timer; deadlines are device-only)
#endif
}

}  // namespace fdk
