// Internal C++ types of the CPU oracle. TEST INFRASTRUCTURE ONLY (see fdref.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <functional>
#include <optional>
#include <string>
#include <vector>

namespace fdref {

double exp2i(int64_t k);
int64_t f2i(double f);
int64_t biased_exp(double q);
size_t limbs_for(uint64_t bits);

struct Fixed {
  bool neg = false;
  std::vector<uint64_t> mag;
  static Fixed parse(const std::string &s, size_t nlimbs);
};

struct Decimal {
  bool neg = false;
  std::vector<uint8_t> digits;
  int64_t exp10 = 0;
  static Decimal parse(const std::string &s);
  double log2_abs() const;
  Fixed to_fixed(size_t nlimbs) const;
};

bool frexp_limbs(bool neg, const uint64_t *mag, size_t l, double &m, int64_t &e);
double to_f64_limbs(bool neg, const uint64_t *mag, size_t l);
void orbit(const Fixed &cr, const Fixed &ci, uint64_t steps, double escape2,
           const std::function<void(double, double)> &emit);

enum class Tier { F64 = 0, Fixed = 1, Scaled = 2 };

struct View {
  std::string center_re, center_im, width;
  double rotation = 0.0;
};

struct Params {
  uint32_t nx = 0, ny = 0, ss = 1;
  uint64_t max_iter = 0;
  double escape_radius = 1e10;
  uint32_t columns = 1;
  int threads = 1;
  std::optional<Tier> tier;
  uint32_t row_first = 0, row_step = 1;
  uint32_t stripe_window = 16;  // StripeParams (stripe.rs:20-36)
  double stripe_freq = 5.0;
};

struct Plane {
  double c_re, c_im, h_m;
  int64_t h_e;
  Tier tier;
  uint64_t bits;
  double cos, sin, half_x, half_y;
  static Plane make(const View &v, uint32_t nx, uint32_t ny);
  std::string kernel(Tier t) const;
  bool allows(Tier t) const;
  void unit_offset(size_t i, size_t j, double &ux, double &uy) const;
  double h() const;
  void to_screen(double re, double im, double &x, double &y) const;
};

struct Reference {
  std::vector<double> re, im;
  uint32_t bits = 53;
  static const size_t MAX_LEN = 1u << 20;
  static Reference make_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius);
  static Reference from_fixed(const Fixed &cr, const Fixed &ci, uint64_t max_iter);
  std::optional<size_t> nucleus_period() const;
  // reference.rs:122-148: bounds q[m] >= |A_m - Z_m| on each point's distance from the
  // exact orbit of the exact centre; bits: the fixed-point orbit's fraction bits, or none
  // for an f64 orbit from the correctly rounded centre (c_re, c_im)
  std::vector<double> error_radius(std::optional<uint64_t> bits, double c_re, double c_im) const;
  size_t len() const { return re.size(); }
};

struct Block {
  double ar = 0, ai = 0, br = 0, bi = 0, r = 0, alpha = 0, beta = 0;
  bool finite() const;
};

struct Bla {
  double eps = 0, dc_max = 0;
  int64_t dc_exp = 0;
  uint64_t points = 0;
  std::vector<std::vector<Block>> levels;
  std::vector<std::vector<double>> r2;
  static Bla build_scaled(const Reference &r, double eps, double dc_max, int64_t dc_exp);
  const Block *find(size_t m, double d2, uint64_t budget, size_t &len, size_t *level = nullptr,
                    size_t *index = nullptr) const;
};

enum class Kind { Escaped = 0, Interior = 1, Unresolved = 2 };

struct Outcome {
  Kind kind = Kind::Unresolved;
  uint64_t n = 0;
  double zr = 0, zi = 0, dr = 0, di = 0;
  int64_t dexp = 0;
  // error radii of an escaped sample on z and dz/dc (sample.rs:22-26; infinite unless
  // tracked, B)
  double ez = __builtin_inf(), ed = __builtin_inf();
  uint64_t iterations(uint64_t max_iter) const { return kind == Kind::Unresolved ? max_iter : n; }
};

struct Skip {
  uint64_t blocks = 0, skipped = 0;
  double shift = 0.0;
};

// A sample's state after n iterates (sample.rs:69-80): delta (xr, xi) against Z_n and
// dz/dc (dr, di); the default is the ordinary start at Z_0.
struct Start {
  uint64_t n = 0;
  double xr = 0.0, xi = 0.0, dr = 0.0, di = 0.0;
};

// The loop state at the start of a BLA block, from which a stripe replay restarts
// (stripe.rs:39-52).
struct StripeSnap {
  size_t m = 0;
  uint64_t n = 0;
  double xr = 0, xi = 0;
  int64_t delta_exp = 0;
  double scale = 0, dc_r = 0, dc_i = 0;
  uint64_t valid = 0;  // first iterate of the recorded run that reached n
};

// stripe.rs:12-241: the Stripe column's recorder for one sample at a time. Iterates go
// into a ring of the last RING; each block start is kept (the last SNAPS of them) so that
// an escape whose window misses iterates can replay them plainly.
struct Stripe {
  static constexpr size_t RING = 128, SNAPS = 8;
  uint32_t window = 16;
  double freq = 5.0;
  double ring_r[RING] = {}, ring_i[RING] = {};
  uint64_t valid = UINT64_MAX;
  StripeSnap snaps[SNAPS];
  size_t count = 0;
  float value = 0.0f;
  void begin();
  void start(uint64_t n) { valid = n + 1; }
  void record(uint64_t n, double zr, double zi) {
    ring_r[n % RING] = zr;
    ring_i[n % RING] = zi;
  }
  void snap(StripeSnap s, uint64_t landed);
  bool rewind(uint64_t n, StripeSnap &out);
  void finish(uint64_t n, double zr, double zi, double r2);
  double term(double zr, double zi) const;
  bool complete(uint64_t n) const;
};

// q: the orbit's error radii (Reference::error_radius) to track the bounded variant
// (B, ordinary tiers: no BLA, no nucleus gate, no series start); null otherwise.
// trace: the Stripe column's recorder (begun by the caller), or null.
Outcome iterate(bool extended, bool D, bool L, const Reference &r, const Bla *bla, Skip &skip,
                std::optional<std::pair<double, double>> c, double ar, double ai, int64_t offset_exp,
                uint64_t max_iter, double r2, std::optional<size_t> nucleus, const Start &start = Start{},
                const double *q = nullptr, Stripe *trace = nullptr);

// series.rs:26-55
struct SeriesConfig {
  size_t start_order = 8, max_order = 64;
  double grow_at = 1e-4, shift_px = 1e-8, derivative_rel = 1e-6;
};

// series.rs:57-84: an admitted prefix of n iterates for samples with |dc| <= rho.
struct Series {
  uint64_t n = 0;
  double rho = 0.0;
  uint64_t points = 0;
  std::vector<std::pair<double, double>> b;  // b[1..], trimmed
  double state_bound = 0.0, derivative_bound = 0.0, shift_px = 0.0;
  uint64_t built_steps = 0;
  std::string stop = "reference";
  uint64_t coefficient_pairs = 0;
  std::vector<uint64_t> growth;
  static Series build(const Reference &r, double rho, double pixel, uint64_t max_iter, const SeriesConfig &cfg,
                      uint64_t stalled_steps = 32);
  // the state after n iterates for dc = (ar, ai): delta, and dz/dc when D
  Start eval(bool D, double ar, double ai) const;
};

bool in_main_components(double cr, double ci);

}  // namespace fdref
