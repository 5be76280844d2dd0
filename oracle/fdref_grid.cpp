// Oracle part 3: the grid driver (grid.rs), the column encoder (store.rs), the .fds v1
// writer (crates/fd-samples/src/{header,write,wire}.rs) and the C API of fdref.h.
// TEST INFRASTRUCTURE ONLY (see fdref.h).
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>

#include "fdref.h"
#include "fdref_internal.hpp"

namespace fdref {

static const double LN_2 = 0.693147180559945309417232121458176568;
static const double U = 1.1102230246251565e-16;  // sample.rs:54 (EPSILON / 2)
static const double TAU = 6.28318530717958647692528676655900577;

// store.rs:145-150
static float de_px(double az, double log2z, double dr, double di, int64_t dexp, double px_m, int64_t px_e) {
  double lnz = log2z * LN_2;
  double base = 2.0 * az * lnz / (std::hypot(dr, di) * px_m);
  int64_t k = -(dexp + px_e);
  k = std::max<int64_t>(-4000, std::min<int64_t>(4000, k));
  return (float)(base * exp2i(k / 2) * exp2i(k - k / 2));
}

// crates/fd-samples/src/samples.rs:45-48: round(atan2 * 65536/tau) as i64 as u16.
static uint16_t angle(double x, double y) {
  double t = std::atan2(y, x) * (65536.0 / TAU);
  return (uint16_t)(uint64_t)f2i(std::round(t));
}

struct Columns {
  uint8_t *cls = nullptr;
  double *nu = nullptr;
  float *de = nullptr;
  uint16_t *normal = nullptr;
  float *bound = nullptr;
  uint64_t *n = nullptr;
  double *z = nullptr, *dz = nullptr;
  int64_t *dexp = nullptr;
  double *ez = nullptr, *ed = nullptr;  // raw error radii of escaped samples (bounded renders)
  float *stripe = nullptr;              // Stripe column (stripe.rs)
};

// store.rs:115-151: Bounded evidence for an escaped sample with |z| = az, |dz/dc| = ad
// and error radii ez, ed: (de_lo, bound), or false unless the radii prove escape
// (|z| - ez > 2) and ed < ad / 2.
static bool bounds(uint64_t n, double az, double ez, double ad, double ed, double &de_lo_out, double &bound_out) {
  const double lo = az - ez;
  if (!(lo > 2.0 && ed < 0.5 * ad)) return false;
  const double lnz = std::log(az), llo = std::log(lo), lhi = std::log(az + ez);
  // nu = n + 1 - log2(ln|z| / ln 2): |z| within ez moves it by at most
  // log2(ln|z| / ln(|z| - ez)); plus the rounding of nu itself
  const double nu = std::log1p(-std::log1p(-ez / az) / llo) / LN_2 + 8.0 * U * ((double)n + 8.0);
  // Koebe: distance >= e^-G de / 4 with G <= ln|z| 2^-n
  const double g = lhi * std::exp2(-(double)n);
  const double de_lo = (lo * llo) / (az * lnz) * ad / (ad + ed) * std::exp(-g) * (1.0 - 4.0 / (lo * lo)) * (1.0 - 1e-6);
  const double de_hi = ((az + ez) * lhi) / (az * lnz) * ad / (ad - ed) * (1.0 + 1e-6);
  de_lo_out = de_lo;
  bound_out = nu * de_hi / de_lo * (1.0 + 1e-6);
  return true;
}

// store.rs:66-112 (the class byte is kind | evidence << 2: Bounded when the error radii
// prove it, sample.rs:22-26).
static void put(const Plane &pl, uint32_t ss, uint32_t cols, const Outcome &o, size_t idx, Columns &c,
                uint64_t max_iter = 0) {
  if (c.n) c.n[idx] = o.iterations(max_iter);  // Outcome::iterations (sample.rs:45-50)
  if (c.z) {
    c.z[2 * idx] = o.zr;
    c.z[2 * idx + 1] = o.zi;
  }
  if (c.dz) {
    c.dz[2 * idx] = o.dr;
    c.dz[2 * idx + 1] = o.di;
  }
  if (c.dexp) c.dexp[idx] = o.dexp;
  if (o.kind != Kind::Escaped) {
    if (c.cls) c.cls[idx] = (uint8_t)(o.kind == Kind::Unresolved ? 2 : 1);
    return;
  }
  double z2 = o.zr * o.zr + o.zi * o.zi;
  double log2z = 0.5 * std::log2(z2);
  double de_lo = 0.0, bnd = 0.0;
  const bool bounded = bounds(o.n, std::sqrt(z2), o.ez, std::hypot(o.dr, o.di), o.ed, de_lo, bnd);
  if (c.cls) c.cls[idx] = bounded ? 4 : 0;
  if (c.ez) c.ez[idx] = o.ez;
  if (c.ed) c.ed[idx] = o.ed;
  if ((cols & FDREF_COL_NU) && c.nu) c.nu[idx] = (double)o.n + 1.0 - std::log2(log2z);
  if ((cols & FDREF_COL_DE) && c.de) {
    const float d = de_px(std::sqrt(z2), log2z, o.dr, o.di, o.dexp, pl.h_m * (double)ss, pl.h_e);
    c.de[idx] = bounded ? (float)((double)d * de_lo) : d;
  }
  if ((cols & FDREF_COL_BOUND) && c.bound) c.bound[idx] = bounded ? (float)bnd : 0.0f;
  if ((cols & FDREF_COL_NORMAL) && c.normal) {
    double x, y;
    pl.to_screen(o.zr * o.dr + o.zi * o.di, o.zi * o.dr - o.zr * o.di, x, y);
    c.normal[idx] = angle(x, y);
  }
}

struct Stats {
  uint64_t reference_len = 0, iterations = 0, blocks = 0, skipped = 0, fallback = 0, closed = 0;
  double shift = 0.0;
};

// grid.rs:779-799
static std::pair<Plane, Tier> setup(const View &v, const Params &p) {
  if (p.ss == 0 || p.nx % p.ss != 0 || p.ny % p.ss != 0)
    throw std::runtime_error("grid must be a whole number of pixels");
  if ((p.columns & FDREF_COL_STRIPE) &&
      (p.stripe_window < 1 || p.stripe_window > 64 || !std::isfinite(p.stripe_freq)))
    throw std::runtime_error("stripe window must be 1..=64 and the frequency finite");
  Plane plane = Plane::make(v, p.nx, p.ny);
  Tier tier = p.tier ? *p.tier : plane.tier;
  if (!plane.allows(tier)) throw std::runtime_error("tier is not valid at this depth");
  return {plane, tier};
}

// grid.rs:802-815
static Reference compute(const View &v, const Plane &plane, Tier tier, const Params &p) {
  if (tier == Tier::F64) return Reference::make_f64(plane.c_re, plane.c_im, p.max_iter, p.escape_radius);
  size_t l = limbs_for(plane.bits);
  Reference r = Reference::from_fixed(Fixed::parse(v.center_re, l), Fixed::parse(v.center_im, l), p.max_iter);
  r.bits = (uint32_t)plane.bits;
  return r;
}

// grid.rs:818-823
static uint32_t precision(const Plane &plane, Tier tier) { return tier == Tier::F64 ? 53 : (uint32_t)plane.bits; }

// grid.rs:428-444
static std::pair<double, int64_t> dc_bound(const Plane &plane, Tier tier, const Params &p) {
  double half = std::hypot((double)p.nx / 2.0, (double)p.ny / 2.0);
  if (tier == Tier::Scaled) return {plane.h_m * half, plane.h_e};
  return {plane.h() * half, 0};
}

// grid.rs:378-413
static void bla_checks(const Plane &plane, Tier tier, const Params &p, const Reference &r, const Bla &bla) {
  if (bla.points != r.len()) throw std::runtime_error("BLA table covers another orbit length");
  if (std::isnan(p.escape_radius) || p.escape_radius < 4.0)
    throw std::runtime_error("escape radius is below 4: BLA needs escape radius >= 4");
  auto [dc, e] = dc_bound(plane, tier, p);
  bool over = e == bla.dc_exp ? dc > bla.dc_max
                              : std::log2(dc) + (double)e > std::log2(bla.dc_max) + (double)bla.dc_exp;
  if (std::isnan(dc) || over) throw std::runtime_error("view reaches |dc| beyond the BLA table's dc_max");
}

// grid.rs:446-535 + Job::one/one_from/fill (grid.rs:623-775), stripe included. series: a
// start every sample takes (n > 0; Series::render_masked's refusals, grid.rs:341-373,
// checked here); mask: render only samples with mask != 0 (the others keep their columns).
static std::string run(const View &v, const Params &p, const Reference *supplied, const Bla *bla, Columns cols,
                       Stats &st, Reference *computed_out = nullptr, const Series *series = nullptr,
                       const uint8_t *mask = nullptr) {
  auto [plane, tier] = setup(v, p);
  uint32_t need = precision(plane, tier);
  Reference computed;
  const Reference *ref = supplied;
  if (supplied) {
    uint32_t bits = supplied->bits;
    if (bits != need && (tier == Tier::F64 || bits < need))
      throw std::runtime_error("supplied reference has " + std::to_string(bits) + " bits; this view needs " +
                               (tier == Tier::F64 ? "" : "at least ") + std::to_string(need));
    if (supplied->len() == 0 || supplied->re.size() != supplied->im.size() || supplied->re[0] != 0.0 ||
        supplied->im[0] != 0.0)
      throw std::runtime_error("supplied reference orbit must start at Z_0 = 0 with equal re/im lengths");
    plane.bits = bits;
  } else {
    computed = compute(v, plane, tier, p);
    ref = &computed;
  }
  const bool series_given = series != nullptr;
  if (series) {  // grid.rs:350-366
    if (tier == Tier::Scaled || (p.columns & FDREF_COL_BOUND))
      throw std::runtime_error("a series start needs f64 deltas and no Bound column");
    if (series->points != ref->len()) throw std::runtime_error("series built over another orbit");
    const double dc = dc_bound(plane, tier, p).first;
    if (std::isnan(dc) || dc > series->rho) throw std::runtime_error("view reaches |dc| beyond the series radius");
  }
  if (bla && (p.columns & FDREF_COL_BOUND))  // grid.rs:379-384
    throw std::runtime_error("--columns bound certifies every step; BLA remainders are not certified (ACC-02)");
  if (bla) bla_checks(plane, tier, p, *ref, *bla);
  if (series && series->n == 0) series = nullptr;  // grid.rs:491: no admitted prefix, the plain kernel
  // grid.rs:588-593: error radii for the Bound column on the ordinary tiers
  std::vector<double> q;
  if ((p.columns & FDREF_COL_BOUND) && tier != Tier::Scaled)
    q = ref->error_radius(tier == Tier::F64 ? std::nullopt : std::optional<uint64_t>(plane.bits), plane.c_re,
                          plane.c_im);
  const double *qp = q.empty() ? nullptr : q.data();
  const bool D = (p.columns & (FDREF_COL_DE | FDREF_COL_NORMAL)) != 0 || qp;
  const bool L = bla != nullptr;
  const double h = plane.h();
  const double r2 = p.escape_radius * p.escape_radius;
  std::optional<size_t> nucleus = ref->nucleus_period();
  std::atomic<uint32_t> next_row{0};
  std::mutex mu;
  const bool striped = (p.columns & FDREF_COL_STRIPE) != 0;
  auto worker = [&]() {
    Stats local;
    Stripe stripe;  // this thread's recorder (grid.rs:498), begun per sample
    stripe.window = p.stripe_window;
    stripe.freq = p.stripe_freq;
    Stripe *trace = striped ? &stripe : nullptr;
    for (;;) {
      uint64_t jj = (uint64_t)p.row_first + (uint64_t)next_row.fetch_add(1) * p.row_step;
      if (jj >= p.ny) break;
      uint32_t j = (uint32_t)jj;
      for (uint32_t i = 0; i < p.nx; ++i) {
        if (mask && !mask[(size_t)j * p.nx + i]) continue;
        double ux, uy;
        plane.unit_offset(i, j, ux, uy);
        Skip skip;
        // Job::one_from (grid.rs:651-717): the series start on the f64 tiers
        auto one_from = [&](bool use_series) {
          auto start = [&](double ar, double ai) { return series && use_series ? series->eval(D, ar, ai) : Start{}; };
          switch (tier) {
            case Tier::F64: {
              double ar = ux * h, ai = uy * h;
              return iterate(false, D, L, *ref, bla, skip, std::make_pair(plane.c_re + ar, plane.c_im + ai), ar, ai,
                             0, p.max_iter, r2, nucleus, start(ar, ai), qp, trace);
            }
            case Tier::Fixed:
              return iterate(false, D, L, *ref, bla, skip, std::nullopt, ux * h, uy * h, 0, p.max_iter, r2, nucleus,
                             start(ux * h, uy * h), qp, trace);
            case Tier::Scaled:
            default:
              return iterate(true, D, L, *ref, bla, skip, std::nullopt, ux * plane.h_m, uy * plane.h_m, plane.h_e,
                             p.max_iter, r2, nucleus, Start{}, nullptr, trace);
          }
        };
        // Job::one (grid.rs:623-648): the prefix is not counted; an unresolved series start
        // retries from zero (keeping the nucleus heuristic), counting both runs
        if (trace) trace->begin();  // Job::one (grid.rs:630)
        const Outcome first = one_from(true);
        const uint64_t prefix = series && !(first.kind == Kind::Interior && first.n == 0) ? series->n : 0;
        uint64_t spent = first.iterations(p.max_iter) - prefix;
        Outcome o = first;
        if (prefix > 0 && first.kind == Kind::Unresolved) {
          if (trace) trace->begin();  // grid.rs:638
          o = one_from(false);
          spent += o.iterations(p.max_iter);
        }
        if (L) {
          spent = spent - skip.skipped + skip.blocks;
          local.blocks += skip.blocks;
          local.skipped += skip.skipped;
          bool closed = o.kind == Kind::Interior && o.n == 0;
          local.closed += closed;
          local.fallback += (skip.blocks == 0 && !closed);
          local.shift = std::max(local.shift, skip.shift);
        }
        local.iterations += spent;
        put(plane, p.ss, p.columns, o, (size_t)j * p.nx + i, cols, p.max_iter);
        if (trace && cols.stripe) cols.stripe[(size_t)j * p.nx + i] = trace->value;  // grid.rs:772
      }
    }
    std::lock_guard<std::mutex> g(mu);
    st.iterations += local.iterations;
    st.blocks += local.blocks;
    st.skipped += local.skipped;
    st.fallback += local.fallback;
    st.closed += local.closed;
    st.shift = std::max(st.shift, local.shift);
  };
  int threads = std::max(1, std::min<int>(p.threads, (int)p.ny));
  std::vector<std::thread> pool;
  for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  st.reference_len = ref->len();
  // Output pixel = ss samples of spacing h (grid.rs:529-531).
  if (L && D) st.shift = st.shift / (plane.h() * (double)p.ss);
  else st.shift = NAN;
  std::string kernel = plane.kernel(tier);
  if (bla) kernel += " bla/1";
  if (series_given) kernel += " series/0";  // grid.rs:371
  if (computed_out && !supplied) *computed_out = std::move(computed);
  return kernel;
}

// ---------------------------------------------------------------- .fds v1
struct Out {
  std::vector<uint8_t> b;
  void bytes(const void *p, size_t n) { b.insert(b.end(), (const uint8_t *)p, (const uint8_t *)p + n); }
  void u16(uint16_t v) { bytes(&v, 2); }
  void u32(uint32_t v) { bytes(&v, 4); }
  void u64(uint64_t v) { bytes(&v, 8); }
  void f64(double v) { bytes(&v, 8); }
  void str(const std::string &s) {
    if (s.size() > 65535) throw std::runtime_error("string longer than 65535 bytes");
    u16((uint16_t)s.size());
    bytes(s.data(), s.size());
  }
  void pad8() { b.resize((b.size() + 7) & ~(size_t)7, 0); }
};

// header.rs:62-81 + write.rs:8-53 (MAGIC/MAJOR/MINOR lib.rs:21-27).
static std::vector<uint8_t> fds(const View &v, const Params &p, uint32_t colset, const std::string &kernel,
                                const std::vector<uint8_t> &cls, const std::vector<double> &nu,
                                const std::vector<float> &de, const std::vector<uint16_t> &normal,
                                const std::vector<float> &bound, const std::vector<float> &stripe) {
  Out o;
  o.bytes("FDSAMPLE", 8);
  o.u16(1);
  o.u16(1);
  o.u32(colset);
  o.u32(p.nx);
  o.u32(p.ny);
  o.u32(p.ss);
  o.u32(0);
  o.u64(p.max_iter);
  o.f64(p.escape_radius);
  o.f64(v.rotation);
  o.str(v.center_re);
  o.str(v.center_im);
  o.str(v.width);
  o.str(kernel);
  o.pad8();
  o.bytes(cls.data(), cls.size());
  o.pad8();
  if (colset & FDREF_COL_NU) {
    o.bytes(nu.data(), nu.size() * 8);
    o.pad8();
  }
  if (colset & FDREF_COL_DE) {
    o.bytes(de.data(), de.size() * 4);
    o.pad8();
  }
  if (colset & FDREF_COL_NORMAL) {
    o.bytes(normal.data(), normal.size() * 2);
    o.pad8();
  }
  if (colset & FDREF_COL_BOUND) {  // column.rs:18-19, 42: f32, after normal in bit order
    o.bytes(bound.data(), bound.size() * 4);
    o.pad8();
  }
  if (colset & FDREF_COL_STRIPE) {  // column.rs:20-22, 42: f32, last in bit order
    o.bytes(stripe.data(), stripe.size() * 4);
    o.pad8();
  }
  return o.b;
}

}  // namespace fdref

// ================================================================= C API
using namespace fdref;

struct fdref_ref {
  Reference r;
};
struct fdref_bla {
  Bla t;
};
struct fdref_series {
  Series s;
};

static thread_local std::string g_error;

#define FDREF_TRY(...)                \
  try {                               \
    __VA_ARGS__                       \
  } catch (std::exception & e) {      \
    g_error = e.what();               \
  }

static View to_view(const fdref_job *j) {
  View v;
  v.center_re = j->center_re;
  v.center_im = j->center_im;
  v.width = j->width;
  v.rotation = j->rotation;
  return v;
}
static Params to_params(const fdref_job *j) {
  Params p;
  p.nx = j->nx;
  p.ny = j->ny;
  p.ss = j->ss;
  p.max_iter = j->max_iter;
  p.escape_radius = j->escape_radius;
  p.columns = j->columns | FDREF_COL_CLASS;
  p.threads = j->threads;
  if (j->tier >= 0) p.tier = (Tier)j->tier;
  p.row_first = j->row_first;
  p.row_step = j->row_step ? j->row_step : 1;
  p.stripe_window = j->stripe_window ? j->stripe_window : 16;
  p.stripe_freq = j->stripe_freq != 0.0 ? j->stripe_freq : 5.0;
  return p;
}

extern "C" {

const char *fdref_last_error(void) { return g_error.c_str(); }

int fdref_plane(const fdref_job *job, double *h_m, int64_t *h_e, int32_t *tier, uint64_t *bits, double *c_re,
                double *c_im) {
  FDREF_TRY({
    Plane p = Plane::make(to_view(job), job->nx, job->ny);
    *h_m = p.h_m;
    *h_e = p.h_e;
    *tier = (int32_t)p.tier;
    *bits = p.bits;
    *c_re = p.c_re;
    *c_im = p.c_im;
    return 0;
  })
  return -1;
}

fdref_ref *fdref_reference(const fdref_job *job) {
  FDREF_TRY({
    View v = to_view(job);
    Params p = to_params(job);
    auto [plane, tier] = setup(v, p);
    auto *r = new fdref_ref{compute(v, plane, tier, p)};
    r->r.bits = precision(plane, tier);
    return r;
  })
  return nullptr;
}

fdref_ref *fdref_reference_f64(double c_re, double c_im, uint64_t max_iter, double escape_radius) {
  return new fdref_ref{Reference::make_f64(c_re, c_im, max_iter, escape_radius)};
}

fdref_ref *fdref_reference_fixed(const char *re, const char *im, uint64_t bits, uint64_t max_iter) {
  FDREF_TRY({
    size_t l = limbs_for(bits);
    auto *r = new fdref_ref{Reference::from_fixed(Fixed::parse(re, l), Fixed::parse(im, l), max_iter)};
    r->r.bits = (uint32_t)bits;
    return r;
  })
  return nullptr;
}

fdref_ref *fdref_reference_arrays(const double *re, const double *im, uint64_t len, uint32_t bits) {
  auto *r = new fdref_ref;
  r->r.re.assign(re, re + len);
  r->r.im.assign(im, im + len);
  r->r.bits = bits;
  return r;
}

uint64_t fdref_ref_len(const fdref_ref *r) { return r->r.len(); }
uint32_t fdref_ref_bits(const fdref_ref *r) { return r->r.bits; }
void fdref_ref_copy(const fdref_ref *r, double *re, double *im) {
  std::memcpy(re, r->r.re.data(), r->r.len() * 8);
  std::memcpy(im, r->r.im.data(), r->r.len() * 8);
}
int64_t fdref_ref_nucleus_period(const fdref_ref *r) {
  auto p = r->r.nucleus_period();
  return p ? (int64_t)*p : -1;
}
void fdref_ref_free(fdref_ref *r) { delete r; }

fdref_bla *fdref_bla_build(const fdref_ref *r, double eps, double dc_max, int64_t dc_exp) {
  FDREF_TRY({ return new fdref_bla{Bla::build_scaled(r->r, eps, dc_max, dc_exp)}; })
  return nullptr;
}
uint32_t fdref_bla_levels(const fdref_bla *t) { return (uint32_t)t->t.levels.size(); }
uint64_t fdref_bla_block_count(const fdref_bla *t) {
  uint64_t n = 0;
  for (auto &l : t->t.levels) n += l.size();
  return n;
}
void fdref_bla_export(const fdref_bla *t, double *blocks7, uint64_t *level_offsets) {
  uint64_t at = 0;
  for (size_t i = 0; i < t->t.levels.size(); ++i) {
    if (level_offsets) level_offsets[i] = at;
    for (auto &b : t->t.levels[i]) {
      double v[7] = {b.ar, b.ai, b.br, b.bi, b.r, b.alpha, b.beta};
      std::memcpy(blocks7 + 7 * at, v, sizeof v);
      ++at;
    }
  }
  if (level_offsets) level_offsets[t->t.levels.size()] = at;
}
uint64_t fdref_bla_find(const fdref_bla *t, uint64_t m, double d2, uint64_t budget, uint64_t *level,
                        uint64_t *index) {
  size_t len = 0, lv = 0, ix = 0;
  const Block *b = t->t.find((size_t)m, d2, budget, len, &lv, &ix);
  if (!b) return 0;
  if (level) *level = lv;
  if (index) *index = ix;
  return len;
}
void fdref_bla_free(fdref_bla *t) { delete t; }

int fdref_bla_dc_bound(const fdref_job *job, double *dc, int64_t *e) {
  FDREF_TRY({
    auto [plane, tier] = setup(to_view(job), to_params(job));
    auto b = dc_bound(plane, tier, to_params(job));
    *dc = b.first;
    *e = b.second;
    return 0;
  })
  return -1;
}

int fdref_iterate_stripe(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative, double ar,
                         double ai, int64_t offset_exp, uint64_t max_iter, double r2, int64_t nucleus,
                         uint32_t window, double freq, fdref_outcome *out, float *value) {
  FDREF_TRY({
    std::optional<size_t> nuc;
    if (nucleus == -2) nuc = r->r.nucleus_period();
    else if (nucleus >= 0) nuc = (size_t)nucleus;
    Skip skip;
    Stripe t;
    t.window = window;
    t.freq = freq;
    t.begin();
    Outcome o = iterate(extended != 0, derivative != 0, bla != nullptr, r->r, bla ? &bla->t : nullptr, skip,
                        std::nullopt, ar, ai, offset_exp, max_iter, r2, nuc, Start{}, nullptr, &t);
    out->kind = (int32_t)o.kind;
    out->n = o.n;
    out->zr = o.zr;
    out->zi = o.zi;
    out->dr = o.dr;
    out->di = o.di;
    out->dexp = o.dexp;
    out->blocks = skip.blocks;
    out->skipped = skip.skipped;
    out->shift = skip.shift;
    out->ez = o.ez;
    out->ed = o.ed;
    *value = t.value;
    return 0;
  })
  return -1;
}

int fdref_iterate(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative, int has_c, double cr,
                  double ci, double ar, double ai, int64_t offset_exp, uint64_t max_iter, double r2,
                  int64_t nucleus, fdref_outcome *out) {
  return fdref_iterate_from(r, bla, extended, derivative, has_c, cr, ci, ar, ai, offset_exp, max_iter, r2, nucleus, 0,
                            0.0, 0.0, 0.0, 0.0, out);
}

int fdref_iterate_from(const fdref_ref *r, const fdref_bla *bla, int extended, int derivative, int has_c, double cr,
                       double ci, double ar, double ai, int64_t offset_exp, uint64_t max_iter, double r2,
                       int64_t nucleus, uint64_t start_n, double start_xr, double start_xi, double start_dr,
                       double start_di, fdref_outcome *out) {
  FDREF_TRY({
    std::optional<size_t> nuc;
    if (nucleus == -2) nuc = r->r.nucleus_period();
    else if (nucleus >= 0) nuc = (size_t)nucleus;
    std::optional<std::pair<double, double>> c;
    if (has_c) c = std::make_pair(cr, ci);
    Skip skip;
    Start start;
    start.n = start_n;
    start.xr = start_xr;
    start.xi = start_xi;
    start.dr = start_dr;
    start.di = start_di;
    Outcome o = iterate(extended != 0, derivative != 0, bla != nullptr, r->r, bla ? &bla->t : nullptr, skip, c, ar,
                        ai, offset_exp, max_iter, r2, nuc, start);
    out->kind = (int32_t)o.kind;
    out->n = o.n;
    out->zr = o.zr;
    out->zi = o.zi;
    out->dr = o.dr;
    out->di = o.di;
    out->dexp = o.dexp;
    out->blocks = skip.blocks;
    out->skipped = skip.skipped;
    out->shift = skip.shift;
    out->ez = o.ez;
    out->ed = o.ed;
    return 0;
  })
  return -1;
}

int fdref_error_radius(const fdref_ref *r, int64_t bits, double c_re, double c_im, double *q) {
  FDREF_TRY({
    auto v = r->r.error_radius(bits >= 0 ? std::optional<uint64_t>((uint64_t)bits) : std::nullopt, c_re, c_im);
    std::copy(v.begin(), v.end(), q);
    return 0;
  })
  return -1;
}

int fdref_iterate_bounded(const fdref_ref *r, int derivative, int has_c, double cr, double ci, double ar,
                          double ai, uint64_t max_iter, double r2, int64_t bits, double c_re, double c_im,
                          fdref_outcome *out) {
  FDREF_TRY({
    auto q = r->r.error_radius(bits >= 0 ? std::optional<uint64_t>((uint64_t)bits) : std::nullopt, c_re, c_im);
    std::optional<std::pair<double, double>> c;
    if (has_c) c = std::make_pair(cr, ci);
    Skip skip;
    Outcome o = iterate(false, derivative != 0, false, r->r, nullptr, skip, c, ar, ai, 0, max_iter, r2, std::nullopt,
                        Start{}, q.data());
    out->kind = (int32_t)o.kind;
    out->n = o.n;
    out->zr = o.zr;
    out->zi = o.zi;
    out->dr = o.dr;
    out->di = o.di;
    out->dexp = o.dexp;
    out->blocks = skip.blocks;
    out->skipped = skip.skipped;
    out->shift = skip.shift;
    out->ez = o.ez;
    out->ed = o.ed;
    return 0;
  })
  return -1;
}

int fdref_render_columns(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla,
                         const fdref_series *series, const uint8_t *mask, const fdref_columns *out,
                         fdref_stats *stats, char *kernel, size_t kernel_cap) {
  FDREF_TRY({
    Columns c;
    c.cls = out->cls;
    c.nu = out->nu;
    c.de = out->de;
    c.normal = out->normal;
    c.bound = out->bound;
    c.n = out->n;
    c.z = out->z;
    c.dz = out->dz;
    c.dexp = out->dexp;
    c.ez = out->ez;
    c.ed = out->ed;
    c.stripe = out->stripe;
    Stats st;
    std::string k = run(to_view(job), to_params(job), ref ? &ref->r : nullptr, bla ? &bla->t : nullptr, c, st,
                        nullptr, series ? &series->s : nullptr, mask);
    if (stats) {
      stats->reference_len = st.reference_len;
      stats->iterations = st.iterations;
      stats->blocks = st.blocks;
      stats->skipped = st.skipped;
      stats->fallback_samples = st.fallback;
      stats->closed_form_samples = st.closed;
      stats->shift_px = st.shift;
    }
    if (kernel && kernel_cap) {
      std::strncpy(kernel, k.c_str(), kernel_cap - 1);
      kernel[kernel_cap - 1] = 0;
    }
    return 0;
  })
  return -1;
}

int fdref_render(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla, uint8_t *cls, double *nu,
                 float *de, uint16_t *normal, uint64_t *n_out, double *z_out, double *dz_out, int64_t *dexp_out,
                 fdref_stats *stats, char *kernel, size_t kernel_cap) {
  FDREF_TRY({
    Columns c;
    c.cls = cls;
    c.nu = nu;
    c.de = de;
    c.normal = normal;
    c.n = n_out;
    c.z = z_out;
    c.dz = dz_out;
    c.dexp = dexp_out;
    Stats st;
    std::string k = run(to_view(job), to_params(job), ref ? &ref->r : nullptr, bla ? &bla->t : nullptr, c, st);
    if (stats) {
      stats->reference_len = st.reference_len;
      stats->iterations = st.iterations;
      stats->blocks = st.blocks;
      stats->skipped = st.skipped;
      stats->fallback_samples = st.fallback;
      stats->closed_form_samples = st.closed;
      stats->shift_px = st.shift;
    }
    if (kernel && kernel_cap) {
      std::strncpy(kernel, k.c_str(), kernel_cap - 1);
      kernel[kernel_cap - 1] = 0;
    }
    return 0;
  })
  return -1;
}

fdref_series *fdref_series_build(const fdref_ref *r, double rho, double pixel, uint64_t max_iter,
                                 uint64_t stalled_steps) {
  FDREF_TRY({ return new fdref_series{Series::build(r->r, rho, pixel, max_iter, SeriesConfig{}, stalled_steps)}; })
  return nullptr;
}

void fdref_series_get(const fdref_series *s, fdref_series_info *info, double *coeffs) {
  info->n = s->s.n;
  info->points = s->s.points;
  info->built_steps = s->s.built_steps;
  info->coefficient_pairs = s->s.coefficient_pairs;
  info->order = s->s.b.size();
  info->growth_count = s->s.growth.size();
  info->rho = s->s.rho;
  info->state_bound = s->s.state_bound;
  info->derivative_bound = s->s.derivative_bound;
  info->shift_px = s->s.shift_px;
  std::strncpy(info->stop, s->s.stop.c_str(), sizeof(info->stop) - 1);
  info->stop[sizeof(info->stop) - 1] = 0;
  if (coeffs)
    for (size_t k = 0; k < s->s.b.size(); ++k) {
      coeffs[2 * k] = s->s.b[k].first;
      coeffs[2 * k + 1] = s->s.b[k].second;
    }
}

fdref_series *fdref_series_with_n(const fdref_series *s, uint64_t n) {
  FDREF_TRY({
    fdref_series *c = new fdref_series{s->s};
    c->s.n = n;
    return c;
  })
  return nullptr;
}

void fdref_series_eval(const fdref_series *s, int derivative, double ar, double ai, double *out4) {
  Start st = s->s.eval(derivative != 0, ar, ai);
  out4[0] = st.xr;
  out4[1] = st.xi;
  out4[2] = st.dr;
  out4[3] = st.di;
}

void fdref_series_free(fdref_series *s) { delete s; }

int fdref_render_series(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla, const fdref_series *series,
                        const uint8_t *mask, uint8_t *cls, double *nu, float *de, uint16_t *normal, uint64_t *n_out,
                        double *z_out, double *dz_out, int64_t *dexp_out, fdref_stats *stats, char *kernel,
                        size_t kernel_cap) {
  FDREF_TRY({
    if (!series) throw std::runtime_error("no series");
    Columns c;
    c.cls = cls;
    c.nu = nu;
    c.de = de;
    c.normal = normal;
    c.n = n_out;
    c.z = z_out;
    c.dz = dz_out;
    c.dexp = dexp_out;
    Stats st;
    std::string k = run(to_view(job), to_params(job), ref ? &ref->r : nullptr, bla ? &bla->t : nullptr, c, st,
                        nullptr, &series->s, mask);
    if (stats) {
      stats->reference_len = st.reference_len;
      stats->iterations = st.iterations;
      stats->blocks = st.blocks;
      stats->skipped = st.skipped;
      stats->fallback_samples = st.fallback;
      stats->closed_form_samples = st.closed;
      stats->shift_px = st.shift;
    }
    if (kernel && kernel_cap) {
      std::strncpy(kernel, k.c_str(), kernel_cap - 1);
      kernel[kernel_cap - 1] = 0;
    }
    return 0;
  })
  return -1;
}

void fdref_store_escaped(double h_m, int64_t h_e, uint32_t ss, double rotation, uint64_t n, double zr, double zi,
                         double dr, double di, int64_t dexp, double *nu, float *de, uint16_t *normal) {
  Plane pl{};
  pl.h_m = h_m;
  pl.h_e = h_e;
  pl.sin = std::sin(rotation);
  pl.cos = std::cos(rotation);
  Outcome o;
  o.kind = Kind::Escaped;
  o.n = n;
  o.zr = zr;
  o.zi = zi;
  o.dr = dr;
  o.di = di;
  o.dexp = dexp;
  uint8_t cls;
  Columns c;
  c.cls = &cls;
  c.nu = nu;
  c.de = de;
  c.normal = normal;
  put(pl, ss, FDREF_COL_NU | FDREF_COL_DE | FDREF_COL_NORMAL, o, 0, c);
}

int64_t fdref_render_fds(const fdref_job *job, const fdref_ref *ref, const fdref_bla *bla, uint8_t *buf,
                         uint64_t cap) {
  FDREF_TRY({
    View v = to_view(job);
    Params p = to_params(job);
    size_t n = (size_t)p.nx * p.ny;
    std::vector<uint8_t> cls(n, 0);
    std::vector<double> nu((p.columns & FDREF_COL_NU) ? n : 0, 0.0);
    std::vector<float> de((p.columns & FDREF_COL_DE) ? n : 0, 0.0f);
    std::vector<uint16_t> normal((p.columns & FDREF_COL_NORMAL) ? n : 0, 0);
    std::vector<float> bound((p.columns & FDREF_COL_BOUND) ? n : 0, 0.0f);
    std::vector<float> stripe((p.columns & FDREF_COL_STRIPE) ? n : 0, 0.0f);
    Columns c;
    c.cls = cls.data();
    c.nu = nu.empty() ? nullptr : nu.data();
    c.de = de.empty() ? nullptr : de.data();
    c.normal = normal.empty() ? nullptr : normal.data();
    c.bound = bound.empty() ? nullptr : bound.data();
    c.stripe = stripe.empty() ? nullptr : stripe.data();
    Stats st;
    std::string k = run(v, p, ref ? &ref->r : nullptr, bla ? &bla->t : nullptr, c, st);
    std::vector<uint8_t> bytes = fds(v, p, p.columns, k, cls, nu, de, normal, bound, stripe);
    if (buf && cap) std::memcpy(buf, bytes.data(), std::min<uint64_t>(cap, bytes.size()));
    return (int64_t)bytes.size();
  })
  return -1;
}

}  // extern "C"
