// fdref: the parameter-series initializer (crates/fd-kernel/src/series.rs:86-275).
// TEST INFRASTRUCTURE ONLY (see fdref.h). Same operation order as the reference, built
// with -ffp-contract=off, so the coefficients and bounds are the reference's bits.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "fdref_internal.hpp"

namespace fdref {

namespace {

// The last admitted step (series.rs:124-125).
struct Admitted {
  uint64_t n = 0;
  std::vector<std::pair<double, double>> b;
  double e = 0, f = 0, budget_e = 0, budget_f = 0, dmin = 0;
};

}  // namespace

// series.rs:86-245 (Series::build with build_stalled's bound on consecutive rejections)
Series Series::build(const Reference &r, double rho, double pixel, uint64_t max_iter, const SeriesConfig &cfg,
                     uint64_t stalled_steps) {
  const size_t k_max = std::max<size_t>(cfg.max_order, 1);
  size_t active = std::min(std::max<size_t>(cfg.start_order, 1), k_max);
  std::vector<double> br(k_max + 1, 0.0), bi(k_max + 1, 0.0);  // b[k], k = 1..k_max
  std::vector<double> sr(2 * k_max + 1, 0.0), si(2 * k_max + 1, 0.0);
  double e = 0.0, f = 0.0;
  Series out;
  out.rho = rho;
  out.points = r.len();
  const uint64_t len = r.len();
  const uint64_t limit = std::min(len >= 2 ? len - 2 : 0, max_iter >= 1 ? max_iter - 1 : 0);
  bool have = false;
  Admitted best;
  if (!(rho > 0.0 && std::isfinite(rho) && pixel > 0.0)) {
    out.stop = "radius";
    return out;
  }
  const double cap_e = cfg.shift_px * pixel * 2.0 / rho, cap_f = cfg.derivative_rel * 2.0;
  for (uint64_t n = 0; n < limit; ++n) {
    double zr = r.re[n], zi = r.im[n];
    const double az = std::hypot(zr, zi);
    // the square of the active polynomial, with its omitted (degree > active) part
    std::fill(sr.begin(), sr.begin() + 2 * active + 1, 0.0);
    std::fill(si.begin(), si.begin() + 2 * active + 1, 0.0);
    for (size_t i = 1; i <= active; ++i) {
      double ar = br[i], ai = bi[i];
      if (ar == 0.0 && ai == 0.0) continue;
      sr[2 * i] += ar * ar - ai * ai;
      si[2 * i] += 2.0 * ar * ai;
      ar = 2.0 * ar;
      ai = 2.0 * ai;
      for (size_t j = i + 1; j <= active; ++j) {
        sr[i + j] += ar * br[j] - ai * bi[j];
        si[i + j] += ar * bi[j] + ai * br[j];
      }
    }
    out.coefficient_pairs += (uint64_t)(active * (active + 1) / 2);
    double m = 0.0, d = 0.0, t = 0.0, td = 0.0;
    for (size_t k = 1; k <= active; ++k) {
      const double a = std::hypot(br[k], bi[k]);
      m += a;
      d += (double)k * a;
    }
    for (size_t k = active + 1; k <= 2 * active; ++k) {
      const double a = std::hypot(sr[k], si[k]);
      t += a;
      td += (double)k * a;
    }
    const double e_next = 2.0 * (az + m) * e + e * e + t;
    f = 2.0 * (az + m + e) * f + 2.0 * e * d + td;
    e = e_next;
    for (size_t k = 1; k <= active; ++k) {
      const double xr = br[k], xi = bi[k];
      br[k] = 2.0 * (zr * xr - zi * xi) + sr[k];
      bi[k] = 2.0 * (zr * xi + zi * xr) + si[k];
    }
    br[1] += rho;
    // the state after step n + 1
    const uint64_t step = n + 1;
    out.built_steps = step;
    zr = r.re[step];
    zi = r.im[step];
    double mm = 0.0, tail_d = 0.0;
    for (size_t k = 1; k <= active; ++k) {
      const double a = std::hypot(br[k], bi[k]);
      mm += a;
      if (k >= 2) tail_d += (double)k * a;
    }
    if (!(std::isfinite(e) && std::isfinite(f))) {
      out.stop = "non-finite";
      break;
    }
    if (std::hypot(zr, zi) + mm + e >= 2.0) {
      out.stop = "escape";
      break;
    }
    const double dmin = std::hypot(br[1], bi[1]) - tail_d - f;
    // the absolute state error allowed now: shift_px output pixels through dz/dc
    const double budget = dmin > 0.0 ? cfg.shift_px * pixel * dmin / rho : 0.0;
    if (dmin > 0.0 && e <= budget && f <= cfg.derivative_rel * dmin) {
      have = true;
      best.n = step;
      best.b.clear();
      for (size_t k = 1; k <= active; ++k) best.b.emplace_back(br[k], bi[k]);
      best.e = e;
      best.f = f;
      best.budget_e = budget;
      best.budget_f = cfg.derivative_rel * dmin;
      best.dmin = dmin;
    } else if (e > cap_e || f > cap_f) {
      out.stop = "budget";  // |b1| <= M < 2 caps every later budget
      break;
    }
    if (active < k_max && e > cfg.grow_at * budget) {
      active = std::min(2 * active, k_max);
      out.growth.push_back(step);
    }
    if (stalled_steps > 0 && have && step - best.n >= stalled_steps) {
      out.stop = "stall";
      break;
    }
  }
  if (have) {
    // trim high orders whose norms fit in half the remaining slack of each bound
    const double slack_e = best.budget_e - best.e, slack_f = best.budget_f - best.f;
    double te = 0.0, tf = 0.0;
    while (best.b.size() > 1) {
      const size_t k = best.b.size();
      const double a = std::hypot(best.b[k - 1].first, best.b[k - 1].second);
      if (te + a > 0.5 * slack_e || tf + (double)k * a > 0.5 * slack_f) break;
      te += a;
      tf += (double)k * a;
      best.b.pop_back();
    }
    out.n = best.n;
    out.b = std::move(best.b);
    out.state_bound = best.e + te;
    out.derivative_bound = best.f + tf;
    out.shift_px = out.state_bound * rho / (best.dmin * pixel);
  }
  return out;
}

// series.rs:247-271: Horner on x = dc / rho; S = x p, dz/dc = (p + x p') / rho.
Start Series::eval(bool D, double ar, double ai) const {
  const double s = 1.0 / rho;
  const double xr = ar * s, xi = ai * s;
  double pr = 0.0, pi = 0.0, qr = 0.0, qi = 0.0;
  for (auto it = b.rbegin(); it != b.rend(); ++it) {
    const double cr = it->first, ci = it->second;
    if (D) {
      const double nr = qr * xr - qi * xi + pr, ni = qr * xi + qi * xr + pi;
      qr = nr;
      qi = ni;
    }
    const double nr = pr * xr - pi * xi + cr, ni = pr * xi + pi * xr + ci;
    pr = nr;
    pi = ni;
  }
  Start st;
  st.n = n;
  st.xr = pr * xr - pi * xi;
  st.xi = pr * xi + pi * xr;
  if (D) {
    const double dr = pr + qr * xr - qi * xi, di = pi + qr * xi + qi * xr;
    st.dr = dr * s;
    st.di = di * s;
  }
  return st;
}

}  // namespace fdref
