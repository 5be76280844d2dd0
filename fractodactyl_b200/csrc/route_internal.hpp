// Host helpers shared by the route's C++ translation units.
#pragma once
#include <cstdint>
#include <cstring>
#include <limits>

namespace fdroute {

// 2^k as f64, exact where representable (crates/fd-fixed/src/lib.rs:32-42).
inline double exp2i(int64_t k) {
  uint64_t b;
  if (k > 1023) return std::numeric_limits<double>::infinity();
  if (k >= -1022)
    b = (uint64_t)(k + 1023) << 52;
  else if (k >= -1074)
    b = 1ull << (k + 1074);
  else
    return 0.0;
  double d;
  std::memcpy(&d, &b, 8);
  return d;
}

// Unbiased exponent field of a normal double.
inline int64_t exponent_field(double q) {
  uint64_t b;
  std::memcpy(&b, &q, 8);
  return (int64_t)((b >> 52) & 0x7ff) - 1023;
}

}  // namespace fdroute
