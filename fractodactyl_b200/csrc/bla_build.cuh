// BLA levels built on the device from an uploaded orbit: Bla::build_scaled
// (crates/fd-kernel/src/bla.rs:161-216) with Block::single and Block::merge
// (bla.rs:72-112), giving the same blocks, bit for bit, as the host builder
// (host.cpp's bla_levels). Every operation is an IEEE binary64 operation in the reference's
// order (compile with -fmad=false); the one library call of the reference, f64::hypot
// (the host C library's hypot), is restated below.
#pragma once
#include <cstdint>

#include "fd_device.cuh"

namespace fdk {

// hypot(x, y) as the host C library (glibc 2.35 and later) rounds it. The method is
// C. F. Borges, "An Improved Algorithm for hypot(a, b)", ACM TOMS 47(1), 2021, in its form
// without a fused multiply-add: h = sqrt(x^2 + y^2) for x >= y >= 0, then one Newton
// correction h - (h^2 - x^2 - y^2) / (2h) whose residual is assembled from terms that are
// exact in one of two cases (h <= 2y: d = h - y; otherwise d = h - x). Inputs are scaled by
// 2^-600 when x > 2^500 (x^2 would overflow) and by 2^600 when both are below the range
// where y^2 and the residual keep their bits; powers of two scale exactly, so scaling does
// not change the rounding. Checked against the host library on 24 million random pairs
// across the whole exponent range, subnormals included, and on the special values.
__host__ __device__ __forceinline__ double hypot_corrected(double ax, double ay) {  // ax >= ay >= 0
  const double h = sqrt(ax * ax + ay * ay);
  double t1, t2;
  if (h <= 2.0 * ay) {
    const double d = h - ay;
    t1 = ax * (2.0 * d - ax);
    t2 = (d - 2.0 * (ax - ay)) * d;
  } else {
    const double d = h - ax;
    t1 = 2.0 * d * (ax - 2.0 * ay);
    t2 = (4.0 * d - ay) * ay + d * d;
  }
  return h - (t1 + t2) / (2.0 * h);
}

__host__ __device__ __forceinline__ double libm_hypot(double x, double y) {
  if (!isfinite(x) || !isfinite(y)) return (isinf(x) || isinf(y)) ? INFINITY : x + y;
  double ax = fabs(x), ay = fabs(y);
  if (ax < ay) {
    const double t = ax;
    ax = ay;
    ay = t;
  }
  if (ay == 0.0) return ax;
  if (ax > 0x1p500) return hypot_corrected(ax * 0x1p-600, ay * 0x1p-600) * 0x1p600;
  if (ay < 0x1p-500 && ax < 0x1p-400) return hypot_corrected(ax * 0x1p600, ay * 0x1p600) * 0x1p-600;
  return hypot_corrected(ax, ay);
}

// A block in the table's export form ([f64; 7]: a.re, a.im, b.re, b.im, r, alpha, beta).
struct Block7 {
  double ar, ai, br, bi, r, alpha, beta;
};

// Block::single (bla.rs:72-85): one step at Z_m; the zero block where r is not positive or
// |Z| > 2.
__device__ __forceinline__ Block7 block_single(double zr, double zi, double eps) {
  const double az = libm_hypot(zr, zi);
  const double r = 2.0 * eps * az;
  if (!(r > 0.0 && az <= 2.0)) return Block7{0, 0, 0, 0, 0, 0, 0};
  return Block7{2.0 * zr + 0.0, 2.0 * zi + 0.0, 1.0, 0.0, r, r, 0.0};
}

// v * 2^e for the dc bound's exponent (bla.rs:115-121): in two factors below 2^-1022.
__device__ __forceinline__ double times_exp2(double v, int64_t e) {
  return e >= -1022 ? v * exp2i(e) : v * exp2i((int64_t)-1022) * exp2i(e + 1022);
}

// Block::merge (bla.rs:91-112): x then y; the zero block if either is, or where the merged
// radius is not positive or a field is not finite. Rust's f64::min ignores a NaN operand.
__device__ __forceinline__ Block7 block_merge(const Block7 &x, const Block7 &y, double c, int64_t ce) {
  if (x.r == 0.0 || y.r == 0.0) return Block7{0, 0, 0, 0, 0, 0, 0};
  const double ax = libm_hypot(x.ar, x.ai), ay = libm_hypot(y.ar, y.ai);
  const double ahat = ax + x.alpha;
  const double bhat = libm_hypot(x.br, x.bi) + x.beta;
  const double lim = (y.r - times_exp2(bhat * c, ce)) / ahat;
  const double r = isnan(x.r) ? lim : (isnan(lim) ? x.r : (x.r < lim ? x.r : lim));
  Block7 z;
  z.ar = y.ar * x.ar - y.ai * x.ai + 0.0 + 0.0;
  z.ai = y.ar * x.ai + y.ai * x.ar + 0.0 + 0.0;
  z.br = y.ar * x.br - y.ai * x.bi + y.br + 0.0;
  z.bi = y.ar * x.bi + y.ai * x.br + y.bi + 0.0;
  z.r = r;
  z.alpha = ay * x.alpha + y.alpha * ahat;
  z.beta = ay * x.beta + y.alpha * bhat + y.beta;
  const bool fin = isfinite(z.ar) && isfinite(z.ai) && isfinite(z.br) && isfinite(z.bi) && isfinite(z.r) &&
                   isfinite(z.alpha) && isfinite(z.beta);
  if (r > 0.0 && fin) return z;
  return Block7{0, 0, 0, 0, 0, 0, 0};
}

__device__ __forceinline__ Block7 load7(const double *p) {
  return Block7{p[0], p[1], p[2], p[3], p[4], p[5], p[6]};
}

__device__ __forceinline__ void store7(double *p, const Block7 &b) {
  p[0] = b.ar;
  p[1] = b.ai;
  p[2] = b.br;
  p[3] = b.bi;
  p[4] = b.r;
  p[5] = b.alpha;
  p[6] = b.beta;
}

// Level `level` of the table (blocks of 2^(level+1) steps, n of them) into out7: level 0
// from pairs of singles over Z_1..Z_2n (z: the orbit), a later level by merging pairs of
// the level before (in7). valid[level] = 1 when the level holds a block with r > 0. A level
// after one without a valid block is not built (valid[level - 1] == 0: the build stopped
// there), so the launches for every possible level can be queued at once.
__global__ void bla_level(const double2 *__restrict__ z, const double *__restrict__ in7, uint64_t n, uint32_t level,
                          double eps, double c, int64_t ce, double *__restrict__ out7, unsigned *valid) {
  if (level > 0 && !*(volatile unsigned *)(valid + level - 1)) return;
  bool any = false;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    Block7 b;
    if (level == 0) {
      const double2 p = z[2 * t + 1], q = z[2 * t + 2];
      b = block_merge(block_single(p.x, p.y, eps), block_single(q.x, q.y, eps), c, ce);
    } else {
      b = block_merge(load7(in7 + 14 * t), load7(in7 + 14 * t + 7), c, ce);
    }
    store7(out7 + 7 * t, b);
    any = any || b.r > 0.0;
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31u) == 0) atomicOr(valid + level, 1u);
}

}  // namespace fdk
