// Host stand-ins for the CUDA builtins the plain-form kernel uses, so that its source
// (fractodactyl_b200/csrc/perturb_f64.cuh) compiles as ordinary C++ and its persistent
// kernel runs on one host thread as a single-lane warp: ballots return the lane's own
// bit, shuffles return the lane's own value (0 for the down-shuffles of the counter
// reduction, whose source lanes do not exist), atomics are plain read-modify-writes.
// TEST INFRASTRUCTURE ONLY: the kernel-emulation tests include it; nothing in the
// package does.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
#define __align__(n) alignas(n)

using std::isfinite;
using std::isinf;
using std::isnan;

struct double2 {
  double x, y;
};
inline double2 make_double2(double x, double y) { return double2{x, y}; }

struct Dim3 {
  unsigned x = 0, y = 0, z = 0;
};
static Dim3 threadIdx, blockIdx, blockDim{1, 1, 1}, gridDim{1, 1, 1};

template <class T>
inline T __ldg(const T *p) {
  return *p;
}

inline double __longlong_as_double(long long v) {
  double d;
  std::memcpy(&d, &v, 8);
  return d;
}
inline long long __double_as_longlong(double d) {
  long long v;
  std::memcpy(&v, &d, 8);
  return v;
}
inline double __hiloint2double(int hi, int lo) {
  return __longlong_as_double((long long)(((unsigned long long)(unsigned)hi << 32) | (unsigned)lo));
}
inline float __int_as_float(int v) {
  float f;
  std::memcpy(&f, &v, 4);
  return f;
}
inline unsigned __float_as_uint(float f) {
  unsigned v;
  std::memcpy(&v, &f, 4);
  return v;
}
inline int __double2hiint(double d) { return (int)((unsigned long long)__double_as_longlong(d) >> 32); }
inline int __double2loint(double d) { return (int)(unsigned)(unsigned long long)__double_as_longlong(d); }
// CUDA's integer max / min overloads
inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int __popc(unsigned v) { return __builtin_popcount(v); }
inline int __popcll(unsigned long long v) { return __builtin_popcountll(v); }
inline int __ffs(int v) { return __builtin_ffs(v); }
inline int __clz(int v) { return v == 0 ? 32 : __builtin_clz((unsigned)v); }
inline int __clzll(long long v) { return v == 0 ? 64 : __builtin_clzll((unsigned long long)v); }

inline unsigned __ballot_sync(unsigned, bool pred) { return pred ? 1u : 0u; }
inline bool __any_sync(unsigned, bool pred) { return pred; }
template <class T>
inline T __shfl_sync(unsigned, T v, int) {
  return v;
}
template <class T>
inline T __shfl_down_sync(unsigned, T, unsigned) {
  return T(0);
}

template <class T>
inline T atomicAdd(T *p, T v) {
  T old = *p;
  *p = old + v;
  return old;
}
inline unsigned atomicExch(unsigned *p, unsigned v) {
  unsigned old = *p;
  *p = v;
  return old;
}
inline unsigned long long atomicMax(unsigned long long *p, unsigned long long v) {
  unsigned long long old = *p;
  if (v > old) *p = v;
  return old;
}
inline unsigned atomicOr(unsigned *p, unsigned v) {
  unsigned old = *p;
  *p = old | v;
  return old;
}
