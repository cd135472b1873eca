// Shared helpers for the jaxfun-b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/jfb200.h"

namespace jfb {

// Thread-local last-error message, returned by jfb_last_error().
void set_error(const std::string& msg);
const char* last_error();

#define JFB_CHECK_CUDA(expr)                                                   \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::jfb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));    \
      return JFB_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

#define JFB_CHECK_LAUNCH()                                                     \
  do {                                                                         \
    cudaError_t _e = cudaGetLastError();                                       \
    if (_e != cudaSuccess) {                                                   \
      ::jfb::set_error(std::string("kernel launch: ") + cudaGetErrorString(_e)); \
      return JFB_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

#define JFB_REQUIRE(cond, msg)                                                 \
  do {                                                                         \
    if (!(cond)) {                                                             \
      ::jfb::set_error(msg);                                                   \
      return JFB_ERR_ARG;                                                      \
    }                                                                          \
  } while (0)

// ---------------------------------------------------------------------------
// Complex helpers on interleaved (re, im) pairs.
// ---------------------------------------------------------------------------
template <typename T>
struct cpx {
  T re, im;
};

template <typename T>
__host__ __device__ __forceinline__ cpx<T> cmk(T r, T i) {
  cpx<T> c;
  c.re = r;
  c.im = i;
  return c;
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) {
  return cmk(a.re + b.re, a.im + b.im);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) {
  return cmk(a.re - b.re, a.im - b.im);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) {
  return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> operator*(T s, cpx<T> a) {
  return cmk(s * a.re, s * a.im);
}
template <typename T>
__host__ __device__ __forceinline__ cpx<T> conjc(cpx<T> a) {
  return cmk(a.re, -a.im);
}
// i * a
template <typename T>
__host__ __device__ __forceinline__ cpx<T> mul_i(cpx<T> a) {
  return cmk(-a.im, a.re);
}

using c64 = cpx<double>;
using c32 = cpx<float>;

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace jfb
