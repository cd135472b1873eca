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

// Programmatic dependent launch: let the next kernel on the stream begin its
// prologue (pdl_trigger), and wait until the previous kernel's results are
// complete and visible (pdl_wait; returns at once for a plain launch).
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Phase stamps (off by default; built into libjfb200_stamps.so by
// jaxfun_b200.build with stamps=True): thread 0 of every CTA writes the
// global timer at the phase boundaries of the step kernels into
// g_jfb_stamps[kernel][cta][phase]; jfb_debug_read_stamps copies them out.
constexpr int kStampCTAs = 1024, kStampPhases = 16;
#ifdef JFB_PHASE_STAMPS
static __device__ unsigned long long g_jfb_stamps[4 * kStampCTAs * kStampPhases];
#define JFB_STAMP(kernel, phase)                                                        \
  do {                                                                                  \
    if (threadIdx.x == 0 && blockIdx.x < kStampCTAs) {                                  \
      unsigned long long t_;                                                            \
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_));                           \
      g_jfb_stamps[((size_t)(kernel) * kStampCTAs + blockIdx.x) * kStampPhases + (phase)] = t_; \
    }                                                                                   \
  } while (0)
#else
#define JFB_STAMP(kernel, phase) \
  do {                           \
  } while (0)
#endif

// Bits of a plan's device status word (read and cleared by jfb_kmm_check).
constexpr int kStatusWaitTimeout = 1;  // a bounded device-side wait gave up
constexpr int kStatusNonFinite = 2;    // a solved coefficient was NaN or infinite

__device__ __forceinline__ bool finite_c(c64 v) { return isfinite(v.re) && isfinite(v.im); }
// Records a non-finite value seen by this thread (one atomic, only when set).
__device__ __forceinline__ void flag_nonfinite(int* status, bool bad) {
  if (bad && status) atomicOr(status, kStatusNonFinite);
}

}  // namespace jfb
