// Small mixed-radix (2, 3, 4) Stockham FFTs on columns held in shared memory.
//
// Used for the periodic y / z axes of the Couette grid (lengths 2^a 3^b such
// as 64, 96, 128, 144, 192).  Columns are stored row-major as
// buf[k * ldc + col], k the transform index, so that consecutive threads
// work on consecutive columns (conflict-free 16-byte smem accesses).
// Twiddles come from a host-computed table tw[k] = exp(-2 pi i k / n); the
// inverse transform uses their conjugates.
#pragma once

#include "jfb_common.cuh"

namespace jfb {

struct FFTPlan {
  int n;
  int nrad;
  int rad[12];
};

// Factor n = 4^a 2^b 3^c with as many radix-4 passes as possible.
inline bool make_fft_plan(int n, FFTPlan& p) {
  p.n = n;
  p.nrad = 0;
  int m = n;
  while (m % 4 == 0) {
    p.rad[p.nrad++] = 4;
    m /= 4;
  }
  while (m % 2 == 0) {
    p.rad[p.nrad++] = 2;
    m /= 2;
  }
  while (m % 3 == 0) {
    p.rad[p.nrad++] = 3;
    m /= 3;
  }
  return m == 1 && p.nrad <= 12;
}

// Apply the twiddle of a forward (sign=-1) or inverse (sign=+1) transform.
template <typename T>
__device__ __forceinline__ cpx<T> twiddle(const cpx<T>* __restrict__ tw, int idx,
                                          int sign) {
  cpx<T> w = tw[idx];
  if (sign > 0) w.im = -w.im;
  return w;
}

// One Stockham pass over all columns: reads `a`, writes `b`.
template <typename T>
__device__ __forceinline__ void fft_pass(const cpx<T>* __restrict__ a, cpx<T>* __restrict__ b,
                                         int n, int R, int Ns, int ncol, int ldc,
                                         const cpx<T>* __restrict__ tw, int sign, int tid,
                                         int nthr) {
  const int nb = n / R;
  const int tstride = n / (Ns * R);
  for (int w = tid; w < nb * ncol; w += nthr) {
    const int col = w % ncol;
    const int j = w / ncol;
    const int k = j % Ns;
    cpx<T> v[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      if (r < R) {
        cpx<T> x = a[(j + r * nb) * ldc + col];
        if (r > 0 && k > 0) x = x * twiddle(tw, r * k * tstride, sign);
        v[r] = x;
      }
    }
    cpx<T> o[4];
    if (R == 2) {
      o[0] = v[0] + v[1];
      o[1] = v[0] - v[1];
    } else if (R == 4) {
      // W4 = exp(sign * 2 pi i / 4) = sign * i
      const cpx<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
      const cpx<T> t2 = v[1] + v[3];
      cpx<T> t3 = v[1] - v[3];
      t3 = sign > 0 ? mul_i(t3) : cmk(t3.im, -t3.re);  // sign * i * t3
      o[0] = t0 + t2;
      o[1] = t1 + t3;
      o[2] = t0 - t2;
      o[3] = t1 - t3;
    } else {  // R == 3, W3 = exp(sign * 2 pi i / 3) = tw[n/3] (conj for inverse)
      const cpx<T> w3 = twiddle(tw, n / 3, sign);
      const cpx<T> t1 = v[1] + v[2];
      const cpx<T> t2 = v[1] - v[2];
      const cpx<T> m = cmk(v[0].re + w3.re * t1.re, v[0].im + w3.re * t1.im);
      const cpx<T> s = cmk(-w3.im * t2.im, w3.im * t2.re);  // i * Im(W3) * t2
      o[0] = v[0] + t1;
      o[1] = m + s;
      o[2] = m - s;
    }
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (r < R) b[(idxD + r * Ns) * ldc + col] = o[r];
  }
}

// Full transform of `ncol` columns.  Ping-pongs between a and b with a
// __syncthreads() after each pass; returns the buffer holding the result.
// All threads of the block must call it.
template <typename T>
__device__ cpx<T>* fft_columns(cpx<T>* a, cpx<T>* b, const FFTPlan& plan, int ncol,
                               int ldc, const cpx<T>* __restrict__ tw, int sign) {
  int Ns = 1;
  for (int ps = 0; ps < plan.nrad; ++ps) {
    const int R = plan.rad[ps];
    fft_pass<T>(a, b, plan.n, R, Ns, ncol, ldc, tw, sign, threadIdx.x, blockDim.x);
    __syncthreads();
    cpx<T>* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace jfb
