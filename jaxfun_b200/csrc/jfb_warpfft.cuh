// Register-resident warp FFTs of length N = 32 P (P in {2, 3, 4, 6}): the
// periodic-axis transforms of the Couette grid (64, 96, 128, 192 points).
//
// Four-step split N = P x 32: a P-point DFT in registers, twiddles
// W_N^(lane k1), then a 32-point radix-2 transform across the lanes with
// __shfl_xor_sync butterflies.
//   inverse (natural in -> scrambled out), 32-point part decimation in
//   frequency:  in v[r] at lane l  = Z[32 r + l]
//               out v[k1] at lane l = x[k1 + P bitrev5(l)]
//   forward (scrambled in -> natural out), 32-point part decimation in time:
//               in v[n1] at lane l  = x[n1 + P bitrev5(l)]
//               out v[k1] at lane l = X[32 k1 + l]
// so a pointwise product between an inverse and a forward transform needs no
// reordering.  Twiddles come from the host table tw[k] = exp(-2 pi i k / N);
// the inverse uses their conjugates.  Unnormalised (numpy "forward" norm
// applied by the caller).
#pragma once

#include "jfb_common.cuh"

namespace jfb {

__device__ __forceinline__ int bitrev5(int x) { return (int)(__brev((unsigned)x) >> 27); }

template <typename T>
__device__ __forceinline__ cpx<T> shfl_c(cpx<T> v, int src) {
  cpx<T> o;
  o.re = __shfl_sync(0xffffffffu, v.re, src);
  o.im = __shfl_sync(0xffffffffu, v.im, src);
  return o;
}
template <typename T>
__device__ __forceinline__ cpx<T> shfl_xor_c(cpx<T> v, int m) {
  cpx<T> o;
  o.re = __shfl_xor_sync(0xffffffffu, v.re, m);
  o.im = __shfl_xor_sync(0xffffffffu, v.im, m);
  return o;
}

// Per-lane twiddles of one transform length (forward sign).
template <int P, typename T>
struct WarpTw {
  cpx<T> lane_k1[P];  // W_N^(lane * k1)
  cpx<T> stage[5];    // W_{2h}^(lane mod h), h = 16, 8, 4, 2, 1
  cpx<T> wp[P];       // W_P^m
};

template <int P, typename T>
__device__ __forceinline__ void load_warp_tw(WarpTw<P, T>& w, const cpx<T>* __restrict__ tw,
                                             int lane) {
  constexpr int N = 32 * P;
#pragma unroll
  for (int k1 = 0; k1 < P; ++k1) w.lane_k1[k1] = tw[(lane * k1) % N];
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    w.stage[s] = tw[(lane % h) * (N / (2 * h))];
  }
#pragma unroll
  for (int m = 0; m < P; ++m) w.wp[m] = tw[m * (N / P)];
}

template <typename T>
__device__ __forceinline__ cpx<T> cmul_sign(cpx<T> a, cpx<T> w, bool inverse) {
  if (inverse) w.im = -w.im;
  return a * w;
}

// P-point DFT in registers: out[k] = sum_q in[q] W_P^(+-qk).
template <int P, typename T>
__device__ __forceinline__ void small_dft(cpx<T> (&v)[P], const WarpTw<P, T>& w, bool inverse) {
  if constexpr (P == 2) {
    const cpx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  } else if constexpr (P == 4) {
    const cpx<T> t0 = v[0] + v[2], t1 = v[0] - v[2];
    const cpx<T> t2 = v[1] + v[3];
    cpx<T> t3 = v[1] - v[3];
    t3 = inverse ? mul_i(t3) : cmk(t3.im, -t3.re);
    v[0] = t0 + t2;
    v[1] = t1 + t3;
    v[2] = t0 - t2;
    v[3] = t1 - t3;
  } else if constexpr (P == 3) {
    cpx<T> w3 = w.wp[1];
    if (inverse) w3.im = -w3.im;
    const cpx<T> t1 = v[1] + v[2];
    const cpx<T> t2 = v[1] - v[2];
    const cpx<T> m = cmk(v[0].re + w3.re * t1.re, v[0].im + w3.re * t1.im);
    const cpx<T> s = cmk(-w3.im * t2.im, w3.im * t2.re);
    v[0] = v[0] + t1;
    v[1] = m + s;
    v[2] = m - s;
  } else {
    cpx<T> o[P];
#pragma unroll
    for (int k = 0; k < P; ++k) {
      cpx<T> acc = v[0];
#pragma unroll
      for (int q = 1; q < P; ++q) acc = acc + cmul_sign(v[q], w.wp[(q * k) % P], inverse);
      o[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = o[k];
  }
}

// inverse (sign +1): natural -> scrambled
template <int P, typename T>
__device__ __forceinline__ void warp_fft_inverse(cpx<T> (&v)[P], const WarpTw<P, T>& w,
                                                 int lane) {
  small_dft<P, T>(v, w, true);
#pragma unroll
  for (int k1 = 1; k1 < P; ++k1) v[k1] = cmul_sign(v[k1], w.lane_k1[k1], true);
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const bool bottom = (lane & h) != 0;
    // FP32: top lanes v + p, bottom lanes (p - v) conj(w), formed as
    // (p + sg v) t with (sg, t) = (1, 1) on top, (-1, conj(w)) below
    if constexpr (sizeof(T) == 4) {
      const T sg = bottom ? T(-1) : T(1);
      const cpx<T> t = bottom ? cmk(w.stage[s].re, -w.stage[s].im) : cmk(T(1), T(0));
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const cpx<T> p = shfl_xor_c(v[r], h);
        const cpx<T> d = cmk(p.re + sg * v[r].re, p.im + sg * v[r].im);
        v[r] = d * t;  // t = 1 on the top lanes: exact
      }
    } else {  // FP64: fewer live temporaries (register pressure of its callers)
      cpx<T> tws = w.stage[s];
      tws.im = -tws.im;
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const cpx<T> p = shfl_xor_c(v[r], h);
        v[r] = bottom ? (p - v[r]) * tws : v[r] + p;
      }
    }
  }
}

// forward (sign -1): scrambled -> natural
template <int P, typename T>
__device__ __forceinline__ void warp_fft_forward(cpx<T> (&v)[P], const WarpTw<P, T>& w,
                                                 int lane) {
#pragma unroll
  for (int s = 4; s >= 0; --s) {
    const int h = 16 >> s;
    const bool bottom = (lane & h) != 0;
    const cpx<T> tws = w.stage[s];
    if constexpr (sizeof(T) == 4) {
      const T sg = bottom ? T(-1) : T(1);
#pragma unroll
      for (int r = 0; r < P; ++r) {
        // top lanes: v + p w; bottom lanes: p - v w -- one product per value
        const cpx<T> p = shfl_xor_c(v[r], h);
        const cpx<T> a = bottom ? p : v[r];
        const cpx<T> m = (bottom ? v[r] : p) * tws;
        v[r] = cmk(a.re + sg * m.re, a.im + sg * m.im);
      }
    } else {
#pragma unroll
      for (int r = 0; r < P; ++r) {
        const cpx<T> p = shfl_xor_c(v[r], h);
        v[r] = bottom ? p - v[r] * tws : v[r] + p * tws;
      }
    }
  }
#pragma unroll
  for (int n1 = 1; n1 < P; ++n1) v[n1] = v[n1] * w.lane_k1[n1];
  small_dft<P, T>(v, w, false);
}

}  // namespace jfb
