// Warp-shuffle FFT versions of the periodic-axis kernels of the KMM step
// (used when the transform lengths are 32 P with P in {2, 3, 4, 6}).
#pragma once

#include <cooperative_groups.h>

#include "jfb_kmm_kernels.cuh"
#include "jfb_warpfft.cuh"

namespace jfb {

// ---------------------------------------------------------------------------
// y_backward: per (x-plane, field, kz chunk of KC columns).  The chunk is
// staged in shared memory, each warp transforms whole columns in registers
// (zero padding Ny -> My in the middle of the spectrum), and the padded
// plane is written back with coalesced rows.
// ---------------------------------------------------------------------------
template <int P, typename T>
__device__ __forceinline__ void y_backward_warp_body(const Dims& d, const int KC,
                                                     const cpx<T>* __restrict__ tw,
                                                     const cpx<T>* __restrict__ X,
                                                     cpx<T>* __restrict__ Y, const int j,
                                                     const int f, const int zc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ld = KC + 1;
  cpx<T>* in = reinterpret_cast<cpx<T>*>(smem_raw);  // Ny x ld
  cpx<T>* out = in + d.Ny * ld;                   // My x ld
  const int kc0 = zc * KC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const cpx<T>* src = X + ((size_t)f * d.Nx + j) * d.P + kc0;
  const int kcn = min(KC, d.Kz - kc0);  // columns of this chunk (the last may be partial)
  for (int idx = threadIdx.x; idx < d.Ny * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    in[r * ld + c] = (c < kcn) ? src[(size_t)r * d.Kz + c] : cmk(T(0), T(0));
  }
  WarpTw<P, T> w;
  load_warp_tw<P, T>(w, tw, lane);
  __syncthreads();
  const int half = d.Ny / 2;
  for (int c = warp; c < KC; c += blockDim.x / 32) {
    cpx<T> v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int k = 32 * r + lane;
      cpx<T> z = cmk(T(0), T(0));
      if (k < half) z = in[k * ld + c];
      else if (k >= d.My - half) z = in[(k - d.My + d.Ny) * ld + c];
      v[r] = z;
    }
    warp_fft_inverse<P, T>(v, w, lane);
    const int br = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) out[(k1 + P * br) * ld + c] = v[k1];
  }
  __syncthreads();
  cpx<T>* dst = Y + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    if (c < kcn) dst[(size_t)r * d.Kz + c] = out[r * ld + c];
  }
}

template <int P, typename T>
__global__ void __launch_bounds__(256) y_backward_warp_kernel(const __grid_constant__ Dims d, int KC,
                                                              const cpx<T>* __restrict__ tw,
                                                              const cpx<T>* __restrict__ X,
                                                              cpx<T>* __restrict__ Y) {
  y_backward_warp_body<P, T>(d, KC, tw, X, Y, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// y_forward: per (x-plane, field, kz chunk): forward FFT My along y, keep the
// Ny retained modes (Nyquist zeroed), scale 1/My.
// ---------------------------------------------------------------------------
template <int P, typename T>
__device__ __forceinline__ void y_forward_warp_body(const Dims& d, const int KC,
                                                    const cpx<T>* __restrict__ tw,
                                                    const cpx<T>* __restrict__ HZ,
                                                    cpx<T>* __restrict__ HX,
                                                    const double* __restrict__ xb, const int j,
                                                    const int f, const int zc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ld = KC + 1;
  cpx<T>* in = reinterpret_cast<cpx<T>*>(smem_raw);  // My x ld
  cpx<T>* out = in + d.My * ld;                   // Ny x ld
  const int kc0 = zc * KC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const cpx<T>* src = HZ + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  const int kcn = min(KC, d.Kz - kc0);  // columns of this chunk (the last may be partial)
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    in[r * ld + c] = (c < kcn) ? src[(size_t)r * d.Kz + c] : cmk(T(0), T(0));
  }
  WarpTw<P, T> w;
  load_warp_tw<P, T>(w, tw, lane);
  __syncthreads();
  const int half = d.Ny / 2;
  const T scale = T(1.0 / d.My);
  const int br = bitrev5(lane);
  for (int c = warp; c < KC; c += blockDim.x / 32) {
    cpx<T> v[P];
#pragma unroll
    for (int n1 = 0; n1 < P; ++n1) v[n1] = in[(n1 + P * br) * ld + c];
    warp_fft_forward<P, T>(v, w, lane);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      const int k = 32 * k1 + lane;
      if (k < half) out[k * ld + c] = scale * v[k1];
      else if (k > d.My - half) out[(k - d.My + d.Ny) * ld + c] = scale * v[k1];
      else if (k == d.My - half) out[half * ld + c] = cmk(T(0), T(0));  // Nyquist
    }
  }
  __syncthreads();
  if (xb && f == 0 && kc0 == 0 && threadIdx.x == 0) {
    // base-flow self term -U_b U_wall e_x: its (ky, kz) = (0, 0) mode
    out[0].re += T(-d.uwall * xb[j] * d.uwall);
  }
  __syncthreads();
  cpx<T>* dst = HX + ((size_t)f * d.Nx + j) * d.P + kc0;
  for (int idx = threadIdx.x; idx < d.Ny * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    if (c < kcn) dst[(size_t)r * d.Kz + c] = out[r * ld + c];
  }
}

template <int P, typename T>
__global__ void __launch_bounds__(256) y_forward_warp_kernel(const __grid_constant__ Dims d, int KC,
                                                             const cpx<T>* __restrict__ tw,
                                                             const cpx<T>* __restrict__ HZ,
                                                             cpx<T>* __restrict__ HX,
                                                             const double* __restrict__ xb) {
  y_forward_warp_body<P, T>(d, KC, tw, HZ, HX, xb, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Hermitian-extended packed spectrum Z = A + i B of two real fields whose
// half spectra (k < Kz) are held as A[q], B[q] at lane l (k = 32 q + l).
// Z[r] at lane l is Z_(32 r + l) of the length-N = 32 P transform.
template <int P, int QK, typename T>
__device__ __forceinline__ void build_packed(const cpx<T> (&A)[QK], const cpx<T> (&B)[QK], int Kz,
                                             int lane, cpx<T> (&Z)[P]) {
  constexpr int N = 32 * P;
#pragma unroll
  for (int r = 0; r < P; ++r) {
    const int k = 32 * r + lane;
    cpx<T> z = cmk(T(0), T(0));
    if (r < QK && k < Kz) {
      z = (k == 0) ? cmk(A[r].re, B[r].re) : cmk(A[r].re - B[r].im, A[r].im + B[r].re);
    }
    // mirror kk = N - k: lane >= 1 -> (q = P - r - 1, lane 32 - l); lane 0 -> (q = P - r, lane 0)
    constexpr int dummy = 0;
    (void)dummy;
    const int q1 = P - r - 1, q0 = P - r;
    cpx<T> a1 = cmk(T(0), T(0)), b1 = a1, a0 = a1, b0 = a1;
#pragma unroll
    for (int q = 0; q < QK; ++q) {
      if (q == q1) {
        a1 = shfl_c(A[q], (32 - lane) & 31);
        b1 = shfl_c(B[q], (32 - lane) & 31);
      }
      if (q == q0) {
        a0 = shfl_c(A[q], 0);
        b0 = shfl_c(B[q], 0);
      }
    }
    if (k > N - Kz) {
      const int kk = N - k;
      if (kk < Kz) {
        const cpx<T> a = (lane != 0) ? a1 : a0;
        const cpx<T> b = (lane != 0) ? b1 : b0;
        z = cmk(a.re + b.im, b.re - a.im);
      }
    }
    Z[r] = z;
  }
}

// From a natural-order forward transform F of z = x + i y, the half spectra
// X_k, Y_k at k = 32 q + lane (q < QK): X = (F_k + conj F_{N-k}) / 2,
// Y = (F_k - conj F_{N-k}) / (2 i).
template <int P, int QK, typename T>
__device__ __forceinline__ void unpack_pair(const cpx<T> (&F)[P], int lane, cpx<T> (&Xo)[QK],
                                            cpx<T> (&Yo)[QK]) {
#pragma unroll
  for (int q = 0; q < QK; ++q) {
    const cpx<T> m1 = shfl_c(F[(P - q - 1 + P) % P], (32 - lane) & 31);
    const cpx<T> m0 = shfl_c(F[(P - q) % P], 0);
    const cpx<T> Zm = (lane != 0) ? m1 : m0;
    const cpx<T> Zk = F[q];
    const T h = T(0.5);
    Xo[q] = cmk(h * (Zk.re + Zm.re), h * (Zk.im - Zm.im));
    Yo[q] = cmk(h * (Zk.im + Zm.im), -h * (Zk.re - Zm.re));
  }
}

// ---------------------------------------------------------------------------
// z_cross: one warp per pair of (x, y) rows, everything in registers.
// ---------------------------------------------------------------------------
template <int P, int QK, typename T>
__global__ void __launch_bounds__(256) z_cross_warp_kernel(DevOps o, Dims d,
                                                           const cpx<T>* __restrict__ tw,
                                                           const cpx<T>* __restrict__ Y,
                                                           cpx<T>* __restrict__ HZ) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int nrows = d.Nx * d.My;
  const int rowa = 2 * pair;
  if (rowa >= nrows) return;
  const bool hasb = rowa + 1 < nrows;
  WarpTw<P, T> w;
  load_warp_tw<P, T>(w, tw, lane);
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  T nrm[2][3][P];  // products n0, n1, n2 per row, scrambled layout
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int row = rowa + rb;
    const bool ok = rb == 0 || hasb;
    cpx<T> ph[3][P];
#pragma unroll
    for (int pr = 0; pr < 3; ++pr) {
      cpx<T> A[QK], B[QK];
#pragma unroll
      for (int q = 0; q < QK; ++q) {
        const int k = 32 * q + lane;
        const bool in = ok && k < d.Kz;
        A[q] = in ? Y[(size_t)(2 * pr) * plane + (size_t)row * d.Kz + k] : cmk(T(0), T(0));
        B[q] = in ? Y[(size_t)(2 * pr + 1) * plane + (size_t)row * d.Kz + k] : cmk(T(0), T(0));
      }
      build_packed<P, QK, T>(A, B, d.Kz, lane, ph[pr]);
      warp_fft_inverse<P, T>(ph[pr], w, lane);
    }
    const int j = (ok ? row : rowa) / d.My;
    const T ub = T(d.uwall * o.xphys[j]), uw = T(d.uwall);
#pragma unroll
    for (int r = 0; r < P; ++r) {
      rotational_product(ph[0][r].re, ph[0][r].im, ph[1][r].re, ph[1][r].im, ph[2][r].re,
                         ph[2][r].im, ub, uw, nrm[rb][0][r], nrm[rb][1][r], nrm[rb][2][r]);
    }
  }
  cpx<T> F0[P], F1[P], F2[P];
#pragma unroll
  for (int r = 0; r < P; ++r) {
    F0[r] = cmk(nrm[0][0][r], nrm[0][1][r]);
    F1[r] = cmk(nrm[1][0][r], nrm[1][1][r]);
    F2[r] = cmk(nrm[0][2][r], nrm[1][2][r]);
  }
  warp_fft_forward<P, T>(F0, w, lane);
  warp_fft_forward<P, T>(F1, w, lane);
  warp_fft_forward<P, T>(F2, w, lane);
  cpx<T> xa0[QK], xa1[QK], xb0[QK], xb1[QK], x2a[QK], x2b[QK];
  unpack_pair<P, QK, T>(F0, lane, xa0, xa1);
  unpack_pair<P, QK, T>(F1, lane, xb0, xb1);
  unpack_pair<P, QK, T>(F2, lane, x2a, x2b);
  const T scale = T(1.0 / (32 * P));
#pragma unroll
  for (int q = 0; q < QK; ++q) {
    const int k = 32 * q + lane;
    if (k >= d.Kz) continue;
    HZ[(size_t)0 * plane + (size_t)rowa * d.Kz + k] = scale * xa0[q];
    HZ[(size_t)1 * plane + (size_t)rowa * d.Kz + k] = scale * xa1[q];
    HZ[(size_t)2 * plane + (size_t)rowa * d.Kz + k] = scale * x2a[q];
    if (hasb) {
      HZ[(size_t)0 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb0[q];
      HZ[(size_t)1 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb1[q];
      HZ[(size_t)2 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * x2b[q];
    }
  }
}

// ---------------------------------------------------------------------------
// z_grad: the gradient form's z stage (z_grad_kernel) with warp-shuffle
// transforms, one warp per pair of (x, y) rows.  Per row, the twelve
// real fields u_i, d/dx u_i, d/dy u_i (Y fields 0..8) and d/dz u_i = i kz u_i
// (formed here) go through six packed inverse transforms; the three products
// n_i = u . grad u_i + U_b d/dy u_i (+ u_0 dU_b/dx for i = 1) of the row
// pair go through three packed forward transforms.
// ---------------------------------------------------------------------------
template <int P, int QK, typename T>
__global__ void __launch_bounds__(256) z_grad_warp_kernel(DevOps o, Dims d,
                                                          const cpx<T>* __restrict__ tw,
                                                          const cpx<T>* __restrict__ Y,
                                                          cpx<T>* __restrict__ HZ) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int nrows = d.Nx * d.My;
  const int rowa = 2 * pair;
  if (rowa >= nrows) return;
  const bool hasb = rowa + 1 < nrows;
  WarpTw<P, T> w;
  load_warp_tw<P, T>(w, tw, lane);
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  T nrm[2][3][P];
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int row = rowa + rb;
    const bool ok = rb == 0 || hasb;
    // virtual real field v of the row at spectral index k: Y field v (v < 9)
    // or i kz times Y field v - 9
    auto spec = [&](int v, int k) -> cpx<T> {
      if (!ok || k >= d.Kz) return cmk(T(0), T(0));
      const cpx<T> x = Y[(size_t)(v < 9 ? v : v - 9) * plane + (size_t)row * d.Kz + k];
      return v < 9 ? x : mul_i(T(k * d.dfz) * x);
    };
    cpx<T> ph[6][P];
#pragma unroll
    for (int pr = 0; pr < 6; ++pr) {
      cpx<T> A[QK], B[QK];
#pragma unroll
      for (int q = 0; q < QK; ++q) {
        A[q] = spec(2 * pr, 32 * q + lane);
        B[q] = spec(2 * pr + 1, 32 * q + lane);
      }
      build_packed<P, QK, T>(A, B, d.Kz, lane, ph[pr]);
      warp_fft_inverse<P, T>(ph[pr], w, lane);
    }
    const int j = (ok ? row : rowa) / d.My;
    const T ub = T(d.uwall * o.xphys[j]), uw = T(d.uwall);
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const T u0 = ph[0][r].re, u1 = ph[0][r].im, u2 = ph[1][r].re;
      const T x0 = ph[1][r].im, x1 = ph[2][r].re, x2 = ph[2][r].im;  // d/dx
      const T y0 = ph[3][r].re, y1 = ph[3][r].im, y2 = ph[4][r].re;  // d/dy
      const T z0 = ph[4][r].im, z1 = ph[5][r].re, z2 = ph[5][r].im;  // d/dz
      nrm[rb][0][r] = (u0 * x0 + u1 * y0 + u2 * z0) + ub * y0;
      nrm[rb][1][r] = ((u0 * x1 + u1 * y1 + u2 * z1) + ub * y1) + u0 * uw;
      nrm[rb][2][r] = (u0 * x2 + u1 * y2 + u2 * z2) + ub * y2;
    }
  }
  cpx<T> F0[P], F1[P], F2[P];
#pragma unroll
  for (int r = 0; r < P; ++r) {
    F0[r] = cmk(nrm[0][0][r], nrm[0][1][r]);
    F1[r] = cmk(nrm[1][0][r], nrm[1][1][r]);
    F2[r] = cmk(nrm[0][2][r], nrm[1][2][r]);
  }
  warp_fft_forward<P, T>(F0, w, lane);
  warp_fft_forward<P, T>(F1, w, lane);
  warp_fft_forward<P, T>(F2, w, lane);
  cpx<T> xa0[QK], xa1[QK], xb0[QK], xb1[QK], x2a[QK], x2b[QK];
  unpack_pair<P, QK, T>(F0, lane, xa0, xa1);
  unpack_pair<P, QK, T>(F1, lane, xb0, xb1);
  unpack_pair<P, QK, T>(F2, lane, x2a, x2b);
  const T scale = T(1.0 / (32 * P));
#pragma unroll
  for (int q = 0; q < QK; ++q) {
    const int k = 32 * q + lane;
    if (k >= d.Kz) continue;
    HZ[(size_t)0 * plane + (size_t)rowa * d.Kz + k] = scale * xa0[q];
    HZ[(size_t)1 * plane + (size_t)rowa * d.Kz + k] = scale * xa1[q];
    HZ[(size_t)2 * plane + (size_t)rowa * d.Kz + k] = scale * x2a[q];
    if (hasb) {
      HZ[(size_t)0 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb0[q];
      HZ[(size_t)1 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb1[q];
      HZ[(size_t)2 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * x2b[q];
    }
  }
}

// ---------------------------------------------------------------------------
// z_forward_real: three real fields (Nx, Ny, Nz) -> half spectra along z,
// scaled 1/Nz.  One warp per pair of rows.
// ---------------------------------------------------------------------------
template <int P, int QK>
__global__ void __launch_bounds__(256) z_forward_real_warp_kernel(
    Dims d, const c64* __restrict__ tw, const double* __restrict__ f0,
    const double* __restrict__ f1, const double* __restrict__ f2, c64* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int nrows = d.Nx * d.Ny;
  const int rowa = 2 * pair;
  if (rowa >= nrows) return;
  const bool hasb = rowa + 1 < nrows;
  constexpr int N = 32 * P;
  WarpTw<P, double> w;
  load_warp_tw<P, double>(w, tw, lane);
  const int br = bitrev5(lane);
  c64 F0[P], F1[P], F2[P];
#pragma unroll
  for (int n1 = 0; n1 < P; ++n1) {
    const int z = n1 + P * br;
    const size_t ea = (size_t)rowa * N + z;
    const size_t eb = (size_t)(rowa + 1) * N + z;
    F0[n1] = cmk(f0[ea], f1[ea]);
    F1[n1] = hasb ? cmk(f0[eb], f1[eb]) : cmk(0.0, 0.0);
    F2[n1] = cmk(f2[ea], hasb ? f2[eb] : 0.0);
  }
  warp_fft_forward<P, double>(F0, w, lane);
  warp_fft_forward<P, double>(F1, w, lane);
  warp_fft_forward<P, double>(F2, w, lane);
  c64 xa0[QK], xa1[QK], xb0[QK], xb1[QK], x2a[QK], x2b[QK];
  unpack_pair<P, QK, double>(F0, lane, xa0, xa1);
  unpack_pair<P, QK, double>(F1, lane, xb0, xb1);
  unpack_pair<P, QK, double>(F2, lane, x2a, x2b);
  const size_t plane = (size_t)d.Nx * d.Ny * d.Kz;
  const double scale = 1.0 / N;
#pragma unroll
  for (int q = 0; q < QK; ++q) {
    const int k = 32 * q + lane;
    if (k >= d.Kz) continue;
    out[(size_t)0 * plane + (size_t)rowa * d.Kz + k] = scale * xa0[q];
    out[(size_t)1 * plane + (size_t)rowa * d.Kz + k] = scale * xa1[q];
    out[(size_t)2 * plane + (size_t)rowa * d.Kz + k] = scale * x2a[q];
    if (hasb) {
      out[(size_t)0 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb0[q];
      out[(size_t)1 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * xb1[q];
      out[(size_t)2 * plane + (size_t)(rowa + 1) * d.Kz + k] = scale * x2b[q];
    }
  }
}


// ---------------------------------------------------------------------------
// plane_cross: y_backward -> z_cross -> y_forward of one x-plane in one
// launch, on a cluster of two CTAs (distributed shared memory, no
// multicast).  CTA `rank` owns kz columns [rank Kz/2, (rank+1) Kz/2) for the
// y transforms and padded rows [rank My/2, (rank+1) My/2) for the z stage:
//   1. inverse y FFT (Ny -> My, zero padded) of the six fields of its
//      columns into Ys[f][y][col] (own shared memory);
//   2. per pair of its rows: the six half spectra along z, half of them read
//      from the peer's Ys, inverse real z FFTs, base flow, -(u x omega),
//      forward real z FFTs -> Hs[f][row][kz] (own shared memory, kz XOR
//      swizzled by row when Kz is a multiple of 8);
//   3. forward y FFT (My -> Ny, truncation, Nyquist zeroed) of the three
//      fields of its columns, rows read from both CTAs' Hs, into HX.
// Cluster barriers separate the stages and keep each CTA's shared memory
// alive until the peer has finished reading it.
// ---------------------------------------------------------------------------
#ifndef JFB_PLANE_THREADS_F64
#define JFB_PLANE_THREADS_F64 384
#endif
// threads per CTA of the plane kernel: twelve warps, whose registers (up to
// 168 per thread) suit the z stage better than sixteen warps at 128 (measured
// at 65x64x64, per CTA: FP64 53.6 us against 58.5 us with sixteen warps and
// 54.6 us with eight; FP32 26.4 us against 27.5 us with sixteen)
#ifndef JFB_PLANE_THREADS_F32
#define JFB_PLANE_THREADS_F32 384
#endif
template <typename T>
__host__ __device__ constexpr int plane_threads() {
  return sizeof(T) == 8 ? JFB_PLANE_THREADS_F64 : JFB_PLANE_THREADS_F32;
}

__host__ __device__ inline size_t plane_smem_bytes(int My, int Kz, size_t elem) {
  return (size_t)6 * My * (Kz / 2 + 1) * elem + (size_t)3 * (My / 2) * Kz * elem;
}

template <int PY, int PZ, int QK, typename T>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(plane_threads<T>(), 1)
    plane_cross_kernel(DevOps o, Dims d, const cpx<T>* __restrict__ twy,
                       const cpx<T>* __restrict__ twz, const cpx<T>* __restrict__ X,
                       cpx<T>* __restrict__ HX) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int MY = 32 * PY, MH = MY / 2, MZ = 32 * PZ;
  const int rank = (int)cluster.block_rank();
  const int j = blockIdx.x >> 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kPlaneThreads = plane_threads<T>();
  constexpr int NW = kPlaneThreads / 32;
  const int Kz = d.Kz, KH = Kz / 2, LDZ = KH + 1;
  const bool swz = (Kz & 7) == 0;
  cpx<T>* Ys = reinterpret_cast<cpx<T>*>(smem_raw);  // [6][MY][LDZ]
  cpx<T>* Hs = Ys + (size_t)6 * MY * LDZ;              // [3][MH][Kz]
  const cpx<T>* Ypeer = cluster.map_shared_rank(Ys, rank ^ 1);
  const cpx<T>* Hpeer = cluster.map_shared_rank(Hs, rank ^ 1);
  const size_t P = (size_t)d.P;
  const int half = d.Ny / 2;
  const int br = bitrev5(lane);
  JFB_STAMP(1, 0);
  pdl_trigger();
  pdl_wait();  // X is written by the previous kernel, HX still read by it
  JFB_STAMP(1, 1);

  // 1. inverse y transforms of this CTA's columns: the six fields staged row
  //    by row (coalesced along kz) into Ys in padded order, then one column
  //    per warp in place
  {
    // half-warp per row (KH <= 16 columns), no per-element index division;
    // FB fields at a time, all loads of a thread before its stores (Ny <=
    // MY <= 96 gives at most three rows per half-warp and field)
    const int hw = threadIdx.x >> 4, cl = threadIdx.x & 15;
    constexpr int RS = kPlaneThreads / 16, RMAX = (MY + RS - 1) / RS;
    constexpr int FB = sizeof(T) == 4 ? 6 : 2;  // register budget of the FP64 form
    if (cl < KH) {
#pragma unroll
      for (int f0 = 0; f0 < 6; f0 += FB) {
        cpx<T> v[FB][RMAX];
#pragma unroll
        for (int f = 0; f < FB; ++f) {
          const cpx<T>* src = X + ((size_t)(f0 + f) * d.Nx + j) * P + rank * KH + cl;
#pragma unroll
          for (int i = 0; i < RMAX; ++i) {
            const int r = hw + RS * i;
            v[f][i] = (r < d.Ny && r != half) ? src[(size_t)r * Kz] : cmk(T(0), T(0));
          }
        }
#pragma unroll
        for (int f = 0; f < FB; ++f) {
          cpx<T>* dst = Ys + (size_t)(f0 + f) * MY * LDZ + cl;
#pragma unroll
          for (int i = 0; i < RMAX; ++i) {
            const int r = hw + RS * i;  // the Nyquist row r == half stays zero
            if (r < d.Ny) dst[(size_t)((r < half) ? r : r - d.Ny + MY) * LDZ] = v[f][i];
          }
          // padding rows half .. MY - half - 1 (row MY - half is the Nyquist
          // row's slot, zeroed above)
          for (int k = half + hw; k < MY - half; k += RS) dst[(size_t)k * LDZ] = cmk(T(0), T(0));
        }
      }
    }
    __syncthreads();
    JFB_STAMP(1, 2);
    WarpTw<PY, T> w;
    load_warp_tw<PY, T>(w, twy, lane);
    for (int t = warp; t < 6 * KH; t += NW) {
      const int f = t / KH, cl = t % KH;
      cpx<T>* col = Ys + (size_t)f * MY * LDZ + cl;
      cpx<T> v[PY];
#pragma unroll
      for (int r = 0; r < PY; ++r) v[r] = col[(size_t)(32 * r + lane) * LDZ];
      __syncwarp();
      warp_fft_inverse<PY, T>(v, w, lane);
#pragma unroll
      for (int k1 = 0; k1 < PY; ++k1) col[(size_t)(k1 + PY * br) * LDZ] = v[k1];
    }
  }
  cluster.sync();
  JFB_STAMP(1, 3);

  // 2. z stage on this CTA's rows (two, or at 96 points three, per warp)
  {
    WarpTw<PZ, T> w;
    load_warp_tw<PZ, T>(w, twz, lane);
    const T ub = T(d.uwall * o.xphys[j]), uw = T(d.uwall);
    const T scale = T(1.0 / MZ);
    // rows ya and (if hasb) ya + 1 of this CTA: inverse real z FFTs of the
    // six fields (two per complex FFT), -(u x omega), forward real z FFTs
    // of the three products (two rows per complex FFT; a lone row pairs its
    // third product with zero)
    auto z_rows = [&](int ya, bool hasb) {
      T nrm[2][3][PZ];
#pragma unroll
      for (int rb = 0; rb < 2; ++rb) {
        if (rb == 1 && !hasb) {
#pragma unroll
          for (int r = 0; r < PZ; ++r) nrm[1][0][r] = nrm[1][1][r] = nrm[1][2][r] = T(0);
          break;
        }
        const int y = rank * MH + ya + rb;
        cpx<T> ph[3][PZ];
#pragma unroll
        for (int pr = 0; pr < 3; ++pr) {
          cpx<T> A[QK], B[QK];
#pragma unroll
          for (int q = 0; q < QK; ++q) {
            const int kz = 32 * q + lane;
            A[q] = B[q] = cmk(T(0), T(0));
            if (kz < Kz) {
              const int own = kz >= KH, cl = kz - own * KH;
              const cpx<T>* base = (own == rank) ? Ys : Ypeer;
              A[q] = base[((size_t)(2 * pr) * MY + y) * LDZ + cl];
              B[q] = base[((size_t)(2 * pr + 1) * MY + y) * LDZ + cl];
            }
          }
          build_packed<PZ, QK, T>(A, B, Kz, lane, ph[pr]);
          warp_fft_inverse<PZ, T>(ph[pr], w, lane);
        }
#pragma unroll
        for (int r = 0; r < PZ; ++r) {
          rotational_product(ph[0][r].re, ph[0][r].im, ph[1][r].re, ph[1][r].im, ph[2][r].re,
                             ph[2][r].im, ub, uw, nrm[rb][0][r], nrm[rb][1][r], nrm[rb][2][r]);
        }
      }
      cpx<T> F0[PZ], F1[PZ], F2[PZ];
#pragma unroll
      for (int r = 0; r < PZ; ++r) {
        F0[r] = cmk(nrm[0][0][r], nrm[0][1][r]);
        F1[r] = cmk(nrm[1][0][r], nrm[1][1][r]);
        F2[r] = cmk(nrm[0][2][r], nrm[1][2][r]);
      }
      warp_fft_forward<PZ, T>(F0, w, lane);
      if (hasb) warp_fft_forward<PZ, T>(F1, w, lane);
      warp_fft_forward<PZ, T>(F2, w, lane);
      cpx<T> xa0[QK], xa1[QK], xb0[QK], xb1[QK], x2a[QK], x2b[QK];
      unpack_pair<PZ, QK, T>(F0, lane, xa0, xa1);
      if (hasb) unpack_pair<PZ, QK, T>(F1, lane, xb0, xb1);
      unpack_pair<PZ, QK, T>(F2, lane, x2a, x2b);
      const int yb = ya + 1;  // local rows
#pragma unroll
      for (int q = 0; q < QK; ++q) {
        const int kz = 32 * q + lane;
        if (kz >= Kz) continue;
        const int ca = swz ? (kz ^ (ya & 7)) : kz, cb = swz ? (kz ^ (yb & 7)) : kz;
        Hs[((size_t)0 * MH + ya) * Kz + ca] = scale * xa0[q];
        Hs[((size_t)1 * MH + ya) * Kz + ca] = scale * xa1[q];
        Hs[((size_t)2 * MH + ya) * Kz + ca] = scale * x2a[q];
        if (hasb) {
          Hs[((size_t)0 * MH + yb) * Kz + cb] = scale * xb0[q];
          Hs[((size_t)1 * MH + yb) * Kz + cb] = scale * xb1[q];
          Hs[((size_t)2 * MH + yb) * Kz + cb] = scale * x2b[q];
        }
      }
    };
    if (MH == 3 * NW) {  // three rows per warp: a pair and a lone row
      z_rows(3 * warp, true);
      z_rows(3 * warp + 2, false);
    } else {
      for (int pair = warp; pair < MH / 2; pair += NW) z_rows(2 * pair, true);
    }
  }
  cluster.sync();
  JFB_STAMP(1, 4);

  // 3. forward y transforms of this CTA's columns into Ys (free once the
  //    peer has passed the barrier above), then row-wise coalesced stores
  {
    WarpTw<PY, T> w;
    load_warp_tw<PY, T>(w, twy, lane);
    const T scale = T(1.0 / MY);
    for (int t = warp; t < 3 * KH; t += NW) {
      const int f = t / KH, cl = t % KH, kz = rank * KH + cl;
      cpx<T> v[PY];
#pragma unroll
      for (int n1 = 0; n1 < PY; ++n1) {
        const int y = n1 + PY * br;
        const int own = y / MH, yl = y - own * MH;
        const cpx<T>* base = (own == rank) ? Hs : Hpeer;
        v[n1] = base[((size_t)f * MH + yl) * Kz + (swz ? (kz ^ (yl & 7)) : kz)];
      }
      warp_fft_forward<PY, T>(v, w, lane);
      cpx<T>* col = Ys + (size_t)f * MY * LDZ + cl;
#pragma unroll
      for (int k1 = 0; k1 < PY; ++k1) col[(size_t)(32 * k1 + lane) * LDZ] = scale * v[k1];
    }
    __syncthreads();
    JFB_STAMP(1, 5);
    for (int e = threadIdx.x; e < 3 * d.Ny * KH; e += kPlaneThreads) {
      const int cl = e % KH, rf = e / KH, r = rf % d.Ny, f = rf / d.Ny;
      const int kz = rank * KH + cl;
      cpx<T> val = cmk(T(0), T(0));  // r == half: Nyquist row
      if (r != half) {
        const int k = (r < half) ? r : r - d.Ny + MY;
        val = Ys[((size_t)f * MY + k) * LDZ + cl];
        if (f == 0 && kz == 0 && r == 0) val.re += T(-d.uwall * o.xphys[j] * d.uwall);
      }
      HX[((size_t)f * d.Nx + j) * P + (size_t)r * Kz + kz] = val;
    }
  }
  JFB_STAMP(1, 6);
  cluster.sync();
  JFB_STAMP(1, 7);
}

}  // namespace jfb
