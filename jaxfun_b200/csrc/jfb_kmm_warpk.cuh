// Warp-shuffle FFT versions of the periodic-axis kernels of the KMM step
// (used when the transform lengths are 32 P with P in {2, 3, 4, 6}).
#pragma once

#include "jfb_kmm_kernels.cuh"
#include "jfb_warpfft.cuh"

namespace jfb {

// ---------------------------------------------------------------------------
// y_backward: per (x-plane, field, kz chunk of KC columns).  The chunk is
// staged in shared memory, each warp transforms whole columns in registers
// (zero padding Ny -> My in the middle of the spectrum), and the padded
// plane is written back with coalesced rows.
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(256) y_backward_warp_kernel(Dims d, int KC,
                                                              const c64* __restrict__ tw,
                                                              const c64* __restrict__ X,
                                                              c64* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ld = KC + 1;
  c64* in = reinterpret_cast<c64*>(smem_raw);  // Ny x ld
  c64* out = in + d.Ny * ld;                   // My x ld
  const int j = blockIdx.x, f = blockIdx.y, kc0 = blockIdx.z * KC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const c64* src = X + ((size_t)f * d.Nx + j) * d.P + kc0;
  for (int idx = threadIdx.x; idx < d.Ny * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    in[r * ld + c] = src[(size_t)r * d.Kz + c];
  }
  WarpTw<P, double> w;
  load_warp_tw<P, double>(w, tw, lane);
  __syncthreads();
  const int half = d.Ny / 2;
  for (int c = warp; c < KC; c += blockDim.x / 32) {
    c64 v[P];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const int k = 32 * r + lane;
      c64 z = cmk(0.0, 0.0);
      if (k < half) z = in[k * ld + c];
      else if (k >= d.My - half) z = in[(k - d.My + d.Ny) * ld + c];
      v[r] = z;
    }
    warp_fft_inverse<P, double>(v, w, lane);
    const int br = bitrev5(lane);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) out[(k1 + P * br) * ld + c] = v[k1];
  }
  __syncthreads();
  c64* dst = Y + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    dst[(size_t)r * d.Kz + c] = out[r * ld + c];
  }
}

// ---------------------------------------------------------------------------
// y_forward: per (x-plane, field, kz chunk): forward FFT My along y, keep the
// Ny retained modes (Nyquist zeroed), scale 1/My.
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(256) y_forward_warp_kernel(Dims d, int KC,
                                                             const c64* __restrict__ tw,
                                                             const c64* __restrict__ HZ,
                                                             c64* __restrict__ HX) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int ld = KC + 1;
  c64* in = reinterpret_cast<c64*>(smem_raw);  // My x ld
  c64* out = in + d.My * ld;                   // Ny x ld
  const int j = blockIdx.x, f = blockIdx.y, kc0 = blockIdx.z * KC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const c64* src = HZ + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    in[r * ld + c] = src[(size_t)r * d.Kz + c];
  }
  WarpTw<P, double> w;
  load_warp_tw<P, double>(w, tw, lane);
  __syncthreads();
  const int half = d.Ny / 2;
  const double scale = 1.0 / d.My;
  const int br = bitrev5(lane);
  for (int c = warp; c < KC; c += blockDim.x / 32) {
    c64 v[P];
#pragma unroll
    for (int n1 = 0; n1 < P; ++n1) v[n1] = in[(n1 + P * br) * ld + c];
    warp_fft_forward<P, double>(v, w, lane);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) {
      const int k = 32 * k1 + lane;
      if (k < half) out[k * ld + c] = scale * v[k1];
      else if (k > d.My - half) out[(k - d.My + d.Ny) * ld + c] = scale * v[k1];
      else if (k == d.My - half) out[half * ld + c] = cmk(0.0, 0.0);  // Nyquist
    }
  }
  __syncthreads();
  c64* dst = HX + ((size_t)f * d.Nx + j) * d.P + kc0;
  for (int idx = threadIdx.x; idx < d.Ny * KC; idx += blockDim.x) {
    const int c = idx % KC, r = idx / KC;
    dst[(size_t)r * d.Kz + c] = out[r * ld + c];
  }
}

// Hermitian-extended packed spectrum Z = A + i B of two real fields whose
// half spectra (k < Kz) are held as A[q], B[q] at lane l (k = 32 q + l).
// Z[r] at lane l is Z_(32 r + l) of the length-N = 32 P transform.
template <int P, int QK>
__device__ __forceinline__ void build_packed(const c64 (&A)[QK], const c64 (&B)[QK], int Kz,
                                             int lane, c64 (&Z)[P]) {
  constexpr int N = 32 * P;
#pragma unroll
  for (int r = 0; r < P; ++r) {
    const int k = 32 * r + lane;
    c64 z = cmk(0.0, 0.0);
    if (r < QK && k < Kz) {
      z = (k == 0) ? cmk(A[r].re, B[r].re) : cmk(A[r].re - B[r].im, A[r].im + B[r].re);
    }
    // mirror kk = N - k: lane >= 1 -> (q = P - r - 1, lane 32 - l); lane 0 -> (q = P - r, lane 0)
    constexpr int dummy = 0;
    (void)dummy;
    const int q1 = P - r - 1, q0 = P - r;
    c64 a1 = cmk(0.0, 0.0), b1 = a1, a0 = a1, b0 = a1;
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
        const c64 a = (lane != 0) ? a1 : a0;
        const c64 b = (lane != 0) ? b1 : b0;
        z = cmk(a.re + b.im, b.re - a.im);
      }
    }
    Z[r] = z;
  }
}

// From a natural-order forward transform F of z = x + i y, the half spectra
// X_k, Y_k at k = 32 q + lane (q < QK): X = (F_k + conj F_{N-k}) / 2,
// Y = (F_k - conj F_{N-k}) / (2 i).
template <int P, int QK>
__device__ __forceinline__ void unpack_pair(const c64 (&F)[P], int lane, c64 (&Xo)[QK],
                                            c64 (&Yo)[QK]) {
#pragma unroll
  for (int q = 0; q < QK; ++q) {
    const c64 m1 = shfl_c(F[(P - q - 1 + P) % P], (32 - lane) & 31);
    const c64 m0 = shfl_c(F[(P - q) % P], 0);
    const c64 Zm = (lane != 0) ? m1 : m0;
    const c64 Zk = F[q];
    Xo[q] = cmk(0.5 * (Zk.re + Zm.re), 0.5 * (Zk.im - Zm.im));
    Yo[q] = cmk(0.5 * (Zk.im + Zm.im), -0.5 * (Zk.re - Zm.re));
  }
}

// ---------------------------------------------------------------------------
// z_cross: one warp per pair of (x, y) rows, everything in registers.
// ---------------------------------------------------------------------------
template <int P, int QK>
__global__ void __launch_bounds__(256) z_cross_warp_kernel(DevOps o, Dims d,
                                                           const c64* __restrict__ tw,
                                                           const c64* __restrict__ Y,
                                                           c64* __restrict__ HZ) {
  const int lane = threadIdx.x & 31;
  const int pair = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int nrows = d.Nx * d.My;
  const int rowa = 2 * pair;
  if (rowa >= nrows) return;
  const bool hasb = rowa + 1 < nrows;
  WarpTw<P, double> w;
  load_warp_tw<P, double>(w, tw, lane);
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  double nrm[2][3][P];  // products n0, n1, n2 per row, scrambled layout
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int row = rowa + rb;
    const bool ok = rb == 0 || hasb;
    c64 ph[3][P];
#pragma unroll
    for (int pr = 0; pr < 3; ++pr) {
      c64 A[QK], B[QK];
#pragma unroll
      for (int q = 0; q < QK; ++q) {
        const int k = 32 * q + lane;
        const bool in = ok && k < d.Kz;
        A[q] = in ? Y[(size_t)(2 * pr) * plane + (size_t)row * d.Kz + k] : cmk(0.0, 0.0);
        B[q] = in ? Y[(size_t)(2 * pr + 1) * plane + (size_t)row * d.Kz + k] : cmk(0.0, 0.0);
      }
      build_packed<P, QK>(A, B, d.Kz, lane, ph[pr]);
      warp_fft_inverse<P, double>(ph[pr], w, lane);
    }
    const int j = (ok ? row : rowa) / d.My;
    const double ub = d.uwall * o.xphys[j];
#pragma unroll
    for (int r = 0; r < P; ++r) {
      const double u0 = ph[0][r].re, u1 = ph[0][r].im + ub, u2 = ph[1][r].re;
      const double w0 = ph[1][r].im, w1 = ph[2][r].re, w2 = ph[2][r].im + d.uwall;
      nrm[rb][0][r] = -(u1 * w2 - u2 * w1);
      nrm[rb][1][r] = -(u2 * w0 - u0 * w2);
      nrm[rb][2][r] = -(u0 * w1 - u1 * w0);
    }
  }
  c64 F0[P], F1[P], F2[P];
#pragma unroll
  for (int r = 0; r < P; ++r) {
    F0[r] = cmk(nrm[0][0][r], nrm[0][1][r]);
    F1[r] = cmk(nrm[1][0][r], nrm[1][1][r]);
    F2[r] = cmk(nrm[0][2][r], nrm[1][2][r]);
  }
  warp_fft_forward<P, double>(F0, w, lane);
  warp_fft_forward<P, double>(F1, w, lane);
  warp_fft_forward<P, double>(F2, w, lane);
  c64 xa0[QK], xa1[QK], xb0[QK], xb1[QK], x2a[QK], x2b[QK];
  unpack_pair<P, QK>(F0, lane, xa0, xa1);
  unpack_pair<P, QK>(F1, lane, xb0, xb1);
  unpack_pair<P, QK>(F2, lane, x2a, x2b);
  const double scale = 1.0 / (32 * P);
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
  unpack_pair<P, QK>(F0, lane, xa0, xa1);
  unpack_pair<P, QK>(F1, lane, xb0, xb1);
  unpack_pair<P, QK>(F2, lane, x2a, x2b);
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

}  // namespace jfb
