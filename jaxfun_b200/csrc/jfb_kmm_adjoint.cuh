// Discrete adjoint of the FP64 plane-Couette step (the reverse-mode
// derivative that jax.grad takes through KMM.solve in
// examples/pcf_minimal_seed_jax.py:111-150).
//
// Inner products: coefficient arrays pair as Re sum conj(a) b over the full
// (Hermitian) spectrum, physical samples as sum a b.  In the half-spectrum
// storage of the step (kz >= 0) the full-spectrum weights (1 at kz = 0, 2 at
// kz > 0) sit on both sides of every per-pencil operator, so a per-pencil
// adjoint is the conjugate transpose of the pencil's operator, and the adjoint
// of the padded periodic-axis chain y_b -> z_b -> product -> z_f -> y_f is the
// same chain with the product replaced by its transpose: the transposes of the
// unnormalised inverse transforms are the forward transforms times My (Mz),
// those of the 1/My (1/Mz) scaled forward transforms the inverse transforms
// over My (Mz), and the factors cancel.
//
// Kernels:
//   pencil_terms_kernel  dst[:, p] (+)= sum_t c_t(ky, kz) Op_t src_t[:, p],
//                        Op_t a real x-matrix, its transpose or the identity
//   band_solve_t_kernel  A^T x = b per wavenumber from the no-pivot LU band of
//                        A (the factors of the forward solves, kept); the
//                        production path is band_solve_t_warp_kernel (a warp
//                        per pencil)
//   z_adjoint_kernel     transposed rotational product: with w the adjoint of
//                        n = -(u_t x omega_t), adj u = w x omega_t and
//                        adj omega = u_t x w
#pragma once

#include "jfb_kmm_kernels.cuh"

namespace jfb {

// One term: coefficient (cre + i cim) ky^a kz^b (k^2)^c, c = -1 meaning 1/k^2
// (zero on the mean pencil).  mat == nullptr is the identity.
struct PTerm {
  const c64* src;
  const double* mat;  // row-major; forward operator of shape (dst_rows x src_rows),
                      // or (src_rows x dst_rows) when trans
  int src_rows;
  int trans;
  double cre, cim;
  int a, b, c;
  int sel;       // 0: every pencil, 1: all but the mean pencil, 2: the mean pencil only
  int realpart;  // keep the real part of the term
};

constexpr int kMaxTerms = 8;

struct PTermList {
  c64* dst;
  int dst_rows;
  int accumulate;
  int n;
  PTerm t[kMaxTerms];
};

// block: 32 pencils (lanes) x 8 warps, each thread kTermRows consecutive
// destination rows of one pencil (every source value it loads serves all of
// them); grid (ceil(P / 32), ceil(dst_rows / (8 kTermRows)))
constexpr int kTermRows = 8;
__global__ void __launch_bounds__(256) pencil_terms_kernel(Dims d, PTermList L) {
  const int p = blockIdx.x * 32 + (threadIdx.x & 31);
  const int r0 = (blockIdx.y * 8 + (threadIdx.x >> 5)) * kTermRows;
  if (p >= d.P || r0 >= L.dst_rows) return;
  const size_t P = (size_t)d.P;
  const int nr = min(kTermRows, L.dst_rows - r0);
  const int row = p / d.Kz, kzi = p % d.Kz;
  c64 acc[kTermRows];
#pragma unroll
  for (int q = 0; q < kTermRows; ++q) acc[q] = cmk(0.0, 0.0);
  if (row != d.Ny / 2) {  // the y Nyquist row stays zero
    const double ky = ((row < d.Ny / 2) ? row : row - d.Ny) * d.dfy;
    const double kz = kzi * d.dfz;
    const double k2 = ky * ky + kz * kz;
    const bool mean = (p == 0);
    for (int t = 0; t < L.n; ++t) {
      const PTerm& T = L.t[t];
      if ((T.sel == 1 && mean) || (T.sel == 2 && !mean)) continue;
      double s = 1.0;
      for (int e = 0; e < T.a; ++e) s *= ky;
      for (int e = 0; e < T.b; ++e) s *= kz;
      if (T.c < 0) {
        if (mean) continue;
        s /= k2;
      } else {
        for (int e = 0; e < T.c; ++e) s *= k2;
      }
      c64 v[kTermRows];
#pragma unroll
      for (int q = 0; q < kTermRows; ++q) v[q] = cmk(0.0, 0.0);
      if (!T.mat) {
#pragma unroll
        for (int q = 0; q < kTermRows; ++q)
          if (q < nr) v[q] = T.src[(size_t)(r0 + q) * P + p];
      } else if (T.trans) {
        for (int k = 0; k < T.src_rows; ++k) {
          const c64 x = T.src[(size_t)k * P + p];
          const double* m = T.mat + (size_t)k * L.dst_rows + r0;
#pragma unroll
          for (int q = 0; q < kTermRows; ++q)
            if (q < nr) v[q] = v[q] + __ldg(m + q) * x;
        }
      } else {
        for (int k = 0; k < T.src_rows; ++k) {
          const c64 x = T.src[(size_t)k * P + p];
#pragma unroll
          for (int q = 0; q < kTermRows; ++q)
            if (q < nr) v[q] = v[q] + __ldg(T.mat + (size_t)(r0 + q) * T.src_rows + k) * x;
        }
      }
      const c64 cf = cmk(T.cre * s, T.cim * s);
#pragma unroll
      for (int q = 0; q < kTermRows; ++q) {
        if (T.realpart) v[q].im = 0.0;
        acc[q] = acc[q] + cf * v[q];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kTermRows; ++q) {
    if (q >= nr) break;
    c64* out = L.dst + (size_t)(r0 + q) * P + p;
    *out = L.accumulate ? *out + acc[q] : acc[q];
  }
}

// A^T x = b for every pencil of the half spectrum, A the system of the
// pencil's wavenumber (mode kyi * Kz + kz, kyi = |ky| index), factored in
// place without pivoting: band[mode][(p + off) * n + j] holds the LU entry
// at (j - off, j) (unit L below the diagonal, U on and above).
// U^T y = b (forward substitution), then L^T x = y (backward), in the output
// array.  mean_only: solve the mean pencil (mode 0) alone.
__global__ void __launch_bounds__(128) band_solve_t_kernel(Dims d, const double* __restrict__ band,
                                                           int p, int q, int n, int mean_only,
                                                           const c64* __restrict__ rhs,
                                                           c64* __restrict__ out) {
  const int pen = blockIdx.x * blockDim.x + threadIdx.x;
  if (pen >= (mean_only ? 1 : d.P)) return;
  const size_t P = (size_t)d.P;
  const int row = pen / d.Kz, kz = pen % d.Kz;
  if (row == d.Ny / 2) {
    for (int i = 0; i < n; ++i) out[(size_t)i * P + pen] = cmk(0.0, 0.0);
    return;
  }
  const int kyi = (row < d.Ny / 2) ? row : d.Ny - row;
  const size_t mode = mean_only ? 0 : (size_t)kyi * d.Kz + kz;
  const double* B = band + mode * (size_t)(p + q + 1) * n;
  auto at = [&](int off, int j) { return B[(size_t)(p + off) * n + j]; };
  for (int i = 0; i < n; ++i) {
    c64 s = rhs[(size_t)i * P + pen];
    const int k0 = max(0, i - q);
    for (int k = k0; k < i; ++k) s = s - at(i - k, i) * out[(size_t)k * P + pen];
    out[(size_t)i * P + pen] = (1.0 / at(0, i)) * s;
  }
  for (int i = n - 1; i >= 0; --i) {
    c64 s = out[(size_t)i * P + pen];
    const int k1 = min(n - 1, i + p);
    for (int k = i + 1; k <= k1; ++k) s = s - at(i - k, i) * out[(size_t)k * P + pen];
    out[(size_t)i * P + pen] = s;
  }
}

// The same solve with a warp per pencil: the vector in shared memory,
// column-oriented substitution (once an unknown is final, lane j applies the
// j-th band entry of its column / row to the unknown j places away; distinct
// targets per lane), the band entries of kBandChunk steps loaded one chunk
// ahead.  U^T y = b: y_k = b_k / U[k][k], then b_{k+j} -= U[k][k+j] y_k
// (j = 1..q); L^T x = y from the bottom: x_{k-j} -= L[k][k-j] x_k (j = 1..p).
constexpr int kBandChunk = 8;
constexpr int kBandWarps = 4;  // pencils per block
__global__ void __launch_bounds__(32 * kBandWarps) band_solve_t_warp_kernel(
    Dims d, const double* __restrict__ band, int p, int q, int n, int mean_only,
    const c64* __restrict__ rhs, c64* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int pen = blockIdx.x * kBandWarps + wib;
  if (pen >= (mean_only ? 1 : d.P)) return;  // whole warps
  c64* x = reinterpret_cast<c64*>(smem_raw) + (size_t)wib * n;
  const size_t P = (size_t)d.P;
  const int row = pen / d.Kz, kz = pen % d.Kz;
  if (row == d.Ny / 2) {
    for (int i = lane; i < n; i += 32) out[(size_t)i * P + pen] = cmk(0.0, 0.0);
    return;
  }
  const int kyi = (row < d.Ny / 2) ? row : d.Ny - row;
  const size_t mode = mean_only ? 0 : (size_t)kyi * d.Kz + kz;
  const double* B = band + mode * (size_t)(p + q + 1) * n;
  auto at = [&](int off, int col) { return __ldg(B + (size_t)(p + off) * n + col); };
  for (int i = lane; i < n; i += 32) x[i] = rhs[(size_t)i * P + pen];
  __syncwarp();
  // U^T y = b.  Lane owns band offsets j0 = lane + 1 and j1 = lane + 33.
  const int j0 = lane + 1, j1 = lane + 33;
  double u0[kBandChunk], u1[kBandChunk], rd[kBandChunk];
  double v0[kBandChunk], v1[kBandChunk], sd[kBandChunk];
  auto uload = [&](int k, double& a, double& b, double& r) {
    a = (k < n && j0 <= q && k + j0 < n) ? at(j0, k + j0) : 0.0;
    b = (k < n && j1 <= q && k + j1 < n) ? at(j1, k + j1) : 0.0;
    r = (k < n) ? 1.0 / at(0, k) : 0.0;
  };
#pragma unroll
  for (int t = 0; t < kBandChunk; ++t) uload(t, u0[t], u1[t], rd[t]);
  for (int k0 = 0; k0 < n; k0 += kBandChunk) {
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) uload(k0 + kBandChunk + t, v0[t], v1[t], sd[t]);
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) {
      const int k = k0 + t;
      if (k >= n) break;
      const c64 b = x[k];
      __syncwarp();
      const c64 y = rd[t] * b;
      if (lane == 0) x[k] = y;
      if (j0 <= q && k + j0 < n) x[k + j0] = x[k + j0] - u0[t] * y;
      if (j1 <= q && k + j1 < n) x[k + j1] = x[k + j1] - u1[t] * y;
      for (int j = lane + 65; j <= q && k + j < n; j += 32) x[k + j] = x[k + j] - at(j, k + j) * y;
      __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) {
      u0[t] = v0[t];
      u1[t] = v1[t];
      rd[t] = sd[t];
    }
  }
  // L^T x = y, k from n - 1 down
  auto lload = [&](int k, double& a, double& b) {
    a = (k >= 0 && j0 <= p && k - j0 >= 0) ? at(-j0, k - j0) : 0.0;
    b = (k >= 0 && j1 <= p && k - j1 >= 0) ? at(-j1, k - j1) : 0.0;
  };
#pragma unroll
  for (int t = 0; t < kBandChunk; ++t) lload(n - 1 - t, u0[t], u1[t]);
  for (int k0 = n - 1; k0 >= 0; k0 -= kBandChunk) {
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) lload(k0 - kBandChunk - t, v0[t], v1[t]);
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) {
      const int k = k0 - t;
      if (k < 0) break;
      const c64 xk = x[k];
      if (j0 <= p && k - j0 >= 0) x[k - j0] = x[k - j0] - u0[t] * xk;
      if (j1 <= p && k - j1 >= 0) x[k - j1] = x[k - j1] - u1[t] * xk;
      for (int j = lane + 65; j <= p && k - j >= 0; j += 32) x[k - j] = x[k - j] - at(-j, k - j) * xk;
      __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < kBandChunk; ++t) {
      u0[t] = v0[t];
      u1[t] = v1[t];
    }
  }
  for (int i = lane; i < n; i += 32) out[(size_t)i * P + pen] = x[i];
}

// Transposed z stage, per group of kZRows (x, y) rows: the forward u, omega
// (six half spectra, padded in y) and the adjoint w of the product (three)
// -> five packed complex inverse FFTs, adj u = w x omega_t, adj omega =
// u_t x w with u_t = u + U_b e_y, omega_t = omega + U_wall e_z, then three
// packed forward transforms into six half spectra (adj u, adj omega).
__global__ void __launch_bounds__(256) z_adjoint_kernel(DevOps o, Dims d, FFTPlan plan,
                                                        const c64* __restrict__ tw,
                                                        const c64* __restrict__ Y,
                                                        const c64* __restrict__ Wa,
                                                        c64* __restrict__ HZ) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NP = 5;              // packed input pairs per row
  constexpr int NC = kZRows * NP;    // packed input columns
  constexpr int NCf = kZRows * 3;    // packed output columns
  c64* A = reinterpret_cast<c64*>(smem_raw);
  c64* B = A + d.Mz * NC;
  const int row0 = blockIdx.x * kZRows;
  const int nrows = d.Nx * d.My;
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  auto field = [&](int f) -> const c64* {  // 0..5 forward u, omega; 6..8 adjoint w; 9 none
    return (f < 6) ? Y + (size_t)f * plane : (f < 9) ? Wa + (size_t)(f - 6) * plane : nullptr;
  };
  // k fastest: a warp reads consecutive spectral values of one row and field
  for (int idx = threadIdx.x; idx < d.Mz * NC; idx += blockDim.x) {
    const int k = idx % d.Mz, c = idx / d.Mz;
    const int rl = c / NP, pr = c % NP;
    const int row = row0 + rl;
    c64 z = cmk(0.0, 0.0);
    if (row < nrows) {
      const c64* fa = field(2 * pr);
      const c64* fb = field(2 * pr + 1);
      auto get = [&](const c64* f, int kk) {
        return f ? f[(size_t)row * d.Kz + kk] : cmk(0.0, 0.0);
      };
      if (k == 0) {
        z = cmk(get(fa, 0).re, get(fb, 0).re);
      } else if (k < d.Kz) {
        const c64 xa = get(fa, k), xb = get(fb, k);
        z = cmk(xa.re - xb.im, xa.im + xb.re);
      } else if (k > d.Mz - d.Kz) {
        const int kk = d.Mz - k;
        const c64 xa = get(fa, kk), xb = get(fb, kk);
        z = cmk(xa.re + xb.im, -xa.im + xb.re);
      }
    }
    A[k * NC + c] = z;
  }
  __syncthreads();
  c64* phys = fft_columns<double>(A, B, plan, NC, NC, tw, +1);
  c64* other = (phys == A) ? B : A;
  for (int idx = threadIdx.x; idx < d.Mz * kZRows; idx += blockDim.x) {
    const int rl = idx % kZRows, n = idx / kZRows;
    const int row = row0 + rl;
    const int j = (row < nrows) ? row / d.My : 0;
    const c64* z = phys + n * NC + rl * NP;
    const double ub = d.uwall * o.xphys[j];
    const double u0 = z[0].re, u1 = z[0].im + ub, u2 = z[1].re;
    const double w0 = z[1].im, w1 = z[2].re, w2 = z[2].im + d.uwall;
    const double a0 = z[3].re, a1 = z[3].im, a2 = z[4].re;
    c64* out = other + n * NCf + rl * 3;
    out[0] = cmk(a1 * w2 - a2 * w1, a2 * w0 - a0 * w2);
    out[1] = cmk(a0 * w1 - a1 * w0, u1 * a2 - u2 * a1);
    out[2] = cmk(u2 * a0 - u0 * a2, u0 * a1 - u1 * a0);
  }
  __syncthreads();
  c64* spec = fft_columns<double>(other, phys, plan, NCf, NCf, tw, -1);
  const double scale = 1.0 / d.Mz;
  for (int idx = threadIdx.x; idx < d.Kz * kZRows * 6; idx += blockDim.x) {
    const int k = idx % d.Kz;
    const int rf = idx / d.Kz;
    const int f = rf % 6, rl = rf / 6;
    const int row = row0 + rl;
    if (row >= nrows) continue;
    const int col = rl * 3 + f / 2;
    const c64 Zk = spec[k * NCf + col];
    const c64 Zm = spec[((d.Mz - k) % d.Mz) * NCf + col];
    c64 v;
    if ((f & 1) == 0) v = cmk(0.5 * (Zk.re + Zm.re), 0.5 * (Zk.im - Zm.im));
    else v = cmk(0.5 * (Zk.im + Zm.im), -0.5 * (Zk.re - Zm.re));
    HZ[(size_t)f * plane + (size_t)row * d.Kz + k] = scale * v;
  }
}

// Elementwise helpers on half-spectrum arrays.
__global__ void axpy_kernel(c64* __restrict__ y, const c64* __restrict__ x, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = y[i] + a * x[i];
}

__global__ void conj_kernel(c64* __restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i].im = -y[i].im;
}

}  // namespace jfb
