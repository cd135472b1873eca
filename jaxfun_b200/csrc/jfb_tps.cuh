// Standalone tensor-product transforms: TensorProductSpace.backward / forward /
// scalar_product (src/jaxfun/galerkin/tensorproductspace.py:253-551) for a
// Chebyshev axis (orthogonal, Dirichlet or biharmonic basis) times one or two
// Fourier axes, on full complex spectra in the reference layout, with the 3/2
// padding of the Fourier axes (Fourier.py:128-184: zero padding in the middle,
// unnormalised inverse, forward scaled 1/M and truncated to the modes
// wavenumbers() keeps, Nyquist included).
//
//   x axis:       dense real operator per axis-0 line (x_apply_kernel)
//   middle axis:  y_backward_kernel / y_forward_kernel (shared with the step)
//   last axis:    fft_rows_kernel (contiguous lines, shared-memory Stockham)
//
// Included at the end of jfb_kmm.cu (one translation unit with the step).
#pragma once

#include "jfb_kmm_kernels.cuh"

namespace jfb {

// out[i][m] = sum_k A[i][k] in[k][m], A real (rows x cols), m < M contiguous.
__global__ void __launch_bounds__(256) x_apply_kernel(const double* __restrict__ A, int rows,
                                                      int cols, const c64* __restrict__ in,
                                                      c64* __restrict__ out, int64_t M) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (m >= M || i >= rows) return;
  const double* a = A + (size_t)i * cols;
  c64 s0 = cmk(0.0, 0.0), s1 = s0;
  int k = 0;
  for (; k + 1 < cols; k += 2) {
    s0 = s0 + __ldg(a + k) * in[(size_t)k * M + m];
    s1 = s1 + __ldg(a + k + 1) * in[(size_t)(k + 1) * M + m];
  }
  if (k < cols) s0 = s0 + __ldg(a + k) * in[(size_t)k * M + m];
  out[(size_t)i * M + m] = s0 + s1;
}

// Per-mode Fourier weight of the separable maps: scale * prod over the
// periodic axes of (i m df)^k, m the FFT-ordered wavenumber, with the Nyquist
// mode zeroed for odd k (Fourier.py:210-223).
struct FourierWeight {
  int n1, n2, k1, k2;
  double df1, df2, scale;
};

__device__ __forceinline__ c64 ipow_times(c64 w, int idx, int n, int k, double df) {
  if (k == 0) return w;
  if ((k & 1) && 2 * idx == n) return cmk(0.0, 0.0);
  const int m = (idx < (n + 1) / 2) ? idx : idx - n;
  double a = 1.0;
  for (int t = 0; t < k; ++t) a *= (double)m * df;
  w = a * w;
  for (int t = 0; t < (k & 3); ++t) w = mul_i(w);  // i^k
  return w;
}

// out[i][m] = w(m) sum_k A[i][k] in[k][m]: an x-axis matrix with per-mode
// Fourier weights (m = i1 n2 + i2 over the periodic axes).
__global__ void __launch_bounds__(256) x_apply_w_kernel(const double* __restrict__ A, int rows,
                                                        int cols, const c64* __restrict__ in,
                                                        c64* __restrict__ out, FourierWeight fw) {
  const int64_t M = (int64_t)fw.n1 * fw.n2;
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (m >= M || i >= rows) return;
  const double* a = A + (size_t)i * cols;
  c64 s0 = cmk(0.0, 0.0), s1 = s0;
  int k = 0;
  for (; k + 1 < cols; k += 2) {
    s0 = s0 + __ldg(a + k) * in[(size_t)k * M + m];
    s1 = s1 + __ldg(a + k + 1) * in[(size_t)(k + 1) * M + m];
  }
  if (k < cols) s0 = s0 + __ldg(a + k) * in[(size_t)k * M + m];
  c64 w = cmk(fw.scale, 0.0);
  w = ipow_times(w, (int)(m / fw.n2), fw.n1, fw.k1, fw.df1);
  w = ipow_times(w, (int)(m % fw.n2), fw.n2, fw.k2, fw.df2);
  out[(size_t)i * M + m] = w * (s0 + s1);
}

// Complex FFT along contiguous lines: `lines` rows of length nin -> nout.
// Inverse (sign +1, transform length nout): pad nin -> nout in the middle,
// unnormalised.  Forward (sign -1, transform length nin): scaled 1/nin,
// truncated to nout modes in FFT order (k < nout/2 and the last nout/2 of
// the spectrum, the -nout/2 mode included).  kTpsRows lines per block.
constexpr int kTpsRows = 8;
__global__ void __launch_bounds__(256) fft_rows_kernel(FFTPlan plan, const c64* __restrict__ tw,
                                                       int sign, const c64* __restrict__ in,
                                                       c64* __restrict__ out, int64_t lines,
                                                       int nin, int nout) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = plan.n;
  c64* A = reinterpret_cast<c64*>(smem_raw);
  c64* B = A + (size_t)n * kTpsRows;
  const int64_t l0 = blockIdx.x * (int64_t)kTpsRows;
  for (int idx = threadIdx.x; idx < n * kTpsRows; idx += blockDim.x) {
    const int c = idx % kTpsRows, k = idx / kTpsRows;
    const int64_t line = l0 + c;
    c64 v = cmk(0.0, 0.0);
    if (line < lines) {
      if (sign > 0) {
        const int h = nin / 2;
        if (k < h) v = in[line * nin + k];
        else if (k >= n - (nin - h)) v = in[line * nin + (k - n + nin)];
      } else {
        v = in[line * nin + k];
      }
    }
    A[k * kTpsRows + c] = v;
  }
  __syncthreads();
  c64* res = fft_columns<double>(A, B, plan, kTpsRows, kTpsRows, tw, sign);
  const double scale = sign > 0 ? 1.0 : 1.0 / n;
  const int h = nout / 2;
  for (int idx = threadIdx.x; idx < nout * kTpsRows; idx += blockDim.x) {
    const int c = idx % kTpsRows, k = idx / kTpsRows;
    const int64_t line = l0 + c;
    if (line >= lines) continue;
    int src = k;
    if (sign < 0 && k >= h) src = k - nout + n;
    out[line * nout + k] = scale * res[src * kTpsRows + c];
  }
}

__global__ void tps_scale_kernel(c64* __restrict__ y, double a, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = a * y[i];
}


// ---------------------------------------------------------------------------
// 2-D Helmholtz solve in one launch (la/solvers.py:22-61 with the per-
// wavenumber solve of tpmatrix.py:1550-1677) on one cluster of kHelmCTAs
// CTAs that keeps the whole (N x n1) problem in distributed shared memory:
// CTA c owns the Fourier columns [c KC, (c+1) KC) for the x-direction work
// (products against the x operators, the per-mode solves) and the x rows
// [c JR, (c+1) JR) for the y transforms; the stages exchange their slices
// through DSMEM reads between cluster barriers, instead of about ten
// launches through global memory.
// ---------------------------------------------------------------------------
constexpr int kHelmMaxDiag = 256;
constexpr int kHelmCTAs = 8;
constexpr int kHelmThreads = 256;
constexpr int kHelmChunk = 8;  // solve columns whose factor entries are loaded together
struct Helm2DArgs {
  const double* BC;  // orthogonal backward, N x N (row j: T_n(x_j))
  const double* SD;  // Dirichlet scalar products, nb x N
  const double* BD;  // Dirichlet backward, N x nb
  const c64* tw;     // n1-point twiddles
  FFTPlan plan;
  const double *L, *U;  // (n1, nL, nb), (n1, nU, nb)
  const double* Uinv;   // optional (n1, nb, nb): U^-1 per mode, entry (r, c) at c nb + r
  int nL, nU, umain;
  int l2, l4;  // indices of the L offsets -2 / -4 (-1: absent) when those are all of L
  int loff[kHelmMaxDiag], uoff[kHelmMaxDiag];
  int N, nb, M, KC, JR, QS;
  double scale;  // Fourier scalar-product weight / fourier_mass / n1
  const c64* f;
  c64* u;
};

__global__ void __cluster_dims__(kHelmCTAs, 1, 1) __launch_bounds__(kHelmThreads, 1)
    helmholtz2d_kernel(const __grid_constant__ Helm2DArgs h) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int N = h.N, M = h.M, nb = h.nb, KC = h.KC, JR = h.JR, QS = h.QS;
  const int k0 = rank * KC, kn = min(KC, M - k0);  // owned Fourier columns
  const int j0 = rank * JR, jn = min(JR, N - j0);  // owned x rows
  c64* A = reinterpret_cast<c64*>(smem_raw);  // [n][kk]: f slice, then gathered columns
  c64* B = A + (size_t)N * KC;                // [j][kk]: x-backward slices
  c64* Q = B + (size_t)N * KC;                // [r][kk] (row stride QS): scalar products -> solutions
  c64* F0 = Q + (size_t)N * h.QS;             // [k][jj]: y-transform lines
  c64* F1 = F0 + (size_t)M * JR;
  double* SdT = reinterpret_cast<double*>(F1 + (size_t)M * JR);  // [j][r]
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < N * KC; i += nt) {
    const int kk = i % KC, n = i / KC;
    A[i] = (kk < kn) ? h.f[(size_t)n * M + k0 + kk] : cmk(0.0, 0.0);
  }
  for (int i = tid; i < nb * N; i += nt) {
    const int j = i % N, r = i / N;
    SdT[j * nb + r] = h.SD[i];
  }
  __syncthreads();
  // x backward (orthogonal) of the owned columns: B[j][kk] = sum_n BC[j][n] f[n][kk]
  for (int i = tid; i < N * KC; i += nt) {
    const int kk = i % KC, j = i / KC;
    const double* a = h.BC + (size_t)j * N;
    c64 s = cmk(0.0, 0.0);
    for (int n = 0; n < N; ++n) s = s + __ldg(a + n) * A[n * KC + kk];
    B[i] = s;
  }
  cluster.sync();
  // y: gather the owned rows across all columns, inverse (unnormalised) then
  // forward transform
  for (int i = tid; i < M * JR; i += nt) {
    const int jj = i % JR, k = i / JR;
    c64 v = cmk(0.0, 0.0);
    if (jj < jn) {
      const c64* src = cluster.map_shared_rank(B, (unsigned)(k / KC));
      v = src[(j0 + jj) * KC + k % KC];
    }
    F0[i] = v;
  }
  __syncthreads();
  c64* P = fft_columns<double>(F0, F1, h.plan, JR, JR, h.tw, +1);
  P = fft_columns<double>(P, (P == F0) ? F1 : F0, h.plan, JR, JR, h.tw, -1);
  cluster.sync();
  // gather the owned columns across all rows (P sits at the same offset in
  // every CTA), then the Dirichlet scalar products Q[r][kk]
  for (int i = tid; i < N * KC; i += nt) {
    const int kk = i % KC, j = i / KC;
    c64 v = cmk(0.0, 0.0);
    if (kk < kn) {
      const c64* src = cluster.map_shared_rank(P, (unsigned)(j / JR));
      v = src[(k0 + kk) * JR + j % JR];
    }
    A[i] = v;
  }
  __syncthreads();
  for (int i = tid; i < nb * KC; i += nt) {
    const int r = i % nb, kk = i / nb;
    c64 s = cmk(0.0, 0.0);
    for (int j = 0; j < N; ++j) s = s + SdT[j * nb + r] * A[j * KC + kk];
    Q[r * QS + kk] = h.scale * s;
  }
  __syncthreads();
  // per-wavenumber solves, a warp per owned mode, column-oriented
  // substitution: once x_c is final each lane applies its diagonals' entries
  // of column c to their rows (distinct rows per diagonal); the entries of
  // diagonals lane and lane + 32 are loaded one column ahead
  if (h.Uinv && h.l2 + h.l4 > -2) {
    // fast form: L with offsets -2 / -4 only is two independent recurrences
    // (one per parity class, lanes 0 and 1, in registers); then x = U^-1 y
    // as a product with the mode's explicit inverse (lanes = rows)
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    for (int kk = warp; kk < kn; kk += nwarps) {
      const int k = k0 + kk;
      const double* Lk = h.L + (size_t)k * h.nL * nb;
      c64* x = Q + kk;  // element c at x[c * QS]
      if (lane < 2) {
        // the right-hand side and the multipliers of the next row are loaded
        // before the current row's update (off the dependent chain)
        auto l2v = [&](int r) { return (h.l2 >= 0 && r >= 2 && r < nb) ? __ldg(Lk + (size_t)h.l2 * nb + r - 2) : 0.0; };
        auto l4v = [&](int r) { return (h.l4 >= 0 && r >= 4 && r < nb) ? __ldg(Lk + (size_t)h.l4 * nb + r - 4) : 0.0; };
        c64 ym2 = cmk(0.0, 0.0), ym4 = cmk(0.0, 0.0);  // y_{r-2}, y_{r-4}
        c64 vn = (lane < nb) ? x[lane * QS] : cmk(0.0, 0.0);
        double an = l2v(lane), bn = l4v(lane);
        for (int r = lane; r < nb; r += 2) {
          const c64 v0 = vn;
          const double a2 = an, a4 = bn;
          if (r + 2 < nb) {
            vn = x[(r + 2) * QS];
            an = l2v(r + 2);
            bn = l4v(r + 2);
          }
          const c64 v = v0 - a2 * ym2 - a4 * ym4;
          x[r * QS] = v;
          ym4 = ym2;
          ym2 = v;
        }
      }
      __syncwarp();
      const double* Ui = h.Uinv + (size_t)k * nb * nb;
      c64 acc0 = cmk(0.0, 0.0), acc1 = cmk(0.0, 0.0);  // rows lane, lane + 32, ...
      c64 acc2 = cmk(0.0, 0.0), acc3 = cmk(0.0, 0.0);
#pragma unroll 8
      for (int c = 0; c < nb; ++c) {
        const c64 y = x[c * QS];
        const double* col = Ui + (size_t)c * nb;
        if (lane <= c) acc0 = acc0 + __ldg(col + lane) * y;
        if (lane + 32 <= c) acc1 = acc1 + __ldg(col + lane + 32) * y;
        if (lane + 64 <= c) acc2 = acc2 + __ldg(col + lane + 64) * y;
        if (lane + 96 <= c) acc3 = acc3 + __ldg(col + lane + 96) * y;
      }
      c64* O = A + kk;
      if (lane < nb) O[lane * KC] = acc0;
      if (lane + 32 < nb) O[(lane + 32) * KC] = acc1;
      if (lane + 64 < nb) O[(lane + 64) * KC] = acc2;
      if (lane + 96 < nb) O[(lane + 96) * KC] = acc3;
    }
  } else {
    const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
    for (int kk = warp; kk < kn; kk += nwarps) {
      const int k = k0 + kk;
      const double* Lk = h.L + (size_t)k * h.nL * nb;
      const double* Uk = h.U + (size_t)k * h.nU * nb;
      c64* x = Q + kk;  // element c at x[c * QS]
      c64* O = A + kk;  // solution, element c at O[c * KC] (A is free after the scalar products)
      auto lld = [&](int d, int c) {
        return (d < h.nL && c < nb) ? __ldg(Lk + (size_t)d * nb + c) : 0.0;
      };
      auto uld = [&](int d, int c) {
        return (d < h.nU && c >= 0) ? __ldg(Uk + (size_t)d * nb + c) : 0.0;
      };
      // row shifts of this lane's diagonals (lane, lane + 32), held in
      // registers: s > 0 below / above the diagonal, 0 when the lane has none
      const int ls0 = lane < h.nL ? -h.loff[lane] : 0;
      const int ls1 = lane + 32 < h.nL ? -h.loff[lane + 32] : 0;
      const int us0 = lane < h.nU ? h.uoff[lane] : 0;
      const int us1 = lane + 32 < h.nU ? h.uoff[lane + 32] : 0;
      // factor entries of diagonals lane and lane + 32, kHelmChunk columns at
      // a time, loaded one chunk ahead (the chunk's work covers the latency)
      double a0[kHelmChunk], a1[kHelmChunk], b0[kHelmChunk], b1[kHelmChunk];
#pragma unroll
      for (int q = 0; q < kHelmChunk; ++q) {
        a0[q] = lld(lane, q);
        a1[q] = lld(lane + 32, q);
      }
      for (int c0 = 0; c0 < nb; c0 += kHelmChunk) {  // unit lower: L[c - s][c] at Lk[d][c], s < 0
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          b0[q] = lld(lane, c0 + kHelmChunk + q);
          b1[q] = lld(lane + 32, c0 + kHelmChunk + q);
        }
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          const int c = c0 + q;
          if (c >= nb) break;
          const c64 y = x[c * QS];
          if (ls0 > 0 && c + ls0 < nb) x[(c + ls0) * QS] = x[(c + ls0) * QS] - a0[q] * y;
          if (ls1 > 0 && c + ls1 < nb) x[(c + ls1) * QS] = x[(c + ls1) * QS] - a1[q] * y;
          for (int d = lane + 64; d < h.nL; d += 32) {
            const int r = c - h.loff[d];
            if (r < nb) x[r * QS] = x[r * QS] - __ldg(Lk + (size_t)d * nb + c) * y;
          }
          __syncwarp();
        }
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          a0[q] = b0[q];
          a1[q] = b1[q];
        }
      }
      // reciprocal main-diagonal entries of the current / next chunk (formed
      // off the dependent chain)
      double g0[kHelmChunk], g1[kHelmChunk];
#pragma unroll
      for (int q = 0; q < kHelmChunk; ++q) {
        a0[q] = uld(lane, nb - 1 - q);
        a1[q] = uld(lane + 32, nb - 1 - q);
        g0[q] = 1.0 / uld(h.umain, nb - 1 - q);
      }
      for (int t0 = 0; t0 < nb; t0 += kHelmChunk) {  // upper: U[c - s][c] at Uk[d][c], s > 0
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          const int c = nb - 1 - (t0 + kHelmChunk + q);
          b0[q] = uld(lane, c);
          b1[q] = uld(lane + 32, c);
          g1[q] = (c >= 0) ? 1.0 / uld(h.umain, c) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          const int c = nb - 1 - (t0 + q);
          if (c < 0) break;
          const c64 v = x[c * QS];
          const c64 xc = cmk(v.re * g0[q], v.im * g0[q]);
          if (lane == 0) O[c * KC] = xc;  // the solution goes to O: x[c] is not written
          if (us0 > 0 && c - us0 >= 0) x[(c - us0) * QS] = x[(c - us0) * QS] - a0[q] * xc;
          if (us1 > 0 && c - us1 >= 0) x[(c - us1) * QS] = x[(c - us1) * QS] - a1[q] * xc;
          for (int d = lane + 64; d < h.nU; d += 32) {
            const int sft = h.uoff[d], r = c - sft;
            if (sft > 0 && r >= 0) x[r * QS] = x[r * QS] - __ldg(Uk + (size_t)d * nb + c) * xc;
          }
          __syncwarp();
        }
#pragma unroll
        for (int q = 0; q < kHelmChunk; ++q) {
          a0[q] = b0[q];
          a1[q] = b1[q];
          g0[q] = g1[q];
        }
      }
    }
  }
  __syncthreads();
  // x backward (Dirichlet) of the owned solutions (in A) into B (its earlier
  // contents were read by the other CTAs before the last cluster barrier)
  for (int i = tid; i < N * KC; i += nt) {
    const int kk = i % KC, j = i / KC;
    const double* a = h.BD + (size_t)j * nb;
    c64 s = cmk(0.0, 0.0);
    for (int r = 0; r < nb; ++r) s = s + __ldg(a + r) * A[r * KC + kk];
    B[i] = s;
  }
  cluster.sync();
  // y: gather the owned rows, inverse transform, store u[j][l]
  for (int i = tid; i < M * JR; i += nt) {
    const int jj = i % JR, k = i / JR;
    c64 v = cmk(0.0, 0.0);
    if (jj < jn) {
      const c64* src = cluster.map_shared_rank(B, (unsigned)(k / KC));
      v = src[(j0 + jj) * KC + k % KC];
    }
    F0[i] = v;
  }
  __syncthreads();
  const c64* R = fft_columns<double>(F0, F1, h.plan, JR, JR, h.tw, +1);
  for (int i = tid; i < jn * M; i += nt) {
    const int l = i % M, jj = i / M;
    h.u[(size_t)(j0 + jj) * M + l] = R[l * JR + jj];
  }
  cluster.sync();  // no CTA leaves while another still reads its slices
}

}  // namespace jfb

struct jfb_tps {
  jfb_tps_config cfg;
  jfb::XBasis xb;  // 1-D wall-normal basis data (long double)
  std::map<int64_t, std::pair<double*, std::pair<int, int>>> xmaps;  // (map, k) -> device matrix
  int nb = 0, N = 0;
  int n1 = 1, n2 = 1, m1 = 1, m2 = 1;  // Fourier modes and padded counts
  double *B = nullptr, *F = nullptr, *Sq = nullptr;
  std::vector<double> G0, G2;
  c64 *tw1n = nullptr, *tw1m = nullptr, *tw2n = nullptr, *tw2m = nullptr;
  FFTPlan f1n, f1m, f2n, f2m;
  c64 *w0 = nullptr, *w1 = nullptr;  // work buffers
  std::vector<void*> allocs;
};

extern "C" int jfb_tps_destroy(jfb_tps* t) {
  if (!t) return JFB_OK;
  for (auto& kv : t->xmaps) cudaFree(kv.second.first);
  for (void* p : t->allocs) cudaFree(p);
  delete t;
  return JFB_OK;
}

extern "C" int jfb_tps_create(const jfb_tps_config* cfg, jfb_tps** out) {
  JFB_REQUIRE(cfg && out, "null pointer");
  *out = nullptr;
  JFB_REQUIRE(cfg->ndim == 2 || cfg->ndim == 3, "ndim must be 2 or 3");
  JFB_REQUIRE(cfg->basis >= 0 && cfg->basis <= 2, "unknown basis");
  JFB_REQUIRE(cfg->family == JFB_FAMILY_CHEBYSHEV || cfg->family == JFB_FAMILY_LEGENDRE,
              "family must be JFB_FAMILY_CHEBYSHEV or JFB_FAMILY_LEGENDRE");
  JFB_REQUIRE(cfg->n[0] >= 8 && cfg->n[0] <= 513, "n[0] out of range [8, 513]");
  for (int a = 1; a < cfg->ndim; ++a)
    JFB_REQUIRE(cfg->n[a] >= 2 && cfg->n[a] % 2 == 0, "Fourier sizes must be even");
  JFB_REQUIRE(cfg->x_hi > cfg->x_lo, "bad domain");
  jfb_tps* t = new jfb_tps();
  t->cfg = *cfg;
  auto fail = [&](int code) {
    jfb_tps_destroy(t);
    return code;
  };
  jfb_kmm_config kc;
  std::memset(&kc, 0, sizeof(kc));
  kc.nx = cfg->n[0];
  kc.ny = 4;
  kc.nz = 4;
  kc.x_lo = cfg->x_lo;
  kc.x_hi = cfg->x_hi;
  kc.ly = kc.lz = 2.0 * M_PI;
  build_x_basis(cfg->family, cfg->basis, cfg->n[0], cfg->x_lo, cfg->x_hi, t->xb);
  TpsX x;
  if (cfg->family == JFB_FAMILY_CHEBYSHEV) {
    HostOperators op;
    build_host_operators(kc, op);
    build_tps_x_operators(op, cfg->basis, x);
  } else {
    // Legendre: backward V S^T, forward M^-1 S Q, scalar product S Q and the
    // Galerkin matrices, all from the Gauss-Legendre Vandermonde matrix
    int r, c;
    x.N = t->xb.N;
    x.nb = t->xb.nb;
    x.B = x_map_matrix(t->xb, kXBackward, 0, &r, &c);
    x.F = x_map_matrix(t->xb, kXForward, 0, &r, &c);
    x.Sq = x_map_matrix(t->xb, kXScalarProd, 0, &r, &c);
    x.G0 = x_map_matrix(t->xb, kXGalerkin, 0, &r, &c);
    x.G2 = x_map_matrix(t->xb, kXGalerkin, 2, &r, &c);
  }
  t->N = x.N;
  t->nb = x.nb;
  t->G0 = x.G0;
  t->G2 = x.G2;
  t->n1 = cfg->n[1];
  t->n2 = cfg->ndim == 3 ? cfg->n[2] : 1;
  t->m1 = std::max(t->n1, (int)(cfg->pad[0] * t->n1));
  t->m2 = cfg->ndim == 3 ? std::max(t->n2, (int)(cfg->pad[1] * t->n2)) : 1;
  if (!make_fft_plan(t->n1, t->f1n) || !make_fft_plan(t->m1, t->f1m) ||
      (cfg->ndim == 3 && (!make_fft_plan(t->n2, t->f2n) || !make_fft_plan(t->m2, t->f2m)))) {
    set_error("Fourier sizes (and padded sizes) must be of the form 2^a 3^b");
    return fail(JFB_ERR_ARG);
  }
  auto up = [&](auto** dst, const auto& v) -> int {
    using E = typename std::decay_t<decltype(v)>::value_type;
    cudaError_t e = cudaMalloc((void**)dst, std::max<size_t>(1, v.size()) * sizeof(E));
    if (e != cudaSuccess) {
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return JFB_ERR_CUDA;
    }
    t->allocs.push_back(*dst);
    e = cudaMemcpy(*dst, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      set_error(std::string("cudaMemcpy: ") + cudaGetErrorString(e));
      return JFB_ERR_CUDA;
    }
    return JFB_OK;
  };
  int st;
  if ((st = up(&t->B, x.B)) || (st = up(&t->F, x.F)) || (st = up(&t->Sq, x.Sq))) return fail(st);
  if ((st = up(&t->tw1n, twiddles(t->n1))) || (st = up(&t->tw1m, twiddles(t->m1))))
    return fail(st);
  if (cfg->ndim == 3 &&
      ((st = up(&t->tw2n, twiddles(t->n2))) || (st = up(&t->tw2m, twiddles(t->m2)))))
    return fail(st);
  const size_t big = (size_t)std::max(t->N, t->nb) * t->m1 * t->m2;
  for (c64** w : {&t->w0, &t->w1}) {
    cudaError_t e = cudaMalloc((void**)w, big * sizeof(c64));
    if (e != cudaSuccess) {
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return fail(JFB_ERR_CUDA);
    }
    t->allocs.push_back(*w);
  }
  if (allow_smem((const void*)y_backward_kernel<double>) != cudaSuccess ||
      allow_smem((const void*)y_forward_kernel<double>) != cudaSuccess ||
      allow_smem((const void*)fft_rows_kernel) != cudaSuccess) {
    set_error("cannot configure the transform kernels");
    return fail(JFB_ERR_CUDA);
  }
  *out = t;
  return JFB_OK;
}

namespace jfb {

// Device copy of one separable x-axis map (built and uploaded on first use).
static int tps_xmap(jfb_tps* t, int map, int k, const double** A, int* rows, int* cols) {
  const int64_t key = (int64_t)map * 64 + k;
  auto it = t->xmaps.find(key);
  if (it == t->xmaps.end()) {
    int r = 0, c = 0;
    const std::vector<double> h = x_map_matrix(t->xb, map, k, &r, &c);
    double* d = nullptr;
    JFB_CHECK_CUDA(cudaMalloc((void**)&d, h.size() * sizeof(double)));
    cudaError_t e = cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(d);
      JFB_CHECK_CUDA(e);
    }
    it = t->xmaps.emplace(key, std::make_pair(d, std::make_pair(r, c))).first;
  }
  *A = it->second.first;
  *rows = it->second.second.first;
  *cols = it->second.second.second;
  return JFB_OK;
}

static double fourier_df(const jfb_tps* t, int a) {
  const double L = t->cfg.l[a];
  return std::fabs(L - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / L;
}

// out = w * (map_k along x) in, w the Fourier weights of orders k1, k2.
static int tps_xw(jfb_tps* t, int map, int kx, int k1, int k2, double scale, const c64* in,
                  c64* out, cudaStream_t s) {
  const double* A;
  int rows, cols;
  int st = tps_xmap(t, map, kx, &A, &rows, &cols);
  if (st) return st;
  FourierWeight fw;
  fw.n1 = t->n1;
  fw.n2 = t->n2;
  fw.k1 = k1;
  fw.k2 = t->cfg.ndim == 3 ? k2 : 0;
  fw.df1 = fourier_df(t, 0);
  fw.df2 = t->cfg.ndim == 3 ? fourier_df(t, 1) : 1.0;
  fw.scale = scale;
  const int64_t M = (int64_t)t->n1 * t->n2;
  dim3 g((unsigned)((M + 255) / 256), rows);
  x_apply_w_kernel<<<g, 256, 0, s>>>(A, rows, cols, in, out, fw);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

static int check_orders(const jfb_tps* t, const int32_t* k) {
  JFB_REQUIRE(k, "null derivative orders");
  for (int a = 0; a < t->cfg.ndim; ++a)
    JFB_REQUIRE(k[a] >= 0 && k[a] < 32, "derivative orders must be in [0, 32)");
  return JFB_OK;
}

static int tps_x(const double* A, int rows, int cols, const c64* in, c64* out, int64_t M,
                 cudaStream_t s) {
  dim3 g((unsigned)((M + 255) / 256), rows);
  x_apply_kernel<<<g, 256, 0, s>>>(A, rows, cols, in, out, M);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

// middle axis of an array (rows, len, inner): the y kernels with Kz = inner
static int tps_y(jfb_tps* t, int sign, int rows, int inner, const c64* in, c64* out,
                 bool padded, cudaStream_t s) {
  Dims d;
  std::memset(&d, 0, sizeof(d));
  d.Nx = rows;
  d.Ny = t->n1;
  d.Kz = inner;
  d.P = t->n1 * inner;
  d.My = padded ? t->m1 : t->n1;
  const FFTPlan& plan = padded ? t->f1m : t->f1n;
  const c64* tw = padded ? t->tw1m : t->tw1n;
  int KC = inner;
  while ((size_t)2 * d.My * KC * sizeof(c64) > 96 * 1024 && KC % 2 == 0) KC /= 2;
  JFB_REQUIRE((size_t)2 * d.My * KC * sizeof(c64) <= 200 * 1024, "Fourier axis too long");
  dim3 g(rows, 1, inner / KC);
  const size_t sm = (size_t)2 * d.My * KC * sizeof(c64);
  if (sign > 0) y_backward_kernel<double><<<g, 256, sm, s>>>(d, plan, KC, tw, in, out);
  else y_forward_kernel<double><<<g, 256, sm, s>>>(d, plan, KC, tw, in, out, nullptr, 1);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

static int tps_z(jfb_tps* t, int sign, int64_t lines, const c64* in, c64* out, bool padded,
                 cudaStream_t s) {
  const int n = t->n2, m = padded ? t->m2 : t->n2;
  const FFTPlan& plan = padded ? t->f2m : t->f2n;
  const c64* tw = padded ? t->tw2m : t->tw2n;
  const size_t sm = (size_t)2 * m * kTpsRows * sizeof(c64);
  JFB_REQUIRE(sm <= 200 * 1024, "Fourier axis too long");
  const int blocks = (int)((lines + kTpsRows - 1) / kTpsRows);
  if (sign > 0) fft_rows_kernel<<<blocks, 256, sm, s>>>(plan, tw, +1, in, out, lines, n, m);
  else fft_rows_kernel<<<blocks, 256, sm, s>>>(plan, tw, -1, in, out, lines, m, n);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

}  // namespace jfb

extern "C" int jfb_tps_backward(jfb_tps* t, const void* coeffs, void* phys, int padded,
                                void* stream) {
  JFB_REQUIRE(t && coeffs && phys, "null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  const bool pad = padded != 0;
  const int m1 = pad ? t->m1 : t->n1;
  int st;
  if (t->cfg.ndim == 2) {
    // x: (nb, n1) -> (N, n1); y: -> (N, m1)
    if ((st = tps_x(t->B, t->N, t->nb, (const c64*)coeffs, t->w0, t->n1, s))) return st;
    return tps_y(t, +1, t->N, 1, t->w0, (c64*)phys, pad, s);
  }
  if ((st = tps_x(t->B, t->N, t->nb, (const c64*)coeffs, t->w0, (int64_t)t->n1 * t->n2, s)))
    return st;
  if ((st = tps_y(t, +1, t->N, t->n2, t->w0, t->w1, pad, s))) return st;
  return tps_z(t, +1, (int64_t)t->N * m1, t->w1, (c64*)phys, pad, s);
}

extern "C" int jfb_tps_forward(jfb_tps* t, const void* phys, void* coeffs, int padded, int kind,
                               void* stream) {
  JFB_REQUIRE(t && phys && coeffs, "null pointer");
  JFB_REQUIRE(kind == 0 || kind == 1, "kind must be 0 (forward) or 1 (scalar product)");
  cudaStream_t s = (cudaStream_t)stream;
  const bool pad = padded != 0;
  const int m1 = pad ? t->m1 : t->n1;
  const double* X = kind ? t->Sq : t->F;
  int st;
  if (t->cfg.ndim == 2) {
    if ((st = tps_y(t, -1, t->N, 1, (const c64*)phys, t->w0, pad, s))) return st;
    if ((st = tps_x(X, t->nb, t->N, t->w0, (c64*)coeffs, t->n1, s))) return st;
  } else {
    if ((st = tps_z(t, -1, (int64_t)t->N * m1, (const c64*)phys, t->w0, pad, s))) return st;
    if ((st = tps_y(t, -1, t->N, t->n2, t->w0, t->w1, pad, s))) return st;
    if ((st = tps_x(X, t->nb, t->N, t->w1, (c64*)coeffs, (int64_t)t->n1 * t->n2, s))) return st;
  }
  if (kind == 1) {
    // scalar products carry the Fourier weight 2 pi / df per periodic axis
    // (Fourier.py:152-167); the forward transform does not
    double w = 1.0;
    for (int a = 0; a + 1 < t->cfg.ndim; ++a) {
      const double L = t->cfg.l[a];
      const double df = std::fabs(L - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / L;
      w *= 2.0 * M_PI / df;
    }
    const size_t n = (size_t)t->nb * t->n1 * t->n2;
    tps_scale_kernel<<<256, 256, 0, s>>>((c64*)coeffs, w, n);
    JFB_CHECK_LAUNCH();
  }
  return JFB_OK;
}

extern "C" int jfb_tps_backward_primitive(jfb_tps* t, const void* coeffs, void* phys,
                                          const int32_t* k, int padded, void* stream) {
  JFB_REQUIRE(t && coeffs && phys, "null pointer");
  int st = check_orders(t, k);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const bool pad = padded != 0;
  const int m1 = pad ? t->m1 : t->n1;
  const int k2 = t->cfg.ndim == 3 ? k[2] : 0;
  if ((st = tps_xw(t, kXBackward, k[0], k[1], k2, 1.0, (const c64*)coeffs, t->w0, s))) return st;
  if (t->cfg.ndim == 2) return tps_y(t, +1, t->N, 1, t->w0, (c64*)phys, pad, s);
  if ((st = tps_y(t, +1, t->N, t->n2, t->w0, t->w1, pad, s))) return st;
  return tps_z(t, +1, (int64_t)t->N * m1, t->w1, (c64*)phys, pad, s);
}

extern "C" int jfb_tps_to_orthogonal(jfb_tps* t, const void* coeffs, void* orth, void* stream) {
  JFB_REQUIRE(t && coeffs && orth, "null pointer");
  return tps_xw(t, kXToOrth, 0, 0, 0, 1.0, (const c64*)coeffs, (c64*)orth,
                (cudaStream_t)stream);
}

extern "C" int jfb_tps_differentiate_orthogonal(jfb_tps* t, const void* orth, void* out,
                                                const int32_t* k, void* stream) {
  JFB_REQUIRE(t && orth && out, "null pointer");
  int st = check_orders(t, k);
  if (st) return st;
  return tps_xw(t, kXDiffOrth, k[0], k[1], t->cfg.ndim == 3 ? k[2] : 0, 1.0, (const c64*)orth,
                (c64*)out, (cudaStream_t)stream);
}

extern "C" int jfb_tps_project_from_orthogonal(jfb_tps* t, const void* orth, void* coeffs,
                                               void* stream) {
  JFB_REQUIRE(t && orth && coeffs, "null pointer");
  return tps_xw(t, kXProjectOrth, 0, 0, 0, 1.0, (const c64*)orth, (c64*)coeffs,
                (cudaStream_t)stream);
}

extern "C" int jfb_tps_scalar_product_from_orthogonal(jfb_tps* t, const void* orth, void* out,
                                                      void* stream) {
  JFB_REQUIRE(t && orth && out, "null pointer");
  double w = 1.0;  // Fourier mass 2 pi / df per periodic axis
  for (int a = 0; a + 1 < t->cfg.ndim; ++a) w *= 2.0 * M_PI / fourier_df(t, a);
  return tps_xw(t, kXSpFromOrth, 0, 0, 0, w, (const c64*)orth, (c64*)out, (cudaStream_t)stream);
}

extern "C" int jfb_tps_galerkin(const jfb_tps* t, int order, double* out) {
  JFB_REQUIRE(t && out, "null pointer");
  JFB_REQUIRE(order == 0 || order == 2, "order must be 0 or 2");
  const std::vector<double>& G = order ? t->G2 : t->G0;
  std::copy(G.begin(), G.end(), out);
  return JFB_OK;
}

extern "C" int jfb_tps_get_sizes(const jfb_tps* t, int32_t* out4) {
  JFB_REQUIRE(t && out4, "null pointer");
  out4[0] = t->nb;
  out4[1] = t->N;
  out4[2] = t->m1;
  out4[3] = t->m2;
  return JFB_OK;
}

extern "C" int jfb_helmholtz2d_solve(const jfb_tps* tc, const jfb_tps* td, const double* L,
                                     const int64_t* L_offsets, int64_t n_L, const double* U,
                                     const int64_t* U_offsets, int64_t n_U, const double* U_inv,
                                     double fourier_mass, const void* f_hat, void* u,
                                     void* stream) {
  JFB_REQUIRE(tc && td && U && U_offsets && f_hat && u, "null pointer");
  JFB_REQUIRE(n_L == 0 || (L && L_offsets), "null L factor");
  JFB_REQUIRE(tc->cfg.ndim == 2 && td->cfg.ndim == 2, "2-D spaces only");
  JFB_REQUIRE(tc->cfg.basis == JFB_BASIS_ORTHOGONAL && td->cfg.basis == JFB_BASIS_DIRICHLET,
              "tc must be orthogonal, td Dirichlet");
  JFB_REQUIRE(tc->N == td->N && tc->n1 == td->n1 && tc->nb == tc->N, "tc, td sizes differ");
  JFB_REQUIRE(tc->cfg.family == td->cfg.family, "tc, td families differ");
  JFB_REQUIRE(fourier_mass != 0.0, "fourier_mass must be nonzero");
  JFB_REQUIRE(n_L >= 0 && n_L <= kHelmMaxDiag && n_U >= 1 && n_U <= kHelmMaxDiag,
              "too many diagonals");
  const int N = td->N, nb = td->nb, M = td->n1;
  const int KC = (M + kHelmCTAs - 1) / kHelmCTAs, JR = (N + kHelmCTAs - 1) / kHelmCTAs;
  // solve vectors: row stride QS = 1 mod 4 complex values, so that the rows
  // one column step updates (even offsets apart) spread over the banks
  const int QS = KC + ((5 - KC % 4) % 4);
  const size_t smem = ((size_t)2 * N * KC + (size_t)N * QS + (size_t)2 * M * JR) * sizeof(c64) +
                      (size_t)nb * N * sizeof(double);
  int dev = 0, optin = 0;
  JFB_CHECK_CUDA(cudaGetDevice(&dev));
  JFB_CHECK_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem > (size_t)optin) {
    set_error("problem too large for the one-cluster Helmholtz solve");
    return JFB_ERR_ARG;
  }
  Helm2DArgs h;
  std::memset(&h, 0, sizeof(h));
  h.nL = (int)n_L;
  h.nU = (int)n_U;
  h.umain = -1;
  for (int d = 0; d < h.nL; ++d) {
    h.loff[d] = (int)L_offsets[d];
    JFB_REQUIRE(h.loff[d] < 0, "L offsets must be < 0");
  }
  for (int d = 0; d < h.nU; ++d) {
    h.uoff[d] = (int)U_offsets[d];
    JFB_REQUIRE(h.uoff[d] >= 0, "U offsets must be >= 0");
    if (h.uoff[d] == 0) h.umain = d;
  }
  JFB_REQUIRE(h.umain >= 0, "U offsets must contain the main diagonal");
  JFB_REQUIRE(!U_inv || td->nb <= 128, "U_inv form: at most 128 unknowns per mode");
  h.Uinv = U_inv;
  h.l2 = h.l4 = -1;
  bool two_four = true;
  for (int d = 0; d < h.nL; ++d) {
    if (h.loff[d] == -2) h.l2 = d;
    else if (h.loff[d] == -4) h.l4 = d;
    else two_four = false;
  }
  if (!two_four) h.l2 = h.l4 = -1;  // the general column-oriented form
  // the column updates of one step write one row per diagonal
  for (int a = 0; a < h.nU; ++a)
    for (int b = a + 1; b < h.nU; ++b) JFB_REQUIRE(h.uoff[a] != h.uoff[b], "repeated U offset");
  for (int a = 0; a < h.nL; ++a)
    for (int b = a + 1; b < h.nL; ++b) JFB_REQUIRE(h.loff[a] != h.loff[b], "repeated L offset");
  h.BC = tc->B;
  h.SD = td->Sq;
  h.BD = td->B;
  h.tw = td->tw1n;
  h.plan = td->f1n;
  h.L = L;
  h.U = U;
  h.N = N;
  h.nb = nb;
  h.M = M;
  h.KC = KC;
  h.JR = JR;
  h.QS = QS;
  // Fourier scalar-product weight 2 pi / df (Fourier.py:152-167), the
  // caller's division by the Fourier mass, the 1/n1 of the forward transform
  const double Ly = td->cfg.l[0];
  const double df = std::fabs(Ly - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / Ly;
  h.scale = (2.0 * M_PI / df) / fourier_mass / M;
  h.f = (const c64*)f_hat;
  h.u = (c64*)u;
  static bool attr = false;
  if (!attr) {
    JFB_CHECK_CUDA(cudaFuncSetAttribute((const void*)helmholtz2d_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    attr = true;
  }
  helmholtz2d_kernel<<<kHelmCTAs, kHelmThreads, smem, (cudaStream_t)stream>>>(h);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}
