// jaxfun.la replacements: DIA matvec / rmatvec, batched no-pivot banded LU and
// the per-wavenumber banded solve, as standalone C-ABI entry points.
//
// Reference semantics:
//   DiaMatrix storage / matvec / rmatvec   src/jaxfun/la/diamatrix.py:100-348
//   no-pivot banded LU kernel              src/jaxfun/la/diamatrix.py:1936-1973
//   batched wavenumber solve               src/jaxfun/la/tpmatrix.py:686-799
#include <climits>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "jfb_common.cuh"

namespace jfb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

constexpr int kMaxOffsets = 512;

struct OffsetTable {
  int n;
  int off[kMaxOffsets];
};

// ---------------------------------------------------------------------------
// DIA matvec:  y[o, i, t] = sum_d data[d, i + k_d] * x[o, i + k_d, t]
// DIA rmatvec: y[o, j, t] = sum_d data[d, j] * x[o, j - k_d, t]
// One thread per output element; t (inner) is the fastest index so that a
// warp reads contiguous x and writes contiguous y.
// ---------------------------------------------------------------------------
template <typename V>
__global__ void dia_matvec_kernel(const double* __restrict__ data, OffsetTable offs,
                                  int64_t n_rows, int64_t n_cols,
                                  const V* __restrict__ x, V* __restrict__ y,
                                  int64_t outer, int64_t inner, int transpose) {
  const int64_t n_out = transpose ? n_cols : n_rows;
  const int64_t n_in = transpose ? n_rows : n_cols;
  const int64_t total = outer * n_out * inner;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = idx % inner;
    const int64_t i = (idx / inner) % n_out;
    const int64_t o = idx / (inner * n_out);
    const V* xo = x + o * n_in * inner;
    double acc_re = 0.0, acc_im = 0.0;
    for (int d = 0; d < offs.n; ++d) {
      const int64_t k = offs.off[d];
      int64_t col, xi;
      if (!transpose) {
        col = i + k;  // A[i, i+k] stored at data[d, i+k]
        xi = col;
        if (col < 0 || col >= n_cols || i >= n_rows) continue;
      } else {
        col = i;      // (x @ A)[j] = sum_d data[d, j] x[j - k]
        xi = i - k;
        if (xi < 0 || xi >= n_rows) continue;
      }
      const double a = data[d * n_cols + col];
      const V xv = xo[xi * inner + t];
      if constexpr (sizeof(V) == sizeof(double)) {
        acc_re += a * (double)xv;
      } else {
        acc_re += a * xv.re;
        acc_im += a * xv.im;
      }
    }
    if constexpr (sizeof(V) == sizeof(double)) {
      y[idx] = acc_re;
    } else {
      y[idx] = cmk(acc_re, acc_im);
    }
  }
}

// ---------------------------------------------------------------------------
// Batched banded LU without pivoting.  One warp per matrix: for each column
// k and each sub-diagonal s the lanes update the trailing row segment in
// parallel (the elimination order per entry is identical to the reference's
// sequential loop: every entry receives its updates in increasing k).
// band[b][p + off][j] = A_b[j - off, j].
// ---------------------------------------------------------------------------
__global__ void banded_lu_kernel(double* __restrict__ band, int64_t n_batch, int p,
                                 int q, int n, int* __restrict__ bad) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= n_batch) return;
  const int bw = p + q + 1;
  double* A = band + b * (int64_t)bw * n;
  auto at = [&](int row, int col) -> double& { return A[(int64_t)row * n + col]; };
  const int c = p;
  for (int k = 0; k < n; ++k) {
    const double pivot = at(c, k);
    if (lane == 0 && (!(fabs(pivot) > 0.0) || !isfinite(pivot))) atomicExch(bad, 1);
    for (int s = 1; s <= p; ++s) {
      if (k + s >= n) break;
      const double f = at(c - s, k) / pivot;
      __syncwarp();
      if (lane == 0) at(c - s, k) = f;
      for (int u = 1 + lane; u <= q; u += 32) {
        const int j = k + u;
        if (j < n) at(c + u - s, j) -= f * at(c + u, j);
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Wavenumber solve.  One thread per (rhs r, Fourier mode f): forward
// elimination with the unit-lower factor, then back substitution.
// rhs/out layout (n_rhs, outer, n_P, inner); mode f = o * inner + t.
// ---------------------------------------------------------------------------
template <typename V>
__global__ void wavenumber_solve_kernel(const double* __restrict__ L, OffsetTable loff,
                                        const double* __restrict__ U, OffsetTable uoff,
                                        int main_idx, int n_P, int64_t outer,
                                        int64_t inner, int64_t n_rhs,
                                        const V* __restrict__ rhs, V* __restrict__ out) {
  const int64_t n_F = outer * inner;
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= n_F * n_rhs) return;
  const int64_t t = gid % inner;
  const int64_t o = (gid / inner) % outer;
  const int64_t r = gid / n_F;
  const int64_t f = o * inner + t;
  const int64_t base = (r * outer + o) * (int64_t)n_P * inner + t;
  const double* Lf = L + f * (int64_t)loff.n * n_P;
  const double* Uf = U + f * (int64_t)uoff.n * n_P;
  const V* b = rhs + base;
  V* x = out + base;
  constexpr bool kCplx = sizeof(V) != sizeof(double);
  // forward: y_i = b_i - sum_s L[i, i-s] y_{i-s};  L[i, i-s] = Ldata[d][i-s]
  for (int i = 0; i < n_P; ++i) {
    double yr, yi = 0.0;
    if constexpr (kCplx) {
      yr = b[(int64_t)i * inner].re;
      yi = b[(int64_t)i * inner].im;
    } else {
      yr = b[(int64_t)i * inner];
    }
    double ar = 0.0, ai = 0.0;
    for (int d = 0; d < loff.n; ++d) {
      const int j = i + loff.off[d];
      if (j < 0) continue;
      const double l = Lf[(int64_t)d * n_P + j];
      if constexpr (kCplx) {
        const V yj = x[(int64_t)j * inner];
        ar += l * yj.re;
        ai += l * yj.im;
      } else {
        ar += l * x[(int64_t)j * inner];
      }
    }
    if constexpr (kCplx) {
      x[(int64_t)i * inner] = cmk(yr - ar, yi - ai);
    } else {
      x[(int64_t)i * inner] = yr - ar;
    }
  }
  // backward: x_i = (y_i - sum_s U[i, i+s] x_{i+s}) / U[i, i]
  for (int i = n_P - 1; i >= 0; --i) {
    double ar = 0.0, ai = 0.0;
    for (int d = 0; d < uoff.n; ++d) {
      const int s = uoff.off[d];
      if (s == 0) continue;
      const int j = i + s;
      if (j >= n_P) continue;
      const double u = Uf[(int64_t)d * n_P + j];
      if constexpr (kCplx) {
        const V xj = x[(int64_t)j * inner];
        ar += u * xj.re;
        ai += u * xj.im;
      } else {
        ar += u * x[(int64_t)j * inner];
      }
    }
    const double diag = Uf[(int64_t)main_idx * n_P + i];
    if constexpr (kCplx) {
      const V yi = x[(int64_t)i * inner];
      x[(int64_t)i * inner] = cmk((yi.re - ar) / diag, (yi.im - ai) / diag);
    } else {
      x[(int64_t)i * inner] = (x[(int64_t)i * inner] - ar) / diag;
    }
  }
}

// Same solve, one warp per (rhs r, Fourier mode f), for factors with many
// diagonals (the dense upper triangles of Chebyshev stiffness matrices).
// Column-oriented substitution on the system's vector in shared memory: once
// x_c is final, lane t applies the column-c entry of diagonal t to that
// diagonal's row (distinct diagonals hit distinct rows, so the updates of one
// column are independent).  The dependent chain is one shared read, (for U)
// a division and one update per column; the factor entries of the next
// column are loaded while the current one is applied.  Reads rhs, writes out
// (in place allowed: a warp reads its whole vector before it writes).
template <typename V>
__global__ void wavenumber_solve_warp_kernel(const double* __restrict__ L, OffsetTable loff,
                                             const double* __restrict__ U, OffsetTable uoff,
                                             int main_idx, int n_P, int64_t outer,
                                             int64_t inner, int64_t n_rhs, const V* rhs,
                                             V* out) {
  extern __shared__ double wsm[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* xr = wsm + (size_t)wib * 2 * n_P;
  double* xi = xr + n_P;
  const int64_t n_F = outer * inner;
  const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (gid >= n_F * n_rhs) return;
  const int64_t t = gid % inner;
  const int64_t o = (gid / inner) % outer;
  const int64_t r = gid / n_F;
  const int64_t f = o * inner + t;
  const int64_t base = (r * outer + o) * (int64_t)n_P * inner + t;
  const double* Lf = L + f * (int64_t)loff.n * n_P;
  const double* Uf = U + f * (int64_t)uoff.n * n_P;
  constexpr bool kCplx = sizeof(V) != sizeof(double);
  for (int i = lane; i < n_P; i += 32) {
    if constexpr (kCplx) {
      const V v = rhs[base + (int64_t)i * inner];
      xr[i] = v.re;
      xi[i] = v.im;
    } else {
      xr[i] = rhs[base + (int64_t)i * inner];
      xi[i] = 0.0;
    }
  }
  __syncwarp();
  // forward: L[i, i + s] (s < 0) sits at column c = i + s, Lf[d * n_P + c]
  const int lrow = (lane < loff.n) ? -loff.off[lane] : n_P;  // row = c + lrow
  double lnext = (lrow < n_P) ? Lf[(int64_t)lane * n_P] : 0.0;
  for (int c = 0; c < n_P; ++c) {
    const double l = lnext;
    if (c + 1 + lrow < n_P) lnext = Lf[(int64_t)lane * n_P + c + 1];
    const double yr = xr[c], yi = xi[c];
    if (c + lrow < n_P) {
      xr[c + lrow] -= l * yr;
      xi[c + lrow] -= l * yi;
    }
    for (int d = lane + 32; d < loff.n; d += 32) {
      const int i = c - loff.off[d];
      if (i >= n_P) continue;
      const double ld = Lf[(int64_t)d * n_P + c];
      xr[i] -= ld * yr;
      xi[i] -= ld * yi;
    }
    __syncwarp();
  }
  // backward: U[i, i + s] (s > 0) sits at column c = i + s, Uf[d * n_P + c]
  const int urow = (lane < uoff.n && uoff.off[lane] != 0) ? uoff.off[lane] : -1;  // row = c - urow
  const double* Ud = Uf + (int64_t)main_idx * n_P;
  double unext = (urow > 0 && n_P - 1 - urow >= 0) ? Uf[(int64_t)lane * n_P + n_P - 1] : 0.0;
  double dnext = Ud[n_P - 1];
  for (int c = n_P - 1; c >= 0; --c) {
    const double u = unext, dg = dnext;
    if (c > 0) {
      dnext = Ud[c - 1];
      if (urow > 0 && c - 1 - urow >= 0) unext = Uf[(int64_t)lane * n_P + c - 1];
    }
    const double x_r = xr[c] / dg, x_i = xi[c] / dg;
    if (lane == (c & 31)) {
      if constexpr (kCplx) out[base + (int64_t)c * inner] = cmk(x_r, x_i);
      else out[base + (int64_t)c * inner] = x_r;
    }
    if (urow > 0 && c - urow >= 0) {
      xr[c - urow] -= u * x_r;
      xi[c - urow] -= u * x_i;
    }
    for (int d = lane + 32; d < uoff.n; d += 32) {
      const int sft = uoff.off[d];
      const int i = c - sft;
      if (sft == 0 || i < 0) continue;
      const double ud = Uf[(int64_t)d * n_P + c];
      xr[i] -= ud * x_r;
      xi[i] -= ud * x_i;
    }
    __syncwarp();
  }
}

static int fill_offsets(OffsetTable& t, const int64_t* offs, int64_t n) {
  if (n < 0 || n > kMaxOffsets) {
    set_error("too many DIA offsets (max 512)");
    return JFB_ERR_ARG;
  }
  t.n = (int)n;
  for (int64_t i = 0; i < n; ++i) t.off[i] = (int)offs[i];
  return JFB_OK;
}

}  // namespace jfb

using namespace jfb;

extern "C" int jfb_version(void) { return 1; }

extern "C" const char* jfb_last_error(void) { return jfb::last_error(); }

extern "C" int jfb_dia_matvec(const double* data, const int64_t* offsets,
                              int64_t n_diags, int64_t n_rows, int64_t n_cols,
                              const double* x, double* y, int64_t outer, int64_t inner,
                              int is_complex, int transpose, void* stream) {
  JFB_REQUIRE(data && offsets && x && y, "null pointer");
  JFB_REQUIRE(n_rows > 0 && n_cols > 0 && outer > 0 && inner > 0, "bad shape");
  OffsetTable t;
  int st = fill_offsets(t, offsets, n_diags);
  if (st) return st;
  const int64_t n_out = transpose ? n_cols : n_rows;
  const int64_t total = outer * n_out * inner;
  const int threads = 256;
  const int blocks = (int)std::min<int64_t>((total + threads - 1) / threads, 148 * 64);
  cudaStream_t s = (cudaStream_t)stream;
  if (is_complex) {
    dia_matvec_kernel<c64><<<blocks, threads, 0, s>>>(
        data, t, n_rows, n_cols, (const c64*)x, (c64*)y, outer, inner, transpose);
  } else {
    dia_matvec_kernel<double><<<blocks, threads, 0, s>>>(
        data, t, n_rows, n_cols, x, y, outer, inner, transpose);
  }
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_banded_lu_factor(double* band, int64_t n_batch, int64_t p, int64_t q,
                                    int64_t n, void* stream) {
  JFB_REQUIRE(band, "null pointer");
  JFB_REQUIRE(n_batch > 0 && p >= 0 && q >= 0 && n > 0, "bad shape");
  cudaStream_t s = (cudaStream_t)stream;
  int* d_bad = nullptr;
  JFB_CHECK_CUDA(cudaMallocAsync((void**)&d_bad, sizeof(int), s));
  JFB_CHECK_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  const int threads = 128;
  const int64_t warps = n_batch;
  const int blocks = (int)((warps * 32 + threads - 1) / threads);
  banded_lu_kernel<<<blocks, threads, 0, s>>>(band, n_batch, (int)p, (int)q, (int)n,
                                              d_bad);
  JFB_CHECK_LAUNCH();
  int h_bad = 0;
  JFB_CHECK_CUDA(cudaMemcpyAsync(&h_bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  JFB_CHECK_CUDA(cudaFreeAsync(d_bad, s));
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  if (h_bad) {
    set_error(
        "Matrix is singular or has a zero/non-finite pivot in LU factorisation "
        "without pivoting");
    return JFB_ERR_SINGULAR;
  }
  return JFB_OK;
}

extern "C" int jfb_wavenumber_solve(const double* L, const int64_t* L_offsets, int64_t n_L,
                                    const double* U, const int64_t* U_offsets, int64_t n_U,
                                    int64_t n_P, int64_t outer, int64_t inner,
                                    int64_t n_rhs, const double* rhs, double* out,
                                    int is_complex, void* stream) {
  JFB_REQUIRE(U && U_offsets && rhs && out, "null pointer");
  JFB_REQUIRE(n_L == 0 || (L && L_offsets), "null L factor");
  JFB_REQUIRE(n_P > 0 && outer > 0 && inner > 0 && n_rhs > 0, "bad shape");
  OffsetTable lt, ut;
  int st = fill_offsets(lt, L_offsets ? L_offsets : (const int64_t*)nullptr, n_L);
  if (st) return st;
  st = fill_offsets(ut, U_offsets, n_U);
  if (st) return st;
  int main_idx = -1;
  for (int d = 0; d < ut.n; ++d) {
    JFB_REQUIRE(ut.off[d] >= 0, "U offsets must be >= 0");
    if (ut.off[d] == 0) main_idx = d;
  }
  for (int d = 0; d < lt.n; ++d) JFB_REQUIRE(lt.off[d] < 0, "L offsets must be < 0");
  JFB_REQUIRE(main_idx >= 0, "U offsets must contain the main diagonal");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t total = n_rhs * outer * inner;
  const int threads = 128;
  if (lt.n + ut.n > 8) {  // wide factors: a warp per system, rhs read in place
    // the column updates of one step write one row per diagonal
    for (int a = 0; a < ut.n; ++a)
      for (int b = a + 1; b < ut.n; ++b) JFB_REQUIRE(ut.off[a] != ut.off[b], "repeated U offset");
    for (int a = 0; a < lt.n; ++a)
      for (int b = a + 1; b < lt.n; ++b) JFB_REQUIRE(lt.off[a] != lt.off[b], "repeated L offset");
    const int64_t wblocks = (total * 32 + threads - 1) / threads;
    const size_t sm = (size_t)(threads / 32) * 2 * n_P * sizeof(double);
    JFB_REQUIRE(sm <= 48 * 1024, "n_P too large for the warp solve (max 768)");
    if (is_complex)
      wavenumber_solve_warp_kernel<c64><<<(unsigned)wblocks, threads, sm, s>>>(
          L, lt, U, ut, main_idx, (int)n_P, outer, inner, n_rhs, (const c64*)rhs, (c64*)out);
    else
      wavenumber_solve_warp_kernel<double><<<(unsigned)wblocks, threads, sm, s>>>(
          L, lt, U, ut, main_idx, (int)n_P, outer, inner, n_rhs, rhs, out);
    JFB_CHECK_LAUNCH();
    return JFB_OK;
  }
  if (rhs != out) {
    const int64_t elems = n_rhs * outer * n_P * inner * (is_complex ? 2 : 1);
    JFB_CHECK_CUDA(cudaMemcpyAsync(out, rhs, elems * sizeof(double),
                                   cudaMemcpyDeviceToDevice, s));
  }
  const int blocks = (int)((total + threads - 1) / threads);
  if (is_complex) {
    wavenumber_solve_kernel<c64><<<blocks, threads, 0, s>>>(
        L, lt, U, ut, main_idx, (int)n_P, outer, inner, n_rhs, (const c64*)out,
        (c64*)out);
  } else {
    wavenumber_solve_kernel<double><<<blocks, threads, 0, s>>>(
        L, lt, U, ut, main_idx, (int)n_P, outer, inner, n_rhs, out, out);
  }
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

// ===========================================================================
// Allocation-free variant of the batched banded LU.
//
// Some callers cannot call cudaMalloc at all: an XLA custom call or another
// framework's operator, whose device memory belongs to that framework's
// allocator, or a process whose caching pool already holds all of the GPU's
// memory.  jfb_banded_lu_factor above allocates its pivot-status word with
// cudaMallocAsync; this entry point keeps the pivot status of every matrix in
// a fixed file-scope device array instead, so it allocates nothing.  The
// array holds JFB_NOALLOC_LU_MAX_BATCH per-matrix flags plus one slot for the
// index of the first singular matrix; every GPU that loads the library holds
// it (256 KiB) until the process exits.  The call reads that index back to
// the host, so it synchronises its stream.
// ===========================================================================

static __device__ __align__(256) int g_noalloc_lu_status[JFB_NOALLOC_LU_MAX_BATCH + 1];

namespace jfb {

// Zero the per-matrix flags of this call and reset the first-singular slot.
__global__ void noalloc_lu_clear_kernel(int* status, int64_t n_batch) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_batch;
       i += (int64_t)gridDim.x * blockDim.x)
    status[i] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) status[JFB_NOALLOC_LU_MAX_BATCH] = INT_MAX;
}

// Same elimination as banded_lu_kernel (one warp per matrix, identical
// operation order); a zero or non-finite pivot sets status[b].
__global__ void noalloc_lu_kernel(double* __restrict__ band, int64_t n_batch, int p, int q,
                                  int n, int* __restrict__ status) {
  const int lane = threadIdx.x & 31;
  const int64_t b = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (b >= n_batch) return;
  double* A = band + b * (int64_t)(p + q + 1) * n;
  auto at = [&](int row, int col) -> double& { return A[(int64_t)row * n + col]; };
  const int c = p;
  for (int k = 0; k < n; ++k) {
    const double pivot = at(c, k);
    if (lane == 0 && (!(fabs(pivot) > 0.0) || !isfinite(pivot))) status[b] = 1;
    for (int s = 1; s <= p; ++s) {
      if (k + s >= n) break;
      const double f = at(c - s, k) / pivot;
      __syncwarp();
      if (lane == 0) at(c - s, k) = f;
      for (int u = 1 + lane; u <= q; u += 32) {
        const int j = k + u;
        if (j < n) at(c + u - s, j) -= f * at(c + u, j);
      }
      __syncwarp();
    }
  }
}

// Lowest index of a singular matrix into the last slot.
__global__ void noalloc_lu_first_kernel(int* status, int64_t n_batch) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_batch;
       i += (int64_t)gridDim.x * blockDim.x)
    if (status[i]) atomicMin(&status[JFB_NOALLOC_LU_MAX_BATCH], (int)i);
}

// Device address of the status array, looked up once per device with that
// device current (the host-side symbol is only a stand-in, not a device
// address, so it must never be passed to a kernel).  The address is kept for
// the life of the process: it is not valid after cudaDeviceReset.
static int noalloc_status_address(int** out) {
  static std::mutex mu;
  static int* addr[128] = {nullptr};
  int dev = 0;
  JFB_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) {
    set_error("device ordinal out of range");
    return JFB_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    int* p = nullptr;
    JFB_CHECK_CUDA(cudaGetSymbolAddress((void**)&p, g_noalloc_lu_status));
    addr[dev] = p;
  }
  *out = addr[dev];
  return JFB_OK;
}

}  // namespace jfb

extern "C" int jfb_banded_lu_factor_noalloc(double* band, int64_t n_batch, int64_t p,
                                            int64_t q, int64_t n, int32_t* first_singular,
                                            void* stream) {
  JFB_REQUIRE(band, "null pointer");
  JFB_REQUIRE(n_batch > 0 && p >= 0 && q >= 0 && n > 0, "bad shape");
  if (n_batch > JFB_NOALLOC_LU_MAX_BATCH) {
    set_error("n_batch exceeds JFB_NOALLOC_LU_MAX_BATCH (65536) of the allocation-free LU");
    return JFB_ERR_ARG;
  }
  int* status = nullptr;
  int st = noalloc_status_address(&status);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const int cblocks = (int)std::min<int64_t>((n_batch + 255) / 256, 1024);
  noalloc_lu_clear_kernel<<<cblocks, 256, 0, s>>>(status, n_batch);
  JFB_CHECK_LAUNCH();
  const int threads = 128;
  const int blocks = (int)((n_batch * 32 + threads - 1) / threads);
  noalloc_lu_kernel<<<blocks, threads, 0, s>>>(band, n_batch, (int)p, (int)q, (int)n, status);
  JFB_CHECK_LAUNCH();
  noalloc_lu_first_kernel<<<cblocks, 256, 0, s>>>(status, n_batch);
  JFB_CHECK_LAUNCH();
  int first = INT_MAX;
  JFB_CHECK_CUDA(cudaMemcpyAsync(&first, status + JFB_NOALLOC_LU_MAX_BATCH, sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  if (first_singular) *first_singular = (first == INT_MAX) ? -1 : first;
  if (first != INT_MAX) {
    set_error("Matrix " + std::to_string(first) +
              " of the batch is singular or has a zero/non-finite pivot in LU "
              "factorisation without pivoting");
    return JFB_ERR_SINGULAR;
  }
  return JFB_OK;
}
