// KMM plane-Couette plan: C-ABI entry points, device set-up (per-wavenumber
// operator assembly, banded LU, packing), state conversion and the step
// driver with CUDA-graph replay of steady SBDF3 steps.
//
// Reference: examples/channelflow_kmm.py (KMM), examples/pcf_fluctuations_jax.py
// (PlaneCouetteFluctuationJax), src/jaxfun/integrators/sbdf3.py, imex_rk.py.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "jfb_common.cuh"
#include "jfb_kmm.h"
#include "jfb_kmm_kernels.cuh"
#include "jfb_kmm_warpk.cuh"
#include "jfb_kmm_gemm.cuh"
#include "jfb_kmm_mhd.cuh"
#include "jfb_kmm_adjoint.cuh"
#include "jfb_kmm_ens.cuh"

#ifdef JFB_PHASE_STAMPS
// Copies the phase stamps (kernel 0: pencil_gemm_kernel, 1: plane_cross_kernel;
// [kernel][cta][phase] global-timer nanoseconds) to host memory.
extern "C" int jfb_debug_read_stamps(unsigned long long* host, int64_t count) {
  JFB_REQUIRE(host && count > 0 && count <= 4 * jfb::kStampCTAs * jfb::kStampPhases,
              "bad stamp buffer");
  JFB_CHECK_CUDA(cudaMemcpyFromSymbol(host, jfb::g_jfb_stamps, (size_t)count * sizeof(*host)));
  return JFB_OK;
}
#endif

namespace jfb {

// IMEXRK3 (Spalart low-storage) tableau, integrators/imex_rk.py:96-125.
static const double kRK3A[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double kRK3B[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
static const double kSBDF3Implicit = 6.0 / 11.0;  // integrators/sbdf3.py:11-12
// ARS IMEXRK222 (imex_rk.py:175-198): implicit diagonal g, explicit weights
// b10 = g, (b20, b21) = (d, 1 - d), explicit linear weight a21 = 1 - g
static const double kG222 = (2.0 - 1.4142135623730950488) / 2.0;
static const double kD222 = 1.0 - 1.0 / (2.0 * kG222);

// ---------------------------------------------------------------------------
// set-up kernels
// ---------------------------------------------------------------------------

// band[m][p + off][j] = a0[m] X0[j-off, j] + a2[m] X2[j-off, j] + a4[m] X4[j-off, j]
__global__ void assemble_band_kernel(const double* __restrict__ X0,
                                     const double* __restrict__ X2,
                                     const double* __restrict__ X4,
                                     const double* __restrict__ coef, int n_modes, int n,
                                     int p, int q, double* __restrict__ band) {
  const int bw = p + q + 1;
  const int64_t total = (int64_t)n_modes * bw * n;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(idx % n);
    const int r = (int)((idx / n) % bw);
    const int m = (int)(idx / ((int64_t)n * bw));
    const int off = r - p;
    const int i = j - off;
    double v = 0.0;
    if (i >= 0 && i < n) {
      const size_t e = (size_t)i * n + j;
      v = coef[3 * m] * X0[e] + coef[3 * m + 1] * X2[e];
      if (X4) v += coef[3 * m + 2] * X4[e];
    }
    band[idx] = v;
  }
}

// Factored band -> packed parity record (see packed_rec_size).
__global__ void pack_factor_kernel(const double* __restrict__ band, int n_modes, int n,
                                   int p, int q, double* __restrict__ out) {
  const int m = blockIdx.x;
  if (m >= n_modes) return;
  const int bw = p + q + 1;
  const double* B = band + (size_t)m * bw * n;
  double* R = out + (size_t)m * packed_rec_size(n);
  auto at = [&](int off, int col) { return B[(size_t)(p + off) * n + col]; };
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    R[2 * i] = (i >= 2 && p >= 2) ? at(-2, i - 2) : 0.0;      // L[i, i-2]
    R[2 * i + 1] = (i >= 4 && p >= 4) ? at(-4, i - 4) : 0.0;  // L[i, i-4]
  }
  const int m0 = (n + 1) / 2, m1 = n / 2;
  double* U0 = R + 2 * n;
  double* U1 = U0 + m0 * (m0 + 1) / 2;
  for (int par = 0; par < 2; ++par) {
    const int mp = par ? m1 : m0;
    double* Up = par ? U1 : U0;
    const int tot = mp * (mp + 1) / 2;
    for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      // invert e -> (r, c) with e = c(c+1)/2 + r, r <= c
      int c = (int)floor((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
      while (c * (c + 1) / 2 > e) --c;
      while ((c + 1) * (c + 2) / 2 <= e) ++c;
      const int r = e - c * (c + 1) / 2;
      const int row = 2 * r + par, col = 2 * c + par;
      const int off = col - row;
      double v = (off <= q) ? at(off, col) : 0.0;
      if (r == c) v = 1.0 / v;
      Up[e] = v;
    }
  }
}

// Factored band -> record of the tensor-core pencil stage: the L pairs as in
// pack_factor_kernel, then per parity class the INVERSE of the upper factor,
// packed column-major (entry (r, c), r <= c, at c (c + 1) / 2 + r).  Column c
// is U^-1 e_c by back substitution (diamatrix.py:1936-1973 gives U).
constexpr int kMaxHalfInv = 64;
__global__ void pack_factor_inv_kernel(const double* __restrict__ band, int n_modes, int n,
                                       int p, int q, double* __restrict__ out) {
  const int mode = blockIdx.x;
  if (mode >= n_modes) return;
  const int bw = p + q + 1;
  const double* B = band + (size_t)mode * bw * n;
  double* R = out + (size_t)mode * packed_rec_size(n);
  auto at = [&](int off, int col) { return B[(size_t)(p + off) * n + col]; };
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    R[2 * i] = (i >= 2 && p >= 2) ? at(-2, i - 2) : 0.0;
    R[2 * i + 1] = (i >= 4 && p >= 4) ? at(-4, i - 4) : 0.0;
  }
  const int m0 = (n + 1) / 2, m1 = n / 2;
  for (int par = 0; par < 2; ++par) {
    const int mp = par ? m1 : m0;
    double* X = R + 2 * n + (par ? m0 * (m0 + 1) / 2 : 0);
    auto U = [&](int r, int k) { return at(2 * (k - r), 2 * k + par); };
    for (int c = threadIdx.x; c < mp; c += blockDim.x) {
      double x[kMaxHalfInv];
      x[c] = 1.0 / U(c, c);
      for (int r = c - 1; r >= 0; --r) {
        double s = 0.0;
        for (int k = r + 1; k <= c && 2 * (k - r) <= q; ++k) s += U(r, k) * x[k];
        x[r] = -s / U(r, r);
      }
      for (int r = 0; r <= c; ++r) X[c * (c + 1) / 2 + r] = x[r];
    }
  }
}

// Reference layout (n, Ny, Nz) complex -> half layout [i][ky][kz < Kz],
// zeroing the y Nyquist row.
__global__ void to_half_kernel(const c64* __restrict__ full, int n, int Ny, int Nz,
                               c64* __restrict__ half) {
  const int Kz = Nz / 2;
  const int64_t total = (int64_t)n * Ny * Kz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int kz = (int)(idx % Kz);
    const int ky = (int)((idx / Kz) % Ny);
    const int i = (int)(idx / ((int64_t)Kz * Ny));
    half[idx] = (ky == Ny / 2) ? cmk(0.0, 0.0) : full[((size_t)i * Ny + ky) * Nz + kz];
  }
}

// Half layout -> full reference layout using c(-ky, -kz) = conj(c(ky, kz));
// the kz = Nz/2 column is zero.
__global__ void to_full_kernel(const c64* __restrict__ half, int n, int Ny, int Nz,
                               c64* __restrict__ full) {
  const int Kz = Nz / 2;
  const int64_t total = (int64_t)n * Ny * Nz;
  for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int kz = (int)(idx % Nz);
    const int ky = (int)((idx / Nz) % Ny);
    const int i = (int)(idx / ((int64_t)Nz * Ny));
    c64 v = cmk(0.0, 0.0);
    if (kz < Kz) {
      v = half[((size_t)i * Ny + ky) * Kz + kz];
    } else if (kz > Kz) {
      const int my = (Ny - ky) % Ny;
      v = conjc(half[((size_t)i * Ny + my) * Kz + (Nz - kz)]);
    }
    full[idx] = v;
  }
}

// Pack / unpack the two real mean-flow vectors into one complex vector.
__global__ void means_in_kernel(const c64* __restrict__ u1, const c64* __restrict__ u2,
                                int n, int Ny, int Nz, c64* __restrict__ vw) {
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    vw[i] = cmk(u1[(size_t)i * Ny * Nz].re, u2[(size_t)i * Ny * Nz].re);
}
__global__ void real_pair_in_kernel(const double* __restrict__ a,
                                    const double* __restrict__ b, int n,
                                    c64* __restrict__ vw) {
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    vw[i] = cmk(a ? a[i] : 0.0, b ? b[i] : 0.0);
}
__global__ void real_pair_out_kernel(const c64* __restrict__ vw, int n, double* a,
                                     double* b) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (a) a[i] = vw[i].re;
    if (b) b[i] = vw[i].im;
  }
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct FactorSet {
  double* su = nullptr;
  double* sg = nullptr;
  double* s00 = nullptr;
  double* s00inv = nullptr;  // explicit inverse of the mean-flow system (tensor-core stage)
  // factored bands kept for the transposed solves of the adjoint (Su, Sg, S00)
  double* band[3] = {nullptr, nullptr, nullptr};
  int bp[3] = {0, 0, 0}, bq[3] = {0, 0, 0};
};

// Real x-matrices of the adjoint (row-major, forward orientation).
struct AdjOps {
  double *A0 = nullptr, *F = nullptr, *R0 = nullptr, *R1 = nullptr, *R2 = nullptr,
         *R3 = nullptr, *B1 = nullptr, *B2 = nullptr, *GB = nullptr, *GD = nullptr,
         *XB0 = nullptr, *XB2 = nullptr, *XB4 = nullptr, *XD0 = nullptr, *XD2 = nullptr;
};

}  // namespace jfb

struct jfb_kmm_plan {
  jfb_kmm_config cfg;
  jfb::HostOperators hop;
  jfb::Dims d;
  jfb::DevOps ops;
  jfb::FFTPlan fy, fz;
  int n_modes = 0, su_rec = 0, sg_rec = 0;
  int KC = 0;
  size_t smem_pencil = 0, smem_y = 0, smem_z = 0;
  std::vector<void*> allocs;
  int64_t device_bytes = 0;
  int* status = nullptr;  // device status word (kStatus* bits), read by jfb_kmm_check
  jfb::FactorSet steady, startup[3];
  jfb::FactorSet rk222;  // IMEXRK222 plans: the factors of gamma = g dt
  jfb::FactorSet cnab2;  // CNAB2 plans: the factors of gamma = dt / 2
  jfb::c64 *U0[3], *G[3], *NU[3], *NG[3], *VW[3], *NVW[3];
  jfb::c64 *NUst, *NGst, *NVWst;
  jfb::c64 *U1S, *U2S;
  jfb::c64 *X, *Y, *HZ, *HX, *HD;
  jfb::c64 *twy, *twz, *twny, *twnz;
  jfb::c32 *twy32 = nullptr, *twz32 = nullptr;  // mixed form: float twiddles
  bool mixed = false;  // X, Y, HZ, HX of the step in complex64
  jfb::FFTPlan fny, fnz;  // unpadded y / z transforms (state_from_physical)
  int py = 0, pz = 0, pnz = 0;  // warp-FFT radix (N = 32 P), 0 = shared-memory Stockham
  int qk = 0;                   // ceil(Kz / 32)
  int KCw = 0;                  // kz columns per warp-FFT y block
  size_t smem_yw_b = 0, smem_yw_f = 0;
  double *diag_partial = nullptr, *diag_mean = nullptr;
  int diag_blocks = 0;
  size_t smem_zf = 0, smem_diag = 0;
  int64_t n = 0;       // ring counter: u^n lives in slot n % 3
  int hist = 0;        // history_steps (0, 1, 2)
  bool have_state = false;
  bool have_H = false;     // HX holds H(u^n)
  bool explicit_u12 = false;  // U1S/U2S hold the current u1, u2
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  cudaStream_t cap = nullptr;  // private stream used only to capture the graphs
  cudaEvent_t* timing_events = nullptr;  // set by jfb_kmm_timed_steps
  bool gemm = false;       // tensor-core pencil stage (pencil_gemm_kernel)
  bool gemm_ok = false, plane_ok = false, tc_ok = false;  // variants this plan can run
  bool pdl = false;        // programmatic dependent launch of the step kernels
  bool plane = false;      // fused periodic-axis transforms (plane_cross_kernel)
  size_t smem_plane = 0;
  size_t smem_zg = 0;      // gradient-form z stage (z_grad_kernel)
  jfb::GemmOps gops;
  size_t smem_gemm = 0;
  // MHD (vector potential A, three Dirichlet components per level)
  bool mhd = false;
  double eta = 0.0;
  jfb::MhdPhys mphys = {0.0, 0.0, 0.0, 0.0, 0.0};
  jfb::MhdOps mops;
  double *sa_steady = nullptr, *sa_startup[3] = {nullptr, nullptr, nullptr};
  jfb::c64 *AR[3], *NA[3], *NAst;
  size_t smem_mhd = 0, smem_zm = 0;
  double* mdiag_partial = nullptr;
  // adjoint: operators and kept factor bands, built on first use
  bool adj_ready = false;
  jfb::AdjOps aops;
  jfb::FactorSet adj_steady, adj_startup[3];
  size_t smem_za = 0;
};

namespace jfb {

// Dynamic shared memory limit of a kernel: the device's opt-in maximum less
// its static shared memory.  The
// attribute is process-wide per kernel, so a per-plan value would let the
// last plan built shrink the limit under an earlier plan's launches.
static cudaError_t allow_smem(const void* fn) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes);
  return e;
}

// Launch with programmatic dependent launch (PDL) when `pdl`: the kernel may
// start while its predecessor on the stream finishes; it runs its read-only
// prologue, then waits in griddepcontrol.wait for the predecessor's results
// (kernels launched this way call pdl_wait() before their first global read
// of a produced array and their first global write).
template <typename... KArgs, typename... Args>
static cudaError_t launch_ex(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block,
                             size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

static int dalloc(jfb_kmm_plan* pl, void** ptr, size_t bytes) {
  JFB_CHECK_CUDA(cudaMalloc(ptr, bytes));
  JFB_CHECK_CUDA(cudaMemset(*ptr, 0, bytes));
  pl->allocs.push_back(*ptr);
  pl->device_bytes += (int64_t)bytes;
  return JFB_OK;
}

template <typename T>
static int upload(jfb_kmm_plan* pl, T** dst, const std::vector<T>& v) {
  int st = dalloc(pl, (void**)dst, std::max<size_t>(1, v.size()) * sizeof(T));
  if (st) return st;
  if (!v.empty())
    JFB_CHECK_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return JFB_OK;
}

static std::vector<c64> twiddles(int n) {
  std::vector<c64> t(n);
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    t[k] = cmk(std::cos(a), std::sin(a));
  }
  return t;
}

// Build, factor and pack the per-wavenumber systems for implicit coefficient
// gamma (tpmatrix.py:1900-2029 assembly, 1105-1149 batched LU).
// Systems sys_first..sys_last (0: Su, 1: Sg, 2: S00) with diffusivity nu;
// inv selects the explicit inverse-factor records (always used by the
// tensor-core pencil stage and the A solves); keep_band keeps the factored
// band instead of packing it (the adjoint's transposed solves).
static int build_factor_set(jfb_kmm_plan* pl, double gamma, FactorSet& fs, double nu,
                            int sys_first, int sys_last, bool inv, bool keep_band = false) {
  const HostOperators& op = pl->hop;
  jfb_kmm_config cfg = pl->cfg;
  cfg.nu = nu;
  const Dims& d = pl->d;
  const int nm = pl->n_modes;
  int st;
  double *dX0 = nullptr, *dX2 = nullptr, *dX4 = nullptr, *dcoef = nullptr, *dband = nullptr;
  auto cleanup = [&]() {
    cudaFree(dX0);
    cudaFree(dX2);
    cudaFree(dX4);
    cudaFree(dcoef);
    cudaFree(dband);
  };
  for (int sys = sys_first; sys <= sys_last; ++sys) {
    // sys 0: Su (biharmonic basis), 1: Sg (Dirichlet), 2: S00 (1-D Dirichlet)
    const bool bih = sys == 0;
    const int n = bih ? d.nB : d.nD;
    const std::vector<double>& X0 = bih ? op.XB0 : op.XD0;
    const std::vector<double>& X2 = bih ? op.XB2 : op.XD2;
    const int modes = (sys == 2) ? 1 : nm;
    std::vector<double> coef((size_t)3 * modes);
    if (sys == 2) {
      coef[0] = 1.0;
      coef[1] = -gamma * cfg.nu;
      coef[2] = 0.0;
    } else {
      for (int a = 0; a < d.Ny / 2; ++a)
        for (int b = 0; b < d.Kz; ++b)
          mode_coefficients(op, cfg, a, b, gamma, bih, &coef[3 * (a * d.Kz + b)]);
    }
    // bandwidths from the nonzero structure of the x-matrices
    int p = 0, q = 0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double v = std::fabs(X0[(size_t)i * n + j]) + std::fabs(X2[(size_t)i * n + j]) +
                         (bih ? std::fabs(op.XB4[(size_t)i * n + j]) : 0.0);
        if (v != 0.0) {
          if (j - i > q) q = j - i;
          if (i - j > p) p = i - j;
          JFB_REQUIRE(((j - i) & 1) == 0, "odd diagonal in a Shen operator");
        }
      }
    JFB_REQUIRE(p <= 4, "unexpected lower bandwidth");
    st = upload(pl, &dX0, X0);
    if (st) return cleanup(), st;
    st = upload(pl, &dX2, X2);
    if (st) return cleanup(), st;
    if (bih) {
      st = upload(pl, &dX4, op.XB4);
      if (st) return cleanup(), st;
    }
    st = upload(pl, &dcoef, coef);
    if (st) return cleanup(), st;
    const size_t band_elems = (size_t)modes * (p + q + 1) * n;
    JFB_CHECK_CUDA(cudaMalloc((void**)&dband, band_elems * sizeof(double)));
    assemble_band_kernel<<<1024, 256>>>(dX0, dX2, bih ? dX4 : nullptr, dcoef, modes, n, p,
                                        q, dband);
    JFB_CHECK_LAUNCH();
    st = jfb_banded_lu_factor(dband, modes, p, q, n, nullptr);
    if (st) return cleanup(), st;
    if (keep_band) {
      fs.band[sys] = dband;
      fs.bp[sys] = p;
      fs.bq[sys] = q;
      pl->allocs.push_back(dband);
      pl->device_bytes += (int64_t)(band_elems * sizeof(double));
      dband = nullptr;
      JFB_CHECK_CUDA(cudaDeviceSynchronize());
      for (void* ptr : {(void*)dX0, (void*)dX2, (void*)dX4, (void*)dcoef}) {
        if (!ptr) continue;
        for (size_t k = 0; k < pl->allocs.size(); ++k)
          if (pl->allocs[k] == ptr) {
            pl->allocs.erase(pl->allocs.begin() + k);
            break;
          }
      }
      pl->device_bytes -= (int64_t)(X0.size() + X2.size() + (bih ? op.XB4.size() : 0) +
                                    coef.size()) *
                          sizeof(double);
      cleanup();
      dX0 = dX2 = dX4 = dcoef = nullptr;
      continue;
    }
    if (sys == 2 && inv) {
      // dense S00 = X0 - gamma nu X2 inverted in long double (Gauss-Jordan,
      // partial pivoting); rows of one parity stay within that parity
      const int nn = n;
      std::vector<long double> Aa((size_t)nn * 2 * nn, 0.0L);
      for (int i = 0; i < nn; ++i) {
        for (int j = 0; j < nn; ++j)
          Aa[(size_t)i * 2 * nn + j] = (long double)coef[0] * X0[(size_t)i * nn + j] +
                                       (long double)coef[1] * X2[(size_t)i * nn + j];
        Aa[(size_t)i * 2 * nn + nn + i] = 1.0L;
      }
      for (int c = 0; c < nn; ++c) {
        int piv = c;
        for (int r = c + 1; r < nn; ++r)
          if (std::fabs(Aa[(size_t)r * 2 * nn + c]) > std::fabs(Aa[(size_t)piv * 2 * nn + c])) piv = r;
        JFB_REQUIRE(Aa[(size_t)piv * 2 * nn + c] != 0.0L, "singular mean-flow system");
        if (piv != c)
          for (int k = 0; k < 2 * nn; ++k) std::swap(Aa[(size_t)c * 2 * nn + k], Aa[(size_t)piv * 2 * nn + k]);
        const long double inv_p = 1.0L / Aa[(size_t)c * 2 * nn + c];
        for (int k = 0; k < 2 * nn; ++k) Aa[(size_t)c * 2 * nn + k] *= inv_p;
        for (int r = 0; r < nn; ++r) {
          if (r == c) continue;
          const long double f = Aa[(size_t)r * 2 * nn + c];
          if (f == 0.0L) continue;
          for (int k = 0; k < 2 * nn; ++k) Aa[(size_t)r * 2 * nn + k] -= f * Aa[(size_t)c * 2 * nn + k];
        }
      }
      std::vector<double> Si((size_t)nn * nn);
      for (int i = 0; i < nn; ++i)
        for (int j = 0; j < nn; ++j) Si[(size_t)i * nn + j] = (double)Aa[(size_t)i * 2 * nn + nn + j];
      st = upload(pl, &fs.s00inv, Si);
      if (st) return cleanup(), st;
    }
    double** dst = (sys == 0) ? &fs.su : (sys == 1) ? &fs.sg : &fs.s00;
    st = dalloc(pl, (void**)dst, (size_t)modes * packed_rec_size(n) * sizeof(double));
    if (st) return cleanup(), st;
    if (inv) {
      JFB_REQUIRE(n <= 2 * kMaxHalfInv, "system too large for the inverse-factor records");
      pack_factor_inv_kernel<<<modes, 64>>>(dband, modes, n, p, q, *dst);
    } else {
      pack_factor_kernel<<<modes, 128>>>(dband, modes, n, p, q, *dst);
    }
    JFB_CHECK_LAUNCH();
    JFB_CHECK_CUDA(cudaDeviceSynchronize());
    // the temporaries were registered as plan allocations by upload(): release them
    for (void* ptr : {(void*)dX0, (void*)dX2, (void*)dX4, (void*)dcoef}) {
      if (!ptr) continue;
      for (size_t k = 0; k < pl->allocs.size(); ++k)
        if (pl->allocs[k] == ptr) {
          pl->allocs.erase(pl->allocs.begin() + k);
          break;
        }
    }
    pl->device_bytes -= (int64_t)(X0.size() + X2.size() + (bih ? op.XB4.size() : 0) +
                                  coef.size()) *
                        sizeof(double);
    cleanup();
    dX0 = dX2 = dX4 = dcoef = dband = nullptr;
  }
  return JFB_OK;
}

static PackedFactors packed(const jfb_kmm_plan* pl, const FactorSet& fs) {
  PackedFactors f;
  f.su = fs.su;
  f.sg = fs.sg;
  f.s00 = fs.s00;
  f.s00inv = fs.s00inv;
  f.su_rec = pl->su_rec;
  f.sg_rec = pl->sg_rec;
  return f;
}

static StageArgs blank_args() {
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  return a;
}

static int launch_pencil(jfb_kmm_plan* pl, const StageArgs& a0, cudaStream_t s) {
  const int blocks = pl->d.Ny * pl->d.nKb;
  StageArgs a = a0;
  a.status = pl->status;
  // one instantiation per register-row count and nonlinear form
  auto* k = pl->d.nD <= 64 ? (pl->d.grad ? pencil_stage_kernel<1, 1> : pencil_stage_kernel<1, 0>)
                           : (pl->d.grad ? pencil_stage_kernel<2, 1> : pencil_stage_kernel<2, 0>);
  k<<<blocks, kNW * 32, pl->smem_pencil, s>>>(pl->ops, pl->d, a);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

// The tensor-core pencil stage's arguments of one implicit stage.
static GemmStageArgs gemm_args(const jfb_kmm_plan* pl, const StageArgs& a) {
  GemmStageArgs g;
  g.HX = a.HX;
  g.c0 = a.c0;
  g.c1 = a.c1;
  g.c2 = a.c2;
  g.d0 = a.d0;
  g.d1 = a.d1;
  g.d2 = a.d2;
  g.slin = a.cL * pl->d.nu;
  g.u0a = a.u0a;
  g.u0b = a.u0b;
  g.u0c = a.u0c;
  g.ga = a.ga;
  g.gb = a.gb;
  g.gc = a.gc;
  g.vwa = a.vwa;
  g.vwb = a.vwb;
  g.vwc = a.vwc;
  g.Nup = a.Nup;
  g.Nuq = a.Nuq;
  g.Ngp = a.Ngp;
  g.Ngq = a.Ngq;
  g.NVWp = a.NVWp;
  g.NVWq = a.NVWq;
  g.Nu_out = a.Nu_out;
  g.Ng_out = a.Ng_out;
  g.NVW_out = a.NVW_out;
  g.su = a.fac.su;
  g.sg = a.fac.sg;
  g.s00 = a.fac.s00;
  g.s00inv = a.fac.s00inv;
  g.su_rec = a.fac.su_rec;
  g.sg_rec = a.fac.sg_rec;
  g.u0_out = a.u0_out;
  g.g_out = a.g_out;
  g.vw_out = a.vw_out;
  g.X = a.X;
  g.x32 = pl->mixed ? 1 : 0;
  g.Xlin = pl->mixed ? reinterpret_cast<const c32*>(pl->X) : nullptr;
  return g;
}

// One implicit stage (mode kImplicit): the tensor-core pencil stage when the
// plan has it, else the warp-per-pencil kernel.
static int launch_implicit(jfb_kmm_plan* pl, const StageArgs& a, cudaStream_t s) {
  if (!pl->gemm) {
    StageArgs b = a;
    b.x32 = pl->mixed ? 1 : 0;
    b.Xlin = pl->mixed ? reinterpret_cast<const c32*>(pl->X) : nullptr;
    return launch_pencil(pl, b, s);
  }
  const GemmStageArgs g = gemm_args(pl, a);
  const int blocks = (pl->d.Ny / 2) * ceil_div(pl->d.Kz, 8);
  // the tcgen05 variant exists for the rotational form only
  auto* k = pl->gops.tc ? pencil_gemm_kernel<true, 0>
            : pl->d.grad ? pencil_gemm_kernel<false, 1>
                         : pencil_gemm_kernel<false, 0>;
  JFB_CHECK_CUDA(launch_ex(pl->pdl, k, dim3(blocks), dim3(kGThreads), pl->smem_gemm, s, pl->d,
                           pl->ops, pl->gops, g));
  return JFB_OK;
}

static int warp_radix(int n) {
  if (n % 32) return 0;
  const int p = n / 32;
  return (p == 2 || p == 3 || p == 4 || p == 6) ? p : 0;
}

// Dimensions handed to the periodic-axis kernels: in the complex64 form the
// base flow is left out of the transforms (the pencil kernels add its terms,
// linear in the perturbation, in FP64 at the x nodes).
template <typename T>
static Dims tdims(const jfb_kmm_plan* pl) {
  Dims d = pl->d;
  if (sizeof(T) == sizeof(float)) d.uwall = 0.0;
  return d;
}

// Step transform buffers and twiddles in the plan's transform precision.
template <typename T> struct Tx;
template <> struct Tx<double> {
  static const c64* twy(const jfb_kmm_plan* pl) { return pl->twy; }
  static const c64* twz(const jfb_kmm_plan* pl) { return pl->twz; }
};
template <> struct Tx<float> {
  static const c32* twy(const jfb_kmm_plan* pl) { return pl->twy32; }
  static const c32* twz(const jfb_kmm_plan* pl) { return pl->twz32; }
};
template <typename T> static cpx<T>* buf(void* p) { return reinterpret_cast<cpx<T>*>(p); }

// Field f of the step's x-physical array X (complex64 in the mixed form).
static c64* x_field(const jfb_kmm_plan* pl, int f) {
  const size_t e = (size_t)f * pl->d.Nx * pl->d.P;
  return pl->mixed ? reinterpret_cast<c64*>(reinterpret_cast<c32*>(pl->X) + e) : pl->X + e;
}
// Field f of the nonlinear array HX (complex64 in the mixed form).
static c64* hx_field(const jfb_kmm_plan* pl, int f) {
  const size_t e = (size_t)f * pl->d.Nx * pl->d.P;
  return pl->mixed ? reinterpret_cast<c64*>(reinterpret_cast<c32*>(pl->HX) + e) : pl->HX + e;
}

// nb / nf: fields transformed backward / forward (6 / 3 for the flow step,
// 12 / 6 for the coupled MHD step)
template <int P, typename T>
static void launch_y_warp(jfb_kmm_plan* pl, cudaStream_t s, bool backward, int nb = 6,
                          int nf = 3, bool self_term = true) {
  const Dims d = tdims<T>(pl);
  const size_t sm = backward ? pl->smem_yw_b : pl->smem_yw_f;
  const size_t smT = sm / sizeof(c64) * sizeof(cpx<T>);
  const int chunks = ceil_div(d.Kz, pl->KCw);
  if (backward) {
    dim3 g(d.Nx, nb, chunks);
    y_backward_warp_kernel<P, T><<<g, 256, smT, s>>>(d, pl->KCw, Tx<T>::twy(pl), buf<T>(pl->X),
                                                       buf<T>(pl->Y));
  } else {
    dim3 g(d.Nx, nf, chunks);
    y_forward_warp_kernel<P, T><<<g, 256, smT, s>>>(d, pl->KCw, Tx<T>::twy(pl), buf<T>(pl->HZ),
                                                      buf<T>(pl->HX),
                                                      self_term ? pl->ops.xphys : nullptr);
  }
}

template <typename T>
static void launch_y_warp_any(jfb_kmm_plan* pl, cudaStream_t s, bool backward, int nb = 6,
                              int nf = 3, bool self_term = true) {
  switch (pl->py) {
    case 2: launch_y_warp<2, T>(pl, s, backward, nb, nf, self_term); break;
    case 3: launch_y_warp<3, T>(pl, s, backward, nb, nf, self_term); break;
    case 4: launch_y_warp<4, T>(pl, s, backward, nb, nf, self_term); break;
    default: launch_y_warp<6, T>(pl, s, backward, nb, nf, self_term); break;
  }
}

template <int P, typename T>
static void launch_zcross_warp(jfb_kmm_plan* pl, cudaStream_t s) {
  const Dims d = tdims<T>(pl);
  const int pairs = ceil_div((int64_t)d.Nx * d.My, 2);
  const int blocks = ceil_div(pairs, 8);
  if (pl->qk == 1)
    z_cross_warp_kernel<P, 1, T><<<blocks, 256, 0, s>>>(pl->ops, d, Tx<T>::twz(pl), buf<T>(pl->Y),
                                                      buf<T>(pl->HZ));
  else
    z_cross_warp_kernel<P, 2, T><<<blocks, 256, 0, s>>>(pl->ops, d, Tx<T>::twz(pl), buf<T>(pl->Y),
                                                      buf<T>(pl->HZ));
}

template <int P>
static void launch_zfwd_warp(jfb_kmm_plan* pl, const double* u0, const double* u1,
                             const double* u2, cudaStream_t s) {
  const Dims& d = pl->d;
  const int pairs = ceil_div((int64_t)d.Nx * d.Ny, 2);
  const int blocks = ceil_div(pairs, 8);
  if (pl->qk == 1)
    z_forward_real_warp_kernel<P, 1><<<blocks, 256, 0, s>>>(d, pl->twnz, u0, u1, u2, pl->HZ);
  else
    z_forward_real_warp_kernel<P, 2><<<blocks, 256, 0, s>>>(d, pl->twnz, u0, u1, u2, pl->HZ);
}

template <int PY, int PZ, typename T>
static cudaError_t launch_plane(jfb_kmm_plan* pl, cudaStream_t s) {
  return launch_ex(pl->pdl, plane_cross_kernel<PY, PZ, 1, T>, dim3(2 * pl->d.Nx),
                   dim3(plane_threads<T>()), plane_smem_bytes(pl->d.My, pl->d.Kz, sizeof(cpx<T>)),
                   s, pl->ops, tdims<T>(pl), Tx<T>::twy(pl), Tx<T>::twz(pl),
                   (const cpx<T>*)buf<T>(pl->X), buf<T>(pl->HX));
}

// y_backward -> z_cross -> y_forward: HX <- H(state whose x-physical fields are in X)
template <typename T>
static int launch_transforms_t(jfb_kmm_plan* pl, cudaStream_t s) {
  const Dims d = tdims<T>(pl);
  if (pl->plane) {
    const int key = pl->py * 10 + pl->pz;
    if (key == 22) JFB_CHECK_CUDA((launch_plane<2, 2, T>(pl, s)));
    else if (key == 23) JFB_CHECK_CUDA((launch_plane<2, 3, T>(pl, s)));
    else if (key == 32) JFB_CHECK_CUDA((launch_plane<3, 2, T>(pl, s)));
    else JFB_CHECK_CUDA((launch_plane<3, 3, T>(pl, s)));
    if (pl->timing_events)
      for (int k = 2; k <= 4; ++k) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[k], s));
    return JFB_OK;
  }
  if (d.grad) {
    // gradient form: u_i, d/dx u_i, d/dy u_i backward in y, the
    // twelve-field z stage, n_i forward in y (no constant base-flow term;
    // complex64 in the mixed form, whose base-flow terms the pencil stage
    // adds in FP64)
    if (pl->py) {
      launch_y_warp_any<T>(pl, s, true, 9);
    } else {
      dim3 gy(d.Nx, 9, d.Kz / pl->KC);
      y_backward_kernel<T><<<gy, 256, pl->smem_y / sizeof(c64) * sizeof(cpx<T>), s>>>(
          d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->X), buf<T>(pl->Y));
    }
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[2], s));
    if (pl->pz) {  // warp-shuffle z transforms (Mz = 32 P, Kz <= 64)
      const int blocks = ceil_div(ceil_div((int64_t)d.Nx * d.My, 2), 8);
      switch (pl->pz * 10 + pl->qk) {
#define JFB_ZG(P, Q)                                                                     \
  case P * 10 + Q:                                                                       \
    z_grad_warp_kernel<P, Q, T><<<blocks, 256, 0, s>>>(pl->ops, d, Tx<T>::twz(pl),              \
                                                        buf<T>(pl->Y), buf<T>(pl->HZ));         \
    break;
        JFB_ZG(2, 1) JFB_ZG(2, 2) JFB_ZG(3, 1) JFB_ZG(3, 2)
        JFB_ZG(4, 1) JFB_ZG(4, 2) JFB_ZG(6, 1) JFB_ZG(6, 2)
#undef JFB_ZG
        default: break;
      }
    } else {
      const int zb = ceil_div((int64_t)d.Nx * d.My, kZRows);
      z_grad_kernel<T><<<zb, 256, pl->smem_zg / sizeof(c64) * sizeof(cpx<T>), s>>>(
          pl->ops, d, pl->fz, Tx<T>::twz(pl), buf<T>(pl->Y), buf<T>(pl->HZ));
    }
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[3], s));
    if (pl->py) {
      launch_y_warp_any<T>(pl, s, false, 9, 3, false);
    } else {
      dim3 gf(d.Nx, 3, d.Kz / pl->KC);
      y_forward_kernel<T><<<gf, 256, pl->smem_y / sizeof(c64) * sizeof(cpx<T>), s>>>(
          d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->HZ), buf<T>(pl->HX), nullptr);
    }
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[4], s));
    return JFB_OK;
  }
  if (pl->py && pl->pz) {
    launch_y_warp_any<T>(pl, s, true);
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[2], s));
    switch (pl->pz) {
      case 2: launch_zcross_warp<2, T>(pl, s); break;
      case 3: launch_zcross_warp<3, T>(pl, s); break;
      case 4: launch_zcross_warp<4, T>(pl, s); break;
      default: launch_zcross_warp<6, T>(pl, s); break;
    }
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[3], s));
    launch_y_warp_any<T>(pl, s, false);
    JFB_CHECK_LAUNCH();
    if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[4], s));
    return JFB_OK;
  }
  dim3 gy(d.Nx, 6, d.Kz / pl->KC);
  const size_t smy = pl->smem_y / sizeof(c64) * sizeof(cpx<T>);
  const size_t smz = pl->smem_z / sizeof(c64) * sizeof(cpx<T>);
  y_backward_kernel<T><<<gy, 256, smy, s>>>(d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->X),
                                            buf<T>(pl->Y));
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[2], s));
  const int zb = ceil_div((int64_t)d.Nx * d.My, kZRows);
  z_cross_kernel<T><<<zb, 256, smz, s>>>(pl->ops, d, pl->fz, Tx<T>::twz(pl), buf<T>(pl->Y),
                                         buf<T>(pl->HZ));
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[3], s));
  dim3 gf(d.Nx, 3, d.Kz / pl->KC);
  y_forward_kernel<T><<<gf, 256, smy, s>>>(d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->HZ),
                                           buf<T>(pl->HX), pl->ops.xphys);
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[4], s));
  return JFB_OK;
}

// The coupled MHD step: twelve fields (u, omega, b, j) backward in y, the z
// stage with the Lorentz force and the EMF, six fields (n, emf) forward in y;
// complex64 in the mixed form (tdims: the flow's base-flow terms are added in
// FP64 by the pencil stage).
template <typename T>
static int launch_transforms_mhd(jfb_kmm_plan* pl, cudaStream_t s) {
  const Dims d = tdims<T>(pl);
  const size_t smy = pl->smem_y / sizeof(c64) * sizeof(cpx<T>);
  if (pl->py) {  // warp-shuffle transforms along y (My = 32 P)
    launch_y_warp_any<T>(pl, s, true, 12, 6);
  } else {
    dim3 gy(d.Nx, 12, d.Kz / pl->KC);
    y_backward_kernel<T><<<gy, 256, smy, s>>>(d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->X),
                                              buf<T>(pl->Y));
  }
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[2], s));
  const int zb = ceil_div((int64_t)d.Nx * d.My, kZRows);
  z_cross_mhd_kernel<T><<<zb, 256, pl->smem_zm / sizeof(c64) * sizeof(cpx<T>), s>>>(
      pl->ops, d, pl->mphys, pl->fz, Tx<T>::twz(pl), buf<T>(pl->Y), buf<T>(pl->HZ));
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[3], s));
  if (pl->py) {
    launch_y_warp_any<T>(pl, s, false, 12, 6);
  } else {
    dim3 gf(d.Nx, 6, d.Kz / pl->KC);
    y_forward_kernel<T><<<gf, 256, smy, s>>>(d, pl->fy, pl->KC, Tx<T>::twy(pl), buf<T>(pl->HZ),
                                             buf<T>(pl->HX), pl->ops.xphys);
  }
  JFB_CHECK_LAUNCH();
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[4], s));
  return JFB_OK;
}

static int launch_transforms(jfb_kmm_plan* pl, cudaStream_t s) {
  if (pl->mhd)
    return pl->mixed ? launch_transforms_mhd<float>(pl, s) : launch_transforms_mhd<double>(pl, s);
  return pl->mixed ? launch_transforms_t<float>(pl, s) : launch_transforms_t<double>(pl, s);
}

static MhdArgs blank_mhd() {
  MhdArgs a;
  std::memset(&a, 0, sizeof(a));
  return a;
}

static int launch_mhd(jfb_kmm_plan* pl, const MhdArgs& a0, cudaStream_t s) {
  const int blocks = (pl->d.Ny / 2) * ceil_div(pl->d.Kz, 8);
  MhdArgs a = a0;
  a.status = pl->status;
  // mixed form: the step's EMF and b, j at the nodes are complex64
  a.x32 = (pl->mixed && a.mode != kMhdFromPhys) ? 1 : 0;
  a.uw_b0z = pl->mphys.uw_emf * pl->mphys.b0z;
  a.uw_b0x = pl->mphys.uw_emf * pl->mphys.b0x;
  mhd_a_kernel<<<blocks, kMhdThreads, pl->smem_mhd, s>>>(pl->d, pl->ops, pl->mops, a);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

// x-physical b and j of A (ring slot c) into X fields 6..11.
static int mhd_fields(jfb_kmm_plan* pl, int c, cudaStream_t s) {
  MhdArgs m = blank_mhd();
  m.mode = kMhdFields;
  m.Aa = pl->AR[c];
  m.XB = x_field(pl, 6);
  return launch_mhd(pl, m, s);
}

static inline int slot(int64_t m) { return (int)(((m % 3) + 3) % 3); }


// u1, u2 of the current state into U1S/U2S (reconstruction).
static int ensure_explicit(jfb_kmm_plan* pl, cudaStream_t s) {
  if (pl->explicit_u12) return JFB_OK;
  StageArgs a = blank_args();
  a.mode = kReconstruct;
  const int c = slot(pl->n);
  a.u0a = pl->U0[c];
  a.ga = pl->G[c];
  a.vwa = pl->VW[c];
  a.X = pl->U1S;   // u1 out
  a.Hd_out = pl->U2S;  // u2 out
  int st = launch_pencil(pl, a, s);
  if (st) return st;
  pl->explicit_u12 = true;
  return JFB_OK;
}

static int ensure_H(jfb_kmm_plan* pl, cudaStream_t s) {
  if (pl->have_H) return JFB_OK;
  int st = ensure_explicit(pl, s);
  if (st) return st;
  StageArgs a = blank_args();
  a.mode = kPrologue;
  a.x32 = pl->mixed ? 1 : 0;
  const int c = slot(pl->n);
  a.pu0 = pl->U0[c];
  a.pu1 = pl->U1S;
  a.pu2 = pl->U2S;
  a.X = pl->X;
  st = launch_pencil(pl, a, s);
  if (st) return st;
  if (pl->mhd && (st = mhd_fields(pl, c, s))) return st;
  st = launch_transforms(pl, s);
  if (st) return st;
  pl->have_H = true;
  return JFB_OK;
}

// Arguments of the pencil stage (a) and, for an MHD plan, of the A stage
// (mm) of one steady SBDF3 step from ring position m (u^m in slot m % 3).
static void steady_args(jfb_kmm_plan* pl, int64_t m, StageArgs& a, MhdArgs& mm) {
  a = blank_args();
  a.mode = kImplicit;
  a.HX = pl->HX;
  const int c = slot(m), o1 = slot(m - 1), o2 = slot(m - 2), nw = slot(m + 1);
  a.c0 = 18.0 / 11.0;
  a.c1 = -9.0 / 11.0;
  a.c2 = 2.0 / 11.0;
  a.cL = 0.0;
  a.d0 = 18.0 / 11.0;
  a.d1 = -18.0 / 11.0;
  a.d2 = 6.0 / 11.0;
  a.u0a = pl->U0[c];
  a.u0b = pl->U0[o1];
  a.u0c = pl->U0[o2];
  a.ga = pl->G[c];
  a.gb = pl->G[o1];
  a.gc = pl->G[o2];
  a.vwa = pl->VW[c];
  a.vwb = pl->VW[o1];
  a.vwc = pl->VW[o2];
  a.Nup = pl->NU[o1];
  a.Nuq = pl->NU[o2];
  a.Ngp = pl->NG[o1];
  a.Ngq = pl->NG[o2];
  a.NVWp = pl->NVW[o1];
  a.NVWq = pl->NVW[o2];
  a.Nu_out = pl->NU[c];
  a.Ng_out = pl->NG[c];
  a.NVW_out = pl->NVW[c];
  a.fac = packed(pl, pl->steady);
  a.u0_out = pl->U0[nw];
  a.g_out = pl->G[nw];
  a.vw_out = pl->VW[nw];
  a.X = pl->X;
  mm = blank_mhd();
  if (pl->mhd) {
    mm.mode = kMhdStep;
    mm.HXA = hx_field(pl, 3);
    mm.c0 = a.c0;
    mm.c1 = a.c1;
    mm.c2 = a.c2;
    mm.d0 = a.d0;
    mm.d1 = a.d1;
    mm.d2 = a.d2;
    mm.Aa = pl->AR[c];
    mm.Ab = pl->AR[o1];
    mm.Ac = pl->AR[o2];
    mm.NAp = pl->NA[o1];
    mm.NAq = pl->NA[o2];
    mm.NA_out = pl->NA[c];
    mm.sa = pl->sa_steady;
    mm.sa_rec = pl->sg_rec;
    mm.A_out = pl->AR[nw];
    mm.XB = x_field(pl, 6);
    mm.status = pl->status;
  }
}

// One steady SBDF3 step from ring position m (u^m in slot m % 3).
static int steady_step(jfb_kmm_plan* pl, int64_t m, cudaStream_t s) {
  StageArgs a;
  MhdArgs mm;
  steady_args(pl, m, a, mm);
  int st = launch_implicit(pl, a, s);
  if (st) return st;
  if (pl->mhd && (st = launch_mhd(pl, mm, s))) return st;
  if (pl->timing_events) JFB_CHECK_CUDA(cudaEventRecord(pl->timing_events[1], s));
  return launch_transforms(pl, s);
}

// steady_step with an event recorded after the pencil kernel and after each
// of the three periodic-axis kernels (ev[1..4]); ev[0] is recorded by the caller.
static int steady_step_timed(jfb_kmm_plan* pl, int64_t m, cudaStream_t s, cudaEvent_t* ev) {
  pl->timing_events = ev;
  const int st = steady_step(pl, m, s);
  pl->timing_events = nullptr;
  return st;
}

// One IMEXRK3 startup step (_step_sbdf3 startup branch).
// rec (optional): receives the stage states after stages 0 and 1 as
// (u0, g, vw) of stage 1 then of stage 2 (the adjoint's linearisation points).
static int startup_step(jfb_kmm_plan* pl, cudaStream_t s, c64* const* rec = nullptr) {
  const int64_t m = pl->n;
  const int c = slot(m), nw = slot(m + 1);
  for (int rk = 0; rk < 3; ++rk) {
    StageArgs a = blank_args();
    a.mode = kImplicit;
    a.HX = pl->HX;
    a.c0 = 1.0;
    a.cL = (kRK3A[rk] + kRK3B[rk]) * pl->cfg.dt / 2.0;
    a.d0 = kRK3A[rk];
    a.d1 = kRK3B[rk];
    const int src = (rk == 0) ? c : nw;
    a.u0a = pl->U0[src];
    a.ga = pl->G[src];
    a.vwa = pl->VW[src];
    if (rk == 1) {
      a.Nup = pl->NU[c];
      a.Ngp = pl->NG[c];
      a.NVWp = pl->NVW[c];
    } else if (rk == 2) {
      a.Nup = pl->NUst;
      a.Ngp = pl->NGst;
      a.NVWp = pl->NVWst;
    }
    if (rk == 0) {
      a.Nu_out = pl->NU[c];
      a.Ng_out = pl->NG[c];
      a.NVW_out = pl->NVW[c];
    } else if (rk == 1) {
      a.Nu_out = pl->NUst;
      a.Ng_out = pl->NGst;
      a.NVW_out = pl->NVWst;
    }
    a.fac = packed(pl, pl->startup[rk]);
    a.u0_out = pl->U0[nw];
    a.g_out = pl->G[nw];
    a.vw_out = pl->VW[nw];
    a.X = pl->X;
    int st = launch_implicit(pl, a, s);
    if (st) return st;
    if (pl->mhd) {
      MhdArgs m = blank_mhd();
      m.mode = kMhdStep;
      m.HXA = hx_field(pl, 3);
      m.c0 = 1.0;
      m.slin = a.cL * pl->eta;
      m.d0 = kRK3A[rk];
      m.d1 = kRK3B[rk];
      m.Aa = pl->AR[src];
      if (rk == 1) m.NAp = pl->NA[c];
      else if (rk == 2) m.NAp = pl->NAst;
      if (rk == 0) m.NA_out = pl->NA[c];
      else if (rk == 1) m.NA_out = pl->NAst;
      m.sa = pl->sa_startup[rk];
      m.sa_rec = pl->sg_rec;
      m.A_out = pl->AR[nw];
      m.XB = x_field(pl, 6);
      if ((st = launch_mhd(pl, m, s))) return st;
    }
    if (rec && rk < 2) {
      const size_t P = pl->d.P;
      JFB_CHECK_CUDA(cudaMemcpyAsync(rec[3 * rk], pl->U0[nw], (size_t)pl->d.nB * P * sizeof(c64),
                                     cudaMemcpyDeviceToDevice, s));
      JFB_CHECK_CUDA(cudaMemcpyAsync(rec[3 * rk + 1], pl->G[nw], (size_t)pl->d.nD * P * sizeof(c64),
                                     cudaMemcpyDeviceToDevice, s));
      JFB_CHECK_CUDA(cudaMemcpyAsync(rec[3 * rk + 2], pl->VW[nw], (size_t)pl->d.nD * sizeof(c64),
                                     cudaMemcpyDeviceToDevice, s));
    }
    st = launch_transforms(pl, s);
    if (st) return st;
  }
  return JFB_OK;
}

// One IMEXRK222 step from ring position m (channelflow_kmm.py:1137-1192,
// integrators/coupled.py:13-44): stage 1 solves
//   M u1 - g dt L u1 = M u^n + dt g N(u^n)
// into the ring slot m - 1 (no history is kept by this integrator), stage 2
//   M u' - g dt L u' = M u^n + dt (d N(u^n) + (1 - d) N(u1)) + dt (1 - g) L u1
// into slot m + 1; each stage is followed by the transforms of its result.
static int imexrk222_step(jfb_kmm_plan* pl, int64_t m, cudaStream_t s) {
  const int c = slot(m), t1 = slot(m - 1), nw = slot(m + 1);
  StageArgs a = blank_args();
  a.mode = kImplicit;
  a.HX = pl->HX;
  a.c0 = 1.0;
  a.d0 = kG222;
  a.u0a = pl->U0[c];
  a.ga = pl->G[c];
  a.vwa = pl->VW[c];
  a.Nu_out = pl->NU[c];
  a.Ng_out = pl->NG[c];
  a.NVW_out = pl->NVW[c];
  a.fac = packed(pl, pl->rk222);
  a.u0_out = pl->U0[t1];
  a.g_out = pl->G[t1];
  a.vw_out = pl->VW[t1];
  a.X = pl->X;
  int st = launch_implicit(pl, a, s);
  if (st || (st = launch_transforms(pl, s))) return st;
  StageArgs b = blank_args();
  b.mode = kImplicit;
  b.HX = pl->HX;
  b.c0 = 0.0;  // the linear term acts on u1 (level a), the mass on u^n (level b)
  b.c1 = 1.0;
  b.cL = (1.0 - kG222) * pl->cfg.dt;
  b.d0 = 1.0 - kD222;
  b.d1 = kD222;
  b.u0a = pl->U0[t1];
  b.ga = pl->G[t1];
  b.vwa = pl->VW[t1];
  b.u0b = pl->U0[c];
  b.gb = pl->G[c];
  b.vwb = pl->VW[c];
  b.Nup = pl->NU[c];
  b.Ngp = pl->NG[c];
  b.NVWp = pl->NVW[c];
  b.fac = packed(pl, pl->rk222);
  b.u0_out = pl->U0[nw];
  b.g_out = pl->G[nw];
  b.vw_out = pl->VW[nw];
  b.X = pl->X;
  if ((st = launch_implicit(pl, b, s))) return st;
  return launch_transforms(pl, s);
}

// One CNAB2 step from ring position m (channelflow_kmm.py:1071-1121,
// integrators/cnab2.py:211-240 with a fixed step, r = dt / previous_dt = 1):
//   (M - dt/2 L) u' = M u^n + dt/2 L u^n + dt N_ab,
//   N_ab = 3/2 N(u^n) - 1/2 N(u^(n-1)), or N(u^n) on the first step.
// N(u^n) goes into the ring slot of u^n, where the next step finds it as
// its previous nonlinear term.
static int cnab2_step(jfb_kmm_plan* pl, int64_t m, cudaStream_t s, bool have_old) {
  const int c = slot(m), o1 = slot(m - 1), nw = slot(m + 1);
  StageArgs a = blank_args();
  a.mode = kImplicit;
  a.HX = pl->HX;
  a.c0 = 1.0;
  a.cL = 0.5 * pl->cfg.dt;
  a.d0 = have_old ? 1.5 : 1.0;
  a.d1 = have_old ? -0.5 : 0.0;
  a.u0a = pl->U0[c];
  a.ga = pl->G[c];
  a.vwa = pl->VW[c];
  if (have_old) {
    a.Nup = pl->NU[o1];
    a.Ngp = pl->NG[o1];
    a.NVWp = pl->NVW[o1];
  }
  a.Nu_out = pl->NU[c];
  a.Ng_out = pl->NG[c];
  a.NVW_out = pl->NVW[c];
  a.fac = packed(pl, pl->cnab2);
  a.u0_out = pl->U0[nw];
  a.g_out = pl->G[nw];
  a.vw_out = pl->VW[nw];
  a.X = pl->X;
  const int st = launch_implicit(pl, a, s);
  if (st) return st;
  return launch_transforms(pl, s);
}

// One step of the plan's integrator once past the SBDF3 / CNAB2 startup (the
// body of the captured step graphs).
static int graph_step(jfb_kmm_plan* pl, int64_t m, cudaStream_t s) {
  switch (pl->cfg.time_integrator) {
    case JFB_INTEGRATOR_IMEXRK3: return startup_step(pl, s);
    case JFB_INTEGRATOR_IMEXRK222: return imexrk222_step(pl, m, s);
    case JFB_INTEGRATOR_CNAB2: return cnab2_step(pl, m, s, true);
    default: return steady_step(pl, m, s);
  }
}

static void destroy_graphs(jfb_kmm_plan* pl) {
  for (int k = 0; k < 3; ++k)
    if (pl->graph[k]) {
      cudaGraphExecDestroy(pl->graph[k]);
      pl->graph[k] = nullptr;
    }
}

}  // namespace jfb

using namespace jfb;

static int create_plan(const jfb_kmm_config* cfg, const jfb_mhd_params* mhd,
                       jfb_kmm_plan** out) {
  JFB_REQUIRE(cfg && out, "null pointer");
  *out = nullptr;
  JFB_REQUIRE(cfg->family == JFB_FAMILY_CHEBYSHEV || cfg->family == JFB_FAMILY_LEGENDRE,
              "family must be JFB_FAMILY_CHEBYSHEV or JFB_FAMILY_LEGENDRE");
  JFB_REQUIRE(cfg->nonlinear_form == JFB_NONLINEAR_ROTATIONAL ||
                  cfg->nonlinear_form == JFB_NONLINEAR_GRADIENT,
              "nonlinear_form must be JFB_NONLINEAR_ROTATIONAL or JFB_NONLINEAR_GRADIENT");
  JFB_REQUIRE(!mhd || (cfg->family == JFB_FAMILY_CHEBYSHEV &&
                       cfg->nonlinear_form == JFB_NONLINEAR_ROTATIONAL),
              "the MHD step is Chebyshev / rotational only");
  JFB_REQUIRE(cfg->precision == JFB_PRECISION_FP64 || cfg->precision == JFB_PRECISION_MIXED,
              "precision must be JFB_PRECISION_FP64 or JFB_PRECISION_MIXED");
  JFB_REQUIRE(cfg->time_integrator >= JFB_INTEGRATOR_SBDF3 &&
                  cfg->time_integrator <= JFB_INTEGRATOR_CNAB2,
              "time_integrator must be SBDF3, IMEXRK3, IMEXRK222 or CNAB2");
  JFB_REQUIRE(!mhd || cfg->time_integrator == JFB_INTEGRATOR_SBDF3,
              "the MHD step is SBDF3 (with its IMEXRK3 startup) only");
  JFB_REQUIRE(cfg->nx >= 9 && cfg->nx <= 64 * kMaxNR + 1, "nx out of range [9, 129]");
  JFB_REQUIRE(cfg->ny >= 4 && cfg->ny % 2 == 0 && cfg->nz >= 4 && cfg->nz % 2 == 0,
              "ny, nz must be even");
  JFB_REQUIRE(cfg->dt > 0 && cfg->nu > 0, "dt and nu must be positive");
  JFB_REQUIRE(cfg->x_hi > cfg->x_lo && cfg->ly > 0 && cfg->lz > 0, "bad domain");
  jfb_kmm_plan* pl = new jfb_kmm_plan();
  pl->cfg = *cfg;
  pl->mhd = mhd != nullptr;
  if (mhd) {
    pl->eta = mhd->eta;
    pl->mphys = MhdPhys{mhd->b0[0], mhd->b0[1], mhd->b0[2], 2.0 * mhd->omega, cfg->u_wall};
  }
  int st = JFB_OK;
  auto fail = [&](int code) {
    jfb_kmm_destroy(pl);
    return code;
  };
  build_host_operators(*cfg, pl->hop);
  Dims& d = pl->d;
  d.Nx = cfg->nx;
  d.nB = cfg->nx - 4;
  d.nD = cfg->nx - 2;
  d.Ny = cfg->ny;
  d.Nz = cfg->nz;
  d.Kz = cfg->nz / 2;
  d.P = d.Ny * d.Kz;
  d.My = std::max(cfg->ny, (int)(cfg->pad_y * cfg->ny));
  d.Mz = std::max(cfg->nz, (int)(cfg->pad_z * cfg->nz));
  d.nKb = ceil_div(d.Kz, kNW);
  d.dfx = pl->hop.dfx;
  d.dfy = pl->hop.dfy;
  d.dfz = pl->hop.dfz;
  d.Myz = (2.0 * M_PI / d.dfy) * (2.0 * M_PI / d.dfz);
  d.nu = cfg->nu;
  d.dt = cfg->dt;
  d.uwall = cfg->u_wall;
  d.family = cfg->family == JFB_FAMILY_LEGENDRE ? 1 : 0;
  d.grad = cfg->nonlinear_form == JFB_NONLINEAR_GRADIENT ? 1 : 0;
  if (!make_fft_plan(d.My, pl->fy) || !make_fft_plan(d.Mz, pl->fz)) {
    set_error("padded sizes must be of the form 2^a 3^b");
    return fail(JFB_ERR_ARG);
  }
  if (d.Mz < d.Nz || d.My < d.Ny) {
    set_error("padding must not truncate");
    return fail(JFB_ERR_ARG);
  }
  if ((st = dalloc(pl, (void**)&pl->status, sizeof(int)))) return fail(st);
  {
    // programmatic dependent launch of the step kernels: off unless
    // JFB200_PDL=1 (measured slower here: the plane kernel's early CTAs and
    // its clusters' placement stretch the transforms)
    const char* env = std::getenv("JFB200_PDL");
    pl->pdl = env && std::string(env) == "1";
  }
  // kz column chunk of the y transforms: two My x KC complex buffers <= 100 KB
  pl->KC = d.Kz;
  while ((size_t)2 * d.My * pl->KC * sizeof(c64) > 100 * 1024 && pl->KC % 2 == 0) pl->KC /= 2;
  pl->smem_y = (size_t)2 * d.My * pl->KC * sizeof(c64);
  pl->smem_z = (size_t)2 * d.Mz * kZRows * 3 * sizeof(c64);
  pl->smem_pencil = (size_t)(6 * d.Nx * kLDW + kNW * 6 * d.Nx + d.Nx) * sizeof(c64);
  pl->smem_zf = (size_t)2 * d.Nz * (kZRows / 2) * 3 * sizeof(c64);
  // warp-shuffle FFT paths (lengths 32 P, P in {2, 3, 4, 6}; Kz <= 64)
  pl->qk = ceil_div(d.Kz, 32);
  pl->py = warp_radix(d.My);
  pl->pz = (pl->qk <= 2) ? warp_radix(d.Mz) : 0;
  pl->pnz = (pl->qk <= 2) ? warp_radix(d.Nz) : 0;
  // kz columns per warp-FFT y block (two per warp; the last chunk may be partial)
  pl->KCw = std::min(16, d.Kz);
  pl->smem_yw_b = (size_t)(d.Ny + d.My) * (pl->KCw + 1) * sizeof(c64);
  pl->smem_yw_f = pl->smem_yw_b;
  // fused plane transforms: warp-FFT lengths 64 or 96 on both periodic axes,
  // Kz even and <= 32, and the plane buffers within one CTA pair
  pl->mixed = cfg->precision == JFB_PRECISION_MIXED;
  pl->smem_plane = plane_smem_bytes(d.My, d.Kz, pl->mixed ? sizeof(c32) : sizeof(c64));
  pl->plane = (pl->py == 2 || pl->py == 3) && (pl->pz == 2 || pl->pz == 3) && d.Kz % 2 == 0 &&
              d.Kz <= 32 && pl->smem_plane <= 227 * 1024 && !pl->mhd && !d.grad;
  // gradient form: nine fields backward in y (u_i, d/dx u_i, d/dy u_i), the
  // twelve-field z stage z_grad_kernel (shared-memory transforms)
  pl->smem_zg = (size_t)2 * d.Mz * kZRows * 6 * sizeof(c64);
  if (d.grad && (pl->smem_zg > 227 * 1024 ||
                 allow_smem((const void*)z_grad_kernel<double>) != cudaSuccess ||
                 allow_smem((const void*)z_grad_kernel<float>) != cudaSuccess)) {
    set_error("grid too large for the gradient-form z stage");
    return fail(JFB_ERR_ARG);
  }
  pl->plane_ok = pl->plane;
  {
    const char* ev = std::getenv("JFB200_TRANSFORMS");
    if (ev && std::string(ev) == "split") pl->plane = false;
  }
  if (pl->mhd) {
    // the coupled step transforms twelve fields with the shared-memory kernels
    pl->plane = false;
    pl->smem_mhd = mhd_smem_bytes(d.nD, d.Nx);
    pl->smem_zm = (size_t)2 * d.Mz * kZRows * 6 * sizeof(c64);
    if (pl->smem_mhd > 227 * 1024 || pl->smem_zm > 227 * 1024 || (d.nD + 1) / 2 > kMaxM) {
      set_error("grid too large for the MHD shared-memory tiling");
      return fail(JFB_ERR_ARG);
    }
    if (allow_smem((const void*)mhd_a_kernel) != cudaSuccess ||
        allow_smem((const void*)z_cross_mhd_kernel<double>) != cudaSuccess ||
        allow_smem((const void*)z_cross_mhd_kernel<float>) != cudaSuccess) {
      set_error("cannot configure the MHD kernels");
      return fail(JFB_ERR_CUDA);
    }
  }
  if (pl->plane) {
    auto attr = [&](const void* fn) { return allow_smem(fn); };
    if (attr((const void*)plane_cross_kernel<2, 2, 1, double>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<2, 3, 1, double>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<3, 2, 1, double>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<3, 3, 1, double>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<2, 2, 1, float>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<2, 3, 1, float>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<3, 2, 1, float>) != cudaSuccess ||
        attr((const void*)plane_cross_kernel<3, 3, 1, float>) != cudaSuccess) {
      set_error("cannot configure the plane transform kernel");
      return fail(JFB_ERR_CUDA);
    }
  }
  pl->smem_diag = (size_t)kNW * 4 * d.Nx * sizeof(c64) + 2 * kNW * sizeof(double);
  if (pl->smem_pencil > 227 * 1024 || pl->smem_y > 227 * 1024 || pl->smem_z > 227 * 1024) {
    set_error("grid too large for the shared-memory tiling");
    return fail(JFB_ERR_ARG);
  }
  allow_smem((const void*)pencil_stage_kernel<1, 0>);
  allow_smem((const void*)pencil_stage_kernel<2, 0>);
  allow_smem((const void*)pencil_stage_kernel<1, 1>);
  allow_smem((const void*)pencil_stage_kernel<2, 1>);
  for (const void* fn : {(const void*)y_backward_kernel<double>, (const void*)y_forward_kernel<double>,
                         (const void*)y_backward_kernel<float>, (const void*)y_forward_kernel<float>})
    allow_smem(fn);
  for (const void* fn : {(const void*)z_cross_kernel<double>, (const void*)z_cross_kernel<float>})
    allow_smem(fn);
  allow_smem((const void*)z_forward_real_kernel);
  allow_smem((const void*)diag_kernel);
#define JFB_YW_ATTR(P)                                                                   \
  for (const void* fn : {(const void*)y_backward_warp_kernel<P, double>,                  \
                         (const void*)y_forward_warp_kernel<P, double>,                   \
                         (const void*)y_backward_warp_kernel<P, float>,                   \
                         (const void*)y_forward_warp_kernel<P, float>})                   \
    allow_smem(fn);
  JFB_YW_ATTR(2)
  JFB_YW_ATTR(3)
  JFB_YW_ATTR(4)
  JFB_YW_ATTR(6)
#undef JFB_YW_ATTR
  JFB_CHECK_LAUNCH();

  // constant operators
  const HostOperators& op = pl->hop;
  double* p;
#define UP(field, vec)                       \
  st = upload(pl, &p, vec);                  \
  if (st) return fail(st);                   \
  pl->ops.field = p;
  UP(Q, op.Q);
  UP(V, op.V);
  {
    const int N = d.Nx, Jh = (N + 1) / 2, Jl = N / 2, Ne = (N + 1) / 2, No = N / 2;
    std::vector<double> VE((size_t)Jh * Ne), VO((size_t)Jh * std::max(1, No)),
        QE((size_t)Ne * Jh), QO((size_t)std::max(1, No) * std::max(1, Jl));
    for (int j = 0; j < Jh; ++j) {
      for (int m = 0; m < Ne; ++m) VE[(size_t)j * Ne + m] = op.V[(size_t)j * N + 2 * m];
      for (int m = 0; m < No; ++m) VO[(size_t)j * No + m] = op.V[(size_t)j * N + 2 * m + 1];
    }
    for (int m = 0; m < Ne; ++m)
      for (int j = 0; j < Jh; ++j) QE[(size_t)m * Jh + j] = op.Q[(size_t)(2 * m) * N + j];
    for (int m = 0; m < No; ++m)
      for (int j = 0; j < Jl; ++j) QO[(size_t)m * Jl + j] = op.Q[(size_t)(2 * m + 1) * N + j];
    UP(VE, VE);
    UP(VO, VO);
    UP(QE, QE);
    UP(QO, QO);
  }
  UP(ns, op.ns);
  UP(sB0, op.SB.s0);
  UP(sB2, op.SB.s2);
  UP(sB4, op.SB.s4);
  UP(mlo, op.mlo);
  UP(mdi, op.mdi);
  UP(mhi, op.mhi);
  std::vector<double> luu_inv(op.lu_u), bu0_inv(op.bu0);
  for (double& v : luu_inv) v = 1.0 / v;
  for (double& v : bu0_inv) v = 1.0 / v;
  UP(lul, op.lu_l);
  UP(luu, luu_inv);
  UP(xphys, op.xphys);
  UP(bl2, op.bl2);
  UP(bl4, op.bl4);
  UP(bu0, bu0_inv);
  UP(bu2, op.bu2);
  UP(bu4, op.bu4);
  UP(fejer, op.fejer);
#undef UP
  st = upload(pl, &pl->twy, twiddles(d.My));
  if (st) return fail(st);
  st = upload(pl, &pl->twz, twiddles(d.Mz));
  if (st) return fail(st);
  if (pl->mixed) {
    auto narrow = [](const std::vector<c64>& t) {
      std::vector<c32> o(t.size());
      for (size_t k = 0; k < t.size(); ++k) o[k] = cmk((float)t[k].re, (float)t[k].im);
      return o;
    };
    if ((st = upload(pl, &pl->twy32, narrow(twiddles(d.My))))) return fail(st);
    if ((st = upload(pl, &pl->twz32, narrow(twiddles(d.Mz))))) return fail(st);
  }
  if (!make_fft_plan(d.Ny, pl->fny) || !make_fft_plan(d.Nz, pl->fnz)) {
    set_error("ny, nz must be of the form 2^a 3^b");
    return fail(JFB_ERR_ARG);
  }
  st = upload(pl, &pl->twny, twiddles(d.Ny));
  if (st) return fail(st);
  st = upload(pl, &pl->twnz, twiddles(d.Nz));
  if (st) return fail(st);

  // tensor-core pencil stage: folded x-operators and its shared-memory plan
  // (JFB200_PENCIL=warp selects the warp-per-pencil kernel instead)
  {
    const int N = d.Nx, Jl = N / 2;
    const int nBe = (d.nB + 1) / 2, nBo = d.nB / 2, nDe = (d.nD + 1) / 2, nDo = d.nD / 2;
    GemmOps& G = pl->gops;
    std::memset(&G, 0, sizeof(G));
    // operand rows: three x-sample blocks (round4(N) + 4 rows each), the
    // mass-row inputs (three segments per parity), the right-hand sides
    const int hb = round4(N) + 4;
    G.oH[0] = 0;
    G.oH[1] = hb;
    G.oH[2] = 2 * hb;
    G.oMUE = 3 * hb;
    G.oMUO = G.oMUE + round4(3 * nBe);
    G.oMGE = G.oMUO + round4(3 * nBo);
    G.oMGO = G.oMGE + round4(3 * nDe);
    G.oRU = G.oMGO + round4(3 * nDo);
    G.oRG = G.oRU + d.nB;
    G.rows = G.oRG + d.nD;
    // velocity operands and the staged velocity operators reuse dead rows
    G.oUE = 0;
    G.oUO = round4(nBe);
    G.oGE = G.oUO + round4(nBo);
    G.oGO = G.oGE + round4(nDe);
    G.oVel = G.oGO + round4(nDo);
    G.oMean = G.rows * kGLd;
    G.oMid = G.oMean + 2 * N + 6 * d.nD;
    const size_t smem = ((size_t)G.oMid + (d.grad ? 6 : 5) * 2 * kGW) * sizeof(double);
    const char* env = std::getenv("JFB200_PENCIL");
    const bool want = !(env && std::string(env) == "warp");
    pl->gemm = smem <= 227 * 1024 && (d.nD + 1) / 2 <= kMaxM && Jl <= kMaxM;
    GemmHost gh;
    if (pl->gemm) {
      std::string err;
      if (!build_gemm_operators(pl->hop, gh, err, d.grad)) {
        set_error(err);
        return fail(JFB_ERR_ARG);
      }
      // unrolled k ranges and the staged velocity operators must fit
      bool fits = (size_t)G.oVel * kGLd + (gh.frag.size() - gh.off[gA0Ee]) <=
                  (size_t)G.oRU * kGLd;
      for (int k = 0; k < gNumSub && fits; ++k)
        for (int mt = 0; mt < gh.mt[k]; ++mt) {
          const int span = gh.krange[gh.kr[k] + 2 * mt + 1] - gh.krange[gh.kr[k] + 2 * mt];
          if ((k <= gNgO && span > kKtN) || (k >= gMuE && k <= gMgO && span > kKtM)) fits = false;
        }
      pl->gemm = fits;  // otherwise the warp-per-pencil kernel handles this size
    }
    pl->gemm_ok = pl->gemm;
    if (pl->gemm) {
      // kReplicas copies of the operators: CTA b reads copy b % kReplicas, so
      // the CTAs that all read every operator line do not queue on the same
      // L2 slices
      constexpr int kReplicas = 16;
      std::vector<double> rep((size_t)kReplicas * gh.frag.size());
      for (int r = 0; r < kReplicas; ++r)
        std::copy(gh.frag.begin(), gh.frag.end(), rep.begin() + (size_t)r * gh.frag.size());
      double *fr, *r3, *x2, *md;
      int* kr;
      if ((st = upload(pl, &fr, rep))) return fail(st);
      if ((st = upload(pl, &kr, gh.krange))) return fail(st);
      if ((st = upload(pl, &r3, gh.R3))) return fail(st);
      if ((st = upload(pl, &x2, gh.X2D))) return fail(st);
      if ((st = upload(pl, &md, gh.mid))) return fail(st);
      G.frag = fr;
      G.krange = kr;
      G.R3 = r3;
      G.X2D = x2;
      G.mid = md;
      G.status = pl->status;
      G.mid_stride = gh.mid_stride;
      G.nfrag = (int)gh.frag.size();
      G.nrep = kReplicas;
      for (int k = 0; k < gNumSub; ++k) G.sub[k] = SubDesc{gh.off[k], gh.mt[k], gh.kt[k], gh.kr[k]};
      G.Jh = gh.Jh;
      G.Jl = gh.Jl;
      G.nBe = gh.nBe;
      G.nBo = gh.nBo;
      G.nDe = gh.nDe;
      G.nDo = gh.nDo;
      G.kt_mu_lin[0] = ceil_div(2 * nBe, 4);
      G.kt_mu_lin[1] = ceil_div(2 * nBo, 4);
      G.kt_mg_lin[0] = ceil_div(nDe, 4);
      G.kt_mg_lin[1] = ceil_div(nDo, 4);
      pl->smem_gemm = smem;
      JFB_CHECK_CUDA(allow_smem((const void*)pencil_gemm_kernel<false, 0>));
      JFB_CHECK_CUDA(allow_smem((const void*)pencil_gemm_kernel<false, 1>));
      JFB_CHECK_CUDA(allow_smem((const void*)pencil_gemm_kernel<true, 0>));
      // mixed form, JFB200_TC=1: the velocity products on the tcgen05
      // tensor cores (split-BF16 operands, FP32 accumulation) when the
      // halves fit the 32-row quarters / 32-deep K blocks and the images fit
      // dead rows.  Off by default: measured slower than the FP64 DMMA
      // products here, and the FP32 accumulation raises the mixed form's
      // distance to FP64 about 30-fold (the base-flow terms are formed from
      // these velocities).
      const char* tce = std::getenv("JFB200_TC");
      const size_t oTA = (size_t)G.oVel * kGLd * sizeof(double);
      const size_t oTB = (size_t)G.oRU * kGLd * sizeof(double);
      const bool tc_fit = Jl <= 32 && nBe <= 32 && nBo <= 32 && nDe <= 32 && nDo <= 32 &&
                          oTA + kTcImgA <= oTB &&
                          oTB + kTcImgB <= (size_t)G.rows * kGLd * sizeof(double) &&
                          (size_t)10 * 32 * kTcStagePitch * sizeof(float) <= (size_t)kTcImgA;
      // (rotational form only: the tcgen05 epilogue forms u and omega)
      if (pl->mixed && tc_fit && !d.grad) {
        std::vector<unsigned char> img(kTcImgA, 0);
        auto bf16_bits = [](float f) -> uint16_t {  // round to nearest even
          uint32_t u;
          std::memcpy(&u, &f, 4);
          u += 0x7FFFu + ((u >> 16) & 1u);
          return (uint16_t)(u >> 16);
        };
        auto bf16_val = [](uint16_t h) -> double {
          const uint32_t u = (uint32_t)h << 16;
          float f;
          std::memcpy(&f, &u, 4);
          return (double)f;
        };
        const int Nn = d.Nx;
        // (group, quarter) -> (matrix N x n, coefficient parity, K offset in the group)
        struct Q {
          const std::vector<double>* M;
          int ncol, par, koff;
        };
        const Q qs[3][4] = {
            {{&gh.A0, d.nB, 0, 0}, {&gh.P2, d.nB, 0, 0}, {&gh.P1, d.nB, 0, 0}, {nullptr, 0, 0, 0}},
            {{&gh.P1, d.nB, 1, 0}, {&gh.A0, d.nB, 1, 0}, {&gh.P2, d.nB, 1, 0}, {nullptr, 0, 0, 0}},
            {{&gh.B1, d.nD, 0, 0}, {&gh.B2, d.nD, 0, 0}, {&gh.B2, d.nD, 1, 32}, {&gh.B1, d.nD, 1, 32}}};
        for (int g = 0; g < 3; ++g)
          for (int q = 0; q < 4; ++q) {
            const Q& e = qs[g][q];
            if (!e.M) continue;
            const int nh = e.par ? e.ncol / 2 : (e.ncol + 1) / 2;
            for (int r = 0; r < Jl; ++r)
              for (int k = 0; k < nh; ++k) {
                double v = (*e.M)[(size_t)r * e.ncol + 2 * k + e.par];
                for (int sp = 0; sp < 3; ++sp) {
                  const uint16_t h = bf16_bits((float)v);
                  v -= bf16_val(h);
                  const size_t o = (size_t)tc_a_off(g, sp) + tc_offset(32 * q + r, e.koff + k, tc_k(g));
                  std::memcpy(&img[o], &h, 2);
                }
              }
          }
        (void)Nn;
        unsigned char* dimg;
        if ((st = upload(pl, &dimg, img))) return fail(st);
        G.tc = (tce && std::string(tce) == "1") ? 1 : 0;
        G.vimg = dimg;
        G.oTA = (int)oTA;
        G.oTB = (int)oTB;
        pl->tc_ok = true;
      }
      // forward-elimination multipliers of the tile's modes, staged at the
      // start of phase C below the right-hand-side rows and above whatever
      // the velocity-operator copy of either variant writes
      {
        const size_t vel_end = std::max(
            oTA + (gh.frag.size() - (size_t)gh.off[gA0Ee]) * sizeof(double),
            pl->tc_ok ? oTA + (size_t)kTcImgA : (size_t)0);
        const size_t lbytes = (size_t)8 * 2 * (d.nB + d.nD) * sizeof(double);
        const size_t top = (size_t)G.oRU * kGLd * sizeof(double);
        G.oL = -1;
        if (top >= lbytes && (top - lbytes) / 16 * 16 >= vel_end)
          G.oL = (int)((top - lbytes) / 16 * 16 / sizeof(double));
      }
    }
    pl->gemm = pl->gemm_ok && want;
  }

  if (pl->mhd) {
    GemmHost gh;
    std::string err;
    if (!build_gemm_operators(pl->hop, gh, err)) {
      set_error(err);
      return fail(JFB_ERR_ARG);
    }
    MhdOps& M = pl->mops;
    double* q;
#define UPM(field, vec)                    \
    if ((st = upload(pl, &q, vec))) return fail(st); \
    M.field = q;
    UPM(R3, gh.R3);
    UPM(X2D, gh.X2D);
    UPM(B1, gh.B1);
    UPM(B2, gh.B2);
    UPM(C1, gh.C1);
    UPM(C2, gh.C2);
#undef UPM
    M.Jh = (d.Nx + 1) / 2;
    M.Jl = d.Nx / 2;
    M.nDe = (d.nD + 1) / 2;
    M.nDo = d.nD / 2;
  }

  // factors: steady SBDF3 and the three IMEXRK3 startup stages
  pl->n_modes = (d.Ny / 2) * d.Kz;
  pl->su_rec = packed_rec_size(d.nB);
  pl->sg_rec = packed_rec_size(d.nD);
  // records with the explicit inverses of the upper factors (both pencil kernels)
  st = build_factor_set(pl, kSBDF3Implicit * cfg->dt, pl->steady, cfg->nu, 0, 2, true);
  if (st) return fail(st);
  for (int rk = 0; rk < 3; ++rk) {
    st = build_factor_set(pl, (kRK3A[rk] + kRK3B[rk]) * cfg->dt / 2.0, pl->startup[rk],
                          cfg->nu, 0, 2, true);
    if (st) return fail(st);
  }
  if (cfg->time_integrator == JFB_INTEGRATOR_CNAB2) {
    // Crank-Nicolson implicit half: gamma = dt / 2 (channelflow_kmm.py:267-274)
    st = build_factor_set(pl, 0.5 * cfg->dt, pl->cnab2, cfg->nu, 0, 2, true);
    if (st) return fail(st);
  }
  if (cfg->time_integrator == JFB_INTEGRATOR_IMEXRK222) {
    st = build_factor_set(pl, kG222 * cfg->dt, pl->rk222, cfg->nu, 0, 2, true);
    if (st) return fail(st);
  }
  if (pl->mhd) {
    // SA = MA - gamma LA: the Sg structure with diffusivity eta
    FactorSet fs;
    st = build_factor_set(pl, kSBDF3Implicit * cfg->dt, fs, pl->eta, 1, 1, true);
    if (st) return fail(st);
    pl->sa_steady = fs.sg;
    for (int rk = 0; rk < 3; ++rk) {
      FactorSet fr;
      st = build_factor_set(pl, (kRK3A[rk] + kRK3B[rk]) * cfg->dt / 2.0, fr, pl->eta, 1, 1, true);
      if (st) return fail(st);
      pl->sa_startup[rk] = fr.sg;
    }
  }

  // state rings and work buffers
  const size_t P = d.P;
  auto cal = [&](c64** ptr, size_t elems) {
    return dalloc(pl, (void**)ptr, std::max<size_t>(1, elems) * sizeof(c64));
  };
  for (int k = 0; k < 3; ++k) {
    if ((st = cal(&pl->U0[k], (size_t)d.nB * P))) return fail(st);
    if ((st = cal(&pl->G[k], (size_t)d.nD * P))) return fail(st);
    if ((st = cal(&pl->NU[k], (size_t)d.nB * P))) return fail(st);
    if ((st = cal(&pl->NG[k], (size_t)d.nD * P))) return fail(st);
    if ((st = cal(&pl->VW[k], d.nD))) return fail(st);
    if ((st = cal(&pl->NVW[k], d.nD))) return fail(st);
  }
  if ((st = cal(&pl->NUst, (size_t)d.nB * P))) return fail(st);
  if ((st = cal(&pl->NGst, (size_t)d.nD * P))) return fail(st);
  if ((st = cal(&pl->NVWst, d.nD))) return fail(st);
  if ((st = cal(&pl->U1S, (size_t)d.nD * P))) return fail(st);
  if ((st = cal(&pl->U2S, (size_t)d.nD * P))) return fail(st);
  // X and Y exist only for the step: half size in the mixed form (complex64);
  // HZ and HX also serve the FP64 state_from_physical path
  // (the coupled MHD step: twelve x-physical fields u, omega, b, j and six
  // nonlinear fields n, emf)
  const size_t xs = pl->mixed ? 2 : 1;
  const size_t nxf = pl->mhd ? 12 : d.grad ? 9 : 6, nhf = pl->mhd ? 6 : 3;
  if ((st = cal(&pl->X, (nxf * d.Nx * P + xs - 1) / xs))) return fail(st);
  if ((st = cal(&pl->Y, (nxf * d.Nx * d.My * d.Kz + xs - 1) / xs))) return fail(st);
  if ((st = cal(&pl->HZ, nhf * d.Nx * d.My * d.Kz))) return fail(st);
  if ((st = cal(&pl->HX, nhf * d.Nx * P))) return fail(st);
  if (pl->mhd) {
    for (int k = 0; k < 3; ++k) {
      if ((st = cal(&pl->AR[k], (size_t)3 * d.nD * P))) return fail(st);
      if ((st = cal(&pl->NA[k], (size_t)3 * d.nD * P))) return fail(st);
    }
    if ((st = cal(&pl->NAst, (size_t)3 * d.nD * P))) return fail(st);
  }
  if ((st = cal(&pl->HD, (size_t)3 * d.nD * P))) return fail(st);
  pl->diag_blocks = d.Ny * d.nKb;
  if ((st = dalloc(pl, (void**)&pl->diag_partial, (size_t)2 * pl->diag_blocks * sizeof(double))))
    return fail(st);
  if ((st = dalloc(pl, (void**)&pl->diag_mean, (size_t)(8 + d.Nx) * sizeof(double))))
    return fail(st);
  if (pl->mhd &&
      (st = dalloc(pl, (void**)&pl->mdiag_partial, (size_t)2 * pl->diag_blocks * sizeof(double))))
    return fail(st);
  JFB_CHECK_CUDA(cudaDeviceSynchronize());
  *out = pl;
  return JFB_OK;
}

extern "C" int jfb_kmm_create(const jfb_kmm_config* cfg, jfb_kmm_plan** out) {
  return create_plan(cfg, nullptr, out);
}

extern "C" int jfb_mhd_create(const jfb_kmm_config* cfg, const jfb_mhd_params* prm,
                              jfb_kmm_plan** out) {
  JFB_REQUIRE(cfg && prm && out, "null pointer");
  *out = nullptr;
  JFB_REQUIRE(prm->eta > 0.0 && std::isfinite(prm->eta), "eta must be positive");
  JFB_REQUIRE(std::isfinite(prm->omega) && std::isfinite(prm->b0[0]) &&
                  std::isfinite(prm->b0[1]) && std::isfinite(prm->b0[2]),
              "omega and b0 must be finite");
  return create_plan(cfg, prm, out);
}

extern "C" int jfb_kmm_destroy(jfb_kmm_plan* pl) {
  if (!pl) return JFB_OK;
  destroy_graphs(pl);
  if (pl->cap) cudaStreamDestroy(pl->cap);
  for (void* ptr : pl->allocs) cudaFree(ptr);
  delete pl;
  return JFB_OK;
}

extern "C" int jfb_kmm_get_info(const jfb_kmm_plan* pl, jfb_kmm_info* info) {
  JFB_REQUIRE(pl && info, "null pointer");
  const Dims& d = pl->d;
  info->n_pencils = d.P;
  info->device_bytes = pl->device_bytes;
  info->launches_per_step = pl->mhd ? 5 : pl->plane ? 2 : 4;
  // stage model: 43 E_s + 18 E_m complex values, E_s = Nx Ny (Nz/2+1), E_m = Nx My (Nz/2+1)
  const int64_t H = d.Nz / 2 + 1;
  const int64_t Es = (int64_t)d.Nx * d.Ny * H, Em = (int64_t)d.Nx * d.My * H;
  info->algorithmic_bytes = (43 * Es + 18 * Em) * 16;
  info->my = d.My;
  info->mz = d.Mz;
  return JFB_OK;
}

extern "C" int jfb_kmm_set_state(jfb_kmm_plan* pl, const jfb_kmm_state* s, void* stream) {
  JFB_REQUIRE(pl && s && s->u0 && s->u1 && s->u2 && s->g, "null pointer");
  JFB_REQUIRE(s->history_steps >= 0 && s->history_steps <= 2, "history_steps in [0, 2]");
  cudaStream_t st = (cudaStream_t)stream;
  const Dims& d = pl->d;
  pl->n = 0;
  const int c = slot(0), o1 = slot(-1), o2 = slot(-2);
  const int blocks = 512;
  auto half = [&](const void* full, int n, c64* dst) {
    if (full) to_half_kernel<<<blocks, 256, 0, st>>>((const c64*)full, n, d.Ny, d.Nz, dst);
    else cudaMemsetAsync(dst, 0, (size_t)n * d.P * sizeof(c64), st);
  };
  half(s->u0, d.nB, pl->U0[c]);
  half(s->g, d.nD, pl->G[c]);
  half(s->u1, d.nD, pl->U1S);
  half(s->u2, d.nD, pl->U2S);
  means_in_kernel<<<1, 128, 0, st>>>((const c64*)s->u1, (const c64*)s->u2, d.nD, d.Ny, d.Nz,
                                     pl->VW[c]);
  const int lv[2] = {o1, o2};
  void* const* sol[2] = {s->solution_old, s->solution_older};
  void* const* nl[2] = {s->nonlinear_old, s->nonlinear_older};
  for (int k = 0; k < 2; ++k) {
    half(sol[k][0], d.nB, pl->U0[lv[k]]);
    half(sol[k][1], d.nD, pl->G[lv[k]]);
    real_pair_in_kernel<<<1, 128, 0, st>>>((const double*)sol[k][2],
                                           (const double*)sol[k][3], d.nD, pl->VW[lv[k]]);
    half(nl[k][0], d.nB, pl->NU[lv[k]]);
    half(nl[k][1], d.nD, pl->NG[lv[k]]);
    real_pair_in_kernel<<<1, 128, 0, st>>>((const double*)nl[k][2], (const double*)nl[k][3],
                                           d.nD, pl->NVW[lv[k]]);
  }
  JFB_CHECK_LAUNCH();
  pl->hist = (int)s->history_steps;
  pl->have_state = true;
  pl->have_H = false;
  pl->explicit_u12 = true;
  return JFB_OK;
}

extern "C" int jfb_kmm_get_state(jfb_kmm_plan* pl, const jfb_kmm_state* s, void* stream) {
  JFB_REQUIRE(pl && s, "null pointer");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const Dims& d = pl->d;
  int rc = ensure_explicit(pl, st);
  if (rc) return rc;
  const int c = slot(pl->n), o1 = slot(pl->n - 1), o2 = slot(pl->n - 2);
  const int blocks = 512;
  auto full = [&](const c64* src, int n, void* dst) {
    if (dst) to_full_kernel<<<blocks, 256, 0, st>>>(src, n, d.Ny, d.Nz, (c64*)dst);
  };
  full(pl->U0[c], d.nB, s->u0);
  full(pl->G[c], d.nD, s->g);
  full(pl->U1S, d.nD, s->u1);
  full(pl->U2S, d.nD, s->u2);
  const int lv[2] = {o1, o2};
  void* const* sol[2] = {s->solution_old, s->solution_older};
  void* const* nl[2] = {s->nonlinear_old, s->nonlinear_older};
  for (int k = 0; k < 2; ++k) {
    full(pl->U0[lv[k]], d.nB, sol[k][0]);
    full(pl->G[lv[k]], d.nD, sol[k][1]);
    real_pair_out_kernel<<<1, 128, 0, st>>>(pl->VW[lv[k]], d.nD, (double*)sol[k][2],
                                            (double*)sol[k][3]);
    full(pl->NU[lv[k]], d.nB, nl[k][0]);
    full(pl->NG[lv[k]], d.nD, nl[k][1]);
    real_pair_out_kernel<<<1, 128, 0, st>>>(pl->NVW[lv[k]], d.nD, (double*)nl[k][2],
                                            (double*)nl[k][3]);
  }
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_kmm_advance(jfb_kmm_plan* pl, int64_t steps, void* stream) {
  JFB_REQUIRE(pl, "null pointer");
  JFB_REQUIRE(steps >= 0, "steps must be >= 0");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_H(pl, s);
  if (st) return st;
  // SBDF3: IMEXRK3 startup steps until two history levels exist; the
  // one-step integrators keep no history
  while (steps > 0 && pl->hist < 2 && pl->cfg.time_integrator == JFB_INTEGRATOR_SBDF3) {
    st = startup_step(pl, s);
    if (st) return st;
    pl->n += 1;
    pl->hist += 1;
    pl->explicit_u12 = false;
    --steps;
  }
  // CNAB2: the first step without a previous nonlinear term (IMEX Euler on
  // the nonlinear part, cnab2.py:185-208); history_steps holds have_old
  while (steps > 0 && pl->hist < 1 && pl->cfg.time_integrator == JFB_INTEGRATOR_CNAB2) {
    st = cnab2_step(pl, pl->n, s, false);
    if (st) return st;
    pl->n += 1;
    pl->hist = 1;
    pl->explicit_u12 = false;
    --steps;
  }
  while (steps > 0) {
    const int k = slot(pl->n);
    if (!pl->graph[k]) {
      // Capture one step for ring phase k on the private stream; the
      // instantiated graph is then launched on the caller's stream (which
      // may be the legacy default stream, where capture is not allowed).
      if (!pl->cap) JFB_CHECK_CUDA(cudaStreamCreateWithFlags(&pl->cap, cudaStreamNonBlocking));
      cudaGraph_t g;
      JFB_CHECK_CUDA(cudaStreamBeginCapture(pl->cap, cudaStreamCaptureModeThreadLocal));
      st = graph_step(pl, pl->n, pl->cap);
      cudaError_t ec = cudaStreamEndCapture(pl->cap, &g);
      if (st) return st;
      JFB_CHECK_CUDA(ec);
      JFB_CHECK_CUDA(cudaGraphInstantiate(&pl->graph[k], g, 0));
      cudaGraphDestroy(g);
    }
    JFB_CHECK_CUDA(cudaGraphLaunch(pl->graph[k], s));
    pl->n += 1;
    pl->explicit_u12 = false;
    --steps;
  }
  return JFB_OK;
}

extern "C" int jfb_kmm_convection(jfb_kmm_plan* pl, void* h0, void* h1, void* h2,
                                  void* stream) {
  JFB_REQUIRE(pl && h0 && h1 && h2, "null pointer");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_H(pl, s);
  if (st) return st;
  StageArgs a = blank_args();
  a.mode = kHOnly;
  a.x32 = pl->mixed ? 1 : 0;
  a.Xlin = pl->mixed ? reinterpret_cast<const c32*>(pl->X) : nullptr;
  a.HX = pl->HX;
  a.Hd_out = pl->HD;
  st = launch_pencil(pl, a, s);
  if (st) return st;
  const Dims& d = pl->d;
  void* outs[3] = {h0, h1, h2};
  for (int f = 0; f < 3; ++f)
    to_full_kernel<<<512, 256, 0, s>>>(pl->HD + (size_t)f * d.nD * d.P, d.nD, d.Ny, d.Nz,
                                       (c64*)outs[f]);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_kmm_state_from_physical(jfb_kmm_plan* pl, const double* u0,
                                           const double* u1, const double* u2,
                                           void* stream) {
  JFB_REQUIRE(pl && u0 && u1 && u2, "null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  Dims d = pl->d;
  const size_t P = d.P;
  // z: real Nz -> Kz half spectrum (into HZ as [f][j][y][kz]), scaled 1/Nz
  if (pl->pnz) {
    switch (pl->pnz) {
      case 2: launch_zfwd_warp<2>(pl, u0, u1, u2, s); break;
      case 3: launch_zfwd_warp<3>(pl, u0, u1, u2, s); break;
      case 4: launch_zfwd_warp<4>(pl, u0, u1, u2, s); break;
      default: launch_zfwd_warp<6>(pl, u0, u1, u2, s); break;
    }
  } else {
    const int zb = ceil_div((int64_t)d.Nx * d.Ny, kZRows);
    z_forward_real_kernel<<<zb, 256, pl->smem_zf, s>>>(d, pl->fnz, pl->twnz, u0, u1, u2,
                                                       pl->HZ);
  }
  JFB_CHECK_LAUNCH();
  // y: forward FFT of length Ny (no truncation), scaled 1/Ny
  Dims dy = d;
  dy.My = d.Ny;
  int KC = d.Kz;
  while ((size_t)2 * d.Ny * KC * sizeof(c64) > 100 * 1024 && KC % 2 == 0) KC /= 2;
  dim3 gf(d.Nx, 3, d.Kz / KC);
  y_forward_kernel<double><<<gf, 256, (size_t)2 * d.Ny * KC * sizeof(c64), s>>>(dy, pl->fny, KC,
                                                                        pl->twny, pl->HZ,
                                                                        pl->HX, nullptr);
  JFB_CHECK_LAUNCH();
  // history reset and x: Shen forward transforms, g = i ky u2 - i kz u1
  pl->n = 0;
  for (int k = 0; k < 3; ++k) {
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->U0[k], 0, (size_t)d.nB * P * sizeof(c64), s));
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->G[k], 0, (size_t)d.nD * P * sizeof(c64), s));
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->NU[k], 0, (size_t)d.nB * P * sizeof(c64), s));
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->NG[k], 0, (size_t)d.nD * P * sizeof(c64), s));
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->VW[k], 0, (size_t)d.nD * sizeof(c64), s));
    JFB_CHECK_CUDA(cudaMemsetAsync(pl->NVW[k], 0, (size_t)d.nD * sizeof(c64), s));
    if (pl->mhd) {
      JFB_CHECK_CUDA(cudaMemsetAsync(pl->AR[k], 0, (size_t)3 * d.nD * P * sizeof(c64), s));
      JFB_CHECK_CUDA(cudaMemsetAsync(pl->NA[k], 0, (size_t)3 * d.nD * P * sizeof(c64), s));
    }
  }
  StageArgs a = blank_args();
  a.mode = kFromPhys;
  a.HX = pl->HX;
  const int c = slot(0);
  a.u0_out = pl->U0[c];
  a.g_out = pl->G[c];
  a.vw_out = pl->VW[c];
  a.u1_out = pl->U1S;
  a.u2_out = pl->U2S;
  int st = launch_pencil(pl, a, s);
  if (st) return st;
  pl->hist = 0;
  pl->have_state = true;
  pl->have_H = false;
  pl->explicit_u12 = true;
  return JFB_OK;
}

extern "C" int jfb_kmm_diagnostics(jfb_kmm_plan* pl, double* out, void* stream) {
  JFB_REQUIRE(pl && out, "null pointer");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_explicit(pl, s);
  if (st) return st;
  const Dims& d = pl->d;
  const int c = slot(pl->n);
  diag_kernel<<<pl->diag_blocks, kNW * 32, pl->smem_diag, s>>>(
      pl->ops, d, pl->U0[c], pl->U1S, pl->U2S, pl->diag_partial, pl->diag_mean);
  JFB_CHECK_LAUNCH();
  diag_finish_kernel<<<1, 32, 0, s>>>(d, pl->diag_partial, pl->diag_blocks, pl->diag_mean,
                                      pl->cfg.ly, pl->cfg.lz, pl->cfg.x_lo, pl->cfg.x_hi,
                                      out, pl->status);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_kmm_check(jfb_kmm_plan* pl, int32_t* flags, void* stream) {
  JFB_REQUIRE(pl, "null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  int word = 0;
  JFB_CHECK_CUDA(cudaMemcpyAsync(&word, pl->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  JFB_CHECK_CUDA(cudaMemsetAsync(pl->status, 0, sizeof(int), s));
  if (flags) *flags = word;
  if (word & kStatusNonFinite) {
    set_error("nonfinite solver state: a solved coefficient or diagnostic was NaN or infinite");
    return JFB_ERR_NONFINITE;
  }
  if (word & kStatusWaitTimeout) {
    set_error("a bounded device-side wait timed out; the step's results are invalid");
    return JFB_ERR_DEVICE;
  }
  return JFB_OK;
}

extern "C" int jfb_kmm_timed_steps(jfb_kmm_plan* pl, int64_t steps, void* flush_buf,
                                   int64_t flush_bytes, double* kernel_ms, double* step_ms,
                                   void* stream) {
  JFB_REQUIRE(pl && kernel_ms && step_ms, "null pointer");
  JFB_REQUIRE(pl->cfg.time_integrator == JFB_INTEGRATOR_SBDF3, "timed steps: SBDF3 plans");
  JFB_REQUIRE(steps >= 0, "steps must be >= 0");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_H(pl, s);
  if (st) return st;
  while (steps > 0 && pl->hist < 2) {  // startup steps are not timed
    st = startup_step(pl, s);
    if (st) return st;
    pl->n += 1;
    pl->hist += 1;
    pl->explicit_u12 = false;
  }
  cudaEvent_t ev[5];
  for (int k = 0; k < 5; ++k) JFB_CHECK_CUDA(cudaEventCreate(&ev[k]));
  for (int k = 0; k < 4; ++k) kernel_ms[k] = 0.0;
  *step_ms = 0.0;
  for (int64_t i = 0; i < steps; ++i) {
    if (flush_buf && flush_bytes > 0)
      JFB_CHECK_CUDA(cudaMemsetAsync(flush_buf, (int)(i & 0xff), (size_t)flush_bytes, s));
    const int64_t m = pl->n;
    // the four launches of steady_step, with an event after each
    JFB_CHECK_CUDA(cudaEventRecord(ev[0], s));
    st = steady_step_timed(pl, m, s, ev);
    if (st) return st;
    JFB_CHECK_CUDA(cudaEventSynchronize(ev[4]));
    float ms;
    for (int k = 0; k < 4; ++k) {
      JFB_CHECK_CUDA(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      kernel_ms[k] += ms;
    }
    JFB_CHECK_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[4]));
    *step_ms += ms;
    pl->n += 1;
    pl->explicit_u12 = false;
  }
  for (int k = 0; k < 5; ++k) cudaEventDestroy(ev[k]);
  return JFB_OK;
}

// ---------------------------------------------------------------------------
// MHD entry points
// ---------------------------------------------------------------------------

extern "C" int jfb_mhd_set_state(jfb_kmm_plan* pl, const jfb_mhd_state* s, void* stream) {
  JFB_REQUIRE(pl && s, "null pointer");
  JFB_REQUIRE(pl->mhd, "not an MHD plan");
  JFB_REQUIRE(s->A[0] && s->A[1] && s->A[2], "null pointer");
  int st = jfb_kmm_set_state(pl, &s->flow, stream);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const Dims& d = pl->d;
  const size_t comp = (size_t)d.nD * d.P;
  auto half3 = [&](void* const* full, c64* dst) {
    for (int k = 0; k < 3; ++k) {
      if (full && full[k])
        to_half_kernel<<<512, 256, 0, cs>>>((const c64*)full[k], d.nD, d.Ny, d.Nz, dst + k * comp);
      else
        cudaMemsetAsync(dst + k * comp, 0, comp * sizeof(c64), cs);
    }
  };
  half3(s->A, pl->AR[slot(0)]);
  half3(s->A_old, pl->AR[slot(-1)]);
  half3(s->A_older, pl->AR[slot(-2)]);
  half3(s->nonlinear_A_old, pl->NA[slot(-1)]);
  half3(s->nonlinear_A_older, pl->NA[slot(-2)]);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_mhd_get_state(jfb_kmm_plan* pl, const jfb_mhd_state* s, void* stream) {
  JFB_REQUIRE(pl && s, "null pointer");
  JFB_REQUIRE(pl->mhd, "not an MHD plan");
  int st = jfb_kmm_get_state(pl, &s->flow, stream);
  if (st) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const Dims& d = pl->d;
  const size_t comp = (size_t)d.nD * d.P;
  auto full3 = [&](const c64* src, void* const* dst) {
    for (int k = 0; k < 3; ++k)
      if (dst[k])
        to_full_kernel<<<512, 256, 0, cs>>>(src + k * comp, d.nD, d.Ny, d.Nz, (c64*)dst[k]);
  };
  full3(pl->AR[slot(pl->n)], s->A);
  full3(pl->AR[slot(pl->n - 1)], s->A_old);
  full3(pl->AR[slot(pl->n - 2)], s->A_older);
  full3(pl->NA[slot(pl->n - 1)], s->nonlinear_A_old);
  full3(pl->NA[slot(pl->n - 2)], s->nonlinear_A_older);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_mhd_potential_from_physical(jfb_kmm_plan* pl, const double* ax,
                                               const double* ay, const double* az, void* a0,
                                               void* a1, void* a2, void* stream) {
  JFB_REQUIRE(pl && ax && ay && az && a0 && a1 && a2, "null pointer");
  JFB_REQUIRE(pl->mhd, "not an MHD plan");
  cudaStream_t s = (cudaStream_t)stream;
  Dims d = pl->d;
  // z then y forward transforms of the three samples into HX (as in
  // jfb_kmm_state_from_physical); HX then no longer holds the state's H
  if (pl->pnz) {
    switch (pl->pnz) {
      case 2: launch_zfwd_warp<2>(pl, ax, ay, az, s); break;
      case 3: launch_zfwd_warp<3>(pl, ax, ay, az, s); break;
      case 4: launch_zfwd_warp<4>(pl, ax, ay, az, s); break;
      default: launch_zfwd_warp<6>(pl, ax, ay, az, s); break;
    }
  } else {
    const int zb = ceil_div((int64_t)d.Nx * d.Ny, kZRows);
    z_forward_real_kernel<<<zb, 256, pl->smem_zf, s>>>(d, pl->fnz, pl->twnz, ax, ay, az, pl->HZ);
  }
  JFB_CHECK_LAUNCH();
  Dims dy = d;
  dy.My = d.Ny;
  int KC = d.Kz;
  while ((size_t)2 * d.Ny * KC * sizeof(c64) > 100 * 1024 && KC % 2 == 0) KC /= 2;
  dim3 gf(d.Nx, 3, d.Kz / KC);
  y_forward_kernel<double><<<gf, 256, (size_t)2 * d.Ny * KC * sizeof(c64), s>>>(
      dy, pl->fny, KC, pl->twny, pl->HZ, pl->HX, nullptr);
  JFB_CHECK_LAUNCH();
  pl->have_H = false;
  MhdArgs m = blank_mhd();
  m.mode = kMhdFromPhys;
  m.HXA = pl->HX;
  m.A_out = pl->HD;
  int st = launch_mhd(pl, m, s);
  if (st) return st;
  void* outs[3] = {a0, a1, a2};
  for (int k = 0; k < 3; ++k)
    to_full_kernel<<<512, 256, 0, s>>>(pl->HD + (size_t)k * d.nD * d.P, d.nD, d.Ny, d.Nz,
                                       (c64*)outs[k]);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

extern "C" int jfb_mhd_convection(jfb_kmm_plan* pl, void* h0, void* h1, void* h2, void* ha0,
                                  void* ha1, void* ha2, void* stream) {
  JFB_REQUIRE(pl && h0 && h1 && h2 && ha0 && ha1 && ha2, "null pointer");
  JFB_REQUIRE(pl->mhd, "not an MHD plan");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  int st = ensure_H(pl, s);
  if (st) return st;
  const Dims& d = pl->d;
  void* outs[6] = {h0, h1, h2, ha0, ha1, ha2};
  for (int half = 0; half < 2; ++half) {
    StageArgs a = blank_args();
    a.mode = kHOnly;
    a.HX = hx_field(pl, 3 * half);
    a.Hd_out = pl->HD;
    // mixed form: complex64 nonlinear fields; the flow's base-flow terms are
    // added in FP64 from the x-physical u, omega (the EMF's are in HX)
    a.x32 = pl->mixed ? 1 : 0;
    a.Xlin = (pl->mixed && half == 0) ? reinterpret_cast<const c32*>(pl->X) : nullptr;
    if (half == 1) {  // the EMF's U_b e_y x B0 (mean mode; the step adds it in the A stage)
      a.emf_b0z = pl->mphys.uw_emf * pl->mphys.b0z;
      a.emf_b0x = pl->mphys.uw_emf * pl->mphys.b0x;
    }
    if ((st = launch_pencil(pl, a, s))) return st;
    for (int f = 0; f < 3; ++f)
      to_full_kernel<<<512, 256, 0, s>>>(pl->HD + (size_t)f * d.nD * d.P, d.nD, d.Ny, d.Nz,
                                         (c64*)outs[3 * half + f]);
    JFB_CHECK_LAUNCH();
  }
  return JFB_OK;
}

extern "C" int jfb_mhd_diagnostics(jfb_kmm_plan* pl, double* out, void* stream) {
  JFB_REQUIRE(pl && out, "null pointer");
  JFB_REQUIRE(pl->mhd, "not an MHD plan");
  int st = jfb_kmm_diagnostics(pl, out, stream);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const Dims& d = pl->d;
  mhd_diag_kernel<<<pl->diag_blocks, kNW * 32, 0, s>>>(pl->ops, d, pl->mops, pl->AR[slot(pl->n)],
                                                       pl->mdiag_partial);
  JFB_CHECK_LAUNCH();
  mhd_diag_finish_kernel<<<1, 32, 0, s>>>(pl->mdiag_partial, pl->diag_blocks, pl->cfg.ly,
                                          pl->cfg.lz, out + 8, pl->status);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

// ---------------------------------------------------------------------------
// Adjoint of the FP64 step: gain E(T)/E(0) and its gradient with respect to
// the initial state (perturbation_gain / gain_and_projected_gradient,
// examples/pcf_minimal_seed_jax.py:111-150, the gradient that jax.grad takes
// through KMM.solve).  State s = (u0, g, v00, w00) as in KMM.primary; the
// explicit initial leaves (u0, u1, u2, g) enter the first nonlinear term
// directly.  Reverse sweep over recomputed segments of `checkpoint` steps.
// ---------------------------------------------------------------------------

namespace jfb {

struct AState {
  c64 *u = nullptr, *g = nullptr, *v = nullptr, *w = nullptr;  // v, w: mean column only
};

struct AdjRun {
  std::vector<void*> mem;
  c64 *XF, *YF, *AH, *AW, *HZ6, *AX, *U1w, *U2w, *EU[3];
  AState S[4], Nn[4], MU, Z, NZ[3];
  int K = 0;
  c64 *TU0, *TG, *TVW;          // states of the segment being reversed, K + 1 slots
  c64* rec[2][6];               // stage states of the two startup steps
  c64 *IU0, *IU1, *IU2, *IG;    // explicit initial leaves
  std::vector<c64*> ck;         // checkpoints: rings + HX
  size_t ck_elems = 0;
  ~AdjRun() {
    for (void* p : mem) cudaFree(p);
  }
  int alloc(c64** p, size_t elems) {
    JFB_CHECK_CUDA(cudaMalloc((void**)p, std::max<size_t>(1, elems) * sizeof(c64)));
    JFB_CHECK_CUDA(cudaMemset(*p, 0, std::max<size_t>(1, elems) * sizeof(c64)));
    mem.push_back(*p);
    return JFB_OK;
  }
};

static int adj_prepare(jfb_kmm_plan* pl) {
  if (pl->adj_ready) return JFB_OK;
  const Dims& d = pl->d;
  GemmHost gh;
  std::string err;
  if (!build_gemm_operators(pl->hop, gh, err)) {
    set_error(err);
    return JFB_ERR_ARG;
  }
  AdjOps& A = pl->aops;
  const HostOperators& op = pl->hop;
  int st;
#define UPA(field, vec) \
  if ((st = upload(pl, &A.field, vec))) return st;
  UPA(A0, gh.A0);
  UPA(F, gh.F);
  UPA(R0, gh.R0);
  UPA(R1, gh.R1);
  UPA(R2, gh.R2);
  UPA(R3, gh.R3);
  UPA(B1, gh.B1);
  UPA(B2, gh.B2);
  UPA(GB, gh.GB);
  UPA(GD, gh.GD);
  UPA(XB0, op.XB0);
  UPA(XB2, op.XB2);
  UPA(XB4, op.XB4);
  UPA(XD0, op.XD0);
  UPA(XD2, op.XD2);
#undef UPA
  const double nu = pl->cfg.nu, dt = pl->cfg.dt;
  if ((st = build_factor_set(pl, kSBDF3Implicit * dt, pl->adj_steady, nu, 0, 2, false, true)))
    return st;
  for (int rk = 0; rk < 3; ++rk)
    if ((st = build_factor_set(pl, (kRK3A[rk] + kRK3B[rk]) * dt / 2.0, pl->adj_startup[rk], nu,
                               0, 2, false, true)))
      return st;
  pl->smem_za = (size_t)2 * d.Mz * kZRows * 5 * sizeof(c64);
  if (pl->smem_za > 227 * 1024) {
    set_error("grid too large for the adjoint z stage");
    return JFB_ERR_ARG;
  }
  JFB_CHECK_CUDA(allow_smem((const void*)z_adjoint_kernel));
  pl->adj_ready = true;
  return JFB_OK;
}

// -- term lists ---------------------------------------------------------------
static PTermList tlist(c64* dst, int rows, bool acc) {
  PTermList L;
  std::memset(&L, 0, sizeof(L));
  L.dst = dst;
  L.dst_rows = rows;
  L.accumulate = acc ? 1 : 0;
  return L;
}

static void term(PTermList& L, const c64* src, const double* mat, int src_rows, int trans,
                 double cre, double cim, int a = 0, int b = 0, int c = 0, int sel = 0,
                 int realpart = 0) {
  if (cre == 0.0 && cim == 0.0) return;
  PTerm& T = L.t[L.n++];
  T.src = src;
  T.mat = mat;
  T.src_rows = src_rows;
  T.trans = trans;
  T.cre = cre;
  T.cim = cim;
  T.a = a;
  T.b = b;
  T.c = c;
  T.sel = sel;
  T.realpart = realpart;
}

static int run(jfb_kmm_plan* pl, const PTermList& L, cudaStream_t s) {
  JFB_REQUIRE(L.n <= kMaxTerms, "term list too long");
  dim3 g(ceil_div(pl->d.P, 32), ceil_div(L.dst_rows, 8 * kTermRows));
  pencil_terms_kernel<<<g, 256, 0, s>>>(pl->d, L);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

#define JFB_RUN(L) \
  if ((st = run(pl, L, s))) return st;

// explicit adjoint (a_u0, a_u1, a_u2) = pro^H (adjoint of the six x-physical
// fields u, omega of the prologue map)
static int adj_pro(jfb_kmm_plan* pl, AdjRun& R, cudaStream_t s) {
  const Dims& d = pl->d;
  const AdjOps& A = pl->aops;
  const size_t f = (size_t)d.Nx * d.P;
  const c64* X = R.AX;
  const int N = d.Nx;
  int st;
  PTermList L = tlist(R.EU[0], d.nB, false);
  term(L, X + 0 * f, A.A0, N, 1, 1, 0);
  term(L, X + 4 * f, A.A0, N, 1, 0, -1, 0, 1);  // -i kz
  term(L, X + 5 * f, A.A0, N, 1, 0, 1, 1, 0);   // +i ky
  JFB_RUN(L);
  L = tlist(R.EU[1], d.nD, false);
  term(L, X + 1 * f, A.B1, N, 1, 1, 0);
  term(L, X + 3 * f, A.B1, N, 1, 0, 1, 0, 1);  // +i kz
  term(L, X + 5 * f, A.B2, N, 1, 1, 0);
  JFB_RUN(L);
  L = tlist(R.EU[2], d.nD, false);
  term(L, X + 2 * f, A.B1, N, 1, 1, 0);
  term(L, X + 3 * f, A.B1, N, 1, 0, -1, 1, 0);  // -i ky
  term(L, X + 4 * f, A.B2, N, 1, -1, 0);
  JFB_RUN(L);
  return JFB_OK;
}

// dst (+)= recon^H (EU): reconstruct_velocity (channelflow_kmm.py:855-870)
static int adj_recon(jfb_kmm_plan* pl, AdjRun& R, const AState& dst, bool acc, cudaStream_t s) {
  const Dims& d = pl->d;
  const AdjOps& A = pl->aops;
  int st;
  PTermList L = tlist(dst.u, d.nB, acc);
  term(L, R.EU[0], nullptr, d.nB, 0, 1, 0);
  term(L, R.EU[1], A.F, d.nD, 1, 0, -1, 1, 0, -1);  // -i ky / k^2
  term(L, R.EU[2], A.F, d.nD, 1, 0, -1, 0, 1, -1);  // -i kz / k^2
  JFB_RUN(L);
  L = tlist(dst.g, d.nD, acc);
  term(L, R.EU[1], nullptr, d.nD, 0, 0, -1, 0, 1, -1);  // -i kz / k^2
  term(L, R.EU[2], nullptr, d.nD, 0, 0, 1, 1, 0, -1);   // +i ky / k^2
  JFB_RUN(L);
  L = tlist(dst.v, d.nD, acc);
  term(L, R.EU[1], nullptr, d.nD, 0, 1, 0, 0, 0, 0, 2, 1);
  JFB_RUN(L);
  L = tlist(dst.w, d.nD, acc);
  term(L, R.EU[2], nullptr, d.nD, 0, 1, 0, 0, 0, 0, 2, 1);
  JFB_RUN(L);
  return JFB_OK;
}

// AH = R_n^H mu: adjoint of the nonlinear rows (channelflow_kmm.py:810-829)
static int adj_rows(jfb_kmm_plan* pl, AdjRun& R, const AState& mu, cudaStream_t s) {
  const Dims& d = pl->d;
  const AdjOps& A = pl->aops;
  const size_t f = (size_t)d.Nx * d.P;
  const double myz = d.Myz;
  int st;
  PTermList L = tlist(R.AH, d.Nx, false);
  term(L, mu.u, A.R0, d.nB, 1, myz, 0, 0, 0, 1);  // Myz k^2
  JFB_RUN(L);
  L = tlist(R.AH + f, d.Nx, false);
  term(L, mu.u, A.R1, d.nB, 1, 0, -myz, 1, 0);  // -i ky Myz
  term(L, mu.g, A.R2, d.nD, 1, 0, -myz, 0, 1);  // -i kz Myz
  term(L, mu.v, A.R3, d.nD, 1, -1, 0, 0, 0, 0, 2, 1);
  JFB_RUN(L);
  L = tlist(R.AH + 2 * f, d.Nx, false);
  term(L, mu.u, A.R1, d.nB, 1, 0, -myz, 0, 1);  // -i kz Myz
  term(L, mu.g, A.R2, d.nD, 1, 0, myz, 1, 0);   // +i ky Myz
  term(L, mu.w, A.R3, d.nD, 1, -1, 0, 0, 0, 0, 2, 1);
  JFB_RUN(L);
  return JFB_OK;
}

// dst += cm (M + gamma L)^T mu, gl = gamma nu (mass rows channelflow_kmm.py:261-409)
static int adj_mass(jfb_kmm_plan* pl, const AState& mu, double cm, double gl, const AState& dst,
                    cudaStream_t s) {
  const Dims& d = pl->d;
  const AdjOps& A = pl->aops;
  const double m = cm * d.Myz;
  int st;
  PTermList L = tlist(dst.u, d.nB, true);
  term(L, mu.u, A.XB0, d.nB, 1, -m, 0, 0, 0, 1);
  term(L, mu.u, A.XB0, d.nB, 1, m * gl, 0, 0, 0, 2);
  term(L, mu.u, A.XB2, d.nB, 1, m, 0);
  term(L, mu.u, A.XB2, d.nB, 1, -2.0 * m * gl, 0, 0, 0, 1);
  term(L, mu.u, A.XB4, d.nB, 1, m * gl, 0);
  JFB_RUN(L);
  L = tlist(dst.g, d.nD, true);
  term(L, mu.g, A.XD0, d.nD, 1, m, 0);
  term(L, mu.g, A.XD0, d.nD, 1, -m * gl, 0, 0, 0, 1);
  term(L, mu.g, A.XD2, d.nD, 1, m * gl, 0);
  JFB_RUN(L);
  for (int k = 0; k < 2; ++k) {
    c64* out = k ? dst.w : dst.v;
    const c64* in = k ? mu.w : mu.v;
    L = tlist(out, d.nD, true);
    term(L, in, A.XD0, d.nD, 1, cm, 0, 0, 0, 0, 2);
    term(L, in, A.XD2, d.nD, 1, cm * gl, 0, 0, 0, 0, 2);
    JFB_RUN(L);
  }
  return JFB_OK;
}

// dst = S^-T src with the kept factor bands
static int adj_solve(jfb_kmm_plan* pl, const FactorSet& fs, const AState& src, const AState& dst,
                     cudaStream_t s) {
  const Dims& d = pl->d;
  // a warp per pencil (kBandWarps pencils per block), the vector in shared memory
  const int blocks = ceil_div(d.P, kBandWarps);
  const size_t smB = (size_t)kBandWarps * d.nB * sizeof(c64), smD = (size_t)kBandWarps * d.nD * sizeof(c64);
  band_solve_t_warp_kernel<<<blocks, 32 * kBandWarps, smB, s>>>(d, fs.band[0], fs.bp[0], fs.bq[0],
                                                                d.nB, 0, src.u, dst.u);
  band_solve_t_warp_kernel<<<blocks, 32 * kBandWarps, smD, s>>>(d, fs.band[1], fs.bp[1], fs.bq[1],
                                                                d.nD, 0, src.g, dst.g);
  band_solve_t_warp_kernel<<<1, 32 * kBandWarps, smD, s>>>(d, fs.band[2], fs.bp[2], fs.bq[2], d.nD,
                                                           1, src.v, dst.v);
  band_solve_t_warp_kernel<<<1, 32 * kBandWarps, smD, s>>>(d, fs.band[2], fs.bp[2], fs.bq[2], d.nD,
                                                           1, src.w, dst.w);
  JFB_CHECK_LAUNCH();
  return JFB_OK;
}

static void astate_axpy(const jfb_kmm_plan* pl, const AState& y, const AState& x, double a,
                        cudaStream_t s) {
  const Dims& d = pl->d;
  const size_t P = d.P;
  axpy_kernel<<<256, 256, 0, s>>>(y.u, x.u, a, (size_t)d.nB * P);
  axpy_kernel<<<256, 256, 0, s>>>(y.g, x.g, a, (size_t)d.nD * P);
  axpy_kernel<<<64, 256, 0, s>>>(y.v, x.v, a, (size_t)d.nD * P);
  axpy_kernel<<<64, 256, 0, s>>>(y.w, x.w, a, (size_t)d.nD * P);
}

static int astate_zero(const jfb_kmm_plan* pl, const AState& y, cudaStream_t s) {
  const Dims& d = pl->d;
  const size_t P = d.P;
  JFB_CHECK_CUDA(cudaMemsetAsync(y.u, 0, (size_t)d.nB * P * sizeof(c64), s));
  JFB_CHECK_CUDA(cudaMemsetAsync(y.g, 0, (size_t)d.nD * P * sizeof(c64), s));
  JFB_CHECK_CUDA(cudaMemsetAsync(y.v, 0, (size_t)d.nD * P * sizeof(c64), s));
  JFB_CHECK_CUDA(cudaMemsetAsync(y.w, 0, (size_t)d.nD * P * sizeof(c64), s));
  return JFB_OK;
}

// EU = J^H mu at a linearisation point: the state (u0, g, vw) or, with u1
// and u2 given, the explicit velocity (u0, u1, u2).
static int adj_nonlinear(jfb_kmm_plan* pl, AdjRun& R, const c64* u0, const c64* g, const c64* vw,
                         const c64* u1, const c64* u2, const AState& mu, cudaStream_t s) {
  const Dims& d = pl->d;
  int st;
  if (!u1) {
    StageArgs a = blank_args();
    a.mode = kReconstruct;
    a.u0a = u0;
    a.ga = g;
    a.vwa = vw;
    a.X = R.U1w;
    a.Hd_out = R.U2w;
    if ((st = launch_pencil(pl, a, s))) return st;
    u1 = R.U1w;
    u2 = R.U2w;
  }
  StageArgs a = blank_args();
  a.mode = kPrologue;
  a.pu0 = u0;
  a.pu1 = u1;
  a.pu2 = u2;
  a.X = R.XF;
  if ((st = launch_pencil(pl, a, s))) return st;
  dim3 gy6(d.Nx, 6, d.Kz / pl->KC), gy3(d.Nx, 3, d.Kz / pl->KC);
  y_backward_kernel<double><<<gy6, 256, pl->smem_y, s>>>(d, pl->fy, pl->KC, pl->twy, R.XF, R.YF);
  JFB_CHECK_LAUNCH();
  if ((st = adj_rows(pl, R, mu, s))) return st;
  y_backward_kernel<double><<<gy3, 256, pl->smem_y, s>>>(d, pl->fy, pl->KC, pl->twy, R.AH, R.AW);
  JFB_CHECK_LAUNCH();
  const int zb = ceil_div((int64_t)d.Nx * d.My, kZRows);
  z_adjoint_kernel<<<zb, 256, pl->smem_za, s>>>(pl->ops, d, pl->fz, pl->twz, R.YF, R.AW, R.HZ6);
  JFB_CHECK_LAUNCH();
  y_forward_kernel<double><<<gy6, 256, pl->smem_y, s>>>(d, pl->fy, pl->KC, pl->twy, R.HZ6, R.AX,
                                                        nullptr);
  JFB_CHECK_LAUNCH();
  return adj_pro(pl, R, s);
}

// EU (+)= scale G u (gradient of the perturbation energy, 2 Ly Lz G u)
static int adj_energy(jfb_kmm_plan* pl, AdjRun& R, const c64* u0, const c64* u1, const c64* u2,
                      double scale, bool acc, cudaStream_t s) {
  const Dims& d = pl->d;
  const AdjOps& A = pl->aops;
  int st;
  PTermList L = tlist(R.EU[0], d.nB, acc);
  term(L, u0, A.GB, d.nB, 0, scale, 0);
  JFB_RUN(L);
  L = tlist(R.EU[1], d.nD, acc);
  term(L, u1, A.GD, d.nD, 0, scale, 0);
  JFB_RUN(L);
  L = tlist(R.EU[2], d.nD, acc);
  term(L, u2, A.GD, d.nD, 0, scale, 0);
  JFB_RUN(L);
  return JFB_OK;
}

static int perturbation_energy(jfb_kmm_plan* pl, double* dev8, cudaStream_t s, double* out) {
  int st = jfb_kmm_diagnostics(pl, dev8, s);
  if (st) return st;
  JFB_CHECK_CUDA(cudaMemcpyAsync(out, dev8, sizeof(double), cudaMemcpyDeviceToHost, s));
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  return JFB_OK;
}

// rings + HX of the plan <-> checkpoint buffer
static int checkpoint_io(jfb_kmm_plan* pl, c64* buf, bool save, cudaStream_t s) {
  const Dims& d = pl->d;
  const size_t P = d.P;
  size_t off = 0;
  auto io = [&](c64* arr, size_t n) -> int {
    if (save)
      JFB_CHECK_CUDA(cudaMemcpyAsync(buf + off, arr, n * sizeof(c64), cudaMemcpyDeviceToDevice, s));
    else
      JFB_CHECK_CUDA(cudaMemcpyAsync(arr, buf + off, n * sizeof(c64), cudaMemcpyDeviceToDevice, s));
    off += n;
    return JFB_OK;
  };
  int st;
  for (int k = 0; k < 3; ++k) {
    if ((st = io(pl->U0[k], (size_t)d.nB * P))) return st;
    if ((st = io(pl->G[k], (size_t)d.nD * P))) return st;
    if ((st = io(pl->VW[k], d.nD))) return st;
    if ((st = io(pl->NU[k], (size_t)d.nB * P))) return st;
    if ((st = io(pl->NG[k], (size_t)d.nD * P))) return st;
    if ((st = io(pl->NVW[k], d.nD))) return st;
  }
  return io(pl->HX, (size_t)3 * d.Nx * P);
}

static size_t checkpoint_elems(const jfb_kmm_plan* pl) {
  const Dims& d = pl->d;
  const size_t P = d.P;
  return 3 * (2 * (size_t)d.nB * P + 2 * (size_t)d.nD * P + 2 * (size_t)d.nD) +
         (size_t)3 * d.Nx * P;
}

// One forward step from ring position pl->n (startup while hist < 2),
// recording the startup stage states when rec is given.
static int forward_step(jfb_kmm_plan* pl, cudaStream_t s, c64* const* rec) {
  int st = (pl->hist < 2) ? startup_step(pl, s, rec) : steady_step(pl, pl->n, s);
  if (st) return st;
  pl->n += 1;
  if (pl->hist < 2) pl->hist += 1;
  pl->explicit_u12 = false;
  return JFB_OK;
}

static int record_state(jfb_kmm_plan* pl, AdjRun& R, int slot_idx, cudaStream_t s) {
  const Dims& d = pl->d;
  const size_t P = d.P;
  const int c = slot(pl->n);
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.TU0 + (size_t)slot_idx * d.nB * P, pl->U0[c],
                                 (size_t)d.nB * P * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.TG + (size_t)slot_idx * d.nD * P, pl->G[c],
                                 (size_t)d.nD * P * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.TVW + (size_t)slot_idx * d.nD, pl->VW[c], (size_t)d.nD * sizeof(c64),
                                 cudaMemcpyDeviceToDevice, s));
  return JFB_OK;
}

}  // namespace jfb

extern "C" int jfb_kmm_gain_gradient(jfb_kmm_plan* pl, const jfb_kmm_state* init, int64_t steps,
                                     int64_t checkpoint, double* gain_out,
                                     const jfb_kmm_state* grad, void* stream) {
  JFB_REQUIRE(pl && pl->cfg.time_integrator == JFB_INTEGRATOR_SBDF3,
              "the adjoint differentiates the SBDF3 step");
  JFB_REQUIRE(pl && init && gain_out, "null pointer");
  JFB_REQUIRE(!pl->mhd && !pl->mixed, "the adjoint runs on FP64 flow plans");
  JFB_REQUIRE(pl->d.family == 0 && !pl->d.grad,
              "the adjoint differentiates the Chebyshev rotational-form step");
  JFB_REQUIRE(steps >= 1, "steps must be >= 1");
  JFB_REQUIRE(init->history_steps == 0.0, "the initial state must have history_steps == 0");
  cudaStream_t s = (cudaStream_t)stream;
  const Dims& d = pl->d;
  const size_t P = d.P, nBP = (size_t)d.nB * P, nDP = (size_t)d.nD * P;
  const int64_t T = steps;
  const int K = (int)std::max<int64_t>(1, std::min<int64_t>(checkpoint > 0 ? checkpoint : T, T));
  int st = adj_prepare(pl);
  if (st) return st;
  // the initial state with a zero history
  jfb_kmm_state z = *init;
  for (int k = 0; k < 4; ++k)
    z.nonlinear_old[k] = z.nonlinear_older[k] = z.solution_old[k] = z.solution_older[k] = nullptr;
  if ((st = jfb_kmm_set_state(pl, &z, stream))) return st;

  AdjRun R;
  const size_t f = (size_t)d.Nx * P, fm = (size_t)d.Nx * d.My * d.Kz;
#define AL(p, n) \
  if ((st = R.alloc(&(p), (n)))) return st;
  AL(R.XF, 6 * f);
  AL(R.YF, 6 * fm);
  AL(R.AH, 3 * f);
  AL(R.AW, 3 * fm);
  AL(R.HZ6, 6 * fm);
  AL(R.AX, 6 * f);
  AL(R.U1w, nDP);
  AL(R.U2w, nDP);
  AL(R.EU[0], nBP);
  AL(R.EU[1], nDP);
  AL(R.EU[2], nDP);
  auto alloc_state = [&](AState& a) -> int {
    int e;
    if ((e = R.alloc(&a.u, nBP))) return e;
    if ((e = R.alloc(&a.g, nDP))) return e;
    if ((e = R.alloc(&a.v, nDP))) return e;
    return R.alloc(&a.w, nDP);
  };
  for (int k = 0; k < 4; ++k) {
    if ((st = alloc_state(R.S[k]))) return st;
    if ((st = alloc_state(R.Nn[k]))) return st;
  }
  if ((st = alloc_state(R.MU))) return st;
  if ((st = alloc_state(R.Z))) return st;
  for (int k = 0; k < 3; ++k)
    if ((st = alloc_state(R.NZ[k]))) return st;
  AL(R.TU0, (size_t)(K + 1) * nBP);
  AL(R.TG, (size_t)(K + 1) * nDP);
  AL(R.TVW, (size_t)(K + 1) * d.nD);
  for (int n = 0; n < 2; ++n)
    for (int z1 = 0; z1 < 2; ++z1) {
      AL(R.rec[n][3 * z1], nBP);
      AL(R.rec[n][3 * z1 + 1], nDP);
      AL(R.rec[n][3 * z1 + 2], (size_t)d.nD);
    }
  AL(R.IU0, nBP);
  AL(R.IU1, nDP);
  AL(R.IU2, nDP);
  AL(R.IG, nDP);
  const int nck = (int)((T + K - 1) / K);
  R.ck_elems = checkpoint_elems(pl);
  R.ck.resize(nck);
  for (int k = 0; k < nck; ++k) AL(R.ck[k], R.ck_elems);
  double* dev8 = nullptr;
  JFB_CHECK_CUDA(cudaMalloc((void**)&dev8, 10 * sizeof(double)));
  R.mem.push_back(dev8);
#undef AL

  // explicit initial leaves and E(0)
  const int c0 = slot(0);
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.IU0, pl->U0[c0], nBP * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.IG, pl->G[c0], nDP * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.IU1, pl->U1S, nDP * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  JFB_CHECK_CUDA(cudaMemcpyAsync(R.IU2, pl->U2S, nDP * sizeof(c64), cudaMemcpyDeviceToDevice, s));
  double E0 = 0.0, ET = 0.0;
  if ((st = perturbation_energy(pl, dev8, s, &E0))) return st;
  JFB_REQUIRE(std::isfinite(E0) && E0 > 0.0, "initial energy must be positive");
  if ((st = ensure_H(pl, s))) return st;

  // forward sweep with checkpoints
  for (int64_t m = 0; m < T; ++m) {
    if (m % K == 0) {
      if ((st = checkpoint_io(pl, R.ck[m / K], true, s))) return st;
    }
    if ((st = forward_step(pl, s, nullptr))) return st;
  }
  if ((st = perturbation_energy(pl, dev8, s, &ET))) return st;
  const double gain = ET / E0;
  *gain_out = gain;
  if (!grad) return JFB_OK;

  // terminal adjoint: grad of E(T) / E(0) through the reconstruction of u(T)
  const double area = pl->cfg.ly * pl->cfg.lz;
  for (int k = 0; k < 4; ++k) {
    if ((st = astate_zero(pl, R.S[k], s))) return st;
    if ((st = astate_zero(pl, R.Nn[k], s))) return st;
  }
  {
    const int cT = slot(pl->n);
    if ((st = adj_energy(pl, R, pl->U0[cT], pl->U1S, pl->U2S, 2.0 * area / E0, false, s)))
      return st;
    if ((st = adj_recon(pl, R, R.S[T % 4], false, s))) return st;
  }
  const double dt = pl->cfg.dt;
  const double cS[3] = {18.0 / 11.0, -9.0 / 11.0, 2.0 / 11.0};
  const double dS[3] = {18.0 / 11.0, -18.0 / 11.0, 6.0 / 11.0};
  auto ring = [](int64_t i) { return (int)(((i % 4) + 4) % 4); };
  for (int seg = nck - 1; seg >= 0; --seg) {
    const int64_t a = (int64_t)seg * K, b = std::min<int64_t>(T, a + K);
    // recompute s_a .. s_b
    if ((st = checkpoint_io(pl, R.ck[seg], false, s))) return st;
    pl->n = a;
    pl->hist = (int)std::min<int64_t>(2, a);
    pl->have_H = true;
    pl->explicit_u12 = false;
    if ((st = record_state(pl, R, 0, s))) return st;
    for (int64_t m = a; m < b; ++m) {
      c64* const* rec = (m < 2) ? R.rec[m] : nullptr;
      if ((st = forward_step(pl, s, rec))) return st;
      if ((st = record_state(pl, R, (int)(m + 1 - a), s))) return st;
    }
    auto su0 = [&](int64_t m) { return R.TU0 + (size_t)(m - a) * nBP; };
    auto sg = [&](int64_t m) { return R.TG + (size_t)(m - a) * nDP; };
    auto svw = [&](int64_t m) { return R.TVW + (size_t)(m - a) * d.nD; };
    for (int64_t n = b - 1; n >= a; --n) {
      // the nonlinear term of s_{n+1} is complete: fold it into its state adjoint
      if (n + 1 <= T - 1) {
        if ((st = adj_nonlinear(pl, R, su0(n + 1), sg(n + 1), svw(n + 1), nullptr, nullptr,
                                R.Nn[ring(n + 1)], s)))
          return st;
        if ((st = adj_recon(pl, R, R.S[ring(n + 1)], true, s))) return st;
      }
      if (n >= 2) {
        if ((st = adj_solve(pl, pl->adj_steady, R.S[ring(n + 1)], R.MU, s))) return st;
        for (int l = 0; l < 3; ++l) {
          if ((st = adj_mass(pl, R.MU, cS[l], 0.0, R.S[ring(n - l)], s))) return st;
          astate_axpy(pl, R.Nn[ring(n - l)], R.MU, dt * dS[l], s);
        }
      } else {
        // IMEXRK3 startup step from s_n: stage states z0 = s_n, z1, z2 (rec)
        JFB_CHECK_CUDA(cudaMemcpyAsync(R.Z.u, R.S[ring(n + 1)].u, nBP * sizeof(c64),
                                       cudaMemcpyDeviceToDevice, s));
        JFB_CHECK_CUDA(cudaMemcpyAsync(R.Z.g, R.S[ring(n + 1)].g, nDP * sizeof(c64),
                                       cudaMemcpyDeviceToDevice, s));
        JFB_CHECK_CUDA(cudaMemcpyAsync(R.Z.v, R.S[ring(n + 1)].v, nDP * sizeof(c64),
                                       cudaMemcpyDeviceToDevice, s));
        JFB_CHECK_CUDA(cudaMemcpyAsync(R.Z.w, R.S[ring(n + 1)].w, nDP * sizeof(c64),
                                       cudaMemcpyDeviceToDevice, s));
        for (int k = 0; k < 3; ++k)
          if ((st = astate_zero(pl, R.NZ[k], s))) return st;
        for (int rk = 2; rk >= 0; --rk) {
          const double gl = (kRK3A[rk] + kRK3B[rk]) * dt / 2.0 * pl->cfg.nu;
          if ((st = adj_solve(pl, pl->adj_startup[rk], R.Z, R.MU, s))) return st;
          if ((st = astate_zero(pl, R.Z, s))) return st;
          if ((st = adj_mass(pl, R.MU, 1.0, gl, R.Z, s))) return st;
          astate_axpy(pl, R.NZ[rk], R.MU, dt * kRK3A[rk], s);
          if (rk > 0) astate_axpy(pl, R.NZ[rk - 1], R.MU, dt * kRK3B[rk], s);
          if (rk > 0) {
            // the stage state's own nonlinear term is complete
            c64* const* z = R.rec[n] + 3 * (rk - 1);
            if ((st = adj_nonlinear(pl, R, z[0], z[1], z[2], nullptr, nullptr, R.NZ[rk], s)))
              return st;
            if ((st = adj_recon(pl, R, R.Z, true, s))) return st;
          }
        }
        astate_axpy(pl, R.S[ring(n)], R.Z, 1.0, s);
        astate_axpy(pl, R.Nn[ring(n)], R.NZ[0], 1.0, s);
      }
      // index n + 1 is finished; its ring slot serves index n - 3 next
      if ((st = astate_zero(pl, R.S[ring(n + 1)], s))) return st;
      if ((st = astate_zero(pl, R.Nn[ring(n + 1)], s))) return st;
    }
  }
  // explicit leaves: the first nonlinear term (explicit velocity) ...
  if ((st = adj_nonlinear(pl, R, R.IU0, R.IG, nullptr, R.IU1, R.IU2, R.Nn[ring(0)], s))) return st;
  // ... minus gain * grad E(0) / E(0) ...
  if ((st = adj_energy(pl, R, R.IU0, R.IU1, R.IU2, -2.0 * area * gain / E0, true, s))) return st;
  // ... plus the primary-state adjoint: u0, g, and the means of u1, u2
  const AState& S0 = R.S[ring(0)];
  axpy_kernel<<<256, 256, 0, s>>>(R.EU[0], S0.u, 1.0, nBP);
  {
    PTermList L = tlist(R.EU[1], d.nD, true);
    term(L, S0.v, nullptr, d.nD, 0, 1, 0, 0, 0, 0, 2, 1);
    if ((st = run(pl, L, s))) return st;
    L = tlist(R.EU[2], d.nD, true);
    term(L, S0.w, nullptr, d.nD, 0, 1, 0, 0, 0, 0, 2, 1);
    if ((st = run(pl, L, s))) return st;
  }
  JFB_CHECK_LAUNCH();
  // jax.grad convention (directional derivative Re sum(g d)): conjugate
  const c64* outs_half[4] = {R.EU[0], R.EU[1], R.EU[2], S0.g};
  void* outs[4] = {grad->u0, grad->u1, grad->u2, grad->g};
  const int rows[4] = {d.nB, d.nD, d.nD, d.nD};
  for (int k = 0; k < 4; ++k) {
    if (!outs[k]) continue;
    to_full_kernel<<<512, 256, 0, s>>>(outs_half[k], rows[k], d.Ny, d.Nz, (c64*)outs[k]);
    conj_kernel<<<512, 256, 0, s>>>((c64*)outs[k], (size_t)rows[k] * d.Ny * d.Nz);
  }
  for (int k = 0; k < 4; ++k) {
    void* const lv[4] = {grad->nonlinear_old[k], grad->nonlinear_older[k], grad->solution_old[k],
                         grad->solution_older[k]};
    const size_t bytes = (k < 2) ? (size_t)rows[k == 0 ? 0 : 3] * d.Ny * d.Nz * sizeof(c64)
                                 : (size_t)d.nD * sizeof(double);
    for (void* p : lv)
      if (p) JFB_CHECK_CUDA(cudaMemsetAsync(p, 0, bytes, s));
  }
  JFB_CHECK_LAUNCH();
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  pl->have_state = false;  // the plan's state was consumed by the sweep
  return JFB_OK;
}

extern "C" int jfb_kmm_energy_gradient(jfb_kmm_plan* pl, const jfb_kmm_state* state,
                                       const jfb_kmm_state* grad, void* stream) {
  JFB_REQUIRE(pl && state && grad && grad->u0 && grad->u1 && grad->u2, "null pointer");
  JFB_REQUIRE(!pl->mhd, "flow plans only");
  int st = adj_prepare(pl);
  if (st) return st;
  jfb_kmm_state z = *state;
  for (int k = 0; k < 4; ++k)
    z.nonlinear_old[k] = z.nonlinear_older[k] = z.solution_old[k] = z.solution_older[k] = nullptr;
  z.history_steps = 0.0;
  if ((st = jfb_kmm_set_state(pl, &z, stream))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const Dims& d = pl->d;
  AdjRun R;
  const size_t P = d.P;
  if ((st = R.alloc(&R.EU[0], (size_t)d.nB * P))) return st;
  if ((st = R.alloc(&R.EU[1], (size_t)d.nD * P))) return st;
  if ((st = R.alloc(&R.EU[2], (size_t)d.nD * P))) return st;
  const double area = pl->cfg.ly * pl->cfg.lz;
  if ((st = adj_energy(pl, R, pl->U0[slot(0)], pl->U1S, pl->U2S, 2.0 * area, false, s))) return st;
  void* outs[3] = {grad->u0, grad->u1, grad->u2};
  const int rows[3] = {d.nB, d.nD, d.nD};
  for (int k = 0; k < 3; ++k) {
    to_full_kernel<<<512, 256, 0, s>>>(R.EU[k], rows[k], d.Ny, d.Nz, (c64*)outs[k]);
    conj_kernel<<<512, 256, 0, s>>>((c64*)outs[k], (size_t)rows[k] * d.Ny * d.Nz);
  }
  if (grad->g) JFB_CHECK_CUDA(cudaMemsetAsync(grad->g, 0, (size_t)d.nD * d.Ny * d.Nz * sizeof(c64), s));
  JFB_CHECK_LAUNCH();
  JFB_CHECK_CUDA(cudaStreamSynchronize(s));
  return JFB_OK;
}

// ---------------------------------------------------------------------------
// Ensembles: independent members (any mix of flow / MHD plans and sizes)
// advanced together, one CUDA graph per steady step holding every member's
// step on its own stream (fork / join inside the capture), so members of
// uneven wall-normal size run concurrently.
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Kernel variants and their autotuner
// ---------------------------------------------------------------------------

extern "C" int jfb_kmm_get_variant(const jfb_kmm_plan* pl, jfb_kmm_variant* cur,
                                   jfb_kmm_variant* avail) {
  JFB_REQUIRE(pl, "null pointer");
  if (cur) {
    cur->pencil = pl->gemm ? 1 : 0;
    cur->transforms = pl->plane ? 1 : 0;
    cur->tc_velocity = pl->gops.tc;
    cur->pdl = pl->pdl ? 1 : 0;
    cur->replicas = pl->gemm_ok ? pl->gops.nrep : 0;
  }
  if (avail) {  // the largest value each field accepts
    avail->pencil = pl->gemm_ok ? 1 : 0;
    avail->transforms = pl->plane_ok ? 1 : 0;
    avail->tc_velocity = pl->tc_ok ? 1 : 0;
    avail->pdl = pl->mhd ? 0 : 1;
    avail->replicas = pl->gemm_ok ? 16 : 0;
  }
  return JFB_OK;
}

extern "C" int jfb_kmm_set_variant(jfb_kmm_plan* pl, const jfb_kmm_variant* v) {
  JFB_REQUIRE(pl && v, "null pointer");
  JFB_REQUIRE(v->pencil == 0 || (v->pencil == 1 && pl->gemm_ok), "pencil variant unavailable");
  JFB_REQUIRE(v->transforms == 0 || (v->transforms == 1 && pl->plane_ok),
              "fused plane transforms unavailable for this grid");
  JFB_REQUIRE(v->tc_velocity == 0 || (v->tc_velocity == 1 && pl->tc_ok && v->pencil == 1),
              "tensor-core velocity products need the mixed form and the tensor-core pencil stage");
  JFB_REQUIRE(v->pdl == 0 || (v->pdl == 1 && !pl->mhd), "bad pdl flag");
  JFB_REQUIRE(!pl->gemm_ok || (v->replicas >= 1 && v->replicas <= 16),
              "replicas must be in [1, 16]");
  destroy_graphs(pl);  // the captured steps hold the previous variant
  pl->gemm = v->pencil == 1;
  pl->plane = v->transforms == 1;
  pl->gops.tc = v->tc_velocity;
  pl->pdl = v->pdl == 1;
  if (pl->gemm_ok) pl->gops.nrep = v->replicas;
  return JFB_OK;
}

extern "C" int jfb_kmm_autotune(jfb_kmm_plan* pl, int64_t steps, jfb_kmm_variant* best,
                                double* best_ms, void* stream) {
  JFB_REQUIRE(pl && best && best_ms, "null pointer");
  JFB_REQUIRE(steps >= 1 && steps <= 10000, "steps must be in [1, 10000]");
  JFB_REQUIRE(!pl->mhd, "the autotuner covers flow plans");
  if (!pl->have_state) {
    set_error("no state loaded");
    return JFB_ERR_STATE;
  }
  cudaStream_t s = (cudaStream_t)stream;
  // keep the loaded state: every trial starts from a copy of it
  const size_t ne = checkpoint_elems(pl);
  c64 *save = nullptr, *x_save = nullptr;
  // X: six x-physical fields, complex64 (half the c64 count) in the mixed form
  const size_t nx = ((size_t)(pl->d.grad ? 9 : 6) * pl->d.Nx * pl->d.P + (pl->mixed ? 1 : 0)) /
                    (pl->mixed ? 2 : 1);
  JFB_CHECK_CUDA(cudaMalloc((void**)&save, ne * sizeof(c64)));
  cudaError_t ce = cudaMalloc((void**)&x_save, (nx + 2 * (size_t)pl->d.nD * pl->d.P) * sizeof(c64));
  if (ce != cudaSuccess) {
    cudaFree(save);
    JFB_CHECK_CUDA(ce);
  }
  const int64_t n0 = pl->n;
  const int hist0 = pl->hist;
  const bool haveH0 = pl->have_H, expl0 = pl->explicit_u12;
  jfb_kmm_variant start;
  jfb_kmm_get_variant(pl, &start, nullptr);
  auto restore = [&]() -> int {
    int st = checkpoint_io(pl, save, false, s);
    if (st) return st;
    JFB_CHECK_CUDA(cudaMemcpyAsync(pl->X, x_save, nx * sizeof(c64), cudaMemcpyDeviceToDevice, s));
    JFB_CHECK_CUDA(cudaMemcpyAsync(pl->U1S, x_save + nx, (size_t)pl->d.nD * pl->d.P * sizeof(c64),
                                   cudaMemcpyDeviceToDevice, s));
    JFB_CHECK_CUDA(cudaMemcpyAsync(pl->U2S, x_save + nx + (size_t)pl->d.nD * pl->d.P,
                                   (size_t)pl->d.nD * pl->d.P * sizeof(c64),
                                   cudaMemcpyDeviceToDevice, s));
    pl->n = n0;
    pl->hist = hist0;
    pl->have_H = haveH0;
    pl->explicit_u12 = expl0;
    return JFB_OK;
  };
  int st = checkpoint_io(pl, save, true, s);
  if (!st) {
    cudaError_t e = cudaMemcpyAsync(x_save, pl->X, nx * sizeof(c64), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(x_save + nx, pl->U1S, (size_t)pl->d.nD * pl->d.P * sizeof(c64),
                          cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(x_save + nx + (size_t)pl->d.nD * pl->d.P, pl->U2S,
                          (size_t)pl->d.nD * pl->d.P * sizeof(c64), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
      set_error(std::string("autotune save: ") + cudaGetErrorString(e));
      st = JFB_ERR_CUDA;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!st && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) {
    set_error("autotune: cudaEventCreate failed");
    st = JFB_ERR_CUDA;
  }
  double bms = 1e300;
  jfb_kmm_variant bv = start;
  jfb_kmm_variant avail;
  jfb_kmm_get_variant(pl, nullptr, &avail);
  const int reps[3] = {4, 8, 16};
  for (int pc = avail.pencil; pc >= 0 && !st; --pc)
    for (int tr = avail.transforms; tr >= 0 && !st; --tr)
      for (int tc = (pc ? start.tc_velocity : 0); tc >= (pc ? start.tc_velocity : 0) && !st; --tc)
        for (int pdl = 0; pdl <= avail.pdl && !st; ++pdl)
          for (int ri = 0; ri < (pc ? 3 : 1) && !st; ++ri) {
            jfb_kmm_variant v;
            v.pencil = pc;
            v.transforms = tr;
            v.tc_velocity = tc;
            v.pdl = pdl;
            v.replicas = pl->gemm_ok ? (pc ? reps[ri] : start.replicas) : 0;
            if ((st = jfb_kmm_set_variant(pl, &v))) break;
            if ((st = restore())) break;
            if ((st = jfb_kmm_advance(pl, 5, stream))) break;  // startup, capture, warm-up
            if (cudaEventRecord(e0, s) != cudaSuccess) st = JFB_ERR_CUDA;
            if (!st) st = jfb_kmm_advance(pl, steps, stream);
            if (!st && cudaEventRecord(e1, s) != cudaSuccess) st = JFB_ERR_CUDA;
            float ms = 0.0f;
            if (!st && (cudaEventSynchronize(e1) != cudaSuccess ||
                        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
              st = JFB_ERR_CUDA;
            if (st) {
              if (st == JFB_ERR_CUDA) set_error("autotune: timing failed");
              break;
            }
            const double per = (double)ms / (double)steps;
            if (per < bms) {
              bms = per;
              bv = v;
            }
          }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (!st) st = jfb_kmm_set_variant(pl, &bv);
  else jfb_kmm_set_variant(pl, &start);
  const int rs = restore();
  cudaStreamSynchronize(s);
  cudaFree(save);
  cudaFree(x_save);
  if (st) return st;
  if (rs) return rs;
  *best = bv;
  *best_ms = bms;
  return JFB_OK;
}

// A set of ensemble members whose five stages run as one launch each.
struct EnsGroup {
  std::vector<int> order;  // member indices, in work-list order
  jfb::EnsTiles htiles;
  jfb::EnsTiles* tiles = nullptr;                         // device copy of htiles
  jfb::EnsMember* tab[3] = {nullptr, nullptr, nullptr};  // per ring phase
  size_t smem[5] = {0, 0, 0, 0, 0};
};

struct jfb_ensemble {
  std::vector<jfb_kmm_plan*> m;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> join;
  cudaStream_t cap = nullptr;
  cudaEvent_t fork = nullptr;
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  // batched form: five launches per steady step for each group of members
  // (one group per wall-normal size, or one for all), the groups on
  // parallel branches of the step graph
  bool batched = false;
  int py = 0;
  std::vector<EnsGroup> groups;
};

namespace jfb {

// Every member an MHD plan on the tensor-core pencil stage with warp-FFT y
// transforms of one length: then the five stages batch across members.
static bool ensemble_batchable(const jfb_ensemble* e) {
  const char* env = std::getenv("JFB200_ENSEMBLE");
  if (env && std::string(env) == "streams") return false;
  if (e->m.size() > (size_t)kEnsMax) return false;
  for (const jfb_kmm_plan* pl : e->m)
    if (!pl->mhd || !pl->gemm || pl->py == 0 || pl->py != e->m[0]->py ||
        pl->mixed != e->m[0]->mixed)
      return false;
  return true;
}

template <int P, typename F>
static cudaError_t ens_y_launch(const EnsGroup& G, const EnsMember* tab, bool backward,
                                cudaStream_t s) {
  const int stage = backward ? 2 : 4;
  const int blocks = G.htiles.first[stage][G.htiles.nm];
  if (backward)
    ens_y_backward_kernel<P, F><<<blocks, 256, G.smem[2], s>>>(tab, G.tiles);
  else
    ens_y_forward_kernel<P, F><<<blocks, 256, G.smem[4], s>>>(tab, G.tiles);
  return cudaGetLastError();
}

template <typename F>
static cudaError_t ens_y_any(int py, const EnsGroup& G, const EnsMember* tab, bool backward,
                             cudaStream_t s) {
  switch (py) {
    case 2: return ens_y_launch<2, F>(G, tab, backward, s);
    case 3: return ens_y_launch<3, F>(G, tab, backward, s);
    case 4: return ens_y_launch<4, F>(G, tab, backward, s);
    default: return ens_y_launch<6, F>(G, tab, backward, s);
  }
}

// The five launches of one group's steady step with ring-phase table `tab`.
static int ensemble_group_step(const jfb_ensemble* e, const EnsGroup& G, const EnsMember* tab,
                               cudaStream_t s) {
  const EnsTiles& T = G.htiles;
  ens_pencil_kernel<<<T.first[0][T.nm], kGThreads, G.smem[0], s>>>(tab, G.tiles);
  JFB_CHECK_LAUNCH();
  ens_mhd_a_kernel<<<T.first[1][T.nm], kMhdThreads, G.smem[1], s>>>(tab, G.tiles);
  JFB_CHECK_LAUNCH();
  const bool f32 = e->m[0]->mixed;
  JFB_CHECK_CUDA(f32 ? ens_y_any<float>(e->py, G, tab, true, s)
                     : ens_y_any<double>(e->py, G, tab, true, s));
  if (f32)
    ens_z_cross_kernel<float><<<T.first[3][T.nm], 256, G.smem[3], s>>>(tab, G.tiles);
  else
    ens_z_cross_kernel<double><<<T.first[3][T.nm], 256, G.smem[3], s>>>(tab, G.tiles);
  JFB_CHECK_LAUNCH();
  JFB_CHECK_CUDA(f32 ? ens_y_any<float>(e->py, G, tab, false, s)
                     : ens_y_any<double>(e->py, G, tab, false, s));
  return JFB_OK;
}

// Device table of a group's members' steady-step arguments for ring phase k.
static int ensemble_table(jfb_ensemble* e, EnsGroup& G, int k) {
  if (G.tab[k]) return JFB_OK;
  std::vector<EnsMember> h(G.order.size());
  for (size_t i = 0; i < G.order.size(); ++i) {
    jfb_kmm_plan* pl = e->m[G.order[i]];
    StageArgs a;
    MhdArgs mm;
    steady_args(pl, pl->n, a, mm);
    EnsMember& x = h[i];
    std::memset(&x, 0, sizeof(x));
    x.d = pl->d;
    x.dT = pl->mixed ? tdims<float>(pl) : pl->d;
    x.o = pl->ops;
    x.G = pl->gops;
    x.ga = gemm_args(pl, a);
    x.M = pl->mops;
    x.ma = mm;
    x.ma.x32 = pl->mixed ? 1 : 0;
    x.ma.uw_b0z = pl->mphys.uw_emf * pl->mphys.b0z;
    x.ma.uw_b0x = pl->mphys.uw_emf * pl->mphys.b0x;
    x.ph = pl->mphys;
    x.fz = pl->fz;
    x.twy = pl->mixed ? (const void*)pl->twy32 : (const void*)pl->twy;
    x.twz = pl->mixed ? (const void*)pl->twz32 : (const void*)pl->twz;
    x.X = pl->X;
    x.Y = pl->Y;
    x.HZ = pl->HZ;
    x.HX = pl->HX;
    x.xb = pl->ops.xphys;
    x.KCw = pl->KCw;
    x.chunks = ceil_div(pl->d.Kz, pl->KCw);
  }
  JFB_CHECK_CUDA(cudaMalloc((void**)&G.tab[k], h.size() * sizeof(EnsMember)));
  JFB_CHECK_CUDA(cudaMemcpy(G.tab[k], h.data(), h.size() * sizeof(EnsMember),
                            cudaMemcpyHostToDevice));
  return JFB_OK;
}

// One steady step of a batched ensemble: the groups fork from the capture
// stream onto their own streams and join back.
static int ensemble_batched_step(jfb_ensemble* e, int k, cudaStream_t cap) {
  JFB_CHECK_CUDA(cudaEventRecord(e->fork, cap));
  for (size_t gi = 0; gi < e->groups.size(); ++gi) {
    cudaStream_t s = e->streams[gi];
    JFB_CHECK_CUDA(cudaStreamWaitEvent(s, e->fork, 0));
    int st = ensemble_group_step(e, e->groups[gi], e->groups[gi].tab[k], s);
    if (st) return st;
    JFB_CHECK_CUDA(cudaEventRecord(e->join[gi], s));
    JFB_CHECK_CUDA(cudaStreamWaitEvent(cap, e->join[gi], 0));
  }
  return JFB_OK;
}

}  // namespace jfb

extern "C" int jfb_ensemble_destroy(jfb_ensemble* e) {
  if (!e) return JFB_OK;
  for (auto& g : e->graph)
    if (g) cudaGraphExecDestroy(g);
  for (EnsGroup& G : e->groups) {
    for (auto* t : G.tab)
      if (t) cudaFree(t);
    if (G.tiles) cudaFree(G.tiles);
  }
  for (cudaStream_t s : e->streams) cudaStreamDestroy(s);
  for (cudaEvent_t ev : e->join) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->cap) cudaStreamDestroy(e->cap);
  delete e;
  return JFB_OK;
}

extern "C" int jfb_ensemble_create(jfb_kmm_plan* const* plans, int32_t n, jfb_ensemble** out) {
  JFB_REQUIRE(plans && out && n >= 1, "null pointer or empty ensemble");
  *out = nullptr;
  for (int i = 0; i < n; ++i) JFB_REQUIRE(plans[i], "null member plan");
  for (int i = 0; i < n; ++i)
    JFB_REQUIRE(plans[i]->cfg.time_integrator == JFB_INTEGRATOR_SBDF3,
                "ensemble members step with SBDF3");
  jfb_ensemble* e = new jfb_ensemble();
  e->m.assign(plans, plans + n);
  auto fail = [&](cudaError_t err) {
    set_error(std::string("CUDA error: ") + cudaGetErrorString(err));
    jfb_ensemble_destroy(e);
    return JFB_ERR_CUDA;
  };
  cudaError_t err;
  if ((err = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking)) != cudaSuccess) return fail(err);
  if ((err = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming)) != cudaSuccess) return fail(err);
  e->streams.resize(n, nullptr);
  e->join.resize(n, nullptr);
  for (int i = 0; i < n; ++i) {
    if ((err = cudaStreamCreateWithFlags(&e->streams[i], cudaStreamNonBlocking)) != cudaSuccess)
      return fail(err);
    if ((err = cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming)) != cudaSuccess)
      return fail(err);
  }
  e->batched = ensemble_batchable(e);
  if (e->batched) {
    e->py = e->m[0]->py;
    // one group per wall-normal size (its launches use that size's shared
    // memory and run beside the other sizes'), or JFB200_ENSEMBLE=batched:
    // a single group, largest members first
    const char* env = std::getenv("JFB200_ENSEMBLE");
    const bool single = env && std::string(env) == "batched";
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int a, int b) { return e->m[a]->d.Nx > e->m[b]->d.Nx; });
    // JFB200_ENSEMBLE_GROUP=k: at most k members per group (more groups on
    // parallel branches, so that stages of different kinds overlap)
    const char* genv = std::getenv("JFB200_ENSEMBLE_GROUP");
    const int gmax = genv ? std::max(1, std::atoi(genv)) : n;
    for (int i : idx) {
      if (e->groups.empty() || (int)e->groups.back().order.size() >= gmax ||
          (!single && e->m[e->groups.back().order.back()]->d.Nx != e->m[i]->d.Nx))
        e->groups.emplace_back();
      e->groups.back().order.push_back(i);
    }
    for (EnsGroup& G : e->groups) {
      EnsTiles& T = G.htiles;
      std::memset(&T, 0, sizeof(T));
      T.nm = (int)G.order.size();
      for (int q = 0; q < T.nm; ++q) {
        const jfb_kmm_plan* pl = e->m[G.order[q]];
        const Dims& d = pl->d;
        const int chunks = ceil_div(d.Kz, pl->KCw);
        const int t[5] = {(d.Ny / 2) * ceil_div(d.Kz, 8), (d.Ny / 2) * ceil_div(d.Kz, 8),
                          d.Nx * 12 * chunks, ceil_div((int64_t)d.Nx * d.My, kZRows),
                          d.Nx * 6 * chunks};
        const size_t sm[5] = {pl->smem_gemm, pl->smem_mhd, pl->smem_yw_b, pl->smem_zm,
                              pl->smem_yw_f};
        for (int st = 0; st < 5; ++st) {
          T.first[st][q + 1] = T.first[st][q] + t[st];
          G.smem[st] = std::max(G.smem[st], sm[st]);
        }
      }
      if ((err = cudaMalloc((void**)&G.tiles, sizeof(EnsTiles))) != cudaSuccess) return fail(err);
      if ((err = cudaMemcpy(G.tiles, &T, sizeof(EnsTiles), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(err);
    }
#define JFB_ENS_Y(F)                                                                     \
  (const void*)ens_y_backward_kernel<2, F>, (const void*)ens_y_forward_kernel<2, F>,     \
      (const void*)ens_y_backward_kernel<3, F>, (const void*)ens_y_forward_kernel<3, F>, \
      (const void*)ens_y_backward_kernel<4, F>, (const void*)ens_y_forward_kernel<4, F>, \
      (const void*)ens_y_backward_kernel<6, F>, (const void*)ens_y_forward_kernel<6, F>
    const void* fns[] = {(const void*)ens_pencil_kernel, (const void*)ens_mhd_a_kernel,
                         (const void*)ens_z_cross_kernel<double>,
                         (const void*)ens_z_cross_kernel<float>, JFB_ENS_Y(double),
                         JFB_ENS_Y(float)};
#undef JFB_ENS_Y
    for (const void* f : fns)
      if ((err = allow_smem(f)) != cudaSuccess) return fail(err);
  }
  *out = e;
  return JFB_OK;
}

extern "C" int jfb_ensemble_info(const jfb_ensemble* e, int32_t* batched,
                                 int64_t* launches_per_step) {
  JFB_REQUIRE(e, "null pointer");
  if (batched) *batched = e->batched ? 1 : 0;
  if (launches_per_step) {
    int64_t n = 0;
    for (const jfb_kmm_plan* pl : e->m) n += pl->mhd ? 5 : pl->plane ? 2 : 4;
    *launches_per_step = e->batched ? 5 * (int64_t)e->groups.size() : n;
  }
  return JFB_OK;
}

extern "C" int jfb_ensemble_advance(jfb_ensemble* e, int64_t steps, void* stream) {
  JFB_REQUIRE(e, "null pointer");
  JFB_REQUIRE(steps >= 0, "steps must be >= 0");
  cudaStream_t s = (cudaStream_t)stream;
  const int n = (int)e->m.size();
  for (jfb_kmm_plan* pl : e->m) {
    if (!pl->have_state) {
      set_error("an ensemble member has no state loaded");
      return JFB_ERR_STATE;
    }
    if (slot(pl->n) != slot(e->m[0]->n) || pl->hist != e->m[0]->hist) {
      set_error("ensemble members must share the step phase and history count");
      return JFB_ERR_STATE;
    }
  }
  int st;
  for (jfb_kmm_plan* pl : e->m)
    if ((st = ensure_H(pl, s))) return st;
  while (steps > 0 && e->m[0]->hist < 2) {
    for (jfb_kmm_plan* pl : e->m) {
      if ((st = startup_step(pl, s))) return st;
      pl->n += 1;
      pl->hist += 1;
      pl->explicit_u12 = false;
    }
    --steps;
  }
  while (steps > 0) {
    const int k = slot(e->m[0]->n);
    if (!e->graph[k] && e->batched) {
      // five launches per group; the member tables of this ring phase are
      // built (with blocking copies) before the capture
      for (EnsGroup& G : e->groups)
        if ((st = ensemble_table(e, G, k))) return st;
      cudaGraph_t g;
      JFB_CHECK_CUDA(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal));
      st = ensemble_batched_step(e, k, e->cap);
      cudaError_t ec = cudaStreamEndCapture(e->cap, &g);
      if (st) return st;
      JFB_CHECK_CUDA(ec);
      JFB_CHECK_CUDA(cudaGraphInstantiate(&e->graph[k], g, 0));
      cudaGraphDestroy(g);
    }
    if (!e->graph[k]) {
      cudaGraph_t g;
      JFB_CHECK_CUDA(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal));
      int rc = JFB_OK;
      cudaError_t ce = cudaEventRecord(e->fork, e->cap);
      for (int i = 0; i < n && rc == JFB_OK && ce == cudaSuccess; ++i) {
        ce = cudaStreamWaitEvent(e->streams[i], e->fork, 0);
        if (ce != cudaSuccess) break;
        rc = steady_step(e->m[i], e->m[i]->n, e->streams[i]);
        if (rc) break;
        ce = cudaEventRecord(e->join[i], e->streams[i]);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->cap, e->join[i], 0);
      }
      cudaError_t ec = cudaStreamEndCapture(e->cap, &g);
      if (rc) return rc;
      JFB_CHECK_CUDA(ce);
      JFB_CHECK_CUDA(ec);
      JFB_CHECK_CUDA(cudaGraphInstantiate(&e->graph[k], g, 0));
      cudaGraphDestroy(g);
    }
    JFB_CHECK_CUDA(cudaGraphLaunch(e->graph[k], s));
    for (jfb_kmm_plan* pl : e->m) {
      pl->n += 1;
      pl->explicit_u12 = false;
    }
    --steps;
  }
  return JFB_OK;
}

#include "jfb_tps.cuh"
