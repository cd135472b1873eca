// Host-side construction of the 1-D operators of the KMM plane-Couette step.
//
// Restates, in closed form, the matrices the reference assembles with SymPy
// at set-up time:
//   Gauss-Chebyshev nodes / scalar products   galerkin/Chebyshev.py:159-180, 300-317
//   Shen Dirichlet / biharmonic stencils      galerkin/composite.py:797-864
//   Galerkin matrices (T_i, T_j^(k))_w        galerkin/Chebyshev.py:21-35, 437-487;
//                                             k = 4 by exact quadrature, inner.py:945-960
//   Fourier diagonal matrices                 galerkin/Fourier.py:241-268
//   Helmholtz / Biharmonic operators          la/solvers.py:22-61
//   per-wavenumber weights W[t, k]            la/tpmatrix.py:1900-2029
#include "jfb_kmm.h"

#include <cmath>
#include <cstdint>
#include <stdexcept>

namespace jfb {

static std::vector<double> chebyshev_norm2(int N) {
  std::vector<double> h(N, M_PI / 2);
  h[0] = M_PI;
  return h;
}

// Integer coefficient matrix of d/dX on Chebyshev coefficients:
// (T_j)' = sum_{i<j, j-i odd} (2 / c_i) j T_i, c_0 = 2.
static std::vector<int64_t> chebyshev_d1_int(int N) {
  std::vector<int64_t> D((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; j += 2) D[(size_t)i * N + j] = (i == 0) ? j : 2 * j;
  return D;
}

static std::vector<int64_t> int_matmul(const std::vector<int64_t>& A,
                                       const std::vector<int64_t>& B, int N) {
  std::vector<int64_t> C((size_t)N * N, 0);
  for (int i = 0; i < N; ++i)
    for (int k = i; k < N; ++k) {
      const int64_t a = A[(size_t)i * N + k];
      if (!a) continue;
      for (int j = k; j < N; ++j) C[(size_t)i * N + j] += a * B[(size_t)k * N + j];
    }
  return C;
}

// (T_i, d^k T_j / dX^k)_w as a dense N x N matrix.
static std::vector<double> chebyshev_galerkin(int N, int k) {
  std::vector<int64_t> D((size_t)N * N, 0);
  for (int i = 0; i < N; ++i) D[(size_t)i * N + i] = 1;
  const std::vector<int64_t> D1 = chebyshev_d1_int(N);
  for (int t = 0; t < k; ++t) D = int_matmul(D1, D, N);
  const std::vector<double> h = chebyshev_norm2(N);
  std::vector<double> M((size_t)N * N);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) M[(size_t)i * N + j] = h[i] * (double)D[(size_t)i * N + j];
  return M;
}

// S X S^T for a stencil with diagonals s0, s2, s4 (s4 may be empty).
static std::vector<double> stencil_sandwich(const std::vector<double>& X, int N,
                                            const Stencil& S) {
  const int n = S.n;
  // T = S X  (n x N)
  std::vector<double> T((size_t)n * N, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < N; ++j) {
      double v = S.s0[i] * X[(size_t)i * N + j] + S.s2[i] * X[(size_t)(i + 2) * N + j];
      if (S.width == 4) v += S.s4[i] * X[(size_t)(i + 4) * N + j];
      T[(size_t)i * N + j] = v;
    }
  // R = T S^T (n x n): R[i, m] = sum_j T[i, j] S[m, j]
  std::vector<double> R((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int m = 0; m < n; ++m) {
      double v = S.s0[m] * T[(size_t)i * N + m] + S.s2[m] * T[(size_t)i * N + m + 2];
      if (S.width == 4) v += S.s4[m] * T[(size_t)i * N + m + 4];
      R[(size_t)i * n + m] = v;
    }
  return R;
}

Stencil make_stencil(int N, bool biharmonic) {
  Stencil S;
  S.width = biharmonic ? 4 : 2;
  S.n = N - S.width;
  S.s0.assign(S.n, 1.0);
  S.s2.assign(S.n, -1.0);
  S.s4.assign(S.n, 0.0);
  if (biharmonic) {
    for (int i = 0; i < S.n; ++i) {
      const double n = i;
      S.s2[i] = 2.0 * (-n - 2.0) / (n + 3.0);
      S.s4[i] = (n + 1.0) / (n + 3.0);
    }
  }
  return S;
}

void build_host_operators(const jfb_kmm_config& cfg, HostOperators& op) {
  const int N = cfg.nx;
  op.N = N;
  op.nB = N - 4;
  op.nD = N - 2;
  const double Lx = cfg.x_hi - cfg.x_lo;
  op.dfx = std::fabs(Lx - 2.0) < 1e-12 ? 1.0 : 2.0 / Lx;
  const double Ly = cfg.ly, Lz = cfg.lz;
  op.dfy = std::fabs(Ly - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / Ly;
  op.dfz = std::fabs(Lz - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / Lz;

  // Gauss-Chebyshev nodes X_j = cos(pi + (2j+1) pi / (2N)) and T_n(X_j).
  op.xnodes.resize(N);
  op.xphys.resize(N);
  for (int j = 0; j < N; ++j) {
    op.xnodes[j] = std::cos(M_PI + (2.0 * j + 1.0) * M_PI / (2.0 * N));
    op.xphys[j] = cfg.x_lo + (op.xnodes[j] + 1.0) / op.dfx;
  }
  op.V.assign((size_t)N * N, 0.0);  // V[j][n] = T_n(X_j)
  for (int j = 0; j < N; ++j) {
    double t0 = 1.0, t1 = op.xnodes[j];
    op.V[(size_t)j * N + 0] = 1.0;
    if (N > 1) op.V[(size_t)j * N + 1] = t1;
    for (int n = 2; n < N; ++n) {
      const double t2 = 2.0 * op.xnodes[j] * t1 - t0;
      op.V[(size_t)j * N + n] = t2;
      t0 = t1;
      t1 = t2;
    }
  }
  // Scalar products (T_n, u)_w by Gauss-Chebyshev quadrature: weight pi/N/df.
  op.Q.assign((size_t)N * N, 0.0);
  for (int n = 0; n < N; ++n)
    for (int j = 0; j < N; ++j)
      op.Q[(size_t)n * N + j] = op.V[(size_t)j * N + n] * (M_PI / N) / op.dfx;

  op.ns = chebyshev_norm2(N);
  for (double& v : op.ns) v /= op.dfx;

  op.SB = make_stencil(N, true);
  op.SD = make_stencil(N, false);

  // Galerkin x-matrices (including the df^(k-1) domain scaling).
  const std::vector<double> T0 = chebyshev_galerkin(N, 0);
  const std::vector<double> T2 = chebyshev_galerkin(N, 2);
  const std::vector<double> T4 = chebyshev_galerkin(N, 4);
  auto scaled = [&](std::vector<double> X, int k) {
    const double f = std::pow(op.dfx, k - 1);
    for (double& v : X) v *= f;
    return X;
  };
  op.XB0 = stencil_sandwich(scaled(T0, 0), N, op.SB);
  op.XB2 = stencil_sandwich(scaled(T2, 2), N, op.SB);
  op.XB4 = stencil_sandwich(scaled(T4, 4), N, op.SB);
  op.XD0 = stencil_sandwich(scaled(T0, 0), N, op.SD);
  op.XD2 = stencil_sandwich(scaled(T2, 2), N, op.SD);

  // Dirichlet mass matrix (== M00) tri-band and its no-pivot LU.
  const int nD = op.nD;
  op.mlo.assign(nD, 0.0);
  op.mdi.assign(nD, 0.0);
  op.mhi.assign(nD, 0.0);
  for (int i = 0; i < nD; ++i) {
    op.mdi[i] = op.XD0[(size_t)i * nD + i];
    if (i >= 2) op.mlo[i] = op.XD0[(size_t)i * nD + i - 2];
    if (i + 2 < nD) op.mhi[i] = op.XD0[(size_t)i * nD + i + 2];
  }
  // LU of the tri-band (offsets -2, 0, 2): l[i] = A[i,i-2]/u[i-2], u[i] = d[i] - l[i]*h[i-2]
  op.lu_l.assign(nD, 0.0);
  op.lu_u.assign(nD, 0.0);
  for (int i = 0; i < nD; ++i) {
    double d = op.mdi[i];
    if (i >= 2) {
      op.lu_l[i] = op.mlo[i] / op.lu_u[i - 2];
      d -= op.lu_l[i] * op.mhi[i - 2];
    }
    op.lu_u[i] = d;
  }

  // Biharmonic mass S_B diag(ns) S_B^T (composite.py:395-399) and its no-pivot
  // banded LU (diamatrix.py:1936-1973), offsets {-4, -2, 0, 2, 4}.
  const int nB = op.nB;
  std::vector<double> A(op.XB0);
  for (int k = 0; k < nB; ++k) {
    const double piv = A[(size_t)k * nB + k];
    for (int s = 2; s <= 4; s += 2) {
      if (k + s >= nB) break;
      const double f = A[(size_t)(k + s) * nB + k] / piv;
      A[(size_t)(k + s) * nB + k] = f;
      for (int u = 2; u <= 4; u += 2)
        if (k + u < nB) A[(size_t)(k + s) * nB + k + u] -= f * A[(size_t)k * nB + k + u];
    }
  }
  op.bl2.assign(nB, 0.0);
  op.bl4.assign(nB, 0.0);
  op.bu0.assign(nB, 0.0);
  op.bu2.assign(nB, 0.0);
  op.bu4.assign(nB, 0.0);
  for (int i = 0; i < nB; ++i) {
    if (i >= 2) op.bl2[i] = A[(size_t)i * nB + i - 2];
    if (i >= 4) op.bl4[i] = A[(size_t)i * nB + i - 4];
    op.bu0[i] = A[(size_t)i * nB + i];
    if (i + 2 < nB) op.bu2[i] = A[(size_t)i * nB + i + 2];
    if (i + 4 < nB) op.bu4[i] = A[(size_t)i * nB + i + 4];
  }

  // Fejer-I weights for physical-volume integrals (Chebyshev.py:182-208).
  op.fejer.assign(N, 0.0);
  for (int j = 0; j < N; ++j) {
    const double theta = M_PI + (2.0 * j + 1.0) * M_PI / (2.0 * N);
    double corr = 0.0;
    for (int m = 1; m <= N / 2; ++m)
      corr += 2.0 * std::cos(2.0 * theta * m) / (4.0 * (double)m * m - 1.0);
    op.fejer[j] = (2.0 / N) * (1.0 - corr) / op.dfx;
  }
}

// Coefficients (a0, a2, a4) such that the per-wavenumber matrix of the
// Biharmonic (Su) or Helmholtz (Sg) operator with implicit coefficient
// `gamma` is a0 X0 + a2 X2 + a4 X4.  The Fourier weights follow
// Fourier._matrices: (ik)^j (-ik)^i 2 pi df^(i+j-1).
void mode_coefficients(const HostOperators& op, const jfb_kmm_config& cfg, int ky,
                       int kz, double gamma, bool biharmonic, double out[3]) {
  const double twopi = 2.0 * M_PI;
  const double My = twopi / op.dfy, Mz = twopi / op.dfz;
  const double a2 = (double)ky * ky, b2 = (double)kz * kz;
  const double D2y = -a2 * twopi * op.dfy, D2z = -b2 * twopi * op.dfz;
  const double D4y = a2 * a2 * twopi * op.dfy * op.dfy * op.dfy;
  const double D4z = b2 * b2 * twopi * op.dfz * op.dfz * op.dfz;
  const double nu = cfg.nu;
  if (biharmonic) {
    // (v, lap u) - gamma (v, nu lap lap u)
    out[0] = (D2y * Mz + My * D2z) - gamma * nu * (D4y * Mz + My * D4z + 2.0 * D2y * D2z);
    out[1] = My * Mz - gamma * nu * 2.0 * (D2y * Mz + My * D2z);
    out[2] = -gamma * nu * My * Mz;
  } else {
    // (v, u) - gamma (v, nu lap u)
    out[0] = My * Mz - gamma * nu * (D2y * Mz + My * D2z);
    out[1] = -gamma * nu * My * Mz;
    out[2] = 0.0;
  }
}

}  // namespace jfb
