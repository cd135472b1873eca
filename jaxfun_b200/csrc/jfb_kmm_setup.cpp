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
#include <algorithm>
#include <string>

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

// (L_i, d^k L_j / dX^k)_w of the Legendre polynomials as a dense N x N
// matrix: (L_j)' = sum_{i<j, j-i odd} (2i+1) L_i (Legendre.py:195-227) and
// (L_i, L_i) = 2 / (2i + 1) (Legendre.py:19-33, 229-268).
static std::vector<double> legendre_galerkin(int N, int k) {
  std::vector<int64_t> D((size_t)N * N, 0), D1((size_t)N * N, 0);
  for (int i = 0; i < N; ++i) D[(size_t)i * N + i] = 1;
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; j += 2) D1[(size_t)i * N + j] = 2 * i + 1;
  for (int t = 0; t < k; ++t) D = int_matmul(D1, D, N);
  std::vector<double> M((size_t)N * N);
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j)
      M[(size_t)i * N + j] = 2.0 / (2.0 * i + 1.0) * (double)D[(size_t)i * N + j];
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

// Shen stencils (composite.py:797-864): Dirichlet P_i - P_{i+2} for both
// families; biharmonic T_i - 2(i+2)/(i+3) T_{i+2} + (i+1)/(i+3) T_{i+4} or
// L_i - 2(2i+5)/(2i+7) L_{i+2} + (2i+3)/(2i+7) L_{i+4}.
Stencil make_stencil(int N, bool biharmonic, int family) {
  Stencil S;
  S.width = biharmonic ? 4 : 2;
  S.n = N - S.width;
  S.s0.assign(S.n, 1.0);
  S.s2.assign(S.n, -1.0);
  S.s4.assign(S.n, 0.0);
  if (biharmonic) {
    for (int i = 0; i < S.n; ++i) {
      const double n = i;
      if (family == 0) {
        S.s2[i] = 2.0 * (-n - 2.0) / (n + 3.0);
        S.s4[i] = (n + 1.0) / (n + 3.0);
      } else {
        S.s2[i] = 2.0 * (-2.0 * n - 5.0) / (2.0 * n + 7.0);
        S.s4[i] = (2.0 * n + 3.0) / (2.0 * n + 7.0);
      }
    }
  }
  return S;
}

void build_host_operators(const jfb_kmm_config& cfg, HostOperators& op) {
  const int N = cfg.nx;
  op.N = N;
  op.nB = N - 4;
  op.nD = N - 2;
  op.family = cfg.family == JFB_FAMILY_LEGENDRE ? 1 : 0;
  op.x_lo = cfg.x_lo;
  op.x_hi = cfg.x_hi;
  const double Lx = cfg.x_hi - cfg.x_lo;
  op.dfx = std::fabs(Lx - 2.0) < 1e-12 ? 1.0 : 2.0 / Lx;
  const double Ly = cfg.ly, Lz = cfg.lz;
  op.dfy = std::fabs(Ly - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / Ly;
  op.dfz = std::fabs(Lz - 2.0 * M_PI) < 1e-12 ? 1.0 : 2.0 * M_PI / Lz;

  op.xnodes.resize(N);
  op.xphys.resize(N);
  XBasis leg;  // Legendre: nodes, Vandermonde and quadrature in long double
  if (op.family == 1) {
    build_x_basis(1, 0, N, cfg.x_lo, cfg.x_hi, leg);
    op.V.assign((size_t)N * N, 0.0);
    op.Q.assign((size_t)N * N, 0.0);
    op.ns.assign(N, 0.0);
    for (int j = 0; j < N; ++j) {
      op.xnodes[j] = (double)leg.X[j];
      op.xphys[j] = cfg.x_lo + (op.xnodes[j] + 1.0) / op.dfx;
      op.ns[j] = (double)leg.ns[j];
    }
    for (size_t k = 0; k < op.V.size(); ++k) {
      op.V[k] = (double)leg.V[k];
      op.Q[k] = (double)leg.Q[k];
    }
  } else {
    // Gauss-Chebyshev nodes X_j = cos(pi + (2j+1) pi / (2N)) and T_n(X_j).
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
  }

  op.SB = make_stencil(N, true, op.family);
  op.SD = make_stencil(N, false, op.family);

  // Galerkin x-matrices (including the df^(k-1) domain scaling).
  auto galerkin = op.family == 1 ? legendre_galerkin : chebyshev_galerkin;
  const std::vector<double> T0 = galerkin(N, 0);
  const std::vector<double> T2 = galerkin(N, 2);
  const std::vector<double> T4 = galerkin(N, 4);
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

  op.fejer.assign(N, 0.0);
  if (op.family == 1) {
    // Gauss-Legendre weights / df: Q[0][j] = L_0(X_j) w_j / df
    for (int j = 0; j < N; ++j) op.fejer[j] = (double)leg.Q[j];
    return;
  }
  // Fejer-I weights for physical-volume integrals (Chebyshev.py:182-208).
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


// ---------------------------------------------------------------------------
// Folded x-operators of the step (long double products, rounded once).
//
// Every per-pencil map of the step along x is linear with (ky, kz)-dependent
// scalar weights, so the Shen projections, chebder recurrences and mass
// solves fold into fixed matrices shared by all pencils:
//   Pi = S_D^T M_D^-1 S_D Q      physical -> orthogonal coefficients of P_TD
//   Nu = Myz [R1 (i ky H1 + i kz H2) + k^2 R0 H0],  R0 = S_B W Pi, R1 = S_B W D Pi
//   Ng = Myz R2 (i kz H1 - i ky H2),                R2 = S_D W Pi
//        (channelflow_kmm.py:784-829, coefficient path)
//   u0 = A0 u0,  u1 = i (ky P1 u0 + kz B1 g) / k^2,  u2 = i (kz P1 u0 - ky B1 g) / k^2
//   w0 = B1 g,   w1 = i kz A0 u0 - i (kz P2 u0 - ky B2 g) / k^2,
//   w2 = i (ky P2 u0 + kz B2 g) / k^2 - i ky A0 u0      (channelflow_kmm.py:699-714, 831-870)
// with A0 = V S_B^T, B1 = V S_D^T, B2 = V D S_D^T, F = M_D^-1 S_D W D S_B^T,
// P1 = B1 F, P2 = B2 F, W = diag(norm^2 / df).  Gauss nodes are mirror
// symmetric and T_n has parity n, so each matrix splits into a symmetric and
// an antisymmetric half of half the size.
// ---------------------------------------------------------------------------
namespace {
using LD = long double;
struct LMat {
  int r = 0, c = 0;
  std::vector<LD> v;
  LMat(int r_, int c_) : r(r_), c(c_), v((size_t)r_ * c_, 0.0L) {}
  LD& operator()(int i, int j) { return v[(size_t)i * c + j]; }
  LD operator()(int i, int j) const { return v[(size_t)i * c + j]; }
};
LMat mul(const LMat& A, const LMat& B) {
  LMat C(A.r, B.c);
  for (int i = 0; i < A.r; ++i)
    for (int k = 0; k < A.c; ++k) {
      const LD a = A(i, k);
      if (a == 0.0L) continue;
      for (int j = 0; j < B.c; ++j) C(i, j) += a * B(k, j);
    }
  return C;
}
LMat transpose(const LMat& A) {
  LMat T(A.c, A.r);
  for (int i = 0; i < A.r; ++i)
    for (int j = 0; j < A.c; ++j) T(j, i) = A(i, j);
  return T;
}
// Gauss-Jordan inverse with partial pivoting (small SPD mass matrix).
LMat inverse(const LMat& A) {
  const int n = A.r;
  LMat M = A, I(n, n);
  for (int i = 0; i < n; ++i) I(i, i) = 1.0L;
  for (int k = 0; k < n; ++k) {
    int piv = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs((double)M(i, k)) > std::fabs((double)M(piv, k))) piv = i;
    if (piv != k)
      for (int j = 0; j < n; ++j) {
        std::swap(M(k, j), M(piv, j));
        std::swap(I(k, j), I(piv, j));
      }
    const LD inv = 1.0L / M(k, k);
    for (int j = 0; j < n; ++j) {
      M(k, j) *= inv;
      I(k, j) *= inv;
    }
    for (int i = 0; i < n; ++i) {
      if (i == k) continue;
      const LD f = M(i, k);
      if (f == 0.0L) continue;
      for (int j = 0; j < n; ++j) {
        M(i, j) -= f * M(k, j);
        I(i, j) -= f * I(k, j);
      }
    }
  }
  return I;
}
LMat from_dense(const std::vector<double>& a, int r, int c) {
  LMat M(r, c);
  for (size_t k = 0; k < a.size(); ++k) M.v[k] = a[k];
  return M;
}
// max |M[i][N-1-j] - sign_i M[i][j]| relative to the largest entry of row i
// (rows of a physical-input matrix) is tiny for every row.
bool rows_mirror(const LMat& M, int sign_even_row) {
  const int N = M.c;
  for (int i = 0; i < M.r; ++i) {
    const LD s = (i % 2 == 0) ? sign_even_row : -sign_even_row;
    LD big = 0, bad = 0;
    for (int j = 0; j < N; ++j) big = std::max(big, std::fabs(M(i, j)));
    for (int j = 0; j < N; ++j) bad = std::max(bad, std::fabs(M(i, N - 1 - j) - s * M(i, j)));
    if (bad > 1e-13L * (big + 1e-300L)) return false;
  }
  return true;
}
bool cols_mirror(const LMat& M, int sign_even_col) {
  const int N = M.r;
  for (int c = 0; c < M.c; ++c) {
    const LD s = (c % 2 == 0) ? sign_even_col : -sign_even_col;
    LD big = 0, bad = 0;
    for (int j = 0; j < N; ++j) big = std::max(big, std::fabs(M(j, c)));
    for (int j = 0; j < N; ++j) bad = std::max(bad, std::fabs(M(N - 1 - j, c) - s * M(j, c)));
    if (bad > 1e-13L * (big + 1e-300L)) return false;
  }
  return true;
}
}  // namespace

bool build_gemm_operators(const HostOperators& op, GemmHost& gh, std::string& err,
                          bool gradient) {
  const int N = op.N, nB = op.nB, nD = op.nD;
  const LD pi = std::acos(-1.0L);
  const LD dfx = op.dfx;
  LMat V(N, N), Q(N, N), D(N, N), W(N, N), SB(nB, N), SD(nD, N);
  if (op.family == 1) {
    // Legendre: Gauss-Legendre nodes, L_n(X_j), legder, norms 2/(2n+1)/df
    XBasis xb;
    build_x_basis(1, 2, N, op.x_lo, op.x_hi, xb);
    V.v = xb.V;
    Q.v = xb.Q;
    for (size_t k = 0; k < D.v.size(); ++k) D.v[k] = dfx * xb.D[k];
    for (int n = 0; n < N; ++n) W(n, n) = xb.ns[n];
    for (size_t k = 0; k < SB.v.size(); ++k) SB.v[k] = xb.S[k];
  } else {
    for (int j = 0; j < N; ++j) {
      const LD th = pi + (2.0L * j + 1.0L) * pi / (2.0L * N);
      for (int n = 0; n < N; ++n) V(j, n) = std::cos((LD)n * th);
    }
    for (int n = 0; n < N; ++n)
      for (int j = 0; j < N; ++j) Q(n, j) = V(j, n) * (pi / N) / dfx;
    for (int i = 0; i < N; ++i)
      for (int j = i + 1; j < N; j += 2) D(i, j) = dfx * (LD)((i == 0) ? j : 2 * j);
    for (int n = 0; n < N; ++n) W(n, n) = ((n == 0) ? pi : pi / 2.0L) / dfx;
    for (int i = 0; i < nB; ++i) {
      const LD n = i;
      SB(i, i) = 1.0L;
      SB(i, i + 2) = 2.0L * (-n - 2.0L) / (n + 3.0L);
      SB(i, i + 4) = (n + 1.0L) / (n + 3.0L);
    }
  }
  for (int i = 0; i < nD; ++i) {
    SD(i, i) = 1.0L;
    SD(i, i + 2) = -1.0L;
  }
  const LMat SBt = transpose(SB), SDt = transpose(SD);
  const LMat WD = mul(W, D);
  const LMat MDi = inverse(mul(mul(SD, W), SDt));
  const LMat Pi = mul(mul(mul(SDt, MDi), SD), Q);
  const LMat R0 = mul(mul(SB, W), Pi);
  const LMat R1 = mul(mul(SB, WD), Pi);
  const LMat R2 = mul(mul(SD, W), Pi);
  const LMat R3 = mul(SD, Q);
  const LMat F = mul(mul(mul(MDi, SD), WD), SBt);
  const LMat A0 = mul(V, SBt);
  const LMat B1 = mul(V, SDt);
  const LMat B2 = mul(mul(V, D), SDt);
  const LMat P1 = mul(B1, F);
  const LMat P2 = mul(B2, F);
  const LMat A1 = mul(mul(V, D), SBt);  // d/dx of a TB field at the nodes (gradient form)
  const LMat K0 = from_dense(op.XB0, nB, nB), K2 = from_dense(op.XB2, nB, nB),
             K4 = from_dense(op.XB4, nB, nB);
  const LMat X0D = from_dense(op.XD0, nD, nD), X2D = from_dense(op.XD2, nD, nD);

  if (!rows_mirror(R0, +1) || !rows_mirror(R1, -1) || !rows_mirror(R2, +1) || !rows_mirror(R3, +1) ||
      !cols_mirror(A0, +1) || !cols_mirror(B1, +1) || !cols_mirror(B2, -1) ||
      !cols_mirror(P1, -1) || !cols_mirror(P2, +1) || (gradient && !cols_mirror(A1, -1))) {
    err = "x-operators lack the mirror parity of the Gauss nodes";
    return false;
  }
  for (int i = 0; i < nB; ++i)
    for (int j = 0; j < nB; ++j)
      if ((i - j) % 2 != 0 && (K0(i, j) != 0 || K2(i, j) != 0 || K4(i, j) != 0)) {
        err = "biharmonic Galerkin matrices couple odd offsets";
        return false;
      }

  const int Jh = (N + 1) / 2, Jl = N / 2;
  const int nBe = (nB + 1) / 2, nBo = nB / 2, nDe = (nD + 1) / 2, nDo = nD / 2;
  gh.Jh = Jh;
  gh.Jl = Jl;
  gh.nBe = nBe;
  gh.nBo = nBo;
  gh.nDe = nDe;
  gh.nDo = nDo;
  gh.frag.clear();
  gh.krange.clear();
  auto add = [&](int id, int R, int K, auto val) {
    const int MT = (R + 7) / 8, KT = (K + 3) / 4;
    gh.off[id] = (int)gh.frag.size();
    gh.mt[id] = MT;
    gh.kt[id] = KT;
    gh.kr[id] = (int)gh.krange.size();
    gh.frag.resize(gh.frag.size() + (size_t)MT * KT * 32, 0.0);
    for (int mt = 0; mt < MT; ++mt) {
      int kb = KT, ke = 0;
      for (int kt = 0; kt < KT; ++kt)
        for (int lane = 0; lane < 32; ++lane) {
          const int r = mt * 8 + lane / 4, k = kt * 4 + lane % 4;
          const double v = (r < R && k < K) ? (double)val(r, k) : 0.0;
          gh.frag[gh.off[id] + ((size_t)mt * KT + kt) * 32 + lane] = v;
          if (v != 0.0) {
            kb = std::min(kb, kt);
            ke = std::max(ke, kt + 1);
          }
        }
      if (ke == 0) kb = 0;
      gh.krange.push_back(kb);
      gh.krange.push_back(ke);
    }
  };
  // right-hand sides.  The B operands are the three x-sample blocks after an
  // in-place mirror transform: block 0 row j < Jl holds d(h12)_j and row
  // N-1-j holds s(k2 h0)_j; block 1 row j holds s(h12)_j, row N-1-j d(k2 h0)_j;
  // block 2 row j holds s(hg)_j, row N-1-j d(hg)_j (j = Jl, the middle node of
  // an odd N, holds the sums).  Columns follow that row order.
  add(gNuE, nBe, N,
      [&](int r, int k) { return k < Jl ? R1(2 * r, k) : R0(2 * r, N - 1 - k); });
  add(gNuO, nBo, N,
      [&](int r, int k) { return k < Jh ? R1(2 * r + 1, k) : R0(2 * r + 1, N - 1 - k); });
  add(gNgE, nDe, Jh, [&](int r, int k) { return R2(2 * r, k); });
  add(gNgO, nDo, Jl, [&](int r, int k) { return R2(2 * r + 1, Jl - 1 - k); });
  // mass rows: B rows [v1; v2; v3] against [X2_B | X0_B | X4_B], [w1; w2] against [X0_D | X2_D]
  auto mu = [&](int par, int nh) {
    return [&, par, nh](int r, int k) {
      const int seg = k / nh, c = 2 * (k % nh) + par, i = 2 * r + par;
      return seg == 0 ? K2(i, c) : seg == 1 ? K0(i, c) : K4(i, c);
    };
  };
  add(gMuE, nBe, 3 * nBe, mu(0, nBe));
  add(gMuO, nBo, 3 * nBo, mu(1, nBo));
  auto mg = [&](int par, int nh) {
    return [&, par, nh](int r, int k) {
      const int seg = k / nh, c = 2 * (k % nh) + par, i = 2 * r + par;
      return seg == 0 ? X0D(i, c) : X2D(i, c);
    };
  };
  add(gMgE, nDe, 2 * nDe, mg(0, nDe));
  add(gMgO, nDo, 2 * nDo, mg(1, nDo));
  // velocity / vorticity halves: rows j < Jl; the middle node of an odd N
  // (symmetric half only) is kept apart in `mid`
  auto ph = [&](const LMat& M, int par) {
    return [&, par](int j, int k) -> LD { return M(j, 2 * k + par); };
  };
  add(gA0Ee, Jl, nBe, ph(A0, 0));
  add(gP2Ee, Jl, nBe, ph(P2, 0));
  add(gP1Oe, Jl, nBe, ph(P1, 0));
  add(gP1Eo, Jl, nBo, ph(P1, 1));
  add(gA0Oo, Jl, nBo, ph(A0, 1));
  add(gP2Oo, Jl, nBo, ph(P2, 1));
  add(gB1Ee, Jl, nDe, ph(B1, 0));
  add(gB2Oe, Jl, nDe, ph(B2, 0));
  add(gB2Eo, Jl, nDo, ph(B2, 1));
  add(gB1Oo, Jl, nDo, ph(B1, 1));
  // gradient form: d/dx u0 at the nodes (an even coefficient gives the
  // antisymmetric half); empty sub-matrices otherwise
  add(gA1Oe, gradient ? Jl : 0, gradient ? nBe : 0, ph(A1, 0));
  add(gA1Eo, gradient ? Jl : 0, gradient ? nBo : 0, ph(A1, 1));
  gh.mid_stride = std::max(std::max(nBe, nBo), std::max(nDe, nDo));
  gh.mid.assign((size_t)6 * gh.mid_stride, 0.0);
  if (N % 2 == 1) {
    const int j = Jl;
    for (int k = 0; k < nBe; ++k) {
      gh.mid[0 * gh.mid_stride + k] = (double)A0(j, 2 * k);
      gh.mid[1 * gh.mid_stride + k] = (double)P2(j, 2 * k);
    }
    for (int k = 0; k < nBo; ++k) gh.mid[2 * gh.mid_stride + k] = (double)P1(j, 2 * k + 1);
    for (int k = 0; k < nDe; ++k) gh.mid[3 * gh.mid_stride + k] = (double)B1(j, 2 * k);
    for (int k = 0; k < nDo; ++k) gh.mid[4 * gh.mid_stride + k] = (double)B2(j, 2 * k + 1);
    if (gradient)
      for (int k = 0; k < nBo; ++k) gh.mid[5 * gh.mid_stride + k] = (double)A1(j, 2 * k + 1);
  }

  {
    const LMat WD2 = mul(WD, D);
    const LMat C1 = mul(mul(mul(mul(V, SDt), MDi), mul(SD, WD)), SDt);
    const LMat C2 = mul(mul(mul(mul(V, SDt), MDi), mul(SD, WD2)), SDt);
    auto dense = [&](const LMat& M) {
      std::vector<double> o((size_t)M.r * M.c);
      for (size_t k = 0; k < o.size(); ++k) o[k] = (double)M.v[k];
      return o;
    };
    gh.B1 = dense(B1);
    gh.B2 = dense(B2);
    gh.P1 = dense(P1);
    gh.P2 = dense(P2);
    gh.C1 = dense(C1);
    gh.C2 = dense(C2);
    gh.A0 = dense(A0);
    gh.F = dense(F);
    gh.R0 = dense(R0);
    gh.R1 = dense(R1);
    gh.R2 = dense(R2);
    LMat Wf(N, N);
    for (int j = 0; j < N; ++j) Wf(j, j) = (LD)op.fejer[j];
    gh.GB = dense(mul(mul(transpose(A0), Wf), A0));
    gh.GD = dense(mul(mul(transpose(B1), Wf), B1));
  }
  gh.R3.assign((size_t)nD * N, 0.0);
  for (int i = 0; i < nD; ++i)
    for (int j = 0; j < N; ++j) gh.R3[(size_t)i * N + j] = (double)R3(i, j);
  gh.X2D = op.XD2;
  return true;
}


// ---------------------------------------------------------------------------
// Standalone wall-normal bases (Chebyshev and Legendre) and their separable
// maps, for the tensor-product space entry points.
// ---------------------------------------------------------------------------

// Gauss-Legendre nodes (ascending) and weights in long double: Newton on P_N
// from the Chebyshev-like first guess, w = 2 / ((1 - x^2) P_N'(x)^2)
// (the nodes numpy's leggauss returns, Legendre.py:136-147).
static void gauss_legendre(int N, std::vector<LD>& x, std::vector<LD>& w) {
  x.assign(N, 0.0L);
  w.assign(N, 0.0L);
  const LD pi = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < N; ++i) {
    LD z = std::cos(pi * ((LD)i + 0.75L) / ((LD)N + 0.5L));
    LD dp = 1.0L;
    for (int it = 0; it < 100; ++it) {
      LD p0 = 1.0L, p1 = z;
      for (int n = 2; n <= N; ++n) {
        const LD p2 = ((2 * n - 1) * z * p1 - (n - 1) * p0) / n;
        p0 = p1;
        p1 = p2;
      }
      const LD pN = (N == 1) ? z : p1, pNm1 = (N == 1) ? 1.0L : p0;
      dp = N * (z * pN - pNm1) / (z * z - 1.0L);
      const LD dz = pN / dp;
      z -= dz;
      if (std::fabs((double)dz) < 1e-19) break;
    }
    // recompute the derivative at the converged node for the weight
    LD p0 = 1.0L, p1 = z;
    for (int n = 2; n <= N; ++n) {
      const LD p2 = ((2 * n - 1) * z * p1 - (n - 1) * p0) / n;
      p0 = p1;
      p1 = p2;
    }
    dp = N * (z * p1 - p0) / (z * z - 1.0L);
    x[N - 1 - i] = z;  // the guesses run from +1 down to -1
    w[N - 1 - i] = 2.0L / ((1.0L - z * z) * dp * dp);
  }
}

void build_x_basis(int family, int basis, int N, double x_lo, double x_hi, XBasis& xb) {
  xb.family = family;
  xb.basis = basis;
  xb.N = N;
  xb.nb = basis == 0 ? N : basis == 1 ? N - 2 : N - 4;
  const double Lx = x_hi - x_lo;
  xb.dfx = std::fabs(Lx - 2.0) < 1e-12 ? 1.0 : 2.0 / Lx;
  const LD df = xb.dfx, pi = 3.141592653589793238462643383279502884L;
  std::vector<LD> w(N);
  xb.X.assign(N, 0.0L);
  if (family == 0) {
    for (int j = 0; j < N; ++j) {
      xb.X[j] = std::cos(pi + (2.0L * j + 1.0L) * pi / (2.0L * N));
      w[j] = pi / N;
    }
  } else {
    gauss_legendre(N, xb.X, w);
  }
  xb.V.assign((size_t)N * N, 0.0L);
  for (int j = 0; j < N; ++j) {
    const LD x = xb.X[j];
    LD p0 = 1.0L, p1 = x;
    xb.V[(size_t)j * N] = 1.0L;
    if (N > 1) xb.V[(size_t)j * N + 1] = x;
    for (int n = 2; n < N; ++n) {
      const LD p2 = family == 0 ? 2.0L * x * p1 - p0 : ((2 * n - 1) * x * p1 - (n - 1) * p0) / n;
      xb.V[(size_t)j * N + n] = p2;
      p0 = p1;
      p1 = p2;
    }
  }
  xb.Q.assign((size_t)N * N, 0.0L);
  for (int n = 0; n < N; ++n)
    for (int j = 0; j < N; ++j) xb.Q[(size_t)n * N + j] = xb.V[(size_t)j * N + n] * w[j] / df;
  xb.ns.assign(N, 0.0L);
  for (int n = 0; n < N; ++n)
    xb.ns[n] = (family == 0 ? (n == 0 ? pi : pi / 2.0L) : 2.0L / (2.0L * n + 1.0L)) / df;
  // d/dX on coefficients: Chebyshev (T_j)' = sum_{i<j, j-i odd} (2/c_i) j T_i
  // (Chebyshev.py:319-353); Legendre (P_j)' = sum_{i<j, j-i odd} (2i+1) P_i
  // (Legendre.py:195-227)
  xb.D.assign((size_t)N * N, 0.0L);
  for (int i = 0; i < N; ++i)
    for (int j = i + 1; j < N; j += 2)
      xb.D[(size_t)i * N + j] = family == 0 ? (i == 0 ? (LD)j : 2.0L * j) : 2.0L * i + 1.0L;
  xb.S.assign((size_t)xb.nb * N, 0.0L);
  for (int i = 0; i < xb.nb; ++i) {
    const LD n = i;
    xb.S[(size_t)i * N + i] = 1.0L;
    if (basis == 1) {
      xb.S[(size_t)i * N + i + 2] = -1.0L;
    } else if (basis == 2) {
      if (family == 0) {
        xb.S[(size_t)i * N + i + 2] = 2.0L * (-n - 2.0L) / (n + 3.0L);
        xb.S[(size_t)i * N + i + 4] = (n + 1.0L) / (n + 3.0L);
      } else {
        xb.S[(size_t)i * N + i + 2] = 2.0L * (-2.0L * n - 5.0L) / (2.0L * n + 7.0L);
        xb.S[(size_t)i * N + i + 4] = (2.0L * n + 3.0L) / (2.0L * n + 7.0L);
      }
    }
  }
}

std::vector<double> x_map_matrix(const XBasis& xb, int map, int k, int* rows, int* cols) {
  const int N = xb.N, nb = xb.nb;
  LMat V(N, N), Q(N, N), D(N, N), S(nb, N), W(N, N), Dk(N, N);
  V.v = xb.V;
  Q.v = xb.Q;
  D.v = xb.D;
  S.v = xb.S;
  for (int n = 0; n < N; ++n) {
    W(n, n) = xb.ns[n];
    Dk(n, n) = 1.0L;
  }
  LD scale = 1.0L;
  for (int t = 0; t < k; ++t) {
    Dk = mul(D, Dk);
    scale *= (LD)xb.dfx;
  }
  const LMat St = transpose(S);
  auto mass_inv = [&]() { return inverse(mul(mul(S, W), St)); };
  LMat R(1, 1);
  switch (map) {
    case kXBackward: R = mul(mul(V, Dk), St); break;
    case kXToOrth: R = St; break;
    case kXDiffOrth: R = Dk; break;
    case kXProjectOrth: R = mul(mass_inv(), mul(S, W)); break;
    case kXSpFromOrth: R = mul(S, W); break;
    case kXForward: R = mul(mass_inv(), mul(S, Q)); break;
    case kXScalarProd: R = mul(S, Q); break;
    default: R = mul(mul(mul(S, W), Dk), St); break;  // kXGalerkin
  }
  if (map == kXBackward || map == kXDiffOrth || map == kXGalerkin)
    for (LD& v : R.v) v *= scale;
  *rows = R.r;
  *cols = R.c;
  std::vector<double> o(R.v.size());
  for (size_t i = 0; i < o.size(); ++i) o[i] = (double)R.v[i];
  return o;
}

void build_tps_x_operators(const HostOperators& op, int basis, TpsX& t) {
  const int N = op.N;
  const int nb = basis == 0 ? N : basis == 1 ? N - 2 : N - 4;
  LMat V = from_dense(op.V, N, N), Q = from_dense(op.Q, N, N), W(N, N), S(nb, N);
  for (int n = 0; n < N; ++n) W(n, n) = (LD)op.ns[n];
  if (basis == 0) {
    for (int i = 0; i < N; ++i) S(i, i) = 1.0L;
  } else {
    const Stencil& st = basis == 1 ? op.SD : op.SB;
    for (int i = 0; i < nb; ++i) {
      S(i, i) = st.s0[i];
      S(i, i + 2) = st.s2[i];
      if (basis == 2) S(i, i + 4) = st.s4[i];
    }
  }
  const LMat St = transpose(S);
  const LMat Minv = inverse(mul(mul(S, W), St));
  auto dense = [](const LMat& M) {
    std::vector<double> o((size_t)M.r * M.c);
    for (size_t k = 0; k < o.size(); ++k) o[k] = (double)M.v[k];
    return o;
  };
  t.N = N;
  t.nb = nb;
  t.B = dense(mul(V, St));
  t.Sq = dense(mul(S, Q));
  t.F = dense(mul(Minv, mul(S, Q)));
  if (basis == 0) {
    // (T_i, T_j^(k))_w with the df^(k-1) domain scaling
    std::vector<double> T0 = chebyshev_galerkin(N, 0), T2 = chebyshev_galerkin(N, 2);
    for (double& v : T0) v /= op.dfx;
    for (double& v : T2) v *= op.dfx;
    t.G0 = T0;
    t.G2 = T2;
  } else if (basis == 1) {
    t.G0 = op.XD0;
    t.G2 = op.XD2;
  } else {
    t.G0 = op.XB0;
    t.G2 = op.XB2;
  }
}

}  // namespace jfb
