// Internal declarations of the KMM plane-Couette plan (not part of the C ABI).
#pragma once

#include <string>
#include <vector>

#include "../../include/jfb200.h"

namespace jfb {

struct Stencil {
  int n = 0;      // number of composite dofs (N - width)
  int width = 0;  // 2 (Dirichlet) or 4 (biharmonic)
  std::vector<double> s0, s2, s4;  // S[i, i], S[i, i+2], S[i, i+4]
};

struct HostOperators {
  int N = 0, nB = 0, nD = 0;
  int family = 0;                     // 0 Chebyshev, 1 Legendre (JFB_FAMILY_*)
  double x_lo = -1, x_hi = 1;
  double dfx = 1, dfy = 1, dfz = 1;
  std::vector<double> xnodes, xphys;  // reference / physical Gauss nodes
  std::vector<double> V;              // V[j][n] = P_n(X_j) (T_n or L_n)
  std::vector<double> Q;              // Q[n][j] = P_n(X_j) w_j / df
  std::vector<double> ns;             // norms^2 (P_n, P_n) / df
  Stencil SB, SD;
  std::vector<double> XB0, XB2, XB4, XD0, XD2;  // dense Galerkin x-matrices
  std::vector<double> mlo, mdi, mhi;            // Dirichlet mass (= M00) tri-band
  std::vector<double> lu_l, lu_u;               // its no-pivot LU
  // biharmonic mass (offsets -4..4) no-pivot LU: L[i,i-2], L[i,i-4], U[i,i], U[i,i+2], U[i,i+4]
  std::vector<double> bl2, bl4, bu0, bu2, bu4;
  // physical-volume quadrature weights on the Gauss nodes / df: Fejer-I
  // (Chebyshev.py:182-208) or the Gauss-Legendre weights (Legendre.py:136-147)
  std::vector<double> fejer;
};

// Parity-split x-operators of the step in mma.sync m8n8k4 fragment order.
// Sub-matrix ids (rows x columns in the half spaces; E/O = symmetric /
// antisymmetric physical half, e/o = even / odd coefficient half):
//   Nu/Ng right-hand sides   gNuE, gNuO, gNgE, gNgO   (physical -> coefficient)
//   mass rows of Su / Sg     gMuE, gMuO, gMgE, gMgO   (coefficient -> coefficient)
//   velocity / vorticity     gA0Ee ... gB1Oo          (coefficient -> physical)
//   gradient form: d/dx u0   gA1Oe, gA1Eo (A1 = V D S_B^T; empty otherwise)
enum GemmSub {
  gNuE, gNuO, gNgE, gNgO, gMuE, gMuO, gMgE, gMgO,
  gA0Ee, gP2Ee, gP1Oe, gP1Eo, gA0Oo, gP2Oo, gB1Ee, gB2Oe, gB2Eo, gB1Oo,
  gA1Oe, gA1Eo,
  gNumSub
};

struct GemmHost {
  int Jh = 0, Jl = 0, nBe = 0, nBo = 0, nDe = 0, nDo = 0;
  std::vector<double> frag;   // fragment-tiled sub-matrices
  std::vector<int> krange;    // per sub-matrix and row tile: [first k tile, end k tile)
  int off[gNumSub], mt[gNumSub], kt[gNumSub], kr[gNumSub];
  std::vector<double> R3;     // S_D Q (nD x N): mean-flow nonlinear rows
  std::vector<double> X2D;    // (T_i, phi_j'')_w of the Dirichlet basis (nD x nD)
  // middle Gauss node of an odd N: rows of A0 (even cols), P2 (even), P1 (odd),
  // B1 (even), B2 (odd), A1 (odd; gradient form), each padded to mid_stride
  std::vector<double> mid;
  int mid_stride = 0;
  // MHD: x-physical values (N x nD, row-major) of a Dirichlet-basis field and
  // of TD projections of its derivatives: B1 = V S_D^T, B2 = V D S_D^T,
  // C1 = V S_D^T M_D^-1 S_D W D S_D^T, C2 = V S_D^T M_D^-1 S_D W D^2 S_D^T
  std::vector<double> B1, B2, C1, C2;
  // P1 = B1 F, P2 = B2 F (N x nB, row-major): velocity from u0 (phase D)
  std::vector<double> P1, P2;
  // Adjoint of the step: A0 = V S_B^T (N x nB), F = M_D^-1 S_D W D S_B^T
  // (nD x nB, the TD projection of d/dx of a TB field), the nonlinear-row
  // operators R0 = S_B W Pi, R1 = S_B W D Pi (nB x N), R2 = S_D W Pi (nD x N)
  // with Pi = S_D^T M_D^-1 S_D Q, and the energy Gram matrices
  // GB = A0^T diag(w) A0 (nB x nB), GD = B1^T diag(w) B1 (nD x nD), w the
  // Fejer weights.  All row-major.
  std::vector<double> A0, F, R0, R1, R2, GB, GD;
};

// x-axis operators of a standalone tensor-product space (row-major):
// backward B = V S^T (N x nb), forward (L2 projection) F = M^-1 S Q (nb x N),
// scalar product Sq = S Q (nb x N), Galerkin G0 = (phi_i, phi_j)_w and
// G2 = (phi_i, phi_j'')_w (nb x nb, domain-scaled).  basis: 0 orthogonal
// Chebyshev, 1 Dirichlet (T_k - T_{k+2}), 2 biharmonic.
struct TpsX {
  int N = 0, nb = 0;
  std::vector<double> B, F, Sq, G0, G2;
};
void build_tps_x_operators(const HostOperators& op, int basis, TpsX& t);

// 1-D data of the wall-normal basis of a standalone tensor-product space,
// in long double, row-major: V[j][n] = P_n(X_j) on the family's Gauss nodes,
// Q[n][j] = P_n(X_j) w_j / df (scalar products), ns[n] = (P_n, P_n) / df,
// D[i][j] the coefficients of d/dX (P_j)' = sum_i D[i][j] P_i, and the Shen
// stencil S (nb x N; the identity for the orthogonal basis).
// family: 0 Chebyshev (Chebyshev.py), 1 Legendre (Legendre.py);
// basis: 0 orthogonal, 1 Dirichlet, 2 biharmonic (composite.py:797-864).
struct XBasis {
  int family = 0, basis = 0, N = 0, nb = 0;
  double dfx = 1.0;
  std::vector<long double> X, V, Q, ns, D, S;
};
void build_x_basis(int family, int basis, int N, double x_lo, double x_hi, XBasis& xb);

// Separable x-axis maps of a standalone space (row-major double matrices).
enum XMap {
  kXBackward = 0,      // V D^k S^T df^k            (N x nb)  backward_primitive
  kXToOrth = 1,        // S^T                       (N x nb)  to_orthogonal
  kXDiffOrth = 2,      // D^k df^k                  (N x N)   differentiate_orthogonal_coeffs
  kXProjectOrth = 3,   // M^-1 S diag(ns)           (nb x N)  project_from_orthogonal
  kXSpFromOrth = 4,    // S diag(ns)                (nb x N)  scalar_product_from_orthogonal
  kXForward = 5,       // M^-1 S Q                  (nb x N)  forward (L2 projection)
  kXScalarProd = 6,    // S Q                       (nb x N)  scalar_product
  kXGalerkin = 7,      // S diag(ns) D^k S^T df^k   (nb x nb) (phi_i, phi_j^(k))_w
};
std::vector<double> x_map_matrix(const XBasis& xb, int map, int k, int* rows, int* cols);

Stencil make_stencil(int N, bool biharmonic, int family = 0);
// Builds GemmHost from the 1-D operators; returns false (with a message) if a
// parity property the split relies on does not hold.
bool build_gemm_operators(const HostOperators& op, GemmHost& gh, std::string& err,
                          bool gradient = false);
void build_host_operators(const jfb_kmm_config& cfg, HostOperators& op);
void mode_coefficients(const HostOperators& op, const jfb_kmm_config& cfg, int ky,
                       int kz, double gamma, bool biharmonic, double out[3]);

}  // namespace jfb
