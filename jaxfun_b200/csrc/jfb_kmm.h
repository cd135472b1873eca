// Internal declarations of the KMM plane-Couette plan (not part of the C ABI).
#pragma once

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
  double dfx = 1, dfy = 1, dfz = 1;
  std::vector<double> xnodes, xphys;  // reference / physical Gauss nodes
  std::vector<double> V;              // V[j][n] = T_n(X_j)
  std::vector<double> Q;              // Q[n][j] = T_n(X_j) pi / N / df
  std::vector<double> ns;             // Chebyshev norms^2 / df
  Stencil SB, SD;
  std::vector<double> XB0, XB2, XB4, XD0, XD2;  // dense Galerkin x-matrices
  std::vector<double> mlo, mdi, mhi;            // Dirichlet mass (= M00) tri-band
  std::vector<double> lu_l, lu_u;               // its no-pivot LU
  // biharmonic mass (offsets -4..4) no-pivot LU: L[i,i-2], L[i,i-4], U[i,i], U[i,i+2], U[i,i+4]
  std::vector<double> bl2, bl4, bu0, bu2, bu4;
  std::vector<double> fejer;  // Fejer-I weights on the Gauss nodes / df
};

Stencil make_stencil(int N, bool biharmonic);
void build_host_operators(const jfb_kmm_config& cfg, HostOperators& op);
void mode_coefficients(const HostOperators& op, const jfb_kmm_config& cfg, int ky,
                       int kz, double gamma, bool biharmonic, double out[3]);

}  // namespace jfb
