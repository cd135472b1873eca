// MHD part of the plane-Couette step (examples/pcf_mhd_jax.py, conducting
// walls): the vector potential A in the Dirichlet basis (TD^3), B = curl A in
// (TD, TC, TC), J = curl B in (TC, TD, TD), the Lorentz force -J x B in the
// momentum nonlinear term and the EMF (u + U_b e_y) x B driving A.
//
// mhd_a_kernel, one CTA per 16 pencils (the +ky / -ky x 8 kz tiles of the
// flow kernel), three modes:
//   kMhdStep: N_A = Myz S_D Q EMF per component (_A_mass_rhs of the forward-
//     projected EMF, pcf_mhd_jax.py:157-170, 339-357; the mass of a projection
//     is the scalar product), right-hand sides
//       MA comb + gamma eta Myz (X2_D - k^2 X0_D) A_a + dt (d0 N_A + d1 N_A' + d2 N_A'')
//     (sbdf3.py:15-41, pcf_mhd_jax.py:519-530 and 643-715), the solves with
//     SA = MA - gamma LA per wavenumber (banded forward elimination, then the
//     explicit inverse of the upper factor), then b and j of the new A at the
//     x nodes;
//   kMhdFields: b and j of A as given (the state's own nonlinear terms);
//   kMhdFromPhys: A = TD.forward of physical samples already transformed in
//     y and z (_A_state_from_physical, pcf_mhd_jax.py:210-215): S_D Q v, then
//     the Dirichlet mass solve.
// b and j at the x nodes (update_B_from_A / update_J_from_B,
// pcf_mhd_jax.py:269-312, then a backward transform in x):
//   b_x = B1 (i ky A_z - i kz A_y),   b_y = i kz B1 A_x - B2 A_z,
//   b_z = B2 A_y - i ky B1 A_x,
//   j_x = i ky B2 A_y + k^2 B1 A_x + i kz B2 A_z,
//   j_y = kz^2 B1 A_y - ky kz B1 A_z - C2 A_y + i ky C1 A_x,
//   j_z = i kz C1 A_x - C2 A_z + ky^2 B1 A_z - ky kz B1 A_y,
// with B1 = V S_D^T, B2 = V D S_D^T and C1, C2 the x samples of the TD
// projections of D S_D^T and D^2 S_D^T (TC components need no projection and
// the TD projection of a TD field is the identity).  Rows are evaluated in
// mirror pairs x_j, x_{N-1-j}: a column of B1 or C2 has the parity of its
// index, a column of B2 or C1 the opposite one.
#pragma once

#include "jfb_kmm_gemm.cuh"
#include "jfb_kmm_kernels.cuh"

namespace jfb {

struct MhdOps {
  const double* R3;   // S_D Q, nD x N
  const double* X2D;  // nD x nD
  const double* B1;   // N x nD
  const double* B2;
  const double* C1;
  const double* C2;
  int Jh, Jl, nDe, nDo;
};

enum MhdMode { kMhdStep = 0, kMhdFields = 1, kMhdFromPhys = 2 };

// Imposed uniform field B0 (added to b in the Lorentz force and the EMF) and
// the Coriolis term of a rotating frame, n += -2 Omega e_z x u
// (pcf_mhd_mri_shearpy_jax.py:149-176).
struct MhdPhys {
  double b0x, b0y, b0z;
  double two_omega;
  double uw_emf;  // U_wall of the base flow in the EMF (U_b = uw_emf x)
};

struct MhdArgs {
  int mode;
  const c64* HXA;  // EMF (kMhdStep) or physical samples (kMhdFromPhys): 3 x [Nx][P]
  double c0, c1, c2, d0, d1, d2, slin;  // slin = gamma * eta
  const c64 *Aa, *Ab, *Ac;              // levels: 3 x [nD][P] each
  const c64 *NAp, *NAq;
  c64* NA_out;
  const double* sa;  // SA records: L pairs, inverse upper triangles per parity
  int sa_rec;
  c64* A_out;
  c64* XB;  // b, j at the x nodes: 6 x [Nx][P] (null: not wanted)
  int* status;  // plan status word (kStatusNonFinite)
  int x32;      // mixed form: HXA (the EMF) is read and XB written as complex64
  // U_b e_y x B0 = x (U_wall B0z, 0, -U_wall B0x): a function of x alone, so
  // only the (ky, kz) = (0, 0) mode of the EMF; added here in FP64 (the z
  // stage leaves it out, so that no O(1) constant enters the transforms)
  double uw_b0z, uw_b0x;
};

constexpr int kMhdThreads = 512;
constexpr int kMhdW = 16;  // pencils per CTA

inline size_t mhd_smem_bytes(int nD, int N) {
  // right-hand sides and solutions (3 components x nD rows x 16 pencils),
  // then the tile's x samples (3 components x N rows x 16 pencils)
  return ((size_t)2 * 3 * nD + (size_t)3 * N) * kMhdW * sizeof(c64);
}

// The A stage of tile `bid` (the kernel below, or one member's tile of the
// ensemble kernel).
__device__ __forceinline__ void mhd_a_body(const Dims& d, const DevOps& o, const MhdOps& M,
                                           const MhdArgs& a, const int bid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_p[kMhdW], s_mode[kMhdW];
  __shared__ double s_ky[kMhdW], s_kz[kMhdW];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int NWp = kMhdThreads / 32;
  const int nKc = (d.Kz + 7) / 8;
  const int kyi = bid / nKc, kz0 = (bid % nKc) * 8;
  const int N = d.Nx, nD = d.nD, Jh = M.Jh, Jl = M.Jl;
  const size_t P = (size_t)d.P;
  c64* RHS = reinterpret_cast<c64*>(smem_raw);  // [3][nD][kMhdW], split parity order
  c64* SOL = RHS + (size_t)3 * nD * kMhdW;       // [3][nD][kMhdW], split parity order
  c64* HS = SOL + (size_t)3 * nD * kMhdW;        // [3][N][kMhdW]: the tile's x samples
  // split parity order: even rows first, then odd rows
  auto srow = [&](int i) { return (i & 1) ? M.nDe + (i >> 1) : (i >> 1); };

  if (tid < kMhdW) {
    const int side = tid >> 3, kz = kz0 + (tid & 7);
    int p = -1, mode = 0;
    double kyp = 0.0, kzp = 0.0;
    if (kz < d.Kz && !(side == 1 && kyi == 0)) {
      const int row = side ? d.Ny - kyi : kyi;
      p = row * d.Kz + kz;
      mode = kyi * d.Kz + kz;
      kyp = (side ? -kyi : kyi) * d.dfy;
      kzp = kz * d.dfz;
    }
    s_p[tid] = p;
    s_mode[tid] = mode;
    s_ky[tid] = kyp;
    s_kz[tid] = kzp;
  }
  __syncthreads();

  if (a.mode != kMhdFields) {
    // the tile's x samples, read once into shared memory (every row i of the
    // scalar products uses all of them)
    for (int e = tid; e < 3 * N * kMhdW; e += kMhdThreads) {
      const int w = e % kMhdW, cj = e / kMhdW;  // cj = c N + j
      const int p = s_p[w];
      c64 v = cmk(0.0, 0.0);
      if (p >= 0) {
        if (a.x32) {
          const c32 h = reinterpret_cast<const c32*>(a.HXA)[(size_t)cj * P + p];
          v = cmk((double)h.re, (double)h.im);
        } else {
          v = a.HXA[(size_t)cj * P + p];
        }
        if (p == 0 && a.mode == kMhdStep) {
          const int c = cj / N;
          const double x = o.xphys[cj - c * N];
          if (c == 0) v.re += a.uw_b0z * x;
          else if (c == 2) v.re -= a.uw_b0x * x;
        }
      }
      HS[e] = v;
    }
    __syncthreads();
    // 1. scalar products S_D Q v of the three x profiles (mirror sums), and
    //    for a step the right-hand sides; one thread per (comp, row, pencil)
    const bool step = a.mode == kMhdStep;
    for (int e = tid; e < 3 * nD * kMhdW; e += kMhdThreads) {
      const int w = e % kMhdW, i = (e / kMhdW) % nD, c = e / (kMhdW * nD);
      const int p = s_p[w];
      c64 rhs = cmk(0.0, 0.0);
      if (p >= 0) {
        const c64* h = HS + (size_t)c * N * kMhdW + w;  // row j at h[j kMhdW]
        const double* r3 = M.R3 + (size_t)i * N;
        const double sg = (i & 1) ? -1.0 : 1.0;
        c64 s0 = cmk(0.0, 0.0), s1 = s0;
        for (int j = 0; j < Jl; ++j) {
          const c64 x = h[j * kMhdW] + sg * h[(N - 1 - j) * kMhdW];
          if (j & 1) s1 = s1 + __ldg(r3 + j) * x;
          else s0 = s0 + __ldg(r3 + j) * x;
        }
        if ((N & 1) && !(i & 1)) s0 = s0 + __ldg(r3 + Jl) * h[Jl * kMhdW];
        if (!step) {
          rhs = s0 + s1;
        } else {
          const c64 na = d.Myz * (s0 + s1);
          const size_t gi = ((size_t)c * nD + i) * P + p;
          if (a.NA_out) a.NA_out[gi] = na;
          c64 nl = a.d0 * na;
          if (a.NAp && a.d1 != 0.0) nl = nl + a.d1 * a.NAp[gi];
          if (a.NAq && a.d2 != 0.0) nl = nl + a.d2 * a.NAq[gi];
          auto comb = [&](int k) {
            const size_t gk = ((size_t)c * nD + k) * P + p;
            c64 v = a.c0 * a.Aa[gk];
            if (a.Ab && a.c1 != 0.0) v = v + a.c1 * a.Ab[gk];
            if (a.Ac && a.c2 != 0.0) v = v + a.c2 * a.Ac[gk];
            return v;
          };
          auto aa = [&](int k) { return a.Aa[((size_t)c * nD + k) * P + p]; };
          // X0_D f: the Dirichlet mass tri-band (offsets -2, 0, 2)
          auto band = [&](auto f) {
            c64 r = o.mdi[i] * f(i);
            if (i >= 2) r = r + o.mlo[i] * f(i - 2);
            if (i + 2 < nD) r = r + o.mhi[i] * f(i + 2);
            return r;
          };
          c64 mass = band(comb);
          if (a.slin != 0.0) {
            const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
            c64 x2 = cmk(0.0, 0.0);
            for (int k = i; k < nD; k += 2) x2 = x2 + __ldg(M.X2D + (size_t)i * nD + k) * aa(k);
            mass = mass + a.slin * (x2 - k2 * band(aa));
          }
          rhs = d.Myz * mass + d.dt * nl;
        }
      }
      RHS[((size_t)c * nD + srow(i)) * kMhdW + w] = rhs;
    }
    __syncthreads();
    if (step) {
      // 2a. forward elimination with the unit lower factor (offsets -2, -4 in
      //     the full order = -1, -2 within a parity class), one thread per
      //     (comp, pencil, parity)
      if (tid < 3 * kMhdW * 2) {
        const int w = tid % kMhdW, c = (tid / kMhdW) % 3, par = tid / (3 * kMhdW);
        if (s_p[w] >= 0) {
          const double* rec = a.sa + (size_t)s_mode[w] * a.sa_rec;
          const int m = par ? nD / 2 : (nD + 1) / 2;
          c64* y = RHS + ((size_t)c * nD + (par ? M.nDe : 0)) * kMhdW + w;
          forward_elim(rec, par, m, y, kMhdW);  // multipliers loaded ahead of their rows
        }
      }
      __syncthreads();
      // 2b. x = U^-1 y, one warp per (comp, wavenumber column, parity); the
      //     +ky and -ky pencils of a column share the record; lane = row
      for (int task = warp; task < 3 * 8 * 2; task += NWp) {
        const int ms = task % 8, c = (task / 8) % 3, par = task / 24;
        if (s_p[ms] < 0) continue;
        const int m0 = (nD + 1) / 2, m = par ? nD / 2 : m0;
        const double* tri =
            a.sa + (size_t)s_mode[ms] * a.sa_rec + 2 * nD + (par ? m0 * (m0 + 1) / 2 : 0);
        const c64* y = RHS + ((size_t)c * nD + (par ? M.nDe : 0)) * kMhdW;
        c64* x = SOL + ((size_t)c * nD + (par ? M.nDe : 0)) * kMhdW;
        const bool other = s_p[ms + 8] >= 0;
        for (int r0 = 0; r0 < m; r0 += 32) {
          const int r = r0 + lane;
          c64 s0 = cmk(0.0, 0.0), s1 = s0;
          if (r < m) {
            for (int cc = r; cc < m; ++cc) {
              const double u = __ldg(tri + (size_t)cc * (cc + 1) / 2 + r);
              s0 = s0 + u * y[cc * kMhdW + ms];
              s1 = s1 + u * y[cc * kMhdW + ms + 8];
            }
            x[r * kMhdW + ms] = s0;
            x[r * kMhdW + ms + 8] = other ? s1 : cmk(0.0, 0.0);
          }
        }
      }
    } else {
      // 2. Dirichlet mass solve (tri-band LU), one thread per (comp, pencil, parity)
      if (tid < 3 * kMhdW * 2) {
        const int w = tid % kMhdW, c = (tid / kMhdW) % 3, par = tid / (3 * kMhdW);
        const int m = par ? nD / 2 : (nD + 1) / 2;
        const c64* y = RHS + ((size_t)c * nD + (par ? M.nDe : 0)) * kMhdW + w;
        c64* x = SOL + ((size_t)c * nD + (par ? M.nDe : 0)) * kMhdW + w;
        for (int r = 0; r < m; ++r) {
          const int i = 2 * r + par;
          c64 v = y[r * kMhdW];
          if (r > 0) v = v - o.lul[i] * x[(r - 1) * kMhdW];
          x[r * kMhdW] = v;
        }
        for (int r = m - 1; r >= 0; --r) {
          const int i = 2 * r + par;
          c64 v = x[r * kMhdW];
          if (r + 1 < m) v = v - o.mhi[i] * x[(r + 1) * kMhdW];
          x[r * kMhdW] = o.luu[i] * v;
        }
      }
    }
    __syncthreads();
    bool bad = false;
    for (int e = tid; e < 3 * nD * kMhdW; e += kMhdThreads) {
      const int w = e % kMhdW, i = (e / kMhdW) % nD, c = e / (kMhdW * nD);
      if (s_p[w] >= 0) {
        const c64 v = SOL[((size_t)c * nD + srow(i)) * kMhdW + w];
        bad |= !finite_c(v);
        a.A_out[((size_t)c * nD + i) * P + s_p[w]] = v;
      }
    }
    flag_nonfinite(a.status, bad);
  } else {
    for (int e = tid; e < 3 * nD * kMhdW; e += kMhdThreads) {
      const int w = e % kMhdW, i = (e / kMhdW) % nD, c = e / (kMhdW * nD);
      SOL[((size_t)c * nD + srow(i)) * kMhdW + w] =
          (s_p[w] >= 0) ? a.Aa[((size_t)c * nD + i) * P + s_p[w]] : cmk(0.0, 0.0);
    }
  }
  if (!a.XB) return;
  __syncthreads();

  // 3. b and j at the nodes x_j and x_{N-1-j}, one thread per (j < Jh, pencil)
  for (int e = tid; e < Jh * kMhdW; e += kMhdThreads) {
    const int w = e % kMhdW, j = e / kMhdW, jm = N - 1 - j;
    const int p = s_p[w];
    if (p < 0) continue;
    const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
    c64 S[6], A[6];  // mirror-symmetric and antisymmetric parts
#pragma unroll
    for (int f = 0; f < 6; ++f) S[f] = A[f] = cmk(0.0, 0.0);
    const double* b1r = M.B1 + (size_t)j * nD;
    const double* b2r = M.B2 + (size_t)j * nD;
    const double* c1r = M.C1 + (size_t)j * nD;
    const double* c2r = M.C2 + (size_t)j * nD;
    for (int k = 0; k < nD; ++k) {
      const int rk = srow(k);
      const c64 ax = SOL[((size_t)0 * nD + rk) * kMhdW + w];
      const c64 ay = SOL[((size_t)1 * nD + rk) * kMhdW + w];
      const c64 az = SOL[((size_t)2 * nD + rk) * kMhdW + w];
      const double b1 = __ldg(b1r + k), b2 = __ldg(b2r + k);
      const double c1 = __ldg(c1r + k), c2 = __ldg(c2r + k);
      const c64 zero = cmk(0.0, 0.0);
      // column k's contribution per operator, field order (b_x, b_y, b_z, j_x, j_y, j_z)
      const c64 tB1[6] = {mul_i(ky * az - kz * ay), mul_i(kz * ax), mul_i(-ky * ax), k2 * ax,
                          kz * kz * ay - ky * kz * az, ky * ky * az - ky * kz * ay};
      const c64 tB2[6] = {zero, cmk(-az.re, -az.im), ay, mul_i(ky * ay + kz * az), zero, zero};
      const c64 tC1[6] = {zero, zero, zero, zero, mul_i(ky * ax), mul_i(kz * ax)};
      const c64 tC2[6] = {zero, zero, zero, zero, cmk(-ay.re, -ay.im), cmk(-az.re, -az.im)};
      const bool even = (k & 1) == 0;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        const c64 ev = b1 * tB1[f] + c2 * tC2[f];  // parity of k
        const c64 od = b2 * tB2[f] + c1 * tC1[f];  // parity of k + 1
        if (even) {
          S[f] = S[f] + ev;
          A[f] = A[f] + od;
        } else {
          S[f] = S[f] + od;
          A[f] = A[f] + ev;
        }
      }
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      const size_t e0 = (size_t)f * N * P + p;
      const c64 vj = S[f] + A[f], vm = S[f] - A[f];
      if (a.x32) {
        c32* X = reinterpret_cast<c32*>(a.XB) + e0;
        X[(size_t)j * P] = cmk((float)vj.re, (float)vj.im);
        if (jm != j) X[(size_t)jm * P] = cmk((float)vm.re, (float)vm.im);
      } else {
        c64* X = a.XB + e0;
        X[(size_t)j * P] = vj;
        if (jm != j) X[(size_t)jm * P] = vm;
      }
    }
  }
}

__global__ void __launch_bounds__(kMhdThreads, 1)
    mhd_a_kernel(const __grid_constant__ Dims d, const __grid_constant__ DevOps o,
                 const __grid_constant__ MhdOps M, const __grid_constant__ MhdArgs a) {
  mhd_a_body(d, o, M, a, blockIdx.x);
}

// ---------------------------------------------------------------------------
// z stage of the coupled step, per group of kZRows (x, y) rows: twelve half
// spectra (u, omega, b, j) -> six packed complex inverse FFTs, the products
//   n = -(u_t x omega_t) - j x (b + B0) - 2 Omega e_z x u,
//   emf = (u + U_b e_y) x (b + B0)
// (_mhd_convection, pcf_mhd_jax.py:339-357; the flow part in the split form
// of rotational_product, whose constant base-flow term the y stage adds;
// B0 the imposed field and Omega the rotation of MhdPhys,
// pcf_mhd_mri_shearpy_jax.py:149-176), then three packed forward
// transforms: HZ fields (n_x, n_y, n_z, e_x, e_y, e_z).  The products are
// expanded so that no O(1) value (B0, U_b) is added to a perturbation value
// before a product: in FP32 (the mixed form) every term keeps the
// perturbation's digits.  The EMF's term U_b e_y x B0, a function of x
// alone, is left to mhd_a_kernel (FP64, mean pencil).  In the mixed form the
// flow's base-flow terms are left out here too (d.uwall = 0; the pencil
// stage adds them in FP64), the EMF's U_b e_y x b is not (ph.uw_emf).
// ---------------------------------------------------------------------------
// The z stage of rows [bid kZRows, (bid + 1) kZRows) (the kernel below, or
// one member's rows of the ensemble kernel).
template <typename T>
__device__ __forceinline__ void z_cross_mhd_body(const DevOps& o, const Dims& d,
                                                 const MhdPhys& ph, const FFTPlan& plan,
                                                 const cpx<T>* __restrict__ tw,
                                                 const cpx<T>* __restrict__ Y,
                                                 cpx<T>* __restrict__ HZ, const int bid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = kZRows * 6;   // packed input columns
  constexpr int NCf = kZRows * 3;  // packed output columns
  cpx<T>* A = reinterpret_cast<cpx<T>*>(smem_raw);
  cpx<T>* B = A + d.Mz * NC;
  const int row0 = bid * kZRows;  // row = j * My + y
  const int nrows = d.Nx * d.My;
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  // k fastest: a warp reads consecutive spectral values of one row and field
  for (int idx = threadIdx.x; idx < d.Mz * NC; idx += blockDim.x) {
    const int k = idx % d.Mz, c = idx / d.Mz;
    const int rl = c / 6, pr = c % 6;
    const int row = row0 + rl;
    cpx<T> z = cmk(T(0), T(0));
    if (row < nrows) {
      const cpx<T>* fa = Y + (size_t)(2 * pr) * plane + (size_t)row * d.Kz;
      const cpx<T>* fb = Y + (size_t)(2 * pr + 1) * plane + (size_t)row * d.Kz;
      if (k == 0) {
        z = cmk(fa[0].re, fb[0].re);
      } else if (k < d.Kz) {
        const cpx<T> xa = fa[k], xb = fb[k];
        z = cmk(xa.re - xb.im, xa.im + xb.re);
      } else if (k > d.Mz - d.Kz) {
        const int kk = d.Mz - k;
        const cpx<T> xa = fa[kk], xb = fb[kk];  // conj(xa) + i conj(xb)
        z = cmk(xa.re + xb.im, -xa.im + xb.re);
      }
    }
    A[k * NC + c] = z;
  }
  __syncthreads();
  cpx<T>* phys = fft_columns<T>(A, B, plan, NC, NC, tw, +1);
  cpx<T>* other = (phys == A) ? B : A;
  const T bx = T(ph.b0x), by = T(ph.b0y), bz = T(ph.b0z), tw2 = T(ph.two_omega);
  for (int idx = threadIdx.x; idx < d.Mz * kZRows; idx += blockDim.x) {
    const int rl = idx % kZRows, n = idx / kZRows;
    const int row = row0 + rl;
    const int j = (row < nrows) ? row / d.My : 0;
    const cpx<T>* z = phys + n * NC + rl * 6;
    const T u0 = z[0].re, u1 = z[0].im, u2 = z[1].re;
    const T w0 = z[1].im, w1 = z[2].re, w2 = z[2].im;
    const T b0 = z[3].re, b1 = z[3].im, b2 = z[4].re;
    const T j0 = z[4].im, j1 = z[5].re, j2 = z[5].im;
    const T ub = T(d.uwall * o.xphys[j]), ue = T(ph.uw_emf * o.xphys[j]);
    T n0, n1, n2;
    rotational_product(u0, u1, u2, w0, w1, w2, ub, T(d.uwall), n0, n1, n2);
    n0 -= tw2 * u1;
    n1 += tw2 * u0;
    n0 -= (j1 * b2 - j2 * b1) + (j1 * bz - j2 * by);
    n1 -= (j2 * b0 - j0 * b2) + (j2 * bx - j0 * bz);
    n2 -= (j0 * b1 - j1 * b0) + (j0 * by - j1 * bx);
    const T e0 = (u1 * b2 - u2 * b1) + (u1 * bz - u2 * by) + ue * b2;
    const T e1 = (u2 * b0 - u0 * b2) + (u2 * bx - u0 * bz);
    const T e2 = (u0 * b1 - u1 * b0) + (u0 * by - u1 * bx) - ue * b0;
    cpx<T>* out = other + n * NCf + rl * 3;
    out[0] = cmk(n0, n1);
    out[1] = cmk(n2, e0);
    out[2] = cmk(e1, e2);
  }
  __syncthreads();
  cpx<T>* spec = fft_columns<T>(other, phys, plan, NCf, NCf, tw, -1);
  const T scale = T(1.0 / d.Mz), h = T(0.5);
  for (int idx = threadIdx.x; idx < d.Kz * kZRows * 6; idx += blockDim.x) {
    const int k = idx % d.Kz;
    const int rf = idx / d.Kz;
    const int f = rf % 6, rl = rf / 6;
    const int row = row0 + rl;
    if (row >= nrows) continue;
    const int col = rl * 3 + f / 2;
    const cpx<T> Zk = spec[k * NCf + col];
    const cpx<T> Zm = spec[((d.Mz - k) % d.Mz) * NCf + col];
    // x + i y packed: X_k = (Z_k + conj Z_-k)/2, Y_k = (Z_k - conj Z_-k)/(2i)
    cpx<T> v;
    if ((f & 1) == 0) v = cmk(h * (Zk.re + Zm.re), h * (Zk.im - Zm.im));
    else v = cmk(h * (Zk.im + Zm.im), -h * (Zk.re - Zm.re));
    HZ[(size_t)f * plane + (size_t)row * d.Kz + k] = scale * v;
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
    z_cross_mhd_kernel(const __grid_constant__ DevOps o, const __grid_constant__ Dims d,
                       const __grid_constant__ MhdPhys ph, const __grid_constant__ FFTPlan plan,
                       const cpx<T>* __restrict__ tw, const cpx<T>* __restrict__ Y,
                       cpx<T>* __restrict__ HZ) {
  z_cross_mhd_body<T>(o, d, ph, plan, tw, Y, HZ, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Magnetic diagnostics (pcf_mhd_jax.py:760-790): per pencil (one warp, lanes
// over the x nodes) |b|^2 and |div b|^2 at the nodes from the coefficients of
// A, with div b = d/dx b_x + i ky b_y + i kz b_z evaluated from the projected
// curl (B2 applied to the TD coefficients of b_x).  Fejer weights in x,
// Parseval in y and z (half spectrum: kz > 0 counts twice).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) mhd_diag_kernel(DevOps o, Dims d, MhdOps M,
                                                       const c64* __restrict__ Acoef,
                                                       double* __restrict__ partial) {
  __shared__ double red[2 * kNW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kyi = blockIdx.x / d.nKb;
  const int kz = (blockIdx.x % d.nKb) * kNW + warp;
  const int ky = (kyi < d.Ny / 2) ? kyi : kyi - d.Ny;
  const bool active = kz < d.Kz && kyi != d.Ny / 2;
  const size_t P = (size_t)d.P;
  const int p = kyi * d.Kz + kz;
  const double kyp = ky * d.dfy, kzp = kz * d.dfz;
  double eb = 0.0, ed = 0.0;
  if (active) {
    const c64* Ax = Acoef + p;
    const c64* Ay = Ax + (size_t)d.nD * P;
    const c64* Az = Ay + (size_t)d.nD * P;
    const double mult = (kz == 0) ? 1.0 : 2.0;
    for (int j = lane; j < d.Nx; j += 32) {
      c64 b1x = cmk(0.0, 0.0), b1y = b1x, b1z = b1x, b2y = b1x, b2z = b1x;
      for (int k = 0; k < d.nD; ++k) {
        const double t1 = __ldg(M.B1 + (size_t)j * d.nD + k);
        const double t2 = __ldg(M.B2 + (size_t)j * d.nD + k);
        const c64 ax = Ax[(size_t)k * P], ay = Ay[(size_t)k * P], az = Az[(size_t)k * P];
        b1x = b1x + t1 * ax;
        b1y = b1y + t1 * ay;
        b1z = b1z + t1 * az;
        b2y = b2y + t2 * ay;
        b2z = b2z + t2 * az;
      }
      const c64 bx = mul_i(kyp * b1z - kzp * b1y);
      const c64 by = mul_i(kzp * b1x) - b2z;
      const c64 bz = b2y - mul_i(kyp * b1x);
      const c64 dbx = mul_i(kyp * b2z - kzp * b2y);
      const c64 div = dbx + mul_i(kyp * by + kzp * bz);
      const double w = o.fejer[j] * mult;
      eb += w * (bx.re * bx.re + bx.im * bx.im + by.re * by.re + by.im * by.im +
                 bz.re * bz.re + bz.im * bz.im);
      ed += w * (div.re * div.re + div.im * div.im);
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    eb += __shfl_down_sync(0xffffffffu, eb, off);
    ed += __shfl_down_sync(0xffffffffu, ed, off);
  }
  if (lane == 0) {
    red[2 * warp] = eb;
    red[2 * warp + 1] = ed;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, t = 0.0;
    for (int w = 0; w < kNW; ++w) {
      s += red[2 * w];
      t += red[2 * w + 1];
    }
    partial[2 * blockIdx.x] = s;
    partial[2 * blockIdx.x + 1] = t;
  }
}

// out[0] = divB_L2, out[1] = Emag (fixed-order reduction)
__global__ void mhd_diag_finish_kernel(const double* __restrict__ partial, int nblocks,
                                       double ly, double lz, double* __restrict__ out,
                                       int* status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double eb = 0.0, ed = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    eb += partial[2 * b];
    ed += partial[2 * b + 1];
  }
  out[0] = sqrt(ly * lz * ed);
  out[1] = ly * lz * eb;
  flag_nonfinite(status, !isfinite(out[0]) || !isfinite(out[1]));
}

}  // namespace jfb
