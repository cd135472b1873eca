// Device kernels of the KMM plane-Couette step (FP64 form).
//
// One steady SBDF3 step = four launches:
//   pencil_stage  per (ky, kz>=0) pencil, along the wall-normal axis x:
//                 x-forward of the dealiased nonlinear term, Shen projection,
//                 coefficient-space KMM right-hand sides, SBDF3 (or IMEXRK3
//                 stage) combination, the per-wavenumber banded solves,
//                 velocity reconstruction, vorticity and the x-backward of the
//                 six fields u, omega.
//   y_backward    zero-padded inverse FFT along y (Ny -> My) of six fields.
//   z_cross       inverse real FFT along z (Kz -> Mz), base flow, the
//                 rotational product -(u x omega), forward real FFT (Mz -> Kz).
//   y_forward     forward FFT along y (My -> Ny) with 3/2-rule truncation.
// Spectral arrays are laid out [field][x][ky][kz] with kz in [0, Nz/2): the
// real-field half spectrum (the Nyquist column kz = Nz/2 is masked to zero by
// the reference, tensorproductspace.py:276-293, and is not stored).
#pragma once

#include "jfb_common.cuh"
#include "jfb_fft.cuh"

namespace jfb {

constexpr int kNW = 8;         // pencils (warps) per pencil_stage block
constexpr int kLDW = kNW + 1;  // padded pencil stride in shared memory
constexpr int kMaxNR = 2;      // rows per lane in the register solves (n <= 128)
constexpr int kSolveChunk = 16;  // back-substitution columns per prefetch
constexpr int kLoadBatch = 4;    // staged loads per thread in flight
// Mixed form, warp-per-pencil stage: the FP64 base-flow terms in a separate
// branch-free pass over the sample points (1) or per loaded H value (0).
// The pass took the 97x96x96 stage from 474 to 458 us, 129x128x128 from
// 1173 to 1132 us (events around the launch, steady SBDF3 step).
#ifndef JFB_WARP_XLIN_PASS
#define JFB_WARP_XLIN_PASS 1
#endif

struct DevOps {
  const double* Q;   // [n][j] scalar-product quadrature (Nx x Nx)
  const double* V;   // [j][n] Chebyshev Vandermonde (Nx x Nx)
  const double* VE;  // [j][m] = V[j][2m],   j < ceil(Nx/2)
  const double* VO;  // [j][m] = V[j][2m+1], j < ceil(Nx/2)
  const double* QE;  // [m][j] = Q[2m][j],   j < ceil(Nx/2)
  const double* QO;  // [m][j] = Q[2m+1][j], j < floor(Nx/2)
  const double* ns;  // norm^2 / df (Nx)
  const double* sB0;
  const double* sB2;
  const double* sB4;  // biharmonic stencil diagonals (nB)
  const double* mlo;
  const double* mdi;
  const double* mhi;  // Dirichlet mass tri-band (nD)
  const double* lul;
  const double* luu;    // its LU (nD): multipliers and reciprocal pivots
  const double* xphys;  // physical wall-normal nodes (Nx)
  const double* bl2;
  const double* bl4;
  const double* bu0;
  const double* bu2;
  const double* bu4;     // biharmonic mass LU (nB)
  const double* fejer;   // Fejer-I weights (Nx)
};

struct Dims {
  int Nx, nB, nD, Ny, Nz, Kz, P, My, Mz, nKb;
  double dfx, dfy, dfz, Myz, nu, dt, uwall;
  int family;  // wall-normal family: 0 Chebyshev, 1 Legendre
  int grad;    // nonlinear term in gradient form u . grad u (else rotational)
};

struct PackedFactors {
  const double* su;  // n_modes records of su_rec doubles
  const double* sg;
  const double* s00;  // one record (sg layout, n = nD)
  const double* s00inv;  // the explicit inverse of the mean-flow system (nD x nD)
  int su_rec, sg_rec;
};

enum StageMode { kPrologue = 0, kImplicit = 1, kHOnly = 2, kReconstruct = 3, kFromPhys = 4 };

struct StageArgs {
  int mode;
  const c64* HX;  // phase A input: 3 x [Nx][P]
  double c0, c1, c2, cL, d0, d1, d2;
  const c64 *u0a, *u0b, *u0c;
  const c64 *ga, *gb, *gc;
  const c64 *vwa, *vwb, *vwc;
  const c64 *Nup, *Nuq, *Ngp, *Ngq, *NVWp, *NVWq;
  c64 *Nu_out, *Ng_out, *NVW_out;
  PackedFactors fac;
  c64 *u0_out, *g_out, *vw_out;
  const c64 *pu0, *pu1, *pu2;  // prologue: explicit fields
  c64* X;                      // 6 x [Nx][P]
  c64* Hd_out;                 // kHOnly: 3 x [nD][P]
  c64 *u1_out, *u2_out;        // kFromPhys: tangential velocity (nD x P)
  int x32;  // HX (read, step modes) and X (written by the x-backward) hold complex64
  const c32* Xlin;  // mixed form: u, omega of HX's state; FP64 base-flow terms added here
  int* status;      // plan status word: kStatusNonFinite when a solved value is not finite
  // MHD EMF rows (kHOnly): U_wall B0z, U_wall B0x of the term U_b e_y x B0,
  // added to the (0, 0) mode of components 0 and 2 (the z stage leaves it out)
  double emf_b0z, emf_b0x;
};

__host__ __device__ inline int packed_rec_size(int n) {
  const int m0 = (n + 1) / 2, m1 = n / 2;
  return 2 * n + m0 * (m0 + 1) / 2 + m1 * (m1 + 1) / 2;
}

// ---------------------------------------------------------------------------
// Warp-level helpers (all lanes of the warp call them; arrays in smem).
// ---------------------------------------------------------------------------

// d = scale * d/dX of a length-L coefficient vector; in place allowed.
// Chebyshev (fam 0): d_n = sum_{m > n, m - n odd} 2 m c_m, d_0 halved
// (Chebyshev.py:319-353); Legendre (fam 1): d_n = (2n + 1) sum_{m > n, m - n
// odd} c_m (Legendre.py:195-227).
// Warp-level helpers of the warp-per-pencil stage: inlined, or (with
// JFB_WARP_HELPERS_NOINLINE) one shared copy each, for a smaller kernel.
#ifndef JFB_WARP_HELPERS_NOINLINE
#define JFB_WARP_HELPERS_NOINLINE 0
#endif
#if JFB_WARP_HELPERS_NOINLINE
#define JFB_WARP_HELPER __noinline__
#else
#define JFB_WARP_HELPER __forceinline__
#endif
// chebder_warp has one shared copy (sixteen call sites): the smaller
// warp-per-pencil kernel took 474 instead of 514 us per launch at 97x96x96
// (the other helpers not inlined as well: 527 us)
#ifndef JFB_CHEBDER_NOINLINE
#define JFB_CHEBDER_NOINLINE 1
#endif
#if JFB_CHEBDER_NOINLINE
__device__ __noinline__
#else
__device__
#endif
void chebder_warp(const c64* c, c64* d, int L, double scale, int lane, int fam) {
  const int K = (L + 31) / 32;
  const int lo = lane * K, hi = min(L, lo + K);
  c64 se = cmk(0.0, 0.0), so = cmk(0.0, 0.0);
  for (int m = lo; m < hi; ++m) {
    const c64 e = (fam ? 1.0 : 2.0 * m) * c[m];
    if (m & 1) so = so + e; else se = se + e;
  }
  // inclusive suffix sums over lanes >= lane
  c64 ie = se, io = so;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const double er = __shfl_down_sync(0xffffffffu, ie.re, off);
    const double ei = __shfl_down_sync(0xffffffffu, ie.im, off);
    const double orr = __shfl_down_sync(0xffffffffu, io.re, off);
    const double oi = __shfl_down_sync(0xffffffffu, io.im, off);
    if (lane + off < 32) {
      ie = ie + cmk(er, ei);
      io = io + cmk(orr, oi);
    }
  }
  c64 run_e = ie - se, run_o = io - so;  // sums over lanes > lane
  __syncwarp();
  for (int n = hi - 1; n >= lo; --n) {
    const c64 cn = c[n];
    c64 dn = (n & 1) ? run_e : run_o;
    if (fam) dn = (2.0 * n + 1.0) * dn;
    else if (n == 0) dn = 0.5 * dn;
    d[n] = scale * dn;
    const c64 e = (fam ? 1.0 : 2.0 * n) * cn;
    if (n & 1) run_o = run_o + e; else run_e = run_e + e;
  }
  __syncwarp();
}

// out = S_B^T a  (length Nx from nB)
__device__ JFB_WARP_HELPER void apply_SBT(const DevOps& o, const Dims& d, const c64* a,
                                          c64* out, int lane) {
  for (int n = lane; n < d.Nx; n += 32) {
    c64 v = cmk(0.0, 0.0);
    if (n < d.nB) v = v + o.sB0[n] * a[n];
    if (n >= 2 && n - 2 < d.nB) v = v + o.sB2[n - 2] * a[n - 2];
    if (n >= 4 && n - 4 < d.nB) v = v + o.sB4[n - 4] * a[n - 4];
    out[n] = v;
  }
  __syncwarp();
}
// out = S_D^T a  (length Nx from nD)
__device__ JFB_WARP_HELPER void apply_SDT(const Dims& d, const c64* a, c64* out, int lane) {
  for (int n = lane; n < d.Nx; n += 32) {
    c64 v = cmk(0.0, 0.0);
    if (n < d.nD) v = a[n];
    if (n >= 2 && n - 2 < d.nD) v = v - a[n - 2];
    out[n] = v;
  }
  __syncwarp();
}
// out[i] = scale * (S_B (ns .* c))[i]   (length nB)
__device__ JFB_WARP_HELPER void apply_SB_ns(const DevOps& o, const Dims& d, const c64* c,
                                            c64* out, double scale, int lane) {
  for (int i = lane; i < d.nB; i += 32) {
    c64 v = (o.sB0[i] * o.ns[i]) * c[i];
    v = v + (o.sB2[i] * o.ns[i + 2]) * c[i + 2];
    v = v + (o.sB4[i] * o.ns[i + 4]) * c[i + 4];
    out[i] = scale * v;
  }
  __syncwarp();
}
// out[i] = scale * (S_D (ns .* c))[i]   (length nD)
__device__ JFB_WARP_HELPER void apply_SD_ns(const DevOps& o, const Dims& d, const c64* c,
                                            c64* out, double scale, int lane) {
  for (int i = lane; i < d.nD; i += 32) {
    const c64 v = o.ns[i] * c[i] - o.ns[i + 2] * c[i + 2];
    out[i] = scale * v;
  }
  __syncwarp();
}

// Tri-band (offsets -2, 0, 2) no-pivot LU solve of the Dirichlet mass matrix,
// in place on `b` (length nD).  Two lanes (one per parity) per vector; `which`
// selects the lane pair so several vectors can be solved concurrently.
__device__ __forceinline__ void mass_solve_lane(const DevOps& o, const Dims& d, c64* b,
                                                int par) {
  for (int i = par + 2; i < d.nD; i += 2) b[i] = b[i] - o.lul[i] * b[i - 2];
  int last = d.nD - 1;
  if ((last & 1) != par) last -= 1;
  for (int i = last; i >= 0; i -= 2) {
    c64 v = b[i];
    if (i + 2 < d.nD) v = v - o.mhi[i] * b[i + 2];
    b[i] = o.luu[i] * v;
  }
}

// No-pivot LU solve of the biharmonic mass matrix (offsets -4..4), in place,
// one lane per parity class.
__device__ __forceinline__ void bmass_solve_lane(const DevOps& o, const Dims& d, c64* b,
                                                 int par) {
  for (int i = par; i < d.nB; i += 2) {
    c64 v = b[i];
    if (i >= 2) v = v - o.bl2[i] * b[i - 2];
    if (i >= 4) v = v - o.bl4[i] * b[i - 4];
    b[i] = v;
  }
  int last = d.nB - 1;
  if ((last & 1) != par) last -= 1;
  for (int i = last; i >= 0; i -= 2) {
    c64 v = b[i];
    if (i + 2 < d.nB) v = v - o.bu2[i] * b[i + 2];
    if (i + 4 < d.nB) v = v - o.bu4[i] * b[i + 4];
    b[i] = o.bu0[i] * v;
  }
}

// Solve one parity class of a packed record in registers.  Lane r holds
// row 2r + par (and 2(r+32) + par when m > 32).  Forward elimination with
// the unit-lower factor (L[i, i-2], L[i, i-4]) passes the solved rows down
// the lanes with shuffles; then x = U^-1 y with the record's explicit inverse
// of the parity's upper factor (column-major packed, entry (r, c), r <= c, at
// c (c + 1) / 2 + r): y_c is broadcast and every lane r <= c accumulates
// U^-1[r, c] y_c, kSolveChunk columns of the inverse loaded at a time.  Not
// inlined: the call sites (Su, Sg, S00, two parities each) share one copy in
// the instruction cache.
template <int NR>
__device__ __noinline__ void parity_solve_regs(const double* __restrict__ rec, int n, c64* y,
                                               int par, int lane) {
  const int m0 = (n + 1) / 2;
  const int m = par ? n / 2 : m0;
  const double* __restrict__ Ui = rec + 2 * n + (par ? m0 * (m0 + 1) / 2 : 0);
  c64 yr[NR];
  double l1[NR], l2[NR];
#pragma unroll
  for (int s = 0; s < NR; ++s) {
    const int r = lane + 32 * s;
    const int i = 2 * r + par;
    const bool ok = r < m;
    yr[s] = ok ? y[i] : cmk(0.0, 0.0);
    l1[s] = ok ? __ldg(rec + 2 * i) : 0.0;
    l2[s] = ok ? __ldg(rec + 2 * i + 1) : 0.0;
  }
  // forward elimination: y_r -= l1_r y_{r-1} + l2_r y_{r-2}
  c64 ym1 = cmk(0.0, 0.0), ym2 = cmk(0.0, 0.0);
#pragma unroll
  for (int s = 0; s < NR; ++s) {
    for (int r0 = 0; r0 < 32; ++r0) {
      const int r = r0 + 32 * s;
      if (r >= m) break;
      if (lane == r0) yr[s] = yr[s] - l1[s] * ym1 - l2[s] * ym2;
      c64 t;
      t.re = __shfl_sync(0xffffffffu, yr[s].re, r0);
      t.im = __shfl_sync(0xffffffffu, yr[s].im, r0);
      ym2 = ym1;
      ym1 = t;
    }
  }
  // x = U^-1 y
  c64 acc[NR];
#pragma unroll
  for (int s = 0; s < NR; ++s) acc[s] = cmk(0.0, 0.0);
  for (int ch = 0; ch * kSolveChunk < m; ++ch) {
    double u[NR][kSolveChunk];
#pragma unroll
    for (int s = 0; s < NR; ++s)
#pragma unroll
      for (int cc = 0; cc < kSolveChunk; ++cc) {
        const int c = cc + kSolveChunk * ch;
        const int r = lane + 32 * s;
        u[s][cc] = (c < m && r <= c) ? __ldg(Ui + c * (c + 1) / 2 + r) : 0.0;
      }
#pragma unroll
    for (int cc = 0; cc < kSolveChunk; ++cc) {
      const int c = cc + kSolveChunk * ch;
      if (c >= m) break;
      const int own = c & 31, os = c >> 5;  // lane and slot of row c
      c64 v = yr[0];
#pragma unroll
      for (int s = 1; s < NR; ++s)
        if (s == os) v = yr[s];
      c64 yc;
      yc.re = __shfl_sync(0xffffffffu, v.re, own);
      yc.im = __shfl_sync(0xffffffffu, v.im, own);
#pragma unroll
      for (int s = 0; s < NR; ++s) acc[s] = acc[s] + u[s][cc] * yc;
    }
  }
#pragma unroll
  for (int s = 0; s < NR; ++s) {
    const int r = lane + 32 * s;
    if (r < m) y[2 * r + par] = acc[s];
  }
  __syncwarp();
}

// Solve a packed system of size n <= 64 * NR in place on y (both parities).
template <int NR>
__device__ __forceinline__ void packed_solve_warp(const double* __restrict__ rec, int n,
                                                  c64* y, int lane) {
  parity_solve_regs<NR>(rec, n, y, 0, lane);
  parity_solve_regs<NR>(rec, n, y, 1, lane);
}

// Rows i = lane + 32 t of one pencil (n <= 128: the host limits Nx to 129),
// all global loads of the warp issued before the arithmetic.
// out[i] = c0 x[i] + c1 y[i] + c2 z[i]  (the y, z terms only when c1, c2 != 0)
__device__ JFB_WARP_HELPER void comb_rows(c64* out, const c64* x, const c64* y, const c64* z,
                                          double c0, double c1, double c2, int n, size_t P,
                                          int p, int lane) {
  c64 vx[4], vy[4], vz[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = lane + 32 * t;
    const size_t gi = (size_t)i * P + p;
    vx[t] = vy[t] = vz[t] = cmk(0.0, 0.0);
    if (i < n) {
      vx[t] = x[gi];
      if (c1 != 0.0) vy[t] = y[gi];
      if (c2 != 0.0) vz[t] = z[gi];
    }
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = lane + 32 * t;
    if (i < n) {
      c64 v = c0 * vx[t];
      if (c1 != 0.0) v = v + c1 * vy[t];
      if (c2 != 0.0) v = v + c2 * vz[t];
      out[i] = v;
    }
  }
}
// acc[i] = mass[i] + dt (d0 acc[i] + d1 q1[i] + d2 q2[i])  (q terms when d1, d2 != 0)
__device__ JFB_WARP_HELPER void rhs_rows(c64* acc, const c64* mass, const c64* q1,
                                         const c64* q2, double d0, double d1, double d2,
                                         double dt, int n, size_t P, int p, int lane) {
  c64 v1[4], v2[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = lane + 32 * t;
    const size_t gi = (size_t)i * P + p;
    v1[t] = v2[t] = cmk(0.0, 0.0);
    if (i < n) {
      if (d1 != 0.0) v1[t] = q1[gi];
      if (d2 != 0.0) v2[t] = q2[gi];
    }
  }
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int i = lane + 32 * t;
    if (i < n) {
      c64 nl = d0 * acc[i];
      if (d1 != 0.0) nl = nl + d1 * v1[t];
      if (d2 != 0.0) nl = nl + d2 * v2[t];
      acc[i] = mass[i] + dt * nl;
    }
  }
}

// Velocity reconstruction (channelflow_kmm.py:855-870): from u0 (TB, in A3)
// and g (TD, in A4) form uo0 = S_B^T u0 (-> A5), f = P_TD(d/dx uo0),
// u1 = i(ky f + kz g)/k^2 (-> A0), u2 = i(kz f - ky g)/k^2 (-> A1); the
// ky = kz = 0 pencil takes the real mean-flow vectors (v00, w00) from vw.
#ifndef JFB_CTA_DMMA_NOINLINE
#define JFB_CTA_DMMA_NOINLINE 0
#endif
#if JFB_CTA_DMMA_NOINLINE
#define JFB_CTA_DMMA_INLINE __noinline__
#else
#define JFB_CTA_DMMA_INLINE __forceinline__
#endif
#ifndef JFB_RECON_NOINLINE
#define JFB_RECON_NOINLINE 0
#endif
#if JFB_RECON_NOINLINE
__device__ __noinline__
#else
__device__
#endif
void reconstruct_warp(const DevOps& o, const Dims& d, const c64* A3,
                                 const c64* A4, const c64* vw, bool mean_pencil,
                                 double kyp, double kzp, c64* A0, c64* A1, c64* A2,
                                 c64* A5, int lane) {
  apply_SBT(o, d, A3, A5, lane);            // A5 = uo0 = S_B^T u0
  chebder_warp(A5, A0, d.Nx, d.dfx, lane, d.family);   // A0 = d/dx uo0
  apply_SD_ns(o, d, A0, A2, 1.0, lane);      // A2 = S_D(ns du)
  if (lane < 2) mass_solve_lane(o, d, A2, lane);  // f = projection into TD
  __syncwarp();
  const double k2 = kyp * kyp + kzp * kzp;
  const double inv = (k2 == 0.0) ? 1.0 : 1.0 / k2;
  for (int i = lane; i < d.nD; i += 32) {
    const c64 f = A2[i], g = A4[i];
    c64 u1 = mul_i((kyp * inv) * f + (kzp * inv) * g);
    c64 u2 = mul_i((kzp * inv) * f - (kyp * inv) * g);
    if (mean_pencil) {
      u1 = cmk(vw[i].re, 0.0);
      u2 = cmk(vw[i].im, 0.0);
    }
    A0[i] = u1;
    A1[i] = u2;
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// CTA-level small GEMMs against the x-transform matrices.
// out[(f * R + r) * kLDW + w] = sum_k A[r * K + k] * in(f, k, w)
// ---------------------------------------------------------------------------
template <typename InFn>
__device__ __forceinline__ void cta_gemm(const double* __restrict__ A, int R, int K, int NF,
                                         InFn in, c64* out) {
  const int C = NF * kNW;
  const int G = blockDim.x / C;
  const int t = threadIdx.x;
  const int col = t % C, g = t / C;
  if (g < G) {
    const int f = col / kNW, w = col % kNW;
    for (int r0 = g; r0 < R; r0 += 8 * G) {
      c64 acc[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] = cmk(0.0, 0.0);
      for (int k = 0; k < K; ++k) {
        const c64 x = in(f, k, w);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int r = r0 + q * G;
          if (r < R) {
            const double a = __ldg(A + (size_t)r * K + k);
            acc[q] = cmk(acc[q].re + a * x.re, acc[q].im + a * x.im);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int r = r0 + q * G;
        if (r < R) out[(f * R + r) * kLDW + w] = acc[q];
      }
    }
  }
}

// Parity-split x-backward: with x_{N-1-j} = -x_j and T_n(-x) = (-1)^n T_n(x),
// u(x_j) = E_j + O_j and u(x_{N-1-j}) = E_j - O_j, where E (O) sums the even
// (odd) coefficients.  Halves the Vandermonde work.
// out[(f * N + j) * kLDW + w] for the NF fields of in(f, n, w).
template <typename InFn>
__device__ __forceinline__ void cta_backward_parity(const double* __restrict__ VE,
                                                    const double* __restrict__ VO, int N,
                                                    int NF, InFn in, c64* out) {
  const int C = NF * kNW;
  const int G = blockDim.x / C;
  const int t = threadIdx.x;
  const int col = t % C, g = t / C;
  const int Jh = (N + 1) / 2, Ne = (N + 1) / 2, No = N / 2;
  if (g >= G) return;
  const int f = col / kNW, w = col % kNW;
  for (int j0 = g; j0 < Jh; j0 += 4 * G) {
    c64 E[4], O[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) E[q] = O[q] = cmk(0.0, 0.0);
    for (int m = 0; m < Ne; ++m) {
      const c64 x = in(f, 2 * m, w);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = j0 + q * G;
        if (j < Jh) {
          const double a = __ldg(VE + (size_t)j * Ne + m);
          E[q] = cmk(E[q].re + a * x.re, E[q].im + a * x.im);
        }
      }
    }
    for (int m = 0; m < No; ++m) {
      const c64 x = in(f, 2 * m + 1, w);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int j = j0 + q * G;
        if (j < Jh) {
          const double a = __ldg(VO + (size_t)j * No + m);
          O[q] = cmk(O[q].re + a * x.re, O[q].im + a * x.im);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = j0 + q * G;
      if (j < Jh) {
        out[(f * N + j) * kLDW + w] = E[q] + O[q];
        if (N - 1 - j != j) out[(f * N + N - 1 - j) * kLDW + w] = E[q] - O[q];
      }
    }
  }
}

// Parity-split x-forward scalar products: sp[2m] = sum_j QE[m][j] (u_j +
// u_{N-1-j}) (middle node once), sp[2m+1] = sum_j QO[m][j] (u_j - u_{N-1-j}).
// Input phys(f, j, w); output out[(f * N + n) * kLDW + w].
template <typename InFn>
__device__ __forceinline__ void cta_forward_parity(const double* __restrict__ QE,
                                                   const double* __restrict__ QO, int N,
                                                   int NF, InFn phys, c64* out) {
  const int C = NF * kNW;
  const int G = blockDim.x / C;
  const int t = threadIdx.x;
  const int col = t % C, g = t / C;
  const int Jh = (N + 1) / 2, Jl = N / 2, Ne = (N + 1) / 2, No = N / 2;
  if (g >= G) return;
  const int f = col / kNW, w = col % kNW;
  // virtual rows: [0, Ne) even outputs, [Ne, Ne + No) odd outputs
  const int R = Ne + No;
  for (int r0 = g; r0 < R; r0 += 4 * G) {
    c64 acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = cmk(0.0, 0.0);
    for (int j = 0; j < Jh; ++j) {
      const c64 a = phys(f, j, w);
      const c64 b = (N - 1 - j != j) ? phys(f, N - 1 - j, w) : cmk(0.0, 0.0);
      const c64 sum = a + b, dif = a - b;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = r0 + q * G;
        if (r < Ne) {
          const double c = __ldg(QE + (size_t)r * Jh + j);
          acc[q] = cmk(acc[q].re + c * sum.re, acc[q].im + c * sum.im);
        } else if (r < R && j < Jl) {
          const double c = __ldg(QO + (size_t)(r - Ne) * Jl + j);
          acc[q] = cmk(acc[q].re + c * dif.re, acc[q].im + c * dif.im);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = r0 + q * G;
      if (r < R) {
        const int n = (r < Ne) ? 2 * r : 2 * (r - Ne) + 1;
        out[(f * N + n) * kLDW + w] = acc[q];
      }
    }
  }
}

constexpr int kDmmaChunk = 8;  // k steps whose operands are loaded together
constexpr int kDmmaGroup = 6;  // column tiles sharing one operator fragment load
// doubles per B-operand row of the x-backward: 6 fields x kNW pencils x re/im,
// + 4 so that the four rows of a fragment fall in distinct bank halves
constexpr int kLDB = 2 * 6 * kNW + 4;
// doubles per B-operand row of the x-forward (3 fields): consecutive rows
// fall in opposite bank halves
constexpr int kLDF = 2 * 3 * kNW + 8;

// FP64 tensor-core product D = A B + C for one 8x8x4 tile (mma.sync m8n8k4
// f64).  Fragments: a = A[lane / 4][lane % 4], b = B[lane % 4][lane / 4],
// c/d = C[lane / 4][2 (lane % 4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Parity-split x-backward on the FP64 tensor cores.  Columns of the product
// are (pencil w, field f, re/im) with re/im the lowest bit, so each lane's
// accumulator pair is one complex output value.  E (even coefficients) and O
// (odd) tiles share an output tile; u(x_j) = E + O, u(x_{N-1-j}) = E - O.
// The B operand sits in shared memory as rows Bs[n * kLDB + c], n the
// orthogonal coefficient, c = (w NF + f) 2 + re/im, so the fragment of a
// k step is one 8-byte load per lane from four rows (two wavefronts).
// Output: out[(f N + j) ldo + w].  A warp's unit of work is one 8-row tile of
// the operator against up to kDmmaGroup column tiles: each operator fragment
// (read from L2, shared by all CTAs) is loaded once per unit.
__device__ JFB_CTA_DMMA_INLINE void cta_backward_dmma(const double* __restrict__ VE,
                                                  const double* __restrict__ VO, int N,
                                                  int NF, const double* Bs, c64* out,
                                                  int ldo) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int Jh = (N + 1) / 2, Ne = (N + 1) / 2, No = N / 2;
  const int mt = (Jh + 7) / 8, nt = (NF * kNW * 2) / 8;
  const int ng = (nt + kDmmaGroup - 1) / kDmmaGroup;
  const int g = lane >> 2, t4 = lane & 3;
  for (int unit = warp; unit < mt * ng; unit += nwarps) {
    const int m0 = (unit / ng) * 8, nb = (unit % ng) * kDmmaGroup;
    const int nq = min(kDmmaGroup, nt - nb);
    const int ja = m0 + g;  // A row of the a fragment
    double e0[kDmmaGroup], e1[kDmmaGroup], o0[kDmmaGroup], o1[kDmmaGroup];
#pragma unroll
    for (int q = 0; q < kDmmaGroup; ++q) e0[q] = e1[q] = o0[q] = o1[q] = 0.0;
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      const int K = par ? No : Ne;
      const double* A = par ? VO : VE;
      for (int kb = 0; kb < K; kb += 4 * kDmmaChunk) {
        double av[kDmmaChunk];
#pragma unroll
        for (int u = 0; u < kDmmaChunk; ++u) {
          const int k = kb + 4 * u + t4;
          av[u] = (ja < Jh && k < K) ? __ldg(A + (size_t)ja * K + k) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < kDmmaGroup; ++q) {
          if (q >= nq) break;
          const double* brow = Bs + (nb + q) * 8 + g + par * kLDB;  // + 2 k kLDB
          double bv[kDmmaChunk];
#pragma unroll
          for (int u = 0; u < kDmmaChunk; ++u) {
            const int k = kb + 4 * u + t4;
            bv[u] = (k < K) ? brow[2 * k * kLDB] : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kDmmaChunk; ++u)
            if (kb + 4 * u < K) {
              if (par) dmma_8x8x4(o0[q], o1[q], av[u], bv[u]);
              else dmma_8x8x4(e0[q], e1[q], av[u], bv[u]);
            }
        }
      }
    }
    const int j = m0 + g;
#pragma unroll
    for (int q = 0; q < kDmmaGroup; ++q) {
      if (q >= nq) break;
      const int colc = (nb + q) * 8 + 2 * t4;  // even column: re, next: im
      const int wc = colc / (2 * NF), fc = (colc / 2) % NF;
      if (j < Jh) {
        out[(fc * N + j) * ldo + wc] = cmk(e0[q] + o0[q], e1[q] + o1[q]);
        if (N - 1 - j != j) out[(fc * N + N - 1 - j) * ldo + wc] = cmk(e0[q] - o0[q], e1[q] - o1[q]);
      }
    }
  }
}

// Parity-split x-forward scalar products on the FP64 tensor cores:
// sp[2m] = sum_j QE[m][j] (u_j + u_{N-1-j}), sp[2m+1] = sum_j QO[m][j] (u_j -
// u_{N-1-j}).  The mirror sums (Se, ceil(N/2) rows) and differences (So,
// floor(N/2) rows) sit in shared memory as rows of kLDF doubles, column
// c = (w NF + f) 2 + re/im.  Output: out[(f N + n) kLDW + w].  Units of
// work as in cta_backward_dmma.
__device__ JFB_CTA_DMMA_INLINE void cta_forward_dmma(const double* __restrict__ QE,
                                                 const double* __restrict__ QO, int N, int NF,
                                                 const double* Se, const double* So, c64* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int Jh = (N + 1) / 2, Jl = N / 2, Ne = (N + 1) / 2, No = N / 2;
  const int mte = (Ne + 7) / 8, mto = (No + 7) / 8, nt = (NF * kNW * 2) / 8;
  const int ng = (nt + kDmmaGroup - 1) / kDmmaGroup;
  const int g = lane >> 2, t4 = lane & 3;
  for (int unit = warp; unit < (mte + mto) * ng; unit += nwarps) {
    const int mi = unit / ng, nb = (unit % ng) * kDmmaGroup;
    const int nq = min(kDmmaGroup, nt - nb);
    const bool odd = mi >= mte;
    const int m0 = (odd ? mi - mte : mi) * 8;
    const int M = odd ? No : Ne, K = odd ? Jl : Jh;
    const double* A = odd ? QO : QE;
    const double* B = odd ? So : Se;
    const int ma = m0 + g;
    double d0[kDmmaGroup], d1[kDmmaGroup];
#pragma unroll
    for (int q = 0; q < kDmmaGroup; ++q) d0[q] = d1[q] = 0.0;
    for (int kb = 0; kb < K; kb += 4 * kDmmaChunk) {
      double av[kDmmaChunk];
#pragma unroll
      for (int u = 0; u < kDmmaChunk; ++u) {
        const int k = kb + 4 * u + t4;
        av[u] = (ma < M && k < K) ? __ldg(A + (size_t)ma * K + k) : 0.0;
      }
#pragma unroll
      for (int q = 0; q < kDmmaGroup; ++q) {
        if (q >= nq) break;
        const double* brow = B + (nb + q) * 8 + g;
        double bv[kDmmaChunk];
#pragma unroll
        for (int u = 0; u < kDmmaChunk; ++u) {
          const int k = kb + 4 * u + t4;
          bv[u] = (k < K) ? brow[k * kLDF] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kDmmaChunk; ++u)
          if (kb + 4 * u < K) dmma_8x8x4(d0[q], d1[q], av[u], bv[u]);
      }
    }
    const int m = m0 + g;
#pragma unroll
    for (int q = 0; q < kDmmaGroup; ++q) {
      if (q >= nq) break;
      const int colc = (nb + q) * 8 + 2 * t4;
      const int wc = colc / (2 * NF), fc = (colc / 2) % NF;
      if (m < M) {
        const int n = odd ? 2 * m + 1 : 2 * m;
        out[(fc * N + n) * kLDW + wc] = cmk(d0[q], d1[q]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// pencil_stage: see file header.  Block = kNW warps, one pencil per warp.
// ---------------------------------------------------------------------------
// kForm: 0 rotational, 1 gradient (each compiled without the other's code).
template <int NR, int kForm>
__global__ void __launch_bounds__(256, 1) pencil_stage_kernel(DevOps o, Dims d, StageArgs a) {
  const bool grad = kForm == 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c64* R1 = reinterpret_cast<c64*>(smem_raw);  // 6 * Nx * kLDW
  c64* ARR = R1 + 6 * d.Nx * kLDW;              // kNW * 6 * Nx
  c64* sVW = ARR + kNW * 6 * d.Nx;              // Nx

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kyi = blockIdx.x / d.nKb;
  const int kz0 = (blockIdx.x % d.nKb) * kNW;
  const int p0 = kyi * d.Kz + kz0;
  const int nvalid = min(kNW, d.Kz - kz0);
  const int ky = (kyi < d.Ny / 2) ? kyi : kyi - d.Ny;
  const bool nyq = (kyi == d.Ny / 2);
  const int kz = kz0 + warp;
  const bool active = (warp < nvalid) && !nyq;
  const int p = p0 + warp;
  const double kyp = ky * d.dfy, kzp = kz * d.dfz;
  const double k2 = kyp * kyp + kzp * kzp;
  const bool mean_pencil = active && ky == 0 && kz == 0;
  const int mode_idx = (ky < 0 ? -ky : ky) * d.Kz + kz;
  c64* A0 = ARR + (warp * 6 + 0) * d.Nx;
  c64* A1 = A0 + d.Nx;
  c64* A2 = A1 + d.Nx;
  c64* A3 = A2 + d.Nx;
  c64* A4 = A3 + d.Nx;
  c64* A5 = A4 + d.Nx;
  const size_t P = (size_t)d.P;

  // ---------------- reconstruction only (u1, u2 of a stored state) --------
  if (a.mode == kReconstruct) {
    if (active) {
      for (int i = lane; i < d.nB; i += 32) A3[i] = a.u0a[(size_t)i * P + p];
      for (int i = lane; i < d.nD; i += 32) {
        A4[i] = a.ga[(size_t)i * P + p];
        if (mean_pencil) sVW[i] = a.vwa[i];
      }
      __syncwarp();
      reconstruct_warp(o, d, A3, A4, sVW, mean_pencil, kyp, kzp, A0, A1, A2, A5, lane);
      for (int i = lane; i < d.nD; i += 32) {
        a.X[(size_t)i * P + p] = A0[i];
        a.Hd_out[(size_t)i * P + p] = A1[i];
      }
    } else if (warp < nvalid) {
      for (int i = lane; i < d.nD; i += 32) {
        a.X[(size_t)i * P + p] = cmk(0.0, 0.0);
        a.Hd_out[(size_t)i * P + p] = cmk(0.0, 0.0);
      }
    }
    return;
  }

  // ---------------- phase A: nonlinear term of the current state ----------
  if (a.mode != kPrologue) {
    // cooperative load of the x-physical H fields into R1[0..2], kLoadBatch
    // values per thread in flight
    auto load_h = [&](int idx) {
      const int w = idx % kNW, fi = idx / kNW;
      c64 v = cmk(0.0, 0.0);
      if (w < nvalid && !nyq) {
        const size_t e = (size_t)fi * P + p0 + w;
        if (a.x32 && a.mode != kFromPhys) {
          const c32 h = reinterpret_cast<const c32*>(a.HX)[e];
          v = cmk((double)h.re, (double)h.im);
        } else {
          v = a.HX[e];
        }
        if ((a.emf_b0z != 0.0 || a.emf_b0x != 0.0) && p0 + w == 0) {
          const int f = fi / d.Nx, j = fi % d.Nx;
          if (f == 0) v.re += a.emf_b0z * o.xphys[j];
          else if (f == 2) v.re -= a.emf_b0x * o.xphys[j];
        }
        if (!JFB_WARP_XLIN_PASS && a.Xlin && a.mode != kFromPhys) {
          // base-flow terms of the rotational product in FP64 (the complex64
          // transforms carry -(u' x omega') only)
          const int f = fi / d.Nx, j = fi % d.Nx;
          const double uw = d.uwall, ub = d.uwall * o.xphys[j];
          auto ld = [&](int g) {
            const c32 x = a.Xlin[((size_t)g * d.Nx + j) * P + p0 + w];
            return cmk((double)x.re, (double)x.im);
          };
          if (grad) {  // U_b d/dy u_i (+ u_0 dU_b/dx e_y), pcf_fluctuations_jax.py:99-106
            if (f == 0) v = v + ub * ld(6);
            else if (f == 1) v = (v + ub * ld(7)) + uw * ld(0);
            else v = v + ub * ld(8);
          } else if (f == 0) {
            v = v - uw * ld(1) - ub * ld(5);
            if (p0 + w == 0) v.re -= ub * uw;
          } else if (f == 1) {
            v = v + uw * ld(0);
          } else {
            v = v + ub * ld(3);
          }
        }
      }
      return v;
    };
    const int nload = 3 * d.Nx * kNW;
    for (int i0 = threadIdx.x; i0 < nload; i0 += kLoadBatch * blockDim.x) {
      c64 v[kLoadBatch];
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u) {
        const int idx = i0 + u * blockDim.x;
        v[u] = (idx < nload) ? load_h(idx) : cmk(0.0, 0.0);
      }
#pragma unroll
      for (int u = 0; u < kLoadBatch; ++u) {
        const int idx = i0 + u * blockDim.x;
        if (idx < nload) R1[(idx / kNW) * kLDW + idx % kNW] = v[u];
      }
    }
    __syncthreads();
    if (JFB_WARP_XLIN_PASS && a.Xlin && a.mode != kFromPhys && !nyq) {
      // mixed form: the base-flow terms in FP64 (the complex64 transforms
      // carry the perturbation products only), one pass per sample point
      // (j, pencil) with its four complex64 velocity samples loaded without
      // branches, kLoadBatch points per thread in flight; the same sums in
      // the same order as a per-field update of the loaded H values
      const int npt = d.Nx * kNW;
      const int g1 = grad ? 6 : 1, g2 = grad ? 7 : 3, g3 = grad ? 8 : 5;
      for (int i0 = threadIdx.x; i0 < npt; i0 += kLoadBatch * blockDim.x) {
        c64 x[kLoadBatch][4];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
          const int idx = i0 + u * blockDim.x;
          const int w = idx % kNW, j = idx / kNW;
          const bool ok = idx < npt && w < nvalid;
          const int gs[4] = {0, g1, g2, g3};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            c32 v = {0.f, 0.f};
            if (ok) v = a.Xlin[((size_t)gs[k] * d.Nx + j) * P + p0 + w];
            x[u][k] = cmk((double)v.re, (double)v.im);
          }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
          const int idx = i0 + u * blockDim.x;
          const int w = idx % kNW, j = idx / kNW;
          if (idx >= npt || w >= nvalid) continue;
          const double uw = d.uwall, ub = d.uwall * o.xphys[j];
          c64* h0 = R1 + (size_t)j * kLDW + w;
          c64* h1 = h0 + (size_t)d.Nx * kLDW;
          c64* h2 = h1 + (size_t)d.Nx * kLDW;
          if (grad) {  // U_b d/dy u_i (+ u_0 dU_b/dx e_y), pcf_fluctuations_jax.py:99-106
            *h0 = *h0 + ub * x[u][1];
            *h1 = (*h1 + ub * x[u][2]) + uw * x[u][0];
            *h2 = *h2 + ub * x[u][3];
          } else {  // x = (u0, u1, omega0, omega2)
            c64 v = *h0 - uw * x[u][1] - ub * x[u][3];
            if (p0 + w == 0) v.re -= ub * uw;
            *h0 = v;
            *h1 = *h1 + uw * x[u][0];
            *h2 = *h2 + ub * x[u][2];
          }
        }
      }
      __syncthreads();
    }
    // mirror sums / differences of the samples as B-operand rows in ARR
    // (free until the per-pencil work starts)
    {
      const int Jh = (d.Nx + 1) / 2, Jl = d.Nx / 2;
      double* Se = reinterpret_cast<double*>(ARR);
      double* So = Se + (size_t)Jh * kLDF;
      for (int idx = threadIdx.x; idx < Jh * 3 * kNW; idx += blockDim.x) {
        const int wf = idx % (3 * kNW), k = idx / (3 * kNW);
        const int w = wf / 3, f = wf % 3;
        const c64 x = R1[(f * d.Nx + k) * kLDW + w];
        const c64 y = (d.Nx - 1 - k != k) ? R1[(f * d.Nx + d.Nx - 1 - k) * kLDW + w] : cmk(0.0, 0.0);
        const c64 sm = x + y;
        *reinterpret_cast<double2*>(Se + (size_t)k * kLDF + 2 * wf) = make_double2(sm.re, sm.im);
        if (k < Jl) {
          const c64 df = x - y;
          *reinterpret_cast<double2*>(So + (size_t)k * kLDF + 2 * wf) = make_double2(df.re, df.im);
        }
      }
    }
    __syncthreads();
    // scalar products (T_n, H_f)_w for the 3 fields -> R1[3..5]
    c64* sT = R1 + 3 * d.Nx * kLDW;
    cta_forward_dmma(o.QE, o.QO, d.Nx, 3, reinterpret_cast<const double*>(ARR),
                     reinterpret_cast<const double*>(ARR) + (size_t)((d.Nx + 1) / 2) * kLDF, sT);
    __syncthreads();
    if (a.mode == kFromPhys) {
      // TB.forward(u0), TD.forward(u1), TD.forward(u2), mask, g = i ky u2 - i kz u1
      // (channelflow_kmm.py:677-683)
      if (active) {
        for (int i = lane; i < d.nB; i += 32) {
          const c64* t = sT + warp;
          A0[i] = o.sB0[i] * t[i * kLDW] + o.sB2[i] * t[(i + 2) * kLDW] +
                  o.sB4[i] * t[(i + 4) * kLDW];
        }
        for (int f = 1; f < 3; ++f) {
          c64* out = (f == 1) ? A1 : A2;
          for (int i = lane; i < d.nD; i += 32)
            out[i] = sT[(f * d.Nx + i) * kLDW + warp] - sT[(f * d.Nx + i + 2) * kLDW + warp];
        }
        __syncwarp();
        if (lane < 2) bmass_solve_lane(o, d, A0, lane);
        else if (lane < 6) mass_solve_lane(o, d, (lane < 4) ? A1 : A2, lane & 1);
        __syncwarp();
        for (int i = lane; i < d.nB; i += 32) a.u0_out[(size_t)i * P + p] = A0[i];
        for (int i = lane; i < d.nD; i += 32) {
          const c64 u1 = A1[i], u2 = A2[i];
          a.u1_out[(size_t)i * P + p] = u1;
          a.u2_out[(size_t)i * P + p] = u2;
          a.g_out[(size_t)i * P + p] = mul_i(kyp * u2 - kzp * u1);
          if (mean_pencil) a.vw_out[i] = cmk(u1.re, u2.re);
        }
      } else if (warp < nvalid) {
        for (int i = lane; i < d.nD; i += 32) {
          if (i < d.nB) a.u0_out[(size_t)i * P + p] = cmk(0.0, 0.0);
          a.u1_out[(size_t)i * P + p] = cmk(0.0, 0.0);
          a.u2_out[(size_t)i * P + p] = cmk(0.0, 0.0);
          a.g_out[(size_t)i * P + p] = cmk(0.0, 0.0);
        }
      }
      return;
    }
    if (active) {
      // S_D (T_n, H)_w -> A0..A2, then Dirichlet mass solves
      for (int f = 0; f < 3; ++f) {
        c64* out = (f == 0) ? A0 : (f == 1) ? A1 : A2;
        for (int i = lane; i < d.nD; i += 32)
          out[i] = sT[(f * d.Nx + i) * kLDW + warp] - sT[(f * d.Nx + i + 2) * kLDW + warp];
      }
      __syncwarp();
      if (lane < 6) {
        c64* b = (lane >> 1) == 0 ? A0 : (lane >> 1) == 1 ? A1 : A2;
        mass_solve_lane(o, d, b, lane & 1);
      }
      __syncwarp();
    }
    if (a.mode == kHOnly) {
      if (active)
        for (int f = 0; f < 3; ++f) {
          const c64* src = (f == 0) ? A0 : (f == 1) ? A1 : A2;
          for (int i = lane; i < d.nD; i += 32) a.Hd_out[((size_t)f * d.nD + i) * P + p] = src[i];
        }
      else if (warp < nvalid)
        for (int f = 0; f < 3; ++f)
          for (int i = lane; i < d.nD; i += 32)
            a.Hd_out[((size_t)f * d.nD + i) * P + p] = cmk(0.0, 0.0);
      return;
    }
    if (active) {
      // mean-flow nonlinear rows: -(M00 Re H1), -(M00 Re H2)  packed as re/im
      if (mean_pencil) {
        for (int i = lane; i < d.nD; i += 32) {
          double v = o.mdi[i] * A1[i].re, w = o.mdi[i] * A2[i].re;
          if (i >= 2) {
            v += o.mlo[i] * A1[i - 2].re;
            w += o.mlo[i] * A2[i - 2].re;
          }
          if (i + 2 < d.nD) {
            v += o.mhi[i] * A1[i + 2].re;
            w += o.mhi[i] * A2[i + 2].re;
          }
          sVW[i] = cmk(-v, -w);
          if (a.NVW_out) a.NVW_out[i] = cmk(-v, -w);
        }
        __syncwarp();
      }
      // orthogonal coefficients Ho_f = S_D^T H_f : A3 <- Ho0, A4 <- Ho1, A5 <- Ho2
      apply_SDT(d, A0, A3, lane);
      apply_SDT(d, A1, A4, lane);
      apply_SDT(d, A2, A5, lane);
      // t = i ky Ho1 + i kz Ho2  -> A0 ;  Hg = i kz Ho1 - i ky Ho2 -> A1
      for (int n = lane; n < d.Nx; n += 32) {
        const c64 h1 = A4[n], h2 = A5[n];
        A0[n] = mul_i(kyp * h1 + kzp * h2);
        A1[n] = mul_i(kzp * h1 - kyp * h2);
      }
      __syncwarp();
      chebder_warp(A0, A2, d.Nx, d.dfx, lane, d.family);  // A2 = d/dx t
      for (int n = lane; n < d.Nx; n += 32) A2[n] = A2[n] + k2 * A3[n];  // Hu
      __syncwarp();
      // Nu = Myz S_B(ns Hu) -> A3 ; Ng = Myz S_D(ns Hg) -> A4
      apply_SB_ns(o, d, A2, A3, d.Myz, lane);
      apply_SD_ns(o, d, A1, A4, d.Myz, lane);
      if (a.Nu_out)
        for (int i = lane; i < d.nB; i += 32) a.Nu_out[(size_t)i * P + p] = A3[i];
      if (a.Ng_out)
        for (int i = lane; i < d.nD; i += 32) a.Ng_out[(size_t)i * P + p] = A4[i];

      // ---- right-hand side of Su: Mu (c0 ua + c1 ub + c2 uc) + cL Lu ua + dt N ----
      comb_rows(A0, a.u0a, a.u0b, a.u0c, a.c0, a.c1, a.c2, d.nB, P, p, lane);
      __syncwarp();
      apply_SBT(o, d, A0, A2, lane);            // A2 = S_B^T comb
      chebder_warp(A2, A5, d.Nx, d.dfx, lane, d.family);   // A5 = D comb
      chebder_warp(A5, A0, d.Nx, d.dfx, lane, d.family);   // A0 = D^2 comb
      for (int n = lane; n < d.Nx; n += 32) A2[n] = A0[n] - k2 * A2[n];
      __syncwarp();
      if (a.cL != 0.0) {
        // + cL nu (D^4 - 2 k2 D^2 + k2^2) S_B^T ua
        for (int i = lane; i < d.nB; i += 32) A1[i] = a.u0a[(size_t)i * P + p];
        __syncwarp();
        apply_SBT(o, d, A1, A0, lane);           // A0 = w
        chebder_warp(A0, A5, d.Nx, d.dfx, lane, d.family);
        chebder_warp(A5, A1, d.Nx, d.dfx, lane, d.family);  // A1 = D^2 w
        const double s = a.cL * d.nu;
        for (int n = lane; n < d.Nx; n += 32)
          A2[n] = A2[n] + s * (k2 * k2 * A0[n] - (2.0 * k2) * A1[n]);
        __syncwarp();
        chebder_warp(A1, A5, d.Nx, d.dfx, lane, d.family);
        chebder_warp(A5, A0, d.Nx, d.dfx, lane, d.family);  // A0 = D^4 w
        for (int n = lane; n < d.Nx; n += 32) A2[n] = A2[n] + s * A0[n];
        __syncwarp();
      }
      apply_SB_ns(o, d, A2, A0, d.Myz, lane);  // A0 = mass rows (nB)
      rhs_rows(A3, A0, a.Nup, a.Nuq, a.d0, a.d1, a.d2, d.dt, d.nB, P, p, lane);  // rhs_u
      __syncwarp();

      // ---- right-hand side of Sg: Mg comb_g + cL Lg ga + dt N ----
      comb_rows(A0, a.ga, a.gb, a.gc, a.c0, a.c1, a.c2, d.nD, P, p, lane);
      __syncwarp();
      apply_SDT(d, A0, A2, lane);  // A2 = S_D^T comb
      if (a.cL != 0.0) {
        for (int i = lane; i < d.nD; i += 32) A1[i] = a.ga[(size_t)i * P + p];
        __syncwarp();
        apply_SDT(d, A1, A0, lane);  // A0 = w
        chebder_warp(A0, A5, d.Nx, d.dfx, lane, d.family);
        chebder_warp(A5, A1, d.Nx, d.dfx, lane, d.family);  // A1 = D^2 w
        const double s = a.cL * d.nu;
        for (int n = lane; n < d.Nx; n += 32) A2[n] = A2[n] + s * (A1[n] - k2 * A0[n]);
        __syncwarp();
      }
      apply_SD_ns(o, d, A2, A0, d.Myz, lane);
      rhs_rows(A4, A0, a.Ngp, a.Ngq, a.d0, a.d1, a.d2, d.dt, d.nD, P, p, lane);  // rhs_g
      __syncwarp();

      // ---- mean flow (ky = kz = 0): M00 comb + cL L00 + dt N  -> sVW ----
      if (mean_pencil) {
        for (int i = lane; i < d.nD; i += 32) {
          c64 v = a.c0 * a.vwa[i];
          if (a.c1 != 0.0) v = v + a.c1 * a.vwb[i];
          if (a.c2 != 0.0) v = v + a.c2 * a.vwc[i];
          A0[i] = v;
        }
        __syncwarp();
        apply_SDT(d, A0, A2, lane);
        if (a.cL != 0.0) {
          for (int i = lane; i < d.nD; i += 32) A1[i] = a.vwa[i];
          __syncwarp();
          apply_SDT(d, A1, A0, lane);
          chebder_warp(A0, A5, d.Nx, d.dfx, lane, d.family);
          chebder_warp(A5, A1, d.Nx, d.dfx, lane, d.family);
          for (int n = lane; n < d.Nx; n += 32) A2[n] = A2[n] + (a.cL * d.nu) * A1[n];
          __syncwarp();
        }
        apply_SD_ns(o, d, A2, A0, 1.0, lane);
        for (int i = lane; i < d.nD; i += 32) {
          c64 nl = a.d0 * sVW[i];
          if (a.d1 != 0.0) nl = nl + a.d1 * a.NVWp[i];
          if (a.d2 != 0.0) nl = nl + a.d2 * a.NVWq[i];
          sVW[i] = A0[i] + d.dt * nl;
        }
        __syncwarp();
      }

      // ---- solves ----
      const double* rec_u = a.fac.su + (size_t)mode_idx * a.fac.su_rec;
      const double* rec_g = a.fac.sg + (size_t)mode_idx * a.fac.sg_rec;
      packed_solve_warp<NR>(rec_u, d.nB, A3, lane);
      packed_solve_warp<NR>(rec_g, d.nD, A4, lane);
      if (mean_pencil) {
        packed_solve_warp<NR>(a.fac.s00, d.nD, sVW, lane);
        for (int i = lane; i < d.nD; i += 32) a.vw_out[i] = sVW[i];
        __syncwarp();
      }
      bool bad = false;
      for (int i = lane; i < d.nB; i += 32) {
        bad |= !finite_c(A3[i]);
        a.u0_out[(size_t)i * P + p] = A3[i];
      }
      for (int i = lane; i < d.nD; i += 32) {
        bad |= !finite_c(A4[i]);
        a.g_out[(size_t)i * P + p] = A4[i];
      }
      flag_nonfinite(a.status, bad);

      reconstruct_warp(o, d, A3, A4, sVW, mean_pencil, kyp, kzp, A0, A1, A2, A5, lane);
    }
  } else if (active) {
    // prologue: explicit u0, u1, u2
    for (int i = lane; i < d.nB; i += 32) A3[i] = a.pu0[(size_t)i * P + p];
    for (int i = lane; i < d.nD; i += 32) {
      A0[i] = a.pu1[(size_t)i * P + p];
      A1[i] = a.pu2[(size_t)i * P + p];
    }
    __syncwarp();
    apply_SBT(o, d, A3, A5, lane);
  }

  // ---------------- phase B: u and omega in orthogonal coefficients -------
  if (active) {
    // A5 = uo0 (already); uo1 = S_D^T u1 -> A2, uo2 = S_D^T u2 -> A3
    apply_SDT(d, A0, A2, lane);
    apply_SDT(d, A1, A3, lane);
    chebder_warp(A3, A4, d.Nx, d.dfx, lane, d.family);  // A4 = D uo2
    chebder_warp(A2, A0, d.Nx, d.dfx, lane, d.family);  // A0 = D uo1
    if (grad) {
      // gradient form: the x-derivatives of the three components
      // (channelflow_kmm.py:716-740); the y / z derivatives are wavenumber
      // weights applied on the way to the periodic transforms
      chebder_warp(A5, A1, d.Nx, d.dfx, lane, d.family);  // A1 = D uo0
    } else {
      for (int n = lane; n < d.Nx; n += 32) {
        const c64 u0 = A5[n], u1 = A2[n], u2 = A3[n];
        A1[n] = mul_i(kyp * u2 - kzp * u1);        // omega_0
        A4[n] = mul_i(kzp * u0) - A4[n];           // omega_1
        A0[n] = A0[n] - mul_i(kyp * u0);           // omega_2
      }
    }
    __syncwarp();
  } else {
    for (int n = lane; n < 6 * d.Nx; n += 32) A0[n] = cmk(0.0, 0.0);
    __syncwarp();
  }
  __syncthreads();
  // x-backward of the six fields: field order (u0, u1, u2, w0, w1, w2) lives
  // in arrays (A5, A2, A3, A1, A4, A0); in the gradient form (u0, u1, u2,
  // d/dx u0, d/dx u1, d/dx u2) in (A5, A2, A3, A1, A0, A4).  Their B-operand
  // rows go into R1 (dead by now), the product into ARR (dead once the rows
  // are built).
  double* Bs = reinterpret_cast<double*>(R1);
  for (int idx = threadIdx.x; idx < d.Nx * 6 * kNW; idx += blockDim.x) {
    const int n = idx % d.Nx, wf = idx / d.Nx;
    const int w = wf / 6, f = wf % 6;
    const int arr = (f == 0) ? 5 : (f == 1) ? 2 : (f == 2) ? 3 : (f == 3) ? 1
                    : (f == 4) ? (grad ? 0 : 4) : (grad ? 4 : 0);
    const c64 v = ARR[(w * 6 + arr) * d.Nx + n];
    *reinterpret_cast<double2*>(Bs + (size_t)n * kLDB + 2 * wf) = make_double2(v.re, v.im);
  }
  __syncthreads();
  cta_backward_dmma(o.VE, o.VO, d.Nx, 6, Bs, ARR, kNW);
  __syncthreads();
  for (int idx = threadIdx.x; idx < 6 * d.Nx * kNW; idx += blockDim.x) {
    const int w = idx % kNW, fi = idx / kNW;
    if (w < nvalid) {
      const size_t e = (size_t)fi * P + p0 + w;
      const c64 v = ARR[fi * kNW + w];
      if (a.x32) reinterpret_cast<c32*>(a.X)[e] = cmk((float)v.re, (float)v.im);
      else a.X[e] = v;
      if (grad && fi < 3 * d.Nx) {
        // fields 6..8: d/dy u_i = i ky u_i (the CTA's pencils share ky)
        const c64 dy = mul_i(kyp * v);
        const size_t ey = (size_t)(6 * d.Nx + fi) * P + p0 + w;
        if (a.x32) reinterpret_cast<c32*>(a.X)[ey] = cmk((float)dy.re, (float)dy.im);
        else a.X[ey] = dy;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// y_backward: per (x-plane, field): pad Ny -> My (middle zeros), inverse FFT.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) y_backward_kernel(Dims d, FFTPlan plan, int KC,
                                                         const cpx<T>* __restrict__ tw,
                                                         const cpx<T>* __restrict__ X,
                                                         cpx<T>* __restrict__ Y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* A = reinterpret_cast<cpx<T>*>(smem_raw);
  cpx<T>* B = A + d.My * KC;
  const int j = blockIdx.x, f = blockIdx.y, kc0 = blockIdx.z * KC;
  const cpx<T>* src = X + ((size_t)f * d.Nx + j) * d.P + kc0;
  const int half = d.Ny / 2;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int kz = idx % KC, r = idx / KC;
    cpx<T> v = cmk(T(0), T(0));
    if (r < half) v = src[r * d.Kz + kz];
    else if (r >= d.My - half) v = src[(r - d.My + d.Ny) * d.Kz + kz];
    A[idx] = v;
  }
  __syncthreads();
  cpx<T>* res = fft_columns<T>(A, B, plan, KC, KC, tw, +1);
  cpx<T>* dst = Y + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int kz = idx % KC, r = idx / KC;
    dst[(size_t)r * d.Kz + kz] = res[idx];
  }
}

// ---------------------------------------------------------------------------
// z_cross: per group of 4 (x, y) rows.  Six half spectra -> three complex
// inverse FFTs (two real fields packed per transform), base flow, the
// product -(u x omega), then two packed forward transforms per row pair.
// ---------------------------------------------------------------------------
constexpr int kZRows = 4;

// -(u x omega) of the perturbation (u, omega) about the base flow U_b e_y,
// U_wall e_z, expanded so that no O(1) base-flow value is added to a
// perturbation value before the products (FP32 keeps the perturbation's
// digits): -(u' x w') - U_b e_y x w' - U_wall u' x e_z.  The remaining
// base-flow self term -U_b U_wall e_x is constant in (y, z) and is added to
// the (ky, kz) = (0, 0) mode after the forward transforms.
template <typename T>
__device__ __forceinline__ void rotational_product(T u0, T u1, T u2, T w0, T w1, T w2, T ub, T uw,
                                                   T& n0, T& n1, T& n2) {
  n0 = -((u1 * w2 - u2 * w1) + uw * u1 + ub * w2);
  n1 = -((u2 * w0 - u0 * w2) - uw * u0);
  n2 = -((u0 * w1 - u1 * w0) - ub * w0);
}

template <typename T>
__global__ void __launch_bounds__(256) z_cross_kernel(DevOps o, Dims d, FFTPlan plan,
                                                      const cpx<T>* __restrict__ tw,
                                                      const cpx<T>* __restrict__ Y,
                                                      cpx<T>* __restrict__ HZ) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NC = kZRows * 3;  // packed columns
  cpx<T>* A = reinterpret_cast<cpx<T>*>(smem_raw);
  cpx<T>* B = A + d.Mz * NC;
  const int row0 = blockIdx.x * kZRows;  // row = j * My + y
  const int nrows = d.Nx * d.My;
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  // build the Hermitian-extended packed spectra Z = A_f + i A_{f+1}
  // k fastest: a warp reads consecutive spectral values of one row and field
  for (int idx = threadIdx.x; idx < d.Mz * NC; idx += blockDim.x) {
    const int k = idx % d.Mz, c = idx / d.Mz;
    const int rl = c / 3, pr = c % 3;
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
  // products: packed output columns per row pair q: [n0a+i n1a, n0b+i n1b, n2a+i n2b]
  const int NCf = (kZRows / 2) * 3;
  for (int idx = threadIdx.x; idx < d.Mz * kZRows; idx += blockDim.x) {
    const int rl = idx % kZRows, n = idx / kZRows;
    const int row = row0 + rl;
    const int j = (row < nrows) ? row / d.My : 0;
    const cpx<T> z0 = phys[n * NC + rl * 3 + 0];
    const cpx<T> z1 = phys[n * NC + rl * 3 + 1];
    const cpx<T> z2 = phys[n * NC + rl * 3 + 2];
    T n0, n1, n2;
    rotational_product(z0.re, z0.im, z1.re, z1.im, z2.re, z2.im, T(d.uwall * o.xphys[j]),
                       T(d.uwall), n0, n1, n2);
    const int q = rl >> 1, ab = rl & 1;
    other[n * NCf + q * 3 + ab] = cmk(n0, n1);
    if (ab == 0) other[n * NCf + q * 3 + 2].re = n2;
    else other[n * NCf + q * 3 + 2].im = n2;
  }
  __syncthreads();
  cpx<T>* spec = fft_columns<T>(other, phys, plan, NCf, NCf, tw, -1);
  const T scale = T(1.0 / d.Mz);
  for (int idx = threadIdx.x; idx < d.Kz * kZRows * 3; idx += blockDim.x) {
    const int k = idx % d.Kz;
    const int rf = idx / d.Kz;
    const int f = rf % 3, rl = rf / 3;
    const int row = row0 + rl;
    if (row >= nrows) continue;
    const int q = rl >> 1, ab = rl & 1;
    const int col = (f < 2) ? q * 3 + ab : q * 3 + 2;
    const cpx<T> Zk = spec[k * NCf + col];
    const cpx<T> Zm = spec[((d.Mz - k) % d.Mz) * NCf + col];
    // x + i y packed: X_k = (Z_k + conj Z_-k)/2, Y_k = (Z_k - conj Z_-k)/(2i)
    cpx<T> v;
    const bool take_real = (f < 2) ? (f == 0) : (ab == 0);
    const T h = T(0.5);
    if (take_real) v = cmk(h * (Zk.re + Zm.re), h * (Zk.im - Zm.im));
    else v = cmk(h * (Zk.im + Zm.im), -h * (Zk.re - Zm.re));
    HZ[(size_t)f * plane + (size_t)row * d.Kz + k] = scale * v;
  }
}

// ---------------------------------------------------------------------------
// z_grad: the z stage of the gradient form (channelflow_kmm.py:754-770 with
// the base-flow terms of pcf_fluctuations_jax.py:99-106), per group of 4
// (x, y) rows.  Y holds nine y-physical fields (u_i, d/dx u_i, d/dy u_i);
// d/dz u_i = i kz u_i is formed here.  Twelve real fields, two per complex
// inverse transform, give
//   n_i = u_0 d/dx u_i + u_1 d/dy u_i + u_2 d/dz u_i + U_b d/dy u_i
//         (+ u_0 dU_b/dx for i = 1),
// forward transformed two per complex transform (n2 alone).  In complex64
// (the mixed form) d.uwall = 0: the base-flow terms, linear in the
// perturbation, are added in FP64 by the pencil stage.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) z_grad_kernel(DevOps o, Dims d, FFTPlan plan,
                                                     const cpx<T>* __restrict__ tw,
                                                     const cpx<T>* __restrict__ Y,
                                                     cpx<T>* __restrict__ HZ) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = kZRows * 6;   // packed input columns
  constexpr int NCf = kZRows * 2;  // packed output columns: (n0 + i n1), (n2 + i 0)
  cpx<T>* A = reinterpret_cast<cpx<T>*>(smem_raw);
  cpx<T>* B = A + d.Mz * NC;
  const int row0 = blockIdx.x * kZRows;  // row = j * My + y
  const int nrows = d.Nx * d.My;
  const size_t plane = (size_t)d.Nx * d.My * d.Kz;
  // virtual real field v: v < 9 is Y field v, v >= 9 is i kz (Y field v - 9)
  auto spec = [&](int v, int row, int k) -> cpx<T> {
    const cpx<T> x = Y[(size_t)(v < 9 ? v : v - 9) * plane + (size_t)row * d.Kz + k];
    return v < 9 ? x : mul_i(T(k * d.dfz) * x);
  };
  for (int idx = threadIdx.x; idx < d.Mz * NC; idx += blockDim.x) {
    const int k = idx % d.Mz, c = idx / d.Mz;
    const int rl = c / 6, pr = c % 6;
    const int row = row0 + rl;
    cpx<T> z = cmk(T(0), T(0));
    if (row < nrows) {
      if (k == 0) {
        z = cmk(spec(2 * pr, row, 0).re, spec(2 * pr + 1, row, 0).re);
      } else if (k < d.Kz) {
        const cpx<T> xa = spec(2 * pr, row, k), xb = spec(2 * pr + 1, row, k);
        z = cmk(xa.re - xb.im, xa.im + xb.re);
      } else if (k > d.Mz - d.Kz) {
        const int kk = d.Mz - k;
        const cpx<T> xa = spec(2 * pr, row, kk), xb = spec(2 * pr + 1, row, kk);
        z = cmk(xa.re + xb.im, -xa.im + xb.re);  // conj(xa) + i conj(xb)
      }
    }
    A[k * NC + c] = z;
  }
  __syncthreads();
  cpx<T>* phys = fft_columns<T>(A, B, plan, NC, NC, tw, +1);
  cpx<T>* other = (phys == A) ? B : A;
  for (int idx = threadIdx.x; idx < d.Mz * kZRows; idx += blockDim.x) {
    const int rl = idx % kZRows, n = idx / kZRows;
    const int row = row0 + rl;
    const int j = (row < nrows) ? row / d.My : 0;
    const cpx<T>* z = phys + n * NC + rl * 6;
    const T u0 = z[0].re, u1 = z[0].im, u2 = z[1].re;
    const T x0 = z[1].im, x1 = z[2].re, x2 = z[2].im;  // d/dx
    const T y0 = z[3].re, y1 = z[3].im, y2 = z[4].re;  // d/dy
    const T z0 = z[4].im, z1 = z[5].re, z2 = z[5].im;  // d/dz
    const T ub = T(d.uwall * o.xphys[j]), uw = T(d.uwall);
    const T n0 = (u0 * x0 + u1 * y0 + u2 * z0) + ub * y0;
    const T n1 = ((u0 * x1 + u1 * y1 + u2 * z1) + ub * y1) + u0 * uw;
    const T n2 = (u0 * x2 + u1 * y2 + u2 * z2) + ub * y2;
    cpx<T>* out = other + n * NCf + rl * 2;
    out[0] = cmk(n0, n1);
    out[1] = cmk(n2, T(0));
  }
  __syncthreads();
  cpx<T>* res = fft_columns<T>(other, phys, plan, NCf, NCf, tw, -1);
  const T scale = T(1.0 / d.Mz), h = T(0.5);
  for (int idx = threadIdx.x; idx < d.Kz * kZRows * 3; idx += blockDim.x) {
    const int k = idx % d.Kz;
    const int rf = idx / d.Kz;
    const int f = rf % 3, rl = rf / 3;
    const int row = row0 + rl;
    if (row >= nrows) continue;
    const int col = rl * 2 + f / 2;
    const cpx<T> Zk = res[k * NCf + col];
    const cpx<T> Zm = res[((d.Mz - k) % d.Mz) * NCf + col];
    // x + i y packed: X_k = (Z_k + conj Z_-k)/2, Y_k = (Z_k - conj Z_-k)/(2i)
    cpx<T> v;
    if ((f & 1) == 0) v = cmk(h * (Zk.re + Zm.re), h * (Zk.im - Zm.im));
    else v = cmk(h * (Zk.im + Zm.im), -h * (Zk.re - Zm.re));
    HZ[(size_t)f * plane + (size_t)row * d.Kz + k] = scale * v;
  }
}

// ---------------------------------------------------------------------------
// y_forward: per (x-plane, field): forward FFT My, scale 1/My, keep Ny modes.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) y_forward_kernel(Dims d, FFTPlan plan, int KC,
                                                        const cpx<T>* __restrict__ tw,
                                                        const cpx<T>* __restrict__ HZ,
                                                        cpx<T>* __restrict__ HX,
                                                        const double* __restrict__ xb,
                                                        int keep_nyq = 0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cpx<T>* A = reinterpret_cast<cpx<T>*>(smem_raw);
  cpx<T>* B = A + d.My * KC;
  const int j = blockIdx.x, f = blockIdx.y, kc0 = blockIdx.z * KC;
  const cpx<T>* src = HZ + ((size_t)f * d.Nx + j) * (size_t)d.My * d.Kz + kc0;
  for (int idx = threadIdx.x; idx < d.My * KC; idx += blockDim.x) {
    const int kz = idx % KC, r = idx / KC;
    A[idx] = src[(size_t)r * d.Kz + kz];
  }
  __syncthreads();
  cpx<T>* res = fft_columns<T>(A, B, plan, KC, KC, tw, -1);
  const T scale = T(1.0 / d.My);
  const int half = d.Ny / 2;
  if (xb && f == 0 && kc0 == 0 && threadIdx.x == 0) {
    // base-flow self term -U_b U_wall e_x: its (ky, kz) = (0, 0) mode
    res[0].re += T(-d.uwall * xb[j] * d.uwall * d.My);
  }
  __syncthreads();
  cpx<T>* dst = HX + ((size_t)f * d.Nx + j) * d.P + kc0;
  for (int idx = threadIdx.x; idx < d.Ny * KC; idx += blockDim.x) {
    const int kz = idx % KC, r = idx / KC;
    cpx<T> v = cmk(T(0), T(0));
    if (r < half) v = res[r * KC + kz];
    else if (r > half) v = res[(r - d.Ny + d.My) * KC + kz];
    else if (keep_nyq) v = res[(d.My - half) * KC + kz];  // the -Ny/2 mode (else masked)
    dst[(size_t)r * d.Kz + kz] = scale * v;
  }
}

// ---------------------------------------------------------------------------
// z_forward_real: three real physical fields (Nx, Ny, Nz) -> half spectra
// along z, scaled 1/Nz (Fourier.forward, norm="forward").  Per 4 rows: two
// fields packed per complex transform, third field packed across row pairs.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) z_forward_real_kernel(Dims d, FFTPlan plan,
                                                             const c64* __restrict__ tw,
                                                             const double* __restrict__ f0,
                                                             const double* __restrict__ f1,
                                                             const double* __restrict__ f2,
                                                             c64* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NCf = (kZRows / 2) * 3;
  const int n = d.Nz;
  c64* A = reinterpret_cast<c64*>(smem_raw);
  c64* B = A + n * NCf;
  const int row0 = blockIdx.x * kZRows;
  const int nrows = d.Nx * d.Ny;
  for (int idx = threadIdx.x; idx < n * kZRows; idx += blockDim.x) {
    const int rl = idx % kZRows, z = idx / kZRows;
    const int row = row0 + rl;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    if (row < nrows) {
      const size_t e = (size_t)row * n + z;
      a0 = f0[e];
      a1 = f1[e];
      a2 = f2[e];
    }
    const int q = rl >> 1, ab = rl & 1;
    A[z * NCf + q * 3 + ab] = cmk(a0, a1);
    if (ab == 0) A[z * NCf + q * 3 + 2].re = a2;
    else A[z * NCf + q * 3 + 2].im = a2;
  }
  __syncthreads();
  c64* spec = fft_columns<double>(A, B, plan, NCf, NCf, tw, -1);
  const double scale = 1.0 / n;
  const size_t plane = (size_t)d.Nx * d.Ny * d.Kz;
  for (int idx = threadIdx.x; idx < d.Kz * kZRows * 3; idx += blockDim.x) {
    const int k = idx % d.Kz;
    const int rf = idx / d.Kz;
    const int f = rf % 3, rl = rf / 3;
    const int row = row0 + rl;
    if (row >= nrows) continue;
    const int q = rl >> 1, ab = rl & 1;
    const int col = (f < 2) ? q * 3 + ab : q * 3 + 2;
    const c64 Zk = spec[k * NCf + col];
    const c64 Zm = spec[((n - k) % n) * NCf + col];
    c64 v;
    const bool take_real = (f < 2) ? (f == 0) : (ab == 0);
    if (take_real) v = cmk(0.5 * (Zk.re + Zm.re), 0.5 * (Zk.im - Zm.im));
    else v = cmk(0.5 * (Zk.im + Zm.im), -0.5 * (Zk.re - Zm.re));
    out[(size_t)f * plane + (size_t)row * d.Kz + k] = scale * v;
  }
}

// ---------------------------------------------------------------------------
// Diagnostics of PlaneCouetteFluctuationJax (pcf_fluctuations_jax.py:131-161)
// from the spectral state.  y/z integrals use Parseval (exact for the
// reference's uniform quadrature); x uses the Fejer-I weights of the Gauss
// nodes.  Per block: partial sums of |u|^2 and |div u|^2; the mean pencil
// writes its wall / base-flow terms.  diag_finish_kernel reduces in a fixed
// order (deterministic).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) diag_kernel(DevOps o, Dims d, const c64* __restrict__ u0,
                                                   const c64* __restrict__ u1,
                                                   const c64* __restrict__ u2,
                                                   double* __restrict__ partial,
                                                   double* __restrict__ meanterms) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c64* ARR = reinterpret_cast<c64*>(smem_raw);  // kNW * 4 * Nx
  double* red = reinterpret_cast<double*>(ARR + kNW * 4 * d.Nx);  // kNW * 2
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kyi = blockIdx.x / d.nKb;
  const int kz = (blockIdx.x % d.nKb) * kNW + warp;
  const int ky = (kyi < d.Ny / 2) ? kyi : kyi - d.Ny;
  const bool active = kz < d.Kz && kyi != d.Ny / 2;
  const int p = kyi * d.Kz + kz;
  const size_t P = (size_t)d.P;
  const double kyp = ky * d.dfy, kzp = kz * d.dfz;
  c64* B0 = ARR + warp * 4 * d.Nx;  // uo0
  c64* B1 = B0 + d.Nx;              // uo1
  c64* B2 = B1 + d.Nx;              // uo2
  c64* B3 = B2 + d.Nx;              // div
  double e_u = 0.0, e_div = 0.0;
  if (active) {
    for (int i = lane; i < d.nD; i += 32) {
      B1[i] = u1[(size_t)i * P + p];
      B2[i] = u2[(size_t)i * P + p];
      if (i < d.nB) B3[i] = u0[(size_t)i * P + p];
    }
    __syncwarp();
    apply_SBT(o, d, B3, B0, lane);
    if (lane == 0) {
      for (int n = d.Nx - 1; n >= 0; --n) {
        c64 v = (n < d.nD) ? B1[n] : cmk(0.0, 0.0);
        if (n >= 2) v = v - B1[n - 2];
        B1[n] = v;
      }
    } else if (lane == 1) {
      for (int n = d.Nx - 1; n >= 0; --n) {
        c64 v = (n < d.nD) ? B2[n] : cmk(0.0, 0.0);
        if (n >= 2) v = v - B2[n - 2];
        B2[n] = v;
      }
    }
    __syncwarp();
    chebder_warp(B0, B3, d.Nx, d.dfx, lane, d.family);
    for (int n = lane; n < d.Nx; n += 32) B3[n] = B3[n] + mul_i(kyp * B1[n] + kzp * B2[n]);
    __syncwarp();
    const double mult = (kz == 0) ? 1.0 : 2.0;
    for (int j = lane; j < d.Nx; j += 32) {
      c64 v0 = cmk(0.0, 0.0), v1 = v0, v2 = v0, v3 = v0;
      for (int n = 0; n < d.Nx; ++n) {
        const double t = __ldg(o.V + (size_t)j * d.Nx + n);
        v0 = v0 + t * B0[n];
        v1 = v1 + t * B1[n];
        v2 = v2 + t * B2[n];
        v3 = v3 + t * B3[n];
      }
      const double w = o.fejer[j] * mult;
      e_u += w * (v0.re * v0.re + v0.im * v0.im + v1.re * v1.re + v1.im * v1.im +
                  v2.re * v2.re + v2.im * v2.im);
      e_div += w * (v3.re * v3.re + v3.im * v3.im);
      if (ky == 0 && kz == 0) {
        // base-flow cross term 2 Ub Re(u1_00) + Ub^2 and the mean shear dv/dx
        const double ub = d.uwall * o.xphys[j];
        meanterms[8 + j] = o.fejer[j] * (2.0 * ub * v1.re + ub * ub);
      }
    }
    if (ky == 0 && kz == 0) {
      // wall values and wall derivatives of the mean streamwise velocity
      chebder_warp(B1, B3, d.Nx, d.dfx, lane, d.family);
      if (lane == 0) {
        double top = 0.0, bot = 0.0, stop = 0.0, sbot = 0.0, shear = 0.0;
        for (int n = 0; n < d.Nx; ++n) {
          const double sgn = (n & 1) ? -1.0 : 1.0;
          top += B1[n].re;
          bot += sgn * B1[n].re;
          // d/dX P_n at X = 1: n^2 (Chebyshev), n (n + 1) / 2 (Legendre)
          const double n2 = d.family ? 0.5 * n * (n + 1.0) : (double)n * n;
          stop += n2 * B1[n].re * d.dfx;
          sbot += -sgn * n2 * B1[n].re * d.dfx;
        }
        for (int j = 0; j < d.Nx; ++j) {
          double dv = 0.0;
          for (int n = 0; n < d.Nx; ++n) dv += __ldg(o.V + (size_t)j * d.Nx + n) * B3[n].re;
          shear += o.fejer[j] * dv;
        }
        meanterms[0] = top;
        meanterms[1] = bot;
        meanterms[2] = stop;
        meanterms[3] = sbot;
        meanterms[4] = shear;
      }
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    e_u += __shfl_down_sync(0xffffffffu, e_u, off);
    e_div += __shfl_down_sync(0xffffffffu, e_div, off);
  }
  if (lane == 0) {
    red[2 * warp] = e_u;
    red[2 * warp + 1] = e_div;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kNW; ++w) {
      a += red[2 * w];
      b += red[2 * w + 1];
    }
    partial[2 * blockIdx.x] = a;
    partial[2 * blockIdx.x + 1] = b;
  }
}

// out = (Epert, Etot, divL2, u_top, u_bot, wall_shear_top, wall_shear_bot, mean_shear)
__global__ void diag_finish_kernel(Dims d, const double* __restrict__ partial, int nblocks,
                                   const double* __restrict__ meanterms, double ly, double lz,
                                   double x_lo, double x_hi, double* __restrict__ out,
                                   int* status) {
  const double lx = x_hi - x_lo;
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double eu = 0.0, ed = 0.0, base = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    eu += partial[2 * b];
    ed += partial[2 * b + 1];
  }
  for (int j = 0; j < d.Nx; ++j) base += meanterms[8 + j];
  const double area = ly * lz;
  out[0] = area * eu;
  out[1] = area * (eu + base);
  out[2] = sqrt(area * ed);
  out[3] = meanterms[0] + d.uwall * x_hi;
  out[4] = meanterms[1] + d.uwall * x_lo;
  out[5] = meanterms[2] + d.uwall;
  out[6] = meanterms[3] + d.uwall;
  out[7] = (area * meanterms[4] + d.uwall * lx * area) / (lx * area);
  bool bad = false;
  for (int k = 0; k < 8; ++k) bad |= !isfinite(out[k]);
  flag_nonfinite(status, bad);
}

}  // namespace jfb
