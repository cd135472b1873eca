// Pencil stage of the KMM step as FP64 tensor-core products (mma.sync
// m8n8k4 f64; tcgen05 has no FP64 kind).
//
// One CTA owns a tile of 16 pencils: wavenumbers (+ky, kz0..kz0+7) in columns
// 0-7 and (-ky, kz0..kz0+7) in columns 8-15, so each per-wavenumber factor is
// read once for two pencils.  Per implicit stage (SBDF3 step or IMEXRK3
// stage) the CTA
//   A  stages the x-physical nonlinear samples as mirror sums / differences
//      weighted by (i ky, i kz, k^2), and the mass-row inputs by parity;
//   B  forms Nu, Ng (x-forward, projection, derivative and stencil folded into
//      the R matrices) and the mass rows as products against the parity-split
//      operators, and in the epilogue the time-stepping right-hand sides;
//   C  solves Su, Sg per wavenumber: banded forward elimination with the unit
//      lower factor, then the explicit inverse of the upper factor;
//   D  forms u and omega at the x Gauss nodes as products against the folded
//      reconstruction operators and writes the six fields.
// The ky = kz = 0 pencil also carries the mean-flow system S00.
//
// Operand layout: a sub-matrix of R x K is stored as 8x4 tiles in fragment
// order (one double per lane, coalesced); B operands live in shared memory
// as rows of 16 complex values (32 real columns, re/im interleaved) with a
// 36-double stride so that fragment loads are bank-conflict free.  Inputs are
// staged with 16-byte cp.async copies (thousands of 128-byte bulk copies per
// CTA proved slow: each is one copy-engine operation); the velocity operators
// arrive in one bulk copy into rows that are dead by then.  Every CTA reads
// all operators, so the plan keeps several copies and CTA b reads copy
// b % nrep, spreading those L2 lines.
#pragma once

#include "jfb_kmm.h"
#include "jfb_kmm_kernels.cuh"
#include "jfb_tc.cuh"

namespace jfb {

constexpr int kGW = 16;         // pencils per CTA
constexpr int kGLd = 36;        // doubles per shared row: 2 kGW + 4
// Threads per CTA (a multiple of 128, at least 384: the tcgen05 epilogue
// reads TMEM with twelve warps).  Twelve warps at up to 168 registers took
// 47.7 us per CTA at 65x64x64, sixteen at 128 registers 43.7 us.
// Base-flow samples of the mixed form loaded before the staging copies are
// issued (1) or while they fly (0).  Before: 46.2 us per CTA at 65x64x64,
// while they fly: 44.8 us.
#ifndef JFB_XLIN_EARLY
#define JFB_XLIN_EARLY 0
#endif
#ifndef JFB_GEMM_THREADS
#define JFB_GEMM_THREADS 512
#endif
constexpr int kGThreads = JFB_GEMM_THREADS;
static_assert(kGThreads % 128 == 0 && kGThreads >= 384, "pencil_gemm_kernel thread count");
constexpr int kGWarps = kGThreads / 32;

struct SubDesc {
  int off, mt, kt, kr;
};

struct GemmOps {
  const double* frag;   // nrep copies of the fragment-tiled operators
  const int* krange;
  const double* R3;     // S_D Q (nD x Nx)
  const double* X2D;    // nD x nD
  const double* mid;    // middle-node rows (odd Nx), 5 x mid_stride
  int* status;          // device status word (nonzero: a bounded wait gave up)
  SubDesc sub[gNumSub];
  int Jh, Jl, nBe, nBo, nDe, nDo;
  int kt_mu_lin[2], kt_mg_lin[2];  // k-tile limits when the stage has no linear term
  // shared-memory row offsets (rows of kGLd doubles)
  int oH[3], oMUE, oMUO, oMGE, oMGO, oRU, oRG, oUE, oUO, oGE, oGO, oVel, rows;
  int oMean;    // first double of the mean-flow scratch
  int oMid;     // first double of the middle-node scratch (5 x 2 kGW doubles)
  int nfrag;    // doubles in one copy of frag; the velocity sub-matrices are its tail
  int nrep;     // copies of frag (CTA b reads copy b % nrep)
  int mid_stride;
  // Tensor-core velocity products (mixed form): split-BF16 operator image in
  // the tcgen05 operand layout (kTcImgA bytes), copied into dead shared
  // memory at byte offset oTA; the split state operand goes to byte oTB.
  int tc;
  const unsigned char* vimg;
  int oTA, oTB;
  // forward-elimination multipliers of the tile's wavenumbers, staged into
  // dead shared memory at the start of phase C (first double; -1: read from
  // L2 instead)
  int oL;
};

// Tensor-core velocity stage: three product groups of M = 128 rows (four
// 32-row quarters, one velocity / vorticity half-product each) x N = 32
// columns (16 pencils x re/im), K = 32, 32, 64 coefficient rows:
//   group 0 (B = u0 even): A0Ee, P2Ee, P1Oe, -
//   group 1 (B = u0 odd):  P1Eo, A0Oo, P2Oo, -
//   group 2 (B = [g even; g odd]): B1Ee | 0, B2Oe | 0, 0 | B2Eo, 0 | B1Oo
// Every operand is split into three BF16 parts (hi, mid, lo) and the six
// products of combined order <= 2 are accumulated in FP32 in TMEM.
__host__ __device__ constexpr int tc_k(int g) { return g == 2 ? 64 : 32; }
constexpr int kTcImgA = 3 * 128 * (32 + 32 + 64) * 2;  // 98304 bytes
constexpr int kTcImgB = 3 * 32 * (32 + 32 + 64) * 2;   // 24576 bytes
__host__ __device__ inline int tc_a_off(int g, int s) {
  return 3 * 128 * 2 * (g == 0 ? 0 : g == 1 ? 32 : 64) + s * 128 * 2 * (g == 2 ? 64 : 32);
}
__host__ __device__ inline int tc_b_off(int g, int s) {
  return 3 * 32 * 2 * (g == 0 ? 0 : g == 1 ? 32 : 64) + s * 32 * 2 * (g == 2 ? 64 : 32);
}
// acc slot (velocity_fields argument order, see phase D) of group g, quarter q
__host__ __device__ inline int tc_slot(int g, int q) {
  const int t[3][4] = {{0, 2, 6, -1}, {1, 5, 7, -1}, {3, 9, 4, 8}};
  return t[g][q];
}
constexpr int kTcStagePitch = 33;  // floats per staged row (conflict-free)

// Largest k-tile ranges of the pipelined products (checked on the host).
constexpr int kKtN = 20;   // Nu / Ng products
constexpr int kKtM = 24;   // mass-row products
constexpr int kMaxM = 32;  // rows per parity class of Su / Sg

struct GemmStageArgs {
  const c64* HX;
  double c0, c1, c2, d0, d1, d2, slin;  // slin = (implicit linear coefficient) * nu
  const c64 *u0a, *u0b, *u0c, *ga, *gb, *gc, *vwa, *vwb, *vwc;
  const c64 *Nup, *Nuq, *Ngp, *Ngq, *NVWp, *NVWq;
  c64 *Nu_out, *Ng_out, *NVW_out;
  const double *su, *sg, *s00;  // records: L pairs, then inverse upper triangles
  const double* s00inv;         // mean-flow system inverse (nD x nD, row-major)
  int su_rec, sg_rec;
  c64 *u0_out, *g_out, *vw_out;
  c64* X;
  int x32;  // HX and X hold complex64 values (mixed form)
  // mixed form: x-physical u, omega (complex64) of the state whose nonlinear
  // term is in HX; the FP32 transforms carry only -(u' x omega') and the
  // base-flow terms, linear in u', omega', are added here in FP64
  const c32* Xlin;
};

// Base-flow part of the rotational term at one x node (pcf_fluctuations_jax.py:
// 108-112 with U_b = U_wall x): -U_b e_y x omega' - U_wall u' x e_z, plus the
// constant -U_b U_wall e_x on the mean pencil.  f = field order u0, u1, u2,
// omega0, omega1, omega2 of X.
// x = (u0, u1, omega0, omega2) at the node.
__device__ __forceinline__ void add_base_flow_terms(const c32 (&x)[4], bool mean, double ub,
                                                    double uw, c64 (&h)[3]) {
  auto c = [&](int k) { return cmk((double)x[k].re, (double)x[k].im); };
  h[0] = h[0] - uw * c(1) - ub * c(3);
  h[1] = h[1] + uw * c(0);
  h[2] = h[2] + ub * c(2);
  if (mean) h[0].re -= ub * uw;
}

// Gradient form (pcf_fluctuations_jax.py:99-106): U_b d/dy u_i and
// u_0 dU_b/dx e_y at one x node, from x = (u0, d/dy u0, d/dy u1, d/dy u2)
// (X fields 0, 6, 7, 8).
__device__ __forceinline__ void add_base_convection_terms(const c32 (&x)[4], double ub, double uw,
                                                          c64 (&h)[3]) {
  auto c = [&](int k) { return cmk((double)x[k].re, (double)x[k].im); };
  h[0] = h[0] + ub * c(1);
  h[1] = (h[1] + ub * c(2)) + uw * c(0);
  h[2] = h[2] + ub * c(3);
}

__host__ __device__ inline int round4(int x) { return (x + 3) & ~3; }

// Read-only (non-coherent) load of one complex value.
__device__ __forceinline__ c64 ldg_c(const c64* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return cmk(v.x, v.y);
}

// ---------------------------------------------------------------------------
// asynchronous copies
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// L2 prefetch of [ptr, ptr + bytes) in whole 16-byte units.
__device__ __forceinline__ void prefetch_l2(const void* ptr, size_t bytes) {
  uintptr_t a = reinterpret_cast<uintptr_t>(ptr);
  const uintptr_t lo = a & ~(uintptr_t)15, hi = (a + bytes + 15) & ~(uintptr_t)15;
  for (uintptr_t x = lo; x < hi; x += 32768) {
    const uint32_t n = (uint32_t)min((uintptr_t)32768, hi - x);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(x), "r"(n) : "memory");
  }
}
// 16-byte asynchronous global -> shared copy (L2 only), and its completion.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bulk global -> shared copy (no multicast) completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of `bar` for at most ~2^27 cycles (tens of ms).
// On time-out the status word gets the bit `code`, the wait is repeated once
// with the same limit (the copy in flight targets this CTA's shared memory),
// and false is returned.
__device__ __noinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* status, int code) {
  for (int round = 0; round < 2; ++round) {
    const long long t0 = clock64();
    while (clock64() - t0 < (1ll << 27))
      if (mbar_try(bar, parity)) return round == 0;
    if (round == 0 && status) atomicOr(status, code);
  }
  return false;
}

// acc[nt] += A(rows of one 8-row tile) * B(Bs rows, columns 8 nt ..), k tiles
// [kb, ke) with ke - kb <= KMAX; A fragments are loaded in chunks of 8 k tiles,
// the next chunk in flight while the current one is multiplied.
// The rolled form of the products (JFB_GEMM_COMPACT = 1) is the default:
// its smaller code cut phase B from 12.6 to 9.9 us per CTA at 65x64x64 (the
// unrolled form stalled on instruction fetch).
#ifndef JFB_VEL_UNROLL
#define JFB_VEL_UNROLL 1
#endif
constexpr int kVelUnroll = JFB_VEL_UNROLL;  // k tiles per unrolled step of the velocity products
#ifndef JFB_GEMM_COMPACT
#define JFB_GEMM_COMPACT 1
#endif
template <int NT, int KMAX>
__device__ __forceinline__ void gemm_acc(const double* __restrict__ A, int kb, int ke,
                                         const double* __restrict__ Bs, int lane,
                                         double (&acc)[NT][2]) {
#if JFB_GEMM_COMPACT
  // rolled form: two chunk buffers, the next chunk loading while the current
  // one is multiplied (smaller code than the unrolled form below)
  constexpr int CH = 8;
  const int g = lane >> 2, t4 = lane & 3;
  const double* __restrict__ b = Bs + t4 * kGLd + g;
  double a0[CH], a1[CH];
  auto load = [&](double (&af)[CH], int k0) {
#pragma unroll
    for (int k = 0; k < CH; ++k) af[k] = (k0 + k < ke) ? __ldg(A + (k0 + k) * 32 + lane) : 0.0;
  };
  auto mul = [&](const double (&af)[CH], int k0) {
#pragma unroll
    for (int k = 0; k < CH; ++k)
      if (k0 + k < ke) {
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
          dmma_8x8x4(acc[nt][0], acc[nt][1], af[k], b[(k0 + k) * 4 * kGLd + nt * 8]);
      }
  };
  if (kb >= ke) return;
  load(a0, kb);
#pragma unroll 1
  for (int k0 = kb; k0 < ke; k0 += 2 * CH) {
    if (k0 + CH < ke) load(a1, k0 + CH);
    mul(a0, k0);
    if (k0 + CH >= ke) break;
    if (k0 + 2 * CH < ke) load(a0, k0 + 2 * CH);
    mul(a1, k0 + CH);
  }
#else
  constexpr int CH = 8, NC = (KMAX + CH - 1) / CH;
  const int g = lane >> 2, t4 = lane & 3;
  const double* __restrict__ b = Bs + t4 * kGLd + g;
  double af[2][CH];
#pragma unroll
  for (int k = 0; k < CH; ++k) af[0][k] = (kb + k < ke) ? __ldg(A + (kb + k) * 32 + lane) : 0.0;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (c + 1 < NC) {
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int kk = kb + (c + 1) * CH + k;
        af[(c + 1) & 1][k] = (kk < ke) ? __ldg(A + kk * 32 + lane) : 0.0;
      }
    }
#pragma unroll
    for (int k = 0; k < CH; ++k) {
      const int kk = kb + c * CH + k;
      if (kk < ke) {
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
          dmma_8x8x4(acc[nt][0], acc[nt][1], af[c & 1][k], b[kk * 4 * kGLd + nt * 8]);
      }
    }
  }
#endif
}

__device__ __forceinline__ int2 sub_krange(const GemmOps& G, int id, int mt) {
  const int* kr = G.krange + G.sub[id].kr + 2 * mt;
  return make_int2(kr[0], kr[1]);
}

// u, omega (f[0..5]) of one pencil from the symmetric or antisymmetric
// halves of A0 u0, P1 u0, P2 u0, B1 g, B2 g; for ky = kz = 0 the g slot
// carries the mean flow v + i w.
__device__ __forceinline__ void velocity_fields(double ky, double kz, c64 av, c64 b1, c64 b2,
                                                c64 c1, c64 c2, c64 (&f)[6]) {
  const double k2 = ky * ky + kz * kz;
  f[0] = av;
  if (k2 == 0.0) {
    f[1] = cmk(c1.re, 0.0);
    f[2] = cmk(c1.im, 0.0);
    f[3] = cmk(0.0, 0.0);
    f[4] = cmk(-c2.im, 0.0);
    f[5] = cmk(c2.re, 0.0);
  } else {
    const double inv = 1.0 / k2;
    f[1] = mul_i((ky * inv) * b1 + (kz * inv) * c1);
    f[2] = mul_i((kz * inv) * b1 - (ky * inv) * c1);
    f[3] = c1;
    f[4] = mul_i(kz * av) - mul_i((kz * inv) * b2 - (ky * inv) * c2);
    f[5] = mul_i((ky * inv) * b2 + (kz * inv) * c2) - mul_i(ky * av);
  }
}

// Gradient form: u, d/dx u and d/dy u = i ky u (f[0..8]) of one pencil from
// the symmetric or antisymmetric halves of A0 u0, A1 u0, P1 u0, P2 u0, B1 g,
// B2 g (d/dx u1, d/dx u2 are the terms of omega that velocity_fields forms
// from P2 u0, B2 g); for ky = kz = 0 the g slot carries the mean flow v + i w.
__device__ __forceinline__ void gradient_fields(double ky, double kz, c64 av, c64 a1, c64 b1,
                                                c64 b2, c64 c1, c64 c2, c64 (&f)[9]) {
  const double k2 = ky * ky + kz * kz;
  f[0] = av;
  f[3] = a1;
  if (k2 == 0.0) {
    f[1] = cmk(c1.re, 0.0);
    f[2] = cmk(c1.im, 0.0);
    f[4] = cmk(c2.re, 0.0);
    f[5] = cmk(c2.im, 0.0);
  } else {
    const double inv = 1.0 / k2;
    f[1] = mul_i((ky * inv) * b1 + (kz * inv) * c1);
    f[2] = mul_i((kz * inv) * b1 - (ky * inv) * c1);
    f[4] = mul_i((ky * inv) * b2 + (kz * inv) * c2);
    f[5] = mul_i((kz * inv) * b2 - (ky * inv) * c2);
  }
  f[6] = mul_i(ky * f[0]);
  f[7] = mul_i(ky * f[1]);
  f[8] = mul_i(ky * f[2]);
}

// Forward elimination with the unit lower factor of one parity class, in
// place on y[r * stride] (r < m): y_r -= L[i, i-2] y_{r-1} + L[i, i-4] y_{r-2},
// i = 2 r + par; the multipliers (rec[2 i], rec[2 i + 1]) are loaded eight
// rows ahead of their use.
__device__ __forceinline__ void forward_elim(const double* __restrict__ rec, int par, int m,
                                             c64* y, int stride) {
  constexpr int CH = 8, NC = kMaxM / CH;
  double l1[2][CH], l2[2][CH];
#pragma unroll
  for (int k = 0; k < CH; ++k) {
    const int i = 2 * k + par;
    l1[0][k] = (k < m) ? __ldg(rec + 2 * i) : 0.0;
    l2[0][k] = (k < m) ? __ldg(rec + 2 * i + 1) : 0.0;
  }
  c64 y1 = cmk(0.0, 0.0), y2 = y1;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    if (c + 1 < NC) {
#pragma unroll
      for (int k = 0; k < CH; ++k) {
        const int r = (c + 1) * CH + k, i = 2 * r + par;
        l1[(c + 1) & 1][k] = (r < m) ? __ldg(rec + 2 * i) : 0.0;
        l2[(c + 1) & 1][k] = (r < m) ? __ldg(rec + 2 * i + 1) : 0.0;
      }
    }
#pragma unroll
    for (int k = 0; k < CH; ++k) {
      const int r = c * CH + k;
      if (r < m) {
        c64 v = y[r * stride];
        v = v - l1[c & 1][k] * y1;
        v = v - l2[c & 1][k] * y2;
        y[r * stride] = v;
        y2 = y1;
        y1 = v;
      }
    }
  }
}

// forward_elim with the multipliers staged in shared memory (ls = the first
// 2 n doubles of the record: L[i, i-2], L[i, i-4] for i = 0..n-1).
__device__ __forceinline__ void forward_elim_smem(const double* ls, int par, int m, c64* y,
                                                  int stride) {
  c64 y1 = cmk(0.0, 0.0), y2 = y1;
  for (int r = 0; r < m; ++r) {
    const int i = 2 * r + par;
    c64 v = y[r * stride];
    v = v - ls[2 * i] * y1;
    v = v - ls[2 * i + 1] * y2;
    y[r * stride] = v;
    y2 = y1;
    y1 = v;
  }
}

// Named barrier over `count` threads.
__device__ __forceinline__ void bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Mean-flow system of the ky = kz = 0 pencil (channelflow_kmm.py mean rows)
// on kMeanThreads threads t: N = -(S_D Q Re H1, S_D Q Re H2), rhs = M00 comb
// + slin X2D vwa + dt (d0 N + d1 N' + d2 N''), S00 solve (forward
// elimination, then the inverse upper factor).  Leaves (v, w) in vwx.
constexpr int kMeanThreads = 192;
__device__ void mean_flow(const Dims& d, const DevOps& o, const GemmOps& G,
                          const GemmStageArgs& a, const double* hm, c64* nvw, c64* vw,
                          c64* vwx, int t) {
  const int N = d.Nx, nD = d.nD, Jl = N / 2;
  for (int e = t; e < 2 * nD; e += kMeanThreads) {
    const int i = e >> 1, f = e & 1;
    const double* __restrict__ r3 = G.R3 + (size_t)i * N;
    const double* h = hm + f * N;
    const double sg = (i & 1) ? -1.0 : 1.0;  // rows of S_D Q have the parity of i
    double a0 = 0.0, a1 = 0.0;
#pragma unroll 8
    for (int j = 0; j + 1 < Jl; j += 2) {
      a0 += __ldg(r3 + j) * (h[j] + sg * h[N - 1 - j]);
      a1 += __ldg(r3 + j + 1) * (h[j + 1] + sg * h[N - 2 - j]);
    }
    if (Jl & 1) a0 += __ldg(r3 + Jl - 1) * (h[Jl - 1] + sg * h[N - Jl]);
    if ((N & 1) && !(i & 1)) a1 += __ldg(r3 + Jl) * h[Jl];
    reinterpret_cast<double*>(nvw)[e] = -(a0 + a1);
  }
  bar_sync(1, kMeanThreads);
  for (int i = t; i < nD; i += kMeanThreads) {
    auto comb = [&](int k) {
      c64 v = a.c0 * ldg_c(a.vwa + k);
      if (a.c1 != 0.0) v = v + a.c1 * ldg_c(a.vwb + k);
      if (a.c2 != 0.0) v = v + a.c2 * ldg_c(a.vwc + k);
      return v;
    };
    c64 r = o.mdi[i] * comb(i);
    if (i >= 2) r = r + o.mlo[i] * comb(i - 2);
    if (i + 2 < nD) r = r + o.mhi[i] * comb(i + 2);
    if (a.slin != 0.0) {
      c64 s = cmk(0.0, 0.0);
#pragma unroll 8
      for (int k = 0; k < nD; ++k) s = s + __ldg(G.X2D + (size_t)i * nD + k) * ldg_c(a.vwa + k);
      r = r + a.slin * s;
    }
    c64 nl = a.d0 * nvw[i];
    if (a.d1 != 0.0) nl = nl + a.d1 * ldg_c(a.NVWp + i);
    if (a.d2 != 0.0) nl = nl + a.d2 * ldg_c(a.NVWq + i);
    if (a.NVW_out) a.NVW_out[i] = nvw[i];
    vw[i] = r + d.dt * nl;
  }
  bar_sync(1, kMeanThreads);
  // S00^-1 rhs: rows of parity p couple only to columns of parity p (a
  // sequential elimination on two threads would sit on the kernel's
  // critical path; the inverse makes it one product per row)
  for (int i = t; i < nD; i += kMeanThreads) {
    const double* __restrict__ row = a.s00inv + (size_t)i * nD;
    c64 x0 = cmk(0.0, 0.0), x1 = x0;
    int k = i & 1;
#pragma unroll 4
    for (; k + 2 < nD; k += 4) {
      x0 = x0 + __ldg(row + k) * vw[k];
      x1 = x1 + __ldg(row + k + 2) * vw[k + 2];
    }
    if (k < nD) x0 = x0 + __ldg(row + k) * vw[k];
    const c64 xv = x0 + x1;
    vwx[i] = xv;
    a.vw_out[i] = xv;
    flag_nonfinite(G.status, !finite_c(xv));
  }
}

// One value of the middle-node products (odd N): operator op = e / 32 of
// (A0, P2 | u0 even; P1 | u0 odd; B1 | g even; B2 | g odd; A1 | u0 odd,
// gradient form only), column e % 32.
__device__ __forceinline__ double mid_dot(const GemmOps& G, const double* sm, int e) {
  const int col = e % (2 * kGW), op = e / (2 * kGW);
  const int oB = (op <= 1) ? G.oUE : (op == 2 || op == 5) ? G.oUO : (op == 3) ? G.oGE : G.oGO;
  const int K = (op <= 1) ? G.nBe : (op == 2 || op == 5) ? G.nBo : (op == 3) ? G.nDe : G.nDo;
  const double* row = G.mid + op * G.mid_stride;
  double s = 0.0;
  for (int k = 0; k < K; ++k) s += __ldg(row + k) * sm[(size_t)(oB + k) * kGLd + col];
  return s;
}

// u, omega at the middle node of pencil w from the products md[].
__device__ __forceinline__ void mid_store(const bool grad, const GemmStageArgs& a, const double* md,
                                          const int* s_p, const double* s_ky, const double* s_kz,
                                          int w, int N, int Jl, size_t P) {
  if (s_p[w] < 0) return;
  auto val = [&](int op) { return cmk(md[op * 2 * kGW + 2 * w], md[op * 2 * kGW + 2 * w + 1]); };
  auto put = [&](int q, const c64 v) {
    const size_t e = (size_t)q * N * P + (size_t)Jl * P + s_p[w];
    if (a.x32) reinterpret_cast<c32*>(a.X)[e] = cmk((float)v.re, (float)v.im);
    else a.X[e] = v;
  };
  if (grad) {
    c64 f[9];
    gradient_fields(s_ky[w], s_kz[w], val(0), val(5), val(2), val(1), val(3), val(4), f);
#pragma unroll
    for (int q = 0; q < 9; ++q) put(q, f[q]);
  } else {
    c64 f[6];
    velocity_fields(s_ky[w], s_kz[w], val(0), val(2), val(1), val(3), val(4), f);
#pragma unroll
    for (int q = 0; q < 6; ++q) put(q, f[q]);
  }
}

// The pencil stage of one tile `bid` of `nbid` (the kernel below, or one
// member's tile of the ensemble kernel in jfb_kmm_ens.cuh).
// kTC = false compiles the body without the tcgen05 velocity products (the
// default kernel: a smaller instruction footprint, 78.7 -> 77.4 us per
// mixed step at 65x64x64); kTC = true keeps them behind the plan's runtime
// flag G.tc.  kForm: 0 rotational, 1 gradient (each without the other's
// code), 2 the plan's runtime flag d.grad.
template <bool kTC, int kForm>
__device__ __forceinline__ void pencil_gemm_body(const Dims& d, const DevOps& o, const GemmOps& G,
                                                 const GemmStageArgs& a, const int bid,
                                                 const int nbid) {
  const bool use_tc = kTC && G.tc;
  const bool grad = kForm == 2 ? d.grad != 0 : kForm == 1;
  extern __shared__ __align__(128) double sm[];
  __shared__ int s_p[kGW], s_mode[kGW];
  __shared__ double s_ky[kGW], s_kz[kGW];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ __align__(8) uint64_t s_bar_mma;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int nKc = (d.Kz + 7) / 8;
  const int kyi = bid / nKc, kz0 = (bid % nKc) * 8;
  const int nkz = min(8, d.Kz - kz0);  // valid kz columns per side
  const bool mean_cta = (kyi == 0 && kz0 == 0);
  const int N = d.Nx, Jh = G.Jh, Jl = G.Jl;
  const size_t P = (size_t)d.P;
  const double* __restrict__ frag = G.frag + (size_t)(bid % G.nrep) * G.nfrag;
  c64* rowc = reinterpret_cast<c64*>(sm);  // row r, pencil w: rowc[r * LC + w]
  const int LC = kGLd / 2;
  const double sl = a.slin;
  JFB_STAMP(0, 0);
  pdl_trigger();

  if (tid < kGW) {
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
  } else if (tid == 32) {
    mbar_init(&s_bar, 1);
    mbar_init(&s_bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  } else if (tid == 64) {
    // factor records of this tile's wavenumbers (consecutive modes) into L2
    const size_t m0 = (size_t)kyi * d.Kz + kz0;
    prefetch_l2(a.su + m0 * a.su_rec, (size_t)nkz * a.su_rec * sizeof(double));
    prefetch_l2(a.sg + m0 * a.sg_rec, (size_t)nkz * a.sg_rec * sizeof(double));
  } else if (tid == 96) {
    // this CTA's share of its operator copy
    const int users = (nbid + G.nrep - 1) / G.nrep, slot = bid / G.nrep;
    const int chunk = (G.nfrag + users - 1) / users;
    const int b0 = min(G.nfrag, slot * chunk), b1 = min(G.nfrag, b0 + chunk);
    if (b1 > b0) prefetch_l2(frag + b0, (size_t)(b1 - b0) * sizeof(double));
  } else if (tid == 128 && mean_cta) {
    prefetch_l2(G.R3, (size_t)d.nD * d.Nx * sizeof(double));
    prefetch_l2(a.s00inv, (size_t)d.nD * d.nD * sizeof(double));
    if (sl != 0.0) prefetch_l2(G.X2D, (size_t)d.nD * d.nD * sizeof(double));
  }
  if (use_tc && warp == 3) {  // 128 TMEM columns: the three 32-column accumulators
    __syncwarp();
    tc_alloc(&s_tmem, 128);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = use_tc ? s_tmem : 0u;
  // everything above reads only constant operators and factor records; the
  // arrays below are produced (HX) or still read (X) by the previous kernel
  pdl_wait();
  JFB_STAMP(0, 1);

  // ------------------------------------------------------------------ A --
  // 16-byte asynchronous copies of this tile's values straight into the
  // operand rows (all threads, no registers): H_f row j -> block f row j; u0
  // levels a, b, c -> segments 0, 1, 2 of the parity half of the mass operand
  // (row i -> i / 2), likewise g.  Column = pencil (8 +ky then 8 -ky).
  const bool has_b = (a.c1 != 0.0), has_c = (a.c2 != 0.0);
  const int sides = (kyi == 0) ? 1 : 2;
  // mixed form: (u0, u1, omega0, omega2), gradient form (u0, d/dy u0..2), at
  // rows j, N-1-j of two items
  c32 xl[2][2][4];
  {
    // mixed form: this thread's base-flow samples (before the copies are
    // issued with JFB_XLIN_EARLY, else while they fly)
    auto load_xlin = [&]() {
      if (!a.Xlin) return;
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int idx = tid + it * kGThreads;
        if (idx >= Jh * kGW) continue;
        const int j = idx / kGW, w = idx % kGW, p = s_p[w];
        if (p < 0) continue;
        const int rows[2] = {j, N - 1 - j};
        const int fs[4] = {0, grad ? 6 : 1, grad ? 7 : 3, grad ? 8 : 5};
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            xl[it][s2][k] = a.Xlin[((size_t)fs[k] * N + rows[s2]) * P + p];
      }
    };
    const int lv = 1 + has_b + has_c;
    const int nrow = 3 * N + (d.nB + d.nD) * lv;
    // one half-warp per row (lane & 15 = pencil column), so that the row's
    // source and destination are formed once per row, not per element
    const int hw = tid >> 4, c = tid & 15;
    const int side = c >> 3, kz = c & 7;  // nkz <= 8 columns per side
    const bool col_ok = side < sides && kz < nkz;
    const size_t so = (size_t)(side ? d.Ny - kyi : kyi) * d.Kz + kz0 + kz;
    if (JFB_XLIN_EARLY) load_xlin();
    for (int r = hw; r < nrow; r += kGThreads / 16) {
      if (!col_ok) continue;
      const c64* src;
      int dst_row;
      if (r < 3 * N) {
        const int f = r >= 2 * N ? 2 : r >= N ? 1 : 0, j = r - f * N;
        dst_row = G.oH[f] + j;
        const size_t e = ((size_t)f * N + j) * P + so;
        if (a.x32)  // complex64 sample: lands in the first half of the slot
          cp_async8(rowc + (size_t)dst_row * LC + side * 8 + kz,
                    reinterpret_cast<const c32*>(a.HX) + e);
        else
          cp_async16(rowc + (size_t)dst_row * LC + side * 8 + kz, a.HX + e);
        continue;
      } else if (r < 3 * N + d.nB * lv) {
        int q = r - 3 * N, lvl = 0;
        while (q >= d.nB) { q -= d.nB; ++lvl; }
        const int i = q;
        const int l = (lvl == 0) ? 0 : (lvl == 1 && has_b) ? 1 : 2;
        src = ((l == 0) ? a.u0a : (l == 1) ? a.u0b : a.u0c) + (size_t)i * P;
        const int nh = (i & 1) ? G.nBo : G.nBe;
        dst_row = ((i & 1) ? G.oMUO : G.oMUE) + l * nh + (i >> 1);
      } else {
        int q = r - 3 * N - d.nB * lv, lvl = 0;
        while (q >= d.nD) { q -= d.nD; ++lvl; }
        const int i = q;
        const int l = (lvl == 0) ? 0 : (lvl == 1 && has_b) ? 1 : 2;
        src = ((l == 0) ? a.ga : (l == 1) ? a.gb : a.gc) + (size_t)i * P;
        const int nh = (i & 1) ? G.nDo : G.nDe;
        dst_row = ((i & 1) ? G.oMGO : G.oMGE) + l * nh + (i >> 1);
      }
      cp_async16(rowc + (size_t)dst_row * LC + side * 8 + kz, src + so);
    }
    if (!JFB_XLIN_EARLY) load_xlin();
    cp_async_commit();
    cp_async_wait_all();
  }
  __syncthreads();
  JFB_STAMP(0, 2);

  // in-place transform: mirror sums / differences, (i ky, i kz, k^2) weights
  double* mean = sm + G.oMean;  // mean-flow scratch
  // [0, 2N): Re H1, Re H2 of the mean pencil; [2N, 2N + 2 nD): N (v, w);
  // [2N + 2nD, 2N + 4nD): rhs / forward-eliminated rhs; [2N + 4nD, 2N + 6nD): solution
  c64* m_nvw = reinterpret_cast<c64*>(mean + 2 * N);
  c64* m_vw = reinterpret_cast<c64*>(mean + 2 * N + 2 * d.nD);
  c64* m_x = reinterpret_cast<c64*>(mean + 2 * N + 4 * d.nD);
  // (Jh * kGW <= 2 * kGThreads: the tensor-core path runs for Nx <= 65)
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int idx = tid + it * kGThreads;
    if (idx >= Jh * kGW) break;
    const int j = idx / kGW, w = idx % kGW, jm = N - 1 - j;
    const bool ok = s_p[w] >= 0;
    c64 h[2][3];
    auto slot = [&](int row) {
      const c64* q = rowc + (size_t)row * LC + w;
      if (!a.x32) return *q;
      const c32 v = *reinterpret_cast<const c32*>(q);
      return cmk((double)v.re, (double)v.im);
    };
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      h[0][f] = ok ? slot(G.oH[f] + j) : cmk(0.0, 0.0);
      h[1][f] = (ok && jm != j) ? slot(G.oH[f] + jm) : cmk(0.0, 0.0);
    }
    if (a.Xlin && ok) {
      const bool mean = s_p[w] == 0;
      if (grad) {
        add_base_convection_terms(xl[it][0], d.uwall * o.xphys[j], d.uwall, h[0]);
        if (jm != j) add_base_convection_terms(xl[it][1], d.uwall * o.xphys[jm], d.uwall, h[1]);
      } else {
        add_base_flow_terms(xl[it][0], mean, d.uwall * o.xphys[j], d.uwall, h[0]);
        if (jm != j) add_base_flow_terms(xl[it][1], mean, d.uwall * o.xphys[jm], d.uwall, h[1]);
      }
    }
    if (mean_cta && w == 0) {
      mean[j] = h[0][1].re;
      mean[N + j] = h[0][2].re;
      if (jm != j) {
        mean[jm] = h[1][1].re;
        mean[N + jm] = h[1][2].re;
      }
    }
    const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
    c64 h12[2], k2h0[2], hg[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      h12[s] = mul_i(ky * h[s][1] + kz * h[s][2]);
      k2h0[s] = k2 * h[s][0];
      hg[s] = mul_i(kz * h[s][1] - ky * h[s][2]);
    }
    if (jm != j) {
      rowc[(G.oH[0] + j) * LC + w] = h12[0] - h12[1];
      rowc[(G.oH[0] + jm) * LC + w] = k2h0[0] + k2h0[1];
      rowc[(G.oH[1] + j) * LC + w] = h12[0] + h12[1];
      rowc[(G.oH[1] + jm) * LC + w] = k2h0[0] - k2h0[1];
      rowc[(G.oH[2] + j) * LC + w] = hg[0] + hg[1];
      rowc[(G.oH[2] + jm) * LC + w] = hg[0] - hg[1];
    } else {  // middle node (odd N): sums only
      rowc[(G.oH[0] + j) * LC + w] = k2h0[0];
      rowc[(G.oH[1] + j) * LC + w] = h12[0];
      rowc[(G.oH[2] + j) * LC + w] = hg[0];
    }
  }
  // mass-row inputs: u levels (a, b, c) -> (v1, v2, v3), g levels -> (w1, w2)
  for (int idx = tid; idx < d.nD * kGW; idx += kGThreads) {
    const int i = idx / kGW, w = idx % kGW;
    const bool ok = s_p[w] >= 0;
    const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
    const int par = i & 1, m = i >> 1;
    if (i < d.nB) {
      const int nh = par ? G.nBo : G.nBe;
      c64* x = rowc + (size_t)((par ? G.oMUO : G.oMUE) + m) * LC + w;
      c64 ua = cmk(0.0, 0.0), cu = ua;
      if (ok) {
        ua = x[0];
        cu = a.c0 * ua;
        if (has_b) cu = cu + a.c1 * x[nh * LC];
        if (has_c) cu = cu + a.c2 * x[2 * nh * LC];
      }
      x[0] = cu - (2.0 * sl * k2) * ua;
      x[nh * LC] = (sl * k2 * k2) * ua - k2 * cu;
      x[2 * nh * LC] = sl * ua;
    }
    const int nh = par ? G.nDo : G.nDe;
    c64* x = rowc + (size_t)((par ? G.oMGO : G.oMGE) + m) * LC + w;
    c64 ga = cmk(0.0, 0.0), cg = ga;
    if (ok) {
      ga = x[0];
      cg = a.c0 * ga;
      if (has_b) cg = cg + a.c1 * x[nh * LC];
      if (has_c) cg = cg + a.c2 * x[2 * nh * LC];
    }
    x[0] = cg - (sl * k2) * ga;
    x[nh * LC] = sl * ga;
  }
  // zero the k padding of the operands (rows past the data of each product)
  {
    const int hb = round4(N) + 4;
    const int pads[7][2] = {{G.oH[0] + N, hb - N},
                            {G.oH[1] + N, hb - N},
                            {G.oH[2] + N, hb - N},
                            {G.oMUE + 3 * G.nBe, round4(3 * G.nBe) - 3 * G.nBe},
                            {G.oMUO + 3 * G.nBo, round4(3 * G.nBo) - 3 * G.nBo},
                            {G.oMGE + 2 * G.nDe, round4(3 * G.nDe) - 2 * G.nDe},
                            {G.oMGO + 2 * G.nDo, round4(3 * G.nDo) - 2 * G.nDo}};
    __syncthreads();  // the g transform above reads segment 2 before it is cleared
    for (int q = 0; q < 7; ++q)
      for (int e = tid; e < pads[q][1] * kGLd; e += kGThreads) sm[pads[q][0] * kGLd + e] = 0.0;
  }
  __syncthreads();
  JFB_STAMP(0, 3);

  // ------------------------------------------------------------------ B --
  {
    const int nNu = G.sub[gNuE].mt + G.sub[gNuO].mt;
    const int nTask = nNu + G.sub[gNgE].mt + G.sub[gNgO].mt;
    const bool lin = (sl != 0.0);
    const double Myz = d.Myz, dt = d.dt;
    for (int task = warp; task < nTask; task += kGWarps) {
      const bool isNu = task < nNu;
      int mt = isNu ? task : task - nNu;
      int half = 0;
      const int mtE = isNu ? G.sub[gNuE].mt : G.sub[gNgE].mt;
      if (mt >= mtE) {
        mt -= mtE;
        half = 1;
      }
      const int idN = isNu ? (half ? gNuO : gNuE) : (half ? gNgO : gNgE);
      const int idM = isNu ? (half ? gMuO : gMuE) : (half ? gMgO : gMgE);
      const int oBN = isNu ? G.oH[half] : G.oH[2] + (half ? Jh : 0);
      const int oBM = isNu ? (half ? G.oMUO : G.oMUE) : (half ? G.oMGO : G.oMGE);
      const int nh = isNu ? (half ? G.nBo : G.nBe) : (half ? G.nDo : G.nDe);
      const int r = mt * 8 + g;
      const int i = 2 * r + half;
      // history terms of the epilogue, loaded ahead of the products
      const c64* Np = isNu ? a.Nup : a.Ngp;
      const c64* Nq = isNu ? a.Nuq : a.Ngq;
      c64 hp[4], hq[4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int p = s_p[nt * 4 + t4];
        const bool ok = p >= 0 && r < nh;
        const size_t gi = (size_t)i * P + (ok ? p : 0);
        hp[nt] = (ok && a.d1 != 0.0) ? ldg_c(Np + gi) : cmk(0.0, 0.0);
        hq[nt] = (ok && a.d2 != 0.0) ? ldg_c(Nq + gi) : cmk(0.0, 0.0);
      }
      double accN[4][2], accM[4][2];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) accN[nt][0] = accN[nt][1] = accM[nt][0] = accM[nt][1] = 0.0;
      const SubDesc sN = G.sub[idN], sM = G.sub[idM];
      const int2 krN = sub_krange(G, idN, mt);
      int2 krM = sub_krange(G, idM, mt);
      if (!lin) krM.y = min(krM.y, isNu ? G.kt_mu_lin[half] : G.kt_mg_lin[half]);
      gemm_acc<4, kKtN>(frag + sN.off + (size_t)mt * sN.kt * 32, krN.x, krN.y,
                        sm + (size_t)oBN * kGLd, lane, accN);
      gemm_acc<4, kKtM>(frag + sM.off + (size_t)mt * sM.kt * 32, krM.x, max(krM.x, krM.y),
                        sm + (size_t)oBM * kGLd, lane, accM);
      if (r < nh) {
        const int oR = isNu ? G.oRU + half * G.nBe : G.oRG + half * G.nDe;
        c64* Nout = isNu ? a.Nu_out : a.Ng_out;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int w = nt * 4 + t4;
          const int p = s_p[w];
          c64 rhs = cmk(0.0, 0.0);
          if (p >= 0) {
            const c64 nl0 = cmk(Myz * accN[nt][0], Myz * accN[nt][1]);
            if (Nout) Nout[(size_t)i * P + p] = nl0;
            const c64 nl = a.d0 * nl0 + a.d1 * hp[nt] + a.d2 * hq[nt];
            rhs = cmk(Myz * accM[nt][0], Myz * accM[nt][1]) + dt * nl;
          }
          rowc[(oR + r) * LC + w] = rhs;
        }
      }
    }
  }
  __syncthreads();
  JFB_STAMP(0, 4);

  // ------------------------------------------------------------------ C --
  // stage the velocity operators (tail of the operator copy) into dead rows
  if (tid == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (use_tc) {  // split-BF16 velocity operators in the tcgen05 operand layout
      mbar_arrive_expect(&s_bar, (uint32_t)kTcImgA);
      bulk_g2s(reinterpret_cast<unsigned char*>(sm) + G.oTA, G.vimg, (uint32_t)kTcImgA, &s_bar);
    } else {
      const int voff = G.sub[gA0Ee].off;
      const uint32_t bytes = (uint32_t)(G.nfrag - voff) * sizeof(double);
      mbar_arrive_expect(&s_bar, bytes);
      bulk_g2s(sm + (size_t)G.oVel * kGLd, frag + voff, bytes, &s_bar);
    }
  }
  // the multipliers of the tile's (up to 8) wavenumbers: 8-byte copies by
  // all threads, one latency instead of a chain of dependent chunk loads
  double* Ls = sm + (G.oL >= 0 ? G.oL : 0);
  if (G.oL >= 0) {
    const int per = 2 * (d.nB + d.nD);  // doubles per mode: Su then Sg multipliers
    for (int e = tid; e < 8 * per; e += kGThreads) {
      const int md = e / per, k = e % per;
      if (md >= nkz) continue;
      const size_t mode = (size_t)kyi * d.Kz + kz0 + md;
      const double* src = (k < 2 * d.nB) ? a.su + mode * a.su_rec + k
                                         : a.sg + mode * a.sg_rec + (k - 2 * d.nB);
      cp_async8(Ls + e, src);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
  }
  // C1: forward elimination, one thread per (pencil, system, parity), in place;
  // warps 2..7 of the mean CTA solve the mean-flow system meanwhile
  if (tid < 4 * kGW) {
    const int w = tid & 15, sys = (tid >> 4) & 1, par = tid >> 5;
    const int p = s_p[w];
    if (p >= 0) {
      const int n = sys ? d.nD : d.nB;
      const int m = par ? n / 2 : (n + 1) / 2;
      c64* y = rowc + (size_t)(sys ? G.oRG + par * G.nDe : G.oRU + par * G.nBe) * LC + w;
      if (G.oL >= 0) {
        const int per = 2 * (d.nB + d.nD);
        forward_elim_smem(Ls + (w & 7) * per + (sys ? 2 * d.nB : 0), par, m, y, LC);
      } else {
        const double* __restrict__ rec =
            sys ? a.sg + (size_t)s_mode[w] * a.sg_rec : a.su + (size_t)s_mode[w] * a.su_rec;
        forward_elim(rec, par, m, y, LC);
      }
    }
  } else if (tid < 4 * kGW + kMeanThreads) {
    if (mean_cta) mean_flow(d, o, G, a, mean, m_nvw, m_vw, m_x, tid - 4 * kGW);
  } else {
    const int t2 = tid - 4 * kGW - kMeanThreads, n2 = kGThreads - 4 * kGW - kMeanThreads;
    // zero the k padding of the velocity operands (they alias dead rows)
    const int pads[4][2] = {{G.oUE + G.nBe, round4(G.nBe) - G.nBe},
                            {G.oUO + G.nBo, round4(G.nBo) - G.nBo},
                            {G.oGE + G.nDe, round4(G.nDe) - G.nDe},
                            {G.oGO + G.nDo, round4(G.nDo) - G.nDo}};
    for (int q = 0; q < 4; ++q)
      for (int e = t2; e < pads[q][1] * kGLd; e += n2) sm[pads[q][0] * kGLd + e] = 0.0;
  }
  __syncthreads();
  JFB_STAMP(0, 5);
  // C2: x = U^-1 y for both pencils of a wavenumber; one warp per (pair,
  // system, parity), lane = row
  for (int task = warp; task < 4 * (kGW / 2); task += kGWarps) {
    const int ms = task & 7, sys = (task >> 3) & 1, par = task >> 4;
    if (s_p[ms] < 0) continue;
    const int n = sys ? d.nD : d.nB;
    const int m0 = (n + 1) / 2, m = par ? n / 2 : m0;
    const double* tri =
        (sys ? a.sg + (size_t)s_mode[ms] * a.sg_rec : a.su + (size_t)s_mode[ms] * a.su_rec) + 2 * n +
        (par ? m0 * (m0 + 1) / 2 : 0);
    double u[kMaxM];
#pragma unroll
    for (int c = 0; c < kMaxM; ++c)
      u[c] = (c < m && lane <= c) ? __ldg(tri + c * (c + 1) / 2 + lane) : 0.0;
    const int w0 = ms, w1 = ms + 8;
    const c64* y = rowc + (size_t)(sys ? G.oRG + par * G.nDe : G.oRU + par * G.nBe) * LC;
    c64* x = rowc + (size_t)(sys ? (par ? G.oGO : G.oGE) : (par ? G.oUO : G.oUE)) * LC;
    c64 s0 = cmk(0.0, 0.0), s1 = s0;
#pragma unroll
    for (int c = 0; c < kMaxM; ++c) {
      if (c < m) {
        s0 = s0 + u[c] * y[c * LC + w0];
        s1 = s1 + u[c] * y[c * LC + w1];
      }
    }
    if (lane < m) {
      x[lane * LC + w0] = s0;
      x[lane * LC + w1] = (s_p[w1] >= 0) ? s1 : cmk(0.0, 0.0);
    }
  }
  __syncthreads();
  JFB_STAMP(0, 6);
  // C3: solved coefficients to global memory (coalesced along pencils)
  {
    bool bad = false;
    for (int idx = tid; idx < d.nD * kGW; idx += kGThreads) {
      const int i = idx / kGW, w = idx % kGW;
      const int p = s_p[w];
      if (p < 0) continue;
      const int par = i & 1, m = i >> 1;
      if (i < d.nB) {
        const c64 v = rowc[((par ? G.oUO : G.oUE) + m) * LC + w];
        bad |= !finite_c(v);
        a.u0_out[(size_t)i * P + p] = v;
      }
      const c64 v = rowc[((par ? G.oGO : G.oGE) + m) * LC + w];
      bad |= !finite_c(v);
      a.g_out[(size_t)i * P + p] = v;
    }
    flag_nonfinite(G.status, bad);
  }
  if (mean_cta) {
    // the mean flow (v + i w) replaces g in the velocity operand of pencil 0
    __syncthreads();
    for (int i = tid; i < d.nD; i += kGThreads)
      rowc[(((i & 1) ? G.oGO : G.oGE) + (i >> 1)) * LC + 0] = m_x[i];
  }
  if (Jh > Jl && !use_tc) {
    // middle Gauss node (odd N) while the velocity operators arrive: one FP64
    // dot product per (operator, pencil, re/im)
    __syncthreads();
    if (tid < (grad ? 6 : 5) * 2 * kGW) sm[G.oMid + tid] = mid_dot(G, sm, tid);
  }
  const bool staged = mbar_wait_bounded(&s_bar, 0, G.status, kStatusWaitTimeout);
  // a timed-out copy leaves the velocity operators incomplete: skip D (the
  // status word makes the host call fail)
  const bool skip_d = __syncthreads_or(!staged);
  JFB_STAMP(0, 7);

  // ------------------------------------------------------------------ D --
  if (!skip_d && use_tc) {
    unsigned char* smb = reinterpret_cast<unsigned char*>(sm);
    // state operand: FP64 coefficient rows -> three BF16 parts, K-major
    // (row n = pencil column: 2 w + re/im, k = coefficient row of the half)
    for (int e = tid; e < 32 * 128; e += kGThreads) {
      const int n = e & 31, kk = e >> 5;  // kk over the groups' K: 0-31, 32-63, 64-127
      const int g = kk < 32 ? 0 : kk < 64 ? 1 : 2;
      const int k = kk - (g == 0 ? 0 : g == 1 ? 32 : 64);
      int row = -1;
      if (g == 0) row = k < G.nBe ? G.oUE + k : -1;
      else if (g == 1) row = k < G.nBo ? G.oUO + k : -1;
      else if (k < 32) row = k < G.nDe ? G.oGE + k : -1;
      else row = (k - 32) < G.nDo ? G.oGO + (k - 32) : -1;
      const double v = row >= 0 ? sm[(size_t)row * kGLd + n] : 0.0;
      __nv_bfloat16 b[3];
      bf16_split3(v, b);
      const uint32_t o = tc_offset(n, k, tc_k(g));
#pragma unroll
      for (int sp = 0; sp < 3; ++sp)
        *reinterpret_cast<__nv_bfloat16*>(smb + G.oTB + tc_b_off(g, sp) + o) = b[sp];
    }
    fence_async_smem();
    __syncthreads();
    JFB_STAMP(0, 10);
    if (tid == 0) {
      tc_fence_after();
      // descriptors: a base per operand and group, then constant offsets
      // (start addresses in 16-byte units in the low bits)
      const uint32_t a0 = smem_u32(smb + G.oTA), b0 = smem_u32(smb + G.oTB);
      const uint32_t idesc = tc_idesc_bf16(128, 32);
#pragma unroll
      for (int g = 0; g < 3; ++g) {
        const int K = g == 2 ? 64 : 32;
        const uint64_t ad0 = tc_smem_desc(a0 + tc_a_off(g, 0), (uint32_t)(K / 8) * 128);
        const uint64_t bd0 = tc_smem_desc(b0 + tc_b_off(g, 0), (uint32_t)(K / 8) * 128);
        const uint32_t sa = (uint32_t)(128 * K * 2) >> 4, sb = (uint32_t)(32 * K * 2) >> 4;
#pragma unroll
        for (int t = 0; t < K / 16; ++t)
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            const uint32_t pa = (q == 2 || q == 4) ? 1 : (q == 5) ? 2 : 0;
            const uint32_t pb = (q == 1 || q == 4) ? 1 : (q == 3) ? 2 : 0;
            const uint32_t kt = (uint32_t)(t * 2 * kTcLBO) >> 4;
            tc_mma_bf16(tmem + 32 * g, ad0 + pa * sa + kt, bd0 + pb * sb + kt, idesc,
                        t > 0 || q > 0);
          }
      }
      tc_commit(&s_bar_mma);
    }
    JFB_STAMP(0, 11);
    // middle Gauss node (odd N) on the last four warps while the MMAs run:
    // one FP64 dot product per (operator, pencil, re/im)
    if (Jh > Jl && warp >= kGWarps - 4) {
      for (int e = tid - (kGThreads - 128); e < 5 * 2 * kGW; e += 128)
        sm[G.oMid + e] = mid_dot(G, sm, e);
    }
    const bool done = mbar_wait_bounded(&s_bar_mma, 0, G.status, kStatusWaitTimeout);
    tc_fence_after();
    const bool skip_epi = __syncthreads_or(!done);
    JFB_STAMP(0, 12);
    float* st = reinterpret_cast<float*>(smb + G.oTA);  // [10][32][kTcStagePitch]
    if (!skip_epi) {
      const int g = warp >> 2, q = warp & 3;
      if (g < 3 && tc_slot(g, q) >= 0) {
        float v[32];
        tc_ld32(tmem + ((uint32_t)(32 * q) << 16) + 32 * g, v);
        float* row = st + ((size_t)tc_slot(g, q) * 32 + lane) * kTcStagePitch;
#pragma unroll
        for (int c = 0; c < 32; ++c) row[c] = v[c];
      }
    }
    __syncthreads();
    JFB_STAMP(0, 13);
    if (!skip_epi) {
      constexpr int kEpiIters = (32 * kGW + kGThreads - 1) / kGThreads;
#pragma unroll
      for (int it = 0; it < kEpiIters; ++it) {
      const int e = tid + it * kGThreads;
      if (e >= 32 * kGW) break;
      const int j = e >> 4, w = e & 15;
      const int p = s_p[w];
      if (j < Jl && p >= 0) {
        auto val = [&](int slot) {
          const float* r = st + ((size_t)slot * 32 + j) * kTcStagePitch + 2 * w;
          return cmk((double)r[0], (double)r[1]);
        };
        c64 fe[6], fo[6];
        velocity_fields(s_ky[w], s_kz[w], val(0), val(1), val(2), val(3), val(4), fe);
        velocity_fields(s_ky[w], s_kz[w], val(5), val(6), val(7), val(8), val(9), fo);
        const int jm = N - 1 - j;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const c64 vp = fe[q] + fo[q], vm = fe[q] - fo[q];
          c32* X = reinterpret_cast<c32*>(a.X) + (size_t)q * N * P + p;
          X[(size_t)j * P] = cmk((float)vp.re, (float)vp.im);
          X[(size_t)jm * P] = cmk((float)vm.re, (float)vm.im);
        }
      }
      }
      if (Jh > Jl && tid < kGW) mid_store(grad, a, sm + G.oMid, s_p, s_ky, s_kz, tid, N, Jl, P);
    }
  } else if (!skip_d) {
    const int MTv = G.sub[gA0Ee].mt;
    const double* vs = sm + (size_t)G.oVel * kGLd - G.sub[gA0Ee].off + lane;
    for (int task = warp; task < 4 * MTv; task += kGWarps) {
      const int jt = task >> 2, ncol0 = (task & 3) * 8;
      // accumulators: 0 aE, 1 b1E, 2 b2E, 3 c1E, 4 c2E, 5 aO, 6 b1O, 7 b2O, 8 c1O, 9 c2O,
      // gradient form: 10 a1O (A1 u0 even), 11 a1E (A1 u0 odd)
      double acc[12][2];
#pragma unroll
      for (int q = 0; q < 12; ++q) acc[q][0] = acc[q][1] = 0.0;
      auto group3 = [&](int oB, int s0, int s1, int s2, int q0, int q1, int q2) {
        const double* __restrict__ Bs = sm + (size_t)oB * kGLd + t4 * kGLd + ncol0 + g;
        const SubDesc d0 = G.sub[s0], d1 = G.sub[s1], d2 = G.sub[s2];
        const double* A0 = vs + d0.off + jt * d0.kt * 32;
        const double* A1 = vs + d1.off + jt * d1.kt * 32;
        const double* A2 = vs + d2.off + jt * d2.kt * 32;
#pragma unroll kVelUnroll
        for (int kt = 0; kt < d0.kt; ++kt) {
          const double b = Bs[kt * 4 * kGLd];
          dmma_8x8x4(acc[q0][0], acc[q0][1], A0[kt * 32], b);
          dmma_8x8x4(acc[q1][0], acc[q1][1], A1[kt * 32], b);
          dmma_8x8x4(acc[q2][0], acc[q2][1], A2[kt * 32], b);
        }
      };
      auto group2 = [&](int oB, int s0, int s1, int q0, int q1) {
        const double* __restrict__ Bs = sm + (size_t)oB * kGLd + t4 * kGLd + ncol0 + g;
        const SubDesc d0 = G.sub[s0], d1 = G.sub[s1];
        const double* A0 = vs + d0.off + jt * d0.kt * 32;
        const double* A1 = vs + d1.off + jt * d1.kt * 32;
#pragma unroll kVelUnroll
        for (int kt = 0; kt < d0.kt; ++kt) {
          const double b = Bs[kt * 4 * kGLd];
          dmma_8x8x4(acc[q0][0], acc[q0][1], A0[kt * 32], b);
          dmma_8x8x4(acc[q1][0], acc[q1][1], A1[kt * 32], b);
        }
      };
      group3(G.oUE, gA0Ee, gP2Ee, gP1Oe, 0, 2, 6);
      group3(G.oUO, gP1Eo, gA0Oo, gP2Oo, 1, 5, 7);
      group2(G.oGE, gB1Ee, gB2Oe, 3, 9);
      group2(G.oGO, gB2Eo, gB1Oo, 4, 8);
      if (grad) {  // d/dx u0: A1 on the even and odd coefficient halves
        auto group1 = [&](int oB, int s0, int q0) {
          const double* __restrict__ Bs = sm + (size_t)oB * kGLd + t4 * kGLd + ncol0 + g;
          const SubDesc d0 = G.sub[s0];
          const double* A0 = vs + d0.off + jt * d0.kt * 32;
#pragma unroll 4
          for (int kt = 0; kt < d0.kt; ++kt)
            dmma_8x8x4(acc[q0][0], acc[q0][1], A0[kt * 32], Bs[kt * 4 * kGLd]);
        };
        group1(G.oUE, gA1Oe, 10);
        group1(G.oUO, gA1Eo, 11);
      }
      // epilogue: six fields at x_j and x_{N-1-j}, j < Jl
      const int j = jt * 8 + g;
      const int w = (ncol0 >> 1) + t4;
      const int p = s_p[w];
      if (j < Jl && p >= 0) {
        const int jm = N - 1 - j;
        auto cv = [&](int q) { return cmk(acc[q][0], acc[q][1]); };
        // field q at x_j and x_{N-1-j} from its symmetric and antisymmetric halves
        auto put = [&](int q, const c64 fe, const c64 fo) {
          const c64 vp = fe + fo, vm = fe - fo;
          const size_t e = (size_t)q * N * P + p;
          if (a.x32) {
            c32* X = reinterpret_cast<c32*>(a.X) + e;
            X[(size_t)j * P] = cmk((float)vp.re, (float)vp.im);
            X[(size_t)jm * P] = cmk((float)vm.re, (float)vm.im);
          } else {
            c64* X = a.X + e;
            X[(size_t)j * P] = vp;
            X[(size_t)jm * P] = vm;
          }
        };
        if (grad) {
          c64 fe[9], fo[9];
          gradient_fields(s_ky[w], s_kz[w], cv(0), cv(11), cv(1), cv(2), cv(3), cv(4), fe);
          gradient_fields(s_ky[w], s_kz[w], cv(5), cv(10), cv(6), cv(7), cv(8), cv(9), fo);
#pragma unroll
          for (int q = 0; q < 9; ++q) put(q, fe[q], fo[q]);
        } else {
          c64 fe[6], fo[6];
          velocity_fields(s_ky[w], s_kz[w], cv(0), cv(1), cv(2), cv(3), cv(4), fe);
          velocity_fields(s_ky[w], s_kz[w], cv(5), cv(6), cv(7), cv(8), cv(9), fo);
#pragma unroll
          for (int q = 0; q < 6; ++q) put(q, fe[q], fo[q]);
        }
      }
    }
  }
  JFB_STAMP(0, 8);
  if (Jh > Jl && !skip_d && !use_tc && tid < kGW)  // products formed in C3
    mid_store(grad, a, sm + G.oMid, s_p, s_ky, s_kz, tid, N, Jl, P);
  if (use_tc) {  // free the TMEM columns (every tcgen05 load has completed)
    tc_fence_before();
    __syncthreads();
    if (warp == 3) {
      tc_fence_after();
      tc_dealloc(tmem, 128);
    }
  }
  JFB_STAMP(0, 9);
}

template <bool kTC, int kForm>
__global__ void __launch_bounds__(kGThreads, 1)
    pencil_gemm_kernel(const __grid_constant__ Dims d, const __grid_constant__ DevOps o,
                       const __grid_constant__ GemmOps G, const __grid_constant__ GemmStageArgs a) {
  pencil_gemm_body<kTC, kForm>(d, o, G, a, blockIdx.x, gridDim.x);
}

}  // namespace jfb
