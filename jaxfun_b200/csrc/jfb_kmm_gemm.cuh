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
// 36-double stride so that fragment loads are bank-conflict free.
#pragma once

#include "jfb_kmm.h"
#include "jfb_kmm_kernels.cuh"

namespace jfb {

constexpr int kGW = 16;   // pencils per CTA
constexpr int kGLd = 36;  // doubles per shared row: 2 kGW + 4

struct SubDesc {
  int off, mt, kt, kr;
};

struct GemmOps {
  const double* frag;
  const int* krange;
  const double* R3;   // S_D Q (nD x Nx)
  const double* X2D;  // nD x nD
  SubDesc sub[gNumSub];
  int Jh, Jl, nBe, nBo, nDe, nDo;
  int kt_mu_lin[2], kt_mg_lin[2];  // k-tile limits when the stage has no linear term
  // shared-memory row offsets
  int oHNE, oHNO, oHGE, oHGO, oMUE, oMUO, oMGE, oMGO, oRU, oRG, oUE, oUO, oGE, oGO;
  int rows;     // total rows of kGLd doubles
  int oMean;    // first double of the mean-flow scratch
};

struct GemmStageArgs {
  const c64* HX;
  double c0, c1, c2, d0, d1, d2, slin;  // slin = (implicit linear coefficient) * nu
  const c64 *u0a, *u0b, *u0c, *ga, *gb, *gc, *vwa, *vwb, *vwc;
  const c64 *Nup, *Nuq, *Ngp, *Ngq, *NVWp, *NVWq;
  c64 *Nu_out, *Ng_out, *NVW_out;
  const double *su, *sg, *s00;  // records: L pairs, then inverse upper triangles
  int su_rec, sg_rec;
  c64 *u0_out, *g_out, *vw_out;
  c64* X;
};

__host__ __device__ inline int round4(int x) { return (x + 3) & ~3; }

// acc[nt] += A(sub, mt) * B(rows of Bs, columns 8 nt .. 8 nt + 7), k tiles [kb, ke)
template <int NT>
__device__ __forceinline__ void gemm_acc(const GemmOps& G, int id, int mt, int kb, int ke,
                                         const double* __restrict__ Bs, int ncol0, int lane,
                                         double (&acc)[NT][2]) {
  const SubDesc s = G.sub[id];
  const double* __restrict__ A = G.frag + s.off + (size_t)mt * s.kt * 32 + lane;
  const int g = lane >> 2, t4 = lane & 3;
  const double* __restrict__ b = Bs + t4 * kGLd + ncol0 + g;
#pragma unroll 4
  for (int kt = kb; kt < ke; ++kt) {
    const double a = __ldg(A + kt * 32);
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) dmma_8x8x4(acc[nt][0], acc[nt][1], a, b[kt * 4 * kGLd + nt * 8]);
  }
}

__device__ __forceinline__ int2 sub_krange(const GemmOps& G, int id, int mt) {
  const int* kr = G.krange + G.sub[id].kr + 2 * mt;
  return make_int2(kr[0], kr[1]);
}

__global__ void __launch_bounds__(256, 1) pencil_gemm_kernel(Dims d, DevOps o, GemmOps G,
                                                             GemmStageArgs a) {
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_p[kGW], s_mode[kGW];
  __shared__ double s_ky[kGW], s_kz[kGW];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t4 = lane & 3;
  const int nKc = (d.Kz + 7) / 8;
  const int kyi = blockIdx.x / nKc, kz0 = (blockIdx.x % nKc) * 8;
  const bool mean_cta = (kyi == 0 && kz0 == 0);
  const int N = d.Nx, Jh = G.Jh, Jl = G.Jl;
  const size_t P = (size_t)d.P;

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
  }
  __syncthreads();

  // ------------------------------------------------------------------ A --
  c64* rowc = reinterpret_cast<c64*>(sm);  // row r, pencil w: rowc[r * kGLd / 2 + w]
  const int LC = kGLd / 2;
  for (int idx = tid; idx < Jh * kGW; idx += blockDim.x) {
    const int j = idx / kGW, w = idx % kGW;
    const int p = s_p[w];
    const int jm = N - 1 - j;
    c64 h[2][3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      h[0][f] = (p >= 0) ? a.HX[((size_t)f * N + j) * P + p] : cmk(0.0, 0.0);
      h[1][f] = (p >= 0 && jm != j) ? a.HX[((size_t)f * N + jm) * P + p] : cmk(0.0, 0.0);
    }
    const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
    c64 h12[2], k2h0[2], hg[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      h12[s] = mul_i(ky * h[s][1] + kz * h[s][2]);
      k2h0[s] = k2 * h[s][0];
      hg[s] = mul_i(kz * h[s][1] - ky * h[s][2]);
    }
    if (j < Jl) {
      rowc[(G.oHNE + j) * LC + w] = h12[0] - h12[1];
      rowc[(G.oHNE + Jl + j) * LC + w] = k2h0[0] + k2h0[1];
      rowc[(G.oHNO + j) * LC + w] = h12[0] + h12[1];
      rowc[(G.oHNO + Jh + j) * LC + w] = k2h0[0] - k2h0[1];
      rowc[(G.oHGE + j) * LC + w] = hg[0] + hg[1];
      rowc[(G.oHGO + j) * LC + w] = hg[0] - hg[1];
    } else {  // middle node (odd N): sums only
      rowc[(G.oHNE + Jl + j) * LC + w] = k2h0[0];
      rowc[(G.oHNO + j) * LC + w] = h12[0];
      rowc[(G.oHGE + j) * LC + w] = hg[0];
    }
  }
  // mass-row inputs by parity: [v1; v2; v3] (u) and [w1; w2] (g)
  const double sl = a.slin;
  for (int idx = tid; idx < d.nD * kGW; idx += blockDim.x) {
    const int i = idx / kGW, w = idx % kGW;
    const int p = s_p[w];
    const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
    const int par = i & 1, m = i >> 1;
    if (i < d.nB) {
      c64 ua = cmk(0.0, 0.0), comb = ua;
      if (p >= 0) {
        const size_t gi = (size_t)i * P + p;
        ua = a.u0a[gi];
        comb = a.c0 * ua;
        if (a.c1 != 0.0) comb = comb + a.c1 * a.u0b[gi];
        if (a.c2 != 0.0) comb = comb + a.c2 * a.u0c[gi];
      }
      const int nh = par ? G.nBo : G.nBe;
      const int base = par ? G.oMUO : G.oMUE;
      rowc[(base + m) * LC + w] = comb - (2.0 * sl * k2) * ua;
      rowc[(base + nh + m) * LC + w] = (sl * k2 * k2) * ua - k2 * comb;
      rowc[(base + 2 * nh + m) * LC + w] = sl * ua;
    }
    c64 ga = cmk(0.0, 0.0), comb = ga;
    if (p >= 0) {
      const size_t gi = (size_t)i * P + p;
      ga = a.ga[gi];
      comb = a.c0 * ga;
      if (a.c1 != 0.0) comb = comb + a.c1 * a.gb[gi];
      if (a.c2 != 0.0) comb = comb + a.c2 * a.gc[gi];
    }
    const int nh = par ? G.nDo : G.nDe;
    const int base = par ? G.oMGO : G.oMGE;
    rowc[(base + m) * LC + w] = comb - (sl * k2) * ga;
    rowc[(base + nh + m) * LC + w] = sl * ga;
  }
  // zero the k padding of the B operands
  {
    const int pads[8][2] = {{G.oHNE + N, round4(N) - N},         {G.oHNO + N, round4(N) - N},
                            {G.oHGE + Jh, round4(Jh) - Jh},      {G.oHGO + Jl, round4(Jl) - Jl},
                            {G.oMUE + 3 * G.nBe, round4(3 * G.nBe) - 3 * G.nBe},
                            {G.oMUO + 3 * G.nBo, round4(3 * G.nBo) - 3 * G.nBo},
                            {G.oMGE + 2 * G.nDe, round4(2 * G.nDe) - 2 * G.nDe},
                            {G.oMGO + 2 * G.nDo, round4(2 * G.nDo) - 2 * G.nDo}};
    for (int q = 0; q < 8; ++q)
      for (int e = tid; e < pads[q][1] * kGLd; e += blockDim.x) sm[pads[q][0] * kGLd + e] = 0.0;
  }
  double* mean = sm + G.oMean;  // mean-flow scratch
  // [0, 2N): Re H1, Re H2 of the mean pencil; [2N, 2N + 2 nD): NVW (v, w);
  // [2N + 2nD, 2N + 4nD): rhs / solution (v, w)
  if (mean_cta) {
    for (int j = tid; j < N; j += blockDim.x) {
      mean[j] = a.HX[((size_t)1 * N + j) * P].re;
      mean[N + j] = a.HX[((size_t)2 * N + j) * P].re;
    }
  }
  __syncthreads();

  // ------------------------------------------------------------------ B --
  {
    const int nNu = G.sub[gNuE].mt + G.sub[gNuO].mt;
    const int nTask = nNu + G.sub[gNgE].mt + G.sub[gNgO].mt;
    const bool lin = (sl != 0.0);
    const double Myz = d.Myz, dt = d.dt;
    for (int task = warp; task < nTask; task += 8) {
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
      const int oBN = isNu ? (half ? G.oHNO : G.oHNE) : (half ? G.oHGO : G.oHGE);
      const int oBM = isNu ? (half ? G.oMUO : G.oMUE) : (half ? G.oMGO : G.oMGE);
      double accN[4][2], accM[4][2];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) accN[nt][0] = accN[nt][1] = accM[nt][0] = accM[nt][1] = 0.0;
      int2 kr = sub_krange(G, idN, mt);
      gemm_acc<4>(G, idN, mt, kr.x, kr.y, sm + (size_t)oBN * kGLd, 0, lane, accN);
      kr = sub_krange(G, idM, mt);
      int ke = kr.y;
      if (!lin) ke = min(ke, isNu ? G.kt_mu_lin[half] : G.kt_mg_lin[half]);
      gemm_acc<4>(G, idM, mt, kr.x, ke, sm + (size_t)oBM * kGLd, 0, lane, accM);
      // epilogue: row r of this half, pencils 4 nt + t4
      const int nh = isNu ? (half ? G.nBo : G.nBe) : (half ? G.nDo : G.nDe);
      const int r = mt * 8 + g;
      if (r < nh) {
        const int i = 2 * r + half;
        const int oR = isNu ? G.oRU + half * G.nBe : G.oRG + half * G.nDe;
        c64* Nout = isNu ? a.Nu_out : a.Ng_out;
        const c64* Np = isNu ? a.Nup : a.Ngp;
        const c64* Nq = isNu ? a.Nuq : a.Ngq;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int w = nt * 4 + t4;
          const int p = s_p[w];
          c64 rhs = cmk(0.0, 0.0);
          if (p >= 0) {
            const size_t gi = (size_t)i * P + p;
            const c64 nl0 = cmk(Myz * accN[nt][0], Myz * accN[nt][1]);
            if (Nout) Nout[gi] = nl0;
            c64 nl = a.d0 * nl0;
            if (a.d1 != 0.0) nl = nl + a.d1 * Np[gi];
            if (a.d2 != 0.0) nl = nl + a.d2 * Nq[gi];
            rhs = cmk(Myz * accM[nt][0], Myz * accM[nt][1]) + dt * nl;
          }
          rowc[(oR + r) * LC + w] = rhs;
        }
      }
    }
  }
  __syncthreads();

  // ------------------------------------------------------------------ C --
  // C1: forward elimination, one thread per (pencil, system, parity), in place
  if (tid < 4 * kGW) {
    const int w = tid & 15, sys = (tid >> 4) & 1, par = tid >> 5;
    const int p = s_p[w];
    if (p >= 0) {
      const int n = sys ? d.nD : d.nB;
      const int m = par ? n / 2 : (n + 1) / 2;
      const double* __restrict__ rec =
          sys ? a.sg + (size_t)s_mode[w] * a.sg_rec : a.su + (size_t)s_mode[w] * a.su_rec;
      c64* y = rowc + (size_t)(sys ? G.oRG + par * G.nDe : G.oRU + par * G.nBe) * LC + w;
      c64 y1 = cmk(0.0, 0.0), y2 = y1;
#pragma unroll 4
      for (int r = 0; r < m; ++r) {
        const int i = 2 * r + par;
        const double l1 = __ldg(rec + 2 * i), l2 = __ldg(rec + 2 * i + 1);
        c64 v = y[r * LC];
        v = v - l1 * y1;
        v = v - l2 * y2;
        y[r * LC] = v;
        y2 = y1;
        y1 = v;
      }
    }
  } else {
    // zero the k padding of the velocity operands (they alias dead B rows)
    const int pads[4][2] = {{G.oUE + G.nBe, round4(G.nBe) - G.nBe},
                            {G.oUO + G.nBo, round4(G.nBo) - G.nBo},
                            {G.oGE + G.nDe, round4(G.nDe) - G.nDe},
                            {G.oGO + G.nDo, round4(G.nDo) - G.nDo}};
    for (int q = 0; q < 4; ++q)
      for (int e = tid - 4 * kGW; e < pads[q][1] * kGLd; e += blockDim.x - 4 * kGW)
        sm[pads[q][0] * kGLd + e] = 0.0;
    if (mean_cta) {
      // mean-flow nonlinear rows -(S_D Q Re H1), -(S_D Q Re H2)
      for (int e = tid - 4 * kGW; e < 2 * d.nD; e += blockDim.x - 4 * kGW) {
        const int i = e >> 1, f = e & 1;
        const double* __restrict__ r3 = G.R3 + (size_t)i * N;
        const double* hm = mean + f * N;
        double s = 0.0;
        for (int j = 0; j < N; ++j) s += __ldg(r3 + j) * hm[j];
        mean[2 * N + 2 * i + f] = -s;
      }
    }
  }
  __syncthreads();
  // C2: x = U^-1 y for both pencils of a wavenumber, one warp per (pair, system, parity)
  for (int task = warp; task < 4 * (kGW / 2); task += 8) {
    const int ms = task & 7, sys = (task >> 3) & 1, par = task >> 4;
    const int w0 = ms, w1 = ms + 8;
    if (s_p[w0] < 0) continue;
    const int n = sys ? d.nD : d.nB;
    const int m0 = (n + 1) / 2, m = par ? n / 2 : m0;
    const double* __restrict__ tri = (sys ? a.sg + (size_t)s_mode[w0] * a.sg_rec
                                          : a.su + (size_t)s_mode[w0] * a.su_rec) +
                                     2 * n + (par ? m0 * (m0 + 1) / 2 : 0);
    const c64* y = rowc + (size_t)(sys ? G.oRG + par * G.nDe : G.oRU + par * G.nBe) * LC;
    c64* x = rowc + (size_t)(sys ? (par ? G.oGO : G.oGE) : (par ? G.oUO : G.oUE)) * LC;
    for (int r0 = 0; r0 < m; r0 += 32) {
      const int r = r0 + lane;
      c64 s0 = cmk(0.0, 0.0), s1 = s0;
#pragma unroll 4
      for (int c = r0; c < m; ++c) {
        const c64 ya = y[c * LC + w0], yb = y[c * LC + w1];
        if (r <= c && r < m) {
          const double u = __ldg(tri + c * (c + 1) / 2 + r);
          s0 = s0 + u * ya;
          s1 = s1 + u * yb;
        }
      }
      if (r < m) {
        x[r * LC + w0] = s0;
        x[r * LC + w1] = (s_p[w1] >= 0) ? s1 : cmk(0.0, 0.0);
      }
    }
  }
  __syncthreads();
  // C3: solved coefficients to global memory (coalesced along pencils)
  for (int idx = tid; idx < d.nD * kGW; idx += blockDim.x) {
    const int i = idx / kGW, w = idx % kGW;
    const int p = s_p[w];
    if (p < 0) continue;
    const int par = i & 1, m = i >> 1;
    if (i < d.nB) a.u0_out[(size_t)i * P + p] = rowc[((par ? G.oUO : G.oUE) + m) * LC + w];
    a.g_out[(size_t)i * P + p] = rowc[((par ? G.oGO : G.oGE) + m) * LC + w];
  }
  if (mean_cta) {
    // C4: mean flow: rhs = M00 comb + slin X2D vwa + dt (d0 N + d1 N' + d2 N''),
    // then the S00 solve; (v, w) replaces g in the velocity operand of pencil 0
    c64* vw = reinterpret_cast<c64*>(mean + 2 * N + 2 * d.nD);  // nD complex
    const c64* nvw = reinterpret_cast<const c64*>(mean + 2 * N);
    __syncthreads();
    for (int i = tid; i < d.nD; i += blockDim.x) {
      auto comb = [&](int k) {
        c64 v = a.c0 * a.vwa[k];
        if (a.c1 != 0.0) v = v + a.c1 * a.vwb[k];
        if (a.c2 != 0.0) v = v + a.c2 * a.vwc[k];
        return v;
      };
      c64 r = o.mdi[i] * comb(i);
      if (i >= 2) r = r + o.mlo[i] * comb(i - 2);
      if (i + 2 < d.nD) r = r + o.mhi[i] * comb(i + 2);
      if (sl != 0.0) {
        c64 s = cmk(0.0, 0.0);
        for (int k = 0; k < d.nD; ++k) s = s + __ldg(G.X2D + (size_t)i * d.nD + k) * a.vwa[k];
        r = r + sl * s;
      }
      c64 nl = a.d0 * nvw[i];
      if (a.d1 != 0.0) nl = nl + a.d1 * a.NVWp[i];
      if (a.d2 != 0.0) nl = nl + a.d2 * a.NVWq[i];
      if (a.NVW_out) a.NVW_out[i] = nvw[i];
      vw[i] = r + d.dt * nl;
    }
    __syncthreads();
    if (tid < 2) {
      const int par = tid, n = d.nD, m = par ? n / 2 : (n + 1) / 2;
      c64 y1 = cmk(0.0, 0.0), y2 = y1;
      for (int r = 0; r < m; ++r) {
        const int i = 2 * r + par;
        c64 v = vw[i] - a.s00[2 * i] * y1;
        v = v - a.s00[2 * i + 1] * y2;
        vw[i] = v;
        y2 = y1;
        y1 = v;
      }
    }
    __syncthreads();
    c64 xv = cmk(0.0, 0.0);
    const int i = tid;
    if (i < d.nD) {
      const int n = d.nD, m0 = (n + 1) / 2, par = i & 1, r = i >> 1;
      const int m = par ? n / 2 : m0;
      const double* tri = a.s00 + 2 * n + (par ? m0 * (m0 + 1) / 2 : 0);
      for (int c = r; c < m; ++c) xv = xv + tri[c * (c + 1) / 2 + r] * vw[2 * c + par];
    }
    __syncthreads();
    if (i < d.nD) {
      a.vw_out[i] = xv;
      const int par = i & 1, r = i >> 1;
      rowc[((par ? G.oGO : G.oGE) + r) * LC + 0] = xv;
    }
  }
  __syncthreads();

  // ------------------------------------------------------------------ D --
  {
    const int MTv = G.sub[gA0Ee].mt;
    for (int task = warp; task < 2 * MTv; task += 8) {
      const int jt = task >> 1, ncol0 = (task & 1) * 16;
      // accumulators: 0 aE, 1 b1E, 2 b2E, 3 c1E, 4 c2E, 5 aO, 6 b1O, 7 b2O, 8 c1O, 9 c2O
      double acc[10][2][2];
#pragma unroll
      for (int q = 0; q < 10; ++q)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) acc[q][nt][0] = acc[q][nt][1] = 0.0;
      {
        const double* __restrict__ Bs = sm + (size_t)G.oUE * kGLd + t4 * kGLd + ncol0 + g;
        const double* __restrict__ A0 = G.frag + G.sub[gA0Ee].off + (size_t)jt * G.sub[gA0Ee].kt * 32 + lane;
        const double* __restrict__ A1 = G.frag + G.sub[gP2Ee].off + (size_t)jt * G.sub[gP2Ee].kt * 32 + lane;
        const double* __restrict__ A2 = G.frag + G.sub[gP1Oe].off + (size_t)jt * G.sub[gP1Oe].kt * 32 + lane;
        const int KT = G.sub[gA0Ee].kt;
#pragma unroll 2
        for (int kt = 0; kt < KT; ++kt) {
          const double a0 = __ldg(A0 + kt * 32), a1 = __ldg(A1 + kt * 32), a2 = __ldg(A2 + kt * 32);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const double b = Bs[kt * 4 * kGLd + nt * 8];
            dmma_8x8x4(acc[0][nt][0], acc[0][nt][1], a0, b);
            dmma_8x8x4(acc[2][nt][0], acc[2][nt][1], a1, b);
            dmma_8x8x4(acc[6][nt][0], acc[6][nt][1], a2, b);
          }
        }
      }
      {
        const double* __restrict__ Bs = sm + (size_t)G.oUO * kGLd + t4 * kGLd + ncol0 + g;
        const double* __restrict__ A0 = G.frag + G.sub[gP1Eo].off + (size_t)jt * G.sub[gP1Eo].kt * 32 + lane;
        const double* __restrict__ A1 = G.frag + G.sub[gA0Oo].off + (size_t)jt * G.sub[gA0Oo].kt * 32 + lane;
        const double* __restrict__ A2 = G.frag + G.sub[gP2Oo].off + (size_t)jt * G.sub[gP2Oo].kt * 32 + lane;
        const int KT = G.sub[gP1Eo].kt;
#pragma unroll 2
        for (int kt = 0; kt < KT; ++kt) {
          const double a0 = __ldg(A0 + kt * 32), a1 = __ldg(A1 + kt * 32), a2 = __ldg(A2 + kt * 32);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const double b = Bs[kt * 4 * kGLd + nt * 8];
            dmma_8x8x4(acc[1][nt][0], acc[1][nt][1], a0, b);
            dmma_8x8x4(acc[5][nt][0], acc[5][nt][1], a1, b);
            dmma_8x8x4(acc[7][nt][0], acc[7][nt][1], a2, b);
          }
        }
      }
      {
        const double* __restrict__ Bs = sm + (size_t)G.oGE * kGLd + t4 * kGLd + ncol0 + g;
        const double* __restrict__ A0 = G.frag + G.sub[gB1Ee].off + (size_t)jt * G.sub[gB1Ee].kt * 32 + lane;
        const double* __restrict__ A1 = G.frag + G.sub[gB2Oe].off + (size_t)jt * G.sub[gB2Oe].kt * 32 + lane;
        const int KT = G.sub[gB1Ee].kt;
#pragma unroll 2
        for (int kt = 0; kt < KT; ++kt) {
          const double a0 = __ldg(A0 + kt * 32), a1 = __ldg(A1 + kt * 32);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const double b = Bs[kt * 4 * kGLd + nt * 8];
            dmma_8x8x4(acc[3][nt][0], acc[3][nt][1], a0, b);
            dmma_8x8x4(acc[9][nt][0], acc[9][nt][1], a1, b);
          }
        }
      }
      {
        const double* __restrict__ Bs = sm + (size_t)G.oGO * kGLd + t4 * kGLd + ncol0 + g;
        const double* __restrict__ A0 = G.frag + G.sub[gB2Eo].off + (size_t)jt * G.sub[gB2Eo].kt * 32 + lane;
        const double* __restrict__ A1 = G.frag + G.sub[gB1Oo].off + (size_t)jt * G.sub[gB1Oo].kt * 32 + lane;
        const int KT = G.sub[gB2Eo].kt;
#pragma unroll 2
        for (int kt = 0; kt < KT; ++kt) {
          const double a0 = __ldg(A0 + kt * 32), a1 = __ldg(A1 + kt * 32);
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const double b = Bs[kt * 4 * kGLd + nt * 8];
            dmma_8x8x4(acc[4][nt][0], acc[4][nt][1], a0, b);
            dmma_8x8x4(acc[8][nt][0], acc[8][nt][1], a1, b);
          }
        }
      }
      // epilogue: six fields at x_j and x_{N-1-j}
      const int j = jt * 8 + g;
      if (j < Jh) {
        const int jm = N - 1 - j;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const int w = (ncol0 >> 1) + nt * 4 + t4;
          const int p = s_p[w];
          if (p < 0) continue;
          const double ky = s_ky[w], kz = s_kz[w], k2 = ky * ky + kz * kz;
          const bool meanp = (k2 == 0.0);
          const double inv = meanp ? 0.0 : 1.0 / k2;
          c64 f[2][6];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int q = 5 * h;
            const c64 av = cmk(acc[q + 0][nt][0], acc[q + 0][nt][1]);
            const c64 b1 = cmk(acc[q + 1][nt][0], acc[q + 1][nt][1]);
            const c64 b2 = cmk(acc[q + 2][nt][0], acc[q + 2][nt][1]);
            const c64 c1 = cmk(acc[q + 3][nt][0], acc[q + 3][nt][1]);
            const c64 c2 = cmk(acc[q + 4][nt][0], acc[q + 4][nt][1]);
            f[h][0] = av;
            if (meanp) {  // c1, c2 hold (B1, B2) (v + i w) of the mean flow
              f[h][1] = cmk(c1.re, 0.0);
              f[h][2] = cmk(c1.im, 0.0);
              f[h][3] = cmk(0.0, 0.0);
              f[h][4] = cmk(-c2.im, 0.0);
              f[h][5] = cmk(c2.re, 0.0);
            } else {
              f[h][1] = mul_i((ky * inv) * b1 + (kz * inv) * c1);
              f[h][2] = mul_i((kz * inv) * b1 - (ky * inv) * c1);
              f[h][3] = c1;
              f[h][4] = mul_i(kz * av) - mul_i((kz * inv) * b2 - (ky * inv) * c2);
              f[h][5] = mul_i((ky * inv) * b2 + (kz * inv) * c2) - mul_i(ky * av);
            }
          }
#pragma unroll
          for (int q = 0; q < 6; ++q) {
            c64* X = a.X + (size_t)q * N * P + p;
            X[(size_t)j * P] = f[0][q] + f[1][q];
            if (jm != j) X[(size_t)jm * P] = f[0][q] - f[1][q];
          }
        }
      }
    }
  }
}

}  // namespace jfb
