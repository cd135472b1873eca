// Batched steady step of an ensemble of MHD members of uneven wall-normal
// size: each of the five stages of the coupled step (flow pencil stage, A
// stage, y-inverse of twelve fields, z stage, y-forward of six fields) is ONE
// launch over a group of members, driven by a work list (the host forms one
// group per wall-normal size and runs the groups on parallel branches of the
// step graph, or one group of all members).  Block b of a stage
// belongs to the member m with first[m] <= b < first[m + 1] and processes
// that member's tile b - first[m] with the member's own arguments, read from
// a device table (one table per ring phase, built when the phase's step graph
// is captured).  The per-tile work is the single-plan kernels' bodies, so a
// member's results are bitwise those of its own plan.
#pragma once

#include "jfb_kmm_gemm.cuh"
#include "jfb_kmm_mhd.cuh"
#include "jfb_kmm_warpk.cuh"

namespace jfb {

constexpr int kEnsMax = 64;  // members of a batched ensemble

// One member's arguments of the five stages of a steady step.  The
// transform buffers and twiddles are complex128 (FP64 form) or complex64
// (mixed form: the stage kernels' T = float); dT are the dimensions handed
// to the periodic-axis stages (the mixed form leaves the flow's base flow
// out of them).
struct __align__(16) EnsMember {
  Dims d, dT;
  DevOps o;
  GemmOps G;
  GemmStageArgs ga;
  MhdOps M;
  MhdArgs ma;
  MhdPhys ph;
  FFTPlan fz;
  const void *twy, *twz;
  void *X, *Y, *HZ, *HX;
  const double* xb;
  int KCw, chunks;
};

// Tile prefix sums per stage: stage s of member m owns blocks
// [first[s][m], first[s][m + 1]).
struct EnsTiles {
  int nm;
  int first[5][kEnsMax + 1];
};

__device__ __forceinline__ int ens_member(const EnsTiles* __restrict__ T, int stage, int b) {
  int m = 0;
  while (m + 1 < T->nm && b >= T->first[stage][m + 1]) ++m;
  return m;
}

// The member's arguments copied into shared memory, so that the stage body
// reads them from there (a global-memory reference would be reloaded after
// every global store the body makes).
__device__ __forceinline__ const EnsMember& ens_args(const EnsMember* __restrict__ tab, int m) {
  __shared__ __align__(16) EnsMember s_args;
  const int4* src = reinterpret_cast<const int4*>(tab + m);
  int4* dst = reinterpret_cast<int4*>(&s_args);
  for (int i = threadIdx.x; i < (int)(sizeof(EnsMember) / sizeof(int4)); i += blockDim.x)
    dst[i] = src[i];
  __syncthreads();
  return s_args;
}

__global__ void __launch_bounds__(kGThreads, 1)
    ens_pencil_kernel(const EnsMember* __restrict__ tab, const EnsTiles* __restrict__ T) {
  const int m = ens_member(T, 0, blockIdx.x);
  const EnsMember& e = ens_args(tab, m);
  pencil_gemm_body<true, 2>(e.d, e.o, e.G, e.ga, blockIdx.x - T->first[0][m],
                   T->first[0][m + 1] - T->first[0][m]);
}

__global__ void __launch_bounds__(kMhdThreads, 1)
    ens_mhd_a_kernel(const EnsMember* __restrict__ tab, const EnsTiles* __restrict__ T) {
  const int m = ens_member(T, 1, blockIdx.x);
  const EnsMember& e = ens_args(tab, m);
  mhd_a_body(e.d, e.o, e.M, e.ma, blockIdx.x - T->first[1][m]);
}

// twelve fields (u, omega, b, j) inverse along y: tile = (x-plane, field, kz chunk)
template <int P, typename F>
__global__ void __launch_bounds__(256)
    ens_y_backward_kernel(const EnsMember* __restrict__ tab, const EnsTiles* __restrict__ T) {
  const int m = ens_member(T, 2, blockIdx.x);
  const EnsMember& e = ens_args(tab, m);
  const int t = blockIdx.x - T->first[2][m];
  const int zc = t % e.chunks, f = (t / e.chunks) % 12, j = t / (e.chunks * 12);
  y_backward_warp_body<P, F>(e.dT, e.KCw, static_cast<const cpx<F>*>(e.twy),
                             static_cast<const cpx<F>*>(e.X), static_cast<cpx<F>*>(e.Y), j, f,
                             zc);
}

template <typename F>
__global__ void __launch_bounds__(256)
    ens_z_cross_kernel(const EnsMember* __restrict__ tab, const EnsTiles* __restrict__ T) {
  const int m = ens_member(T, 3, blockIdx.x);
  const EnsMember& e = ens_args(tab, m);
  z_cross_mhd_body<F>(e.o, e.dT, e.ph, e.fz, static_cast<const cpx<F>*>(e.twz),
                      static_cast<const cpx<F>*>(e.Y), static_cast<cpx<F>*>(e.HZ),
                      blockIdx.x - T->first[3][m]);
}

// six fields (n, emf) forward along y
template <int P, typename F>
__global__ void __launch_bounds__(256)
    ens_y_forward_kernel(const EnsMember* __restrict__ tab, const EnsTiles* __restrict__ T) {
  const int m = ens_member(T, 4, blockIdx.x);
  const EnsMember& e = ens_args(tab, m);
  const int t = blockIdx.x - T->first[4][m];
  const int zc = t % e.chunks, f = (t / e.chunks) % 6, j = t / (e.chunks * 6);
  y_forward_warp_body<P, F>(e.dT, e.KCw, static_cast<const cpx<F>*>(e.twy),
                            static_cast<const cpx<F>*>(e.HZ), static_cast<cpx<F>*>(e.HX), e.xb,
                            j, f, zc);
}

}  // namespace jfb
