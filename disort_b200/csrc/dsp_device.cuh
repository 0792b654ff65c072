// dsp_device.cuh — shared device-side definitions of the B200 DISORT engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dsp.h"

// Phase markers for cycle-count instrumentation builds; no-ops otherwise.
#ifndef DSP_PHASE_BEGIN
#define DSP_PHASE_BEGIN
#endif
#ifndef DSP_PHASE
#define DSP_PHASE(k)
#endif

namespace dsp {

__host__ __device__ constexpr int pow2ceil(int x) { return x <= 1 ? 1 : 2 * pow2ceil((x + 1) / 2); }
__host__ __device__ constexpr int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int round4(int x) { return (x + 3) & ~3; }

struct DArr {
  const double* p;
  long long s;
  __device__ __forceinline__ double operator()(long long i, long long k = 0) const { return p[i * s + k]; }
  __device__ __forceinline__ const double* row(long long i) const { return p + i * s; }
};

// Constants of the reference's Planck routine, computed on the host with libm
// exactly as Planck.cpp:18-31 does, so the device uses bit-identical values.
struct PlanckConsts {
  double vmax, sigdpi, conc, c1;
};

// Per-stream-count constant tables (host-computed, FluxSolver.cpp:257-290, :126,
// :442-445): mu[N], wt[N], dsim[NN], dinv[NN], ylm[N][N] = P_l(mu_i) at [l*N+i].
struct Tables {
  const double* base;
  __device__ __forceinline__ const double* mu() const { return base; }
};
__host__ __device__ constexpr int tab_mu(int) { return 0; }
__host__ __device__ constexpr int tab_wt(int N) { return N; }
__host__ __device__ constexpr int tab_dsim(int N) { return 2 * N; }
__host__ __device__ constexpr int tab_dinv(int N) { return 2 * N + N / 2; }
__host__ __device__ constexpr int tab_ylm(int N) { return 3 * N; }
__host__ __device__ constexpr int tab_size(int N) { return 3 * N + N * N; }

// Instance record (doubles) written by the setup kernel.
struct InstLayout {
  int hdr, dtau_s, ssa_s, fsc, sig, mode, tau_s, tauc, btr, pkag, yb, stride;
  __host__ __device__ static InstLayout make(int L, int N) {
    InstLayout o;
    o.hdr = 0;
    o.dtau_s = 16;
    o.ssa_s = o.dtau_s + L;
    o.fsc = o.ssa_s + L;
    o.sig = o.fsc + L;
    o.mode = o.sig + L;
    o.tau_s = o.mode + L;
    o.tauc = o.tau_s + L + 1;
    o.btr = o.tauc + L + 1;
    o.pkag = o.btr + L + 1;
    o.yb = o.pkag + L + 1;
    o.stride = round4(o.yb + N + 1);
    return o;
  }
};
// header slots
enum { H_NCUT = 0, H_LYRCUT, H_PTOP, H_PBOT, H_PBOTD, H_DELTAM, H_DMPLUS, H_FBEAM, H_UMU0, H_ALB,
       H_FISOT, H_FISOB, H_NSLOTS };

// Layer record (doubles) written by the layer kernel:
// G[N][N] | eig[N] | zb[N] | z0[N] | z1[N] | xr0 | xr1
__host__ __device__ constexpr int lrec_G(int) { return 0; }
__host__ __device__ constexpr int lrec_eig(int N) { return N * N; }
__host__ __device__ constexpr int lrec_zb(int N) { return N * N + N; }
__host__ __device__ constexpr int lrec_z0(int N) { return N * N + 2 * N; }
__host__ __device__ constexpr int lrec_z1(int N) { return N * N + 3 * N; }
__host__ __device__ constexpr int lrec_xr(int N) { return N * N + 4 * N; }
__host__ __device__ constexpr int lrec_stride(int N) { return round4(N * N + 4 * N + 2); }
// Elimination record (doubles) written by the BVP kernel: Wt[N][N] (transposed) | d[N]
__host__ __device__ constexpr int brec_stride(int N) { return round4(N * N + N); }

struct FluxParams {
  int n;          // instances in this launch
  int N, L, pc, nmom;
  uint32_t flags;
  DArr wlo, whi, dtau, ssa, pmom, temp, alb, emis, fbeam, umu0, fisot, fisob, ttop, tbot;
  const double* tables;  // tab_* layout for N
  PlanckConsts pk;
  double* inst_rec;
  double* layer_rec;
  double* bvp_rec;
  InstLayout il;
  double* out[8];
  int32_t* status;
};

// Team helpers.  A team is TEAM consecutive threads; TEAM < 32 lives inside a
// warp (synchronised by __syncwarp on its own lanes), TEAM >= 32 is the whole CTA.
template <int TEAM>
__device__ __forceinline__ unsigned team_mask() {
  if constexpr (TEAM >= 32) {
    return 0xffffffffu;
  } else {
    const unsigned lane = threadIdx.x & 31u;
    return ((1u << TEAM) - 1u) << (lane & ~(unsigned)(TEAM - 1));
  }
}

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if constexpr (TEAM >= 32) {
    __syncthreads();
  } else {
    __syncwarp(team_mask<TEAM>());
  }
}

// Arg-max of (v, i) over the team, ties to the smaller index; result to all.
// `red` is team-private shared scratch of 2*(TEAM/32) doubles (unused for TEAM <= 32).
template <int TEAM>
__device__ __forceinline__ void team_argmax(double& v, int& idx, double* red) {
  constexpr int W = TEAM < 32 ? TEAM : 32;
  const unsigned m = team_mask<TEAM>();
#pragma unroll
  for (int off = W / 2; off > 0; off >>= 1) {
    const double ov = __shfl_xor_sync(m, v, off, W);
    const int oi = __shfl_xor_sync(m, idx, off, W);
    if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
  }
  if constexpr (TEAM > 32) {
    constexpr int NW = TEAM / 32;
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
      red[w] = v;
      reinterpret_cast<int*>(red + NW)[w] = idx;
    }
    __syncthreads();
    v = red[0];
    idx = reinterpret_cast<int*>(red + NW)[0];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
      const double ov = red[k];
      const int oi = reinterpret_cast<int*>(red + NW)[k];
      if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void set_status(int32_t* status, int i, int code) {
  if (status) atomicMax(status + i, code);
}

}  // namespace dsp
