// flux_layer.cuh — per-(instance, layer) eigensystem and particular solutions.
//
// Replaces solveEigen (FluxSolver.cpp:459-588), computeBeamSource (:595-643)
// and computeIsotropicSource (:745-831).  One team of TEAM = pow2ceil(N)
// threads per layer task; every matrix lives in the team's shared memory.
//
// Eigenproblem: the reference symmetrises (a+b)(a-b) with D = diag(sqrt(w mu)),
// factors -B_s = L L^T and diagonalises S = L^T (-A_s) L (SelfAdjointEigenSolver).
// Here S is diagonalised with a parallel cyclic Jacobi method (round-robin pair
// ordering, NN/2 disjoint rotations per round, one 2x2 block per thread), which
// yields the same eigenpairs to rounding; eigenvalues are sorted ascending like
// the reference's.  When -B_s is not SPD (the reference's general-eigensolver
// branch, omega' >= 1-1e-12), -A_s = L'L'^T and S' = L'^T(-B_s)L' give the same
// eigenpairs of (a+b)(a-b) with u = D^{-1} L' w.
//
// Shared-memory layout per team: the phase matrix is kept as its unique half
// cc_top (NN x N; C = [[P, Q], [Q, P]] with P = cc_top[:, :NN], Q = cc_top[:, NN:]),
// NN x NN matrices use a padded row stride NS = NN + 1 (conflict-free columns),
// and the N x N LU matrix of the particular solutions overlays the eigen work
// area once the eigenvectors have been written out.
#pragma once

#include "dsp_device.cuh"

namespace dsp {

template <int N, bool GEN = false>
struct LCfg {
  static constexpr int NN = N / 2;
  // 64 streams: a 128-thread team per layer (two threads per stream)
  static constexpr int TEAM = N >= 64 ? 2 * N : (pow2ceil(N) < 4 ? 4 : pow2ceil(N));
  static constexpr int CTA = TEAM >= 32 ? TEAM : 128;
  static constexpr int TPC = CTA / TEAM;
  static constexpr int NNP = NN + (NN & 1);
  static constexpr int NPAIR = NNP / 2;
  static constexpr int BPT = (NPAIR * NPAIR + TEAM - 1) / TEAM;  // Jacobi 2x2 blocks per thread
  static constexpr int NS = NN + 1;  // padded row stride of NN x NN matrices
  static constexpr int MAT = NN * NS;
  // team shared-memory layout (doubles).  The phase matrix is dead once
  // alpha -/+ beta are formed; where it is large enough (N >= 10) the
  // eigenvector matrix V and the vectors b, z are placed over it.
  static constexpr bool OVL = MAT + 2 * N <= NN * N;
  static constexpr int O_CC = 0;                     // cc_top[NN][N]
  static constexpr int O_GL = O_CC + NN * N;         // gl[N]
  static constexpr int O_W = O_GL + N;               // work area: AMB, APB, S0, S1, LC (, V)
  static constexpr int W_SIZE = (OVL ? 5 : 6) * MAT;
  static constexpr int O_V = OVL ? O_CC : O_W + 5 * MAT;
  static constexpr int O_LAM = O_W + W_SIZE;         // NN: k = sqrt|lambda|
  static constexpr int O_LAMR = O_LAM + NN;          // NN: lambda
  static constexpr int O_ROT = O_LAMR + NN;          // c, s, t per pair
  static constexpr int O_B = OVL ? O_CC + MAT : O_ROT + 3 * NPAIR;  // b[N]
  static constexpr int O_Z = O_B + N;                // z[N]
  static constexpr int O_MISC = OVL ? O_ROT + 3 * NPAIR : O_Z + N;  // flags, reduction scratch
  static constexpr int O_PIV = O_MISC + 8;           // N ints
  // general solver: P_l^m(-mu0), then psi0 / p0 / p1 source moments [N] each
  static constexpr int O_GX = O_PIV + N / 2 + 1;
  static constexpr int TEAM_SMEM = round4(O_GX + (GEN ? 4 * N : 0));
  // user angles whose P_l^m columns fit next to W[N][N] in the work area
  static constexpr int UCH = (W_SIZE - N * N) / N;
  static_assert(!GEN || UCH >= 1, "work area too small for the user-angle tables");
  // the Legendre table stays in global memory (L1) for N >= 16, where it would
  // take about as much shared memory as a team
  static constexpr bool Y_GLOBAL = N >= 16;
  static constexpr int TAB = Y_GLOBAL ? tab_ylm(N) : tab_size(N);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(TAB + TPC * TEAM_SMEM); }
  // resident CTAs per SM the register budget is sized for: as many as shared
  // memory admits (228 KB, 1 KB reserved per CTA), never below 80 registers
  static constexpr int MINB_SMEM = (int)((228u * 1024u) / (smem_bytes() + 1024u));
  static constexpr int MINB_REGS = 65536 / (CTA * 80);
  static constexpr int MINB = MINB_SMEM < 1 ? 1 : (MINB_SMEM < MINB_REGS ? MINB_SMEM : MINB_REGS);
};

// Whether the layer stage of an N-stream flux solve is split in three launches:
// the front of the layer kernel (phase matrix, alpha -/+ beta, Cholesky,
// S = L^T M L), the eigensolver with one thread per layer task
// (flux_jacobi_kernel), and the back of the layer kernel (eigenvectors, G,
// particular solutions).  A thread that owns a whole 8 x 8 S and its eigenvector
// matrix in registers runs the rotations of a sweep with no shuffles or
// barriers; the team form spends most of its time waiting on them.
template <int N>
__host__ __device__ constexpr bool layer_split() { return N <= 16; }

// packed lower-triangle index of the symmetric element (r, c)
__host__ __device__ constexpr int tri_idx(int r, int c) {
  return r >= c ? r * (r + 1) / 2 + c : c * (c + 1) / 2 + r;
}

// Hand-off between the three launches of a split layer stage, kept in the
// boundary-value records' area (dead until the boundary-value kernel runs):
// blocks of 32 layer tasks, element e of the block's lane k at
// 32 HS b + e w + k (w = tasks in the block), so that a warp of the
// one-thread-per-task kernels reads or writes an element of 32 tasks in one
// coalesced access.  Per task: flag (0 skipped, 1 primary factorisation,
// 2 fallback), S, the Cholesky factor L, and the odd- and even-order halves
// O, E of the phase sums (all symmetric NN x NN, packed lower; E only with a
// beam), then the eigensolver's diagonal and eigenvector matrix (row-major,
// column j the eigenvector of diagonal entry j).
//   O_ij = sum_{l odd} g'_l P_l(mu_i) P_l(mu_j),  E_ij = sum_{l even} (...),
//   alpha - beta = M^{-1} (O W - I),  alpha + beta = M^{-1} (E W - I)
// with M = diag(mu_1..mu_NN), W = diag(w_1..w_NN): the quadrature is
// symmetric (mu_{NN+j} = -mu_j, P_l(-mu) = (-1)^l P_l(mu)), so the sums over
// the other hemisphere only flip the sign of the odd orders.
template <int NN>
struct Handoff {
  static constexpr int TRI = NN * (NN + 1) / 2;
  static constexpr int S_FLAG = 0, S_S = 1, S_L = 1 + TRI, S_O = 1 + 2 * TRI, S_E = 1 + 3 * TRI;
  static constexpr int S_D = 1 + 4 * TRI, S_V = S_D + NN;
  static constexpr int HS = S_V + NN * NN;
};

// Quadrature tables of an N-stream solve passed by value: kernel parameters
// live in the constant bank, so the one-thread-per-task kernels read them as
// uniform operands with compile-time offsets, no loads.
template <int N>
struct ConstTab {
  double mu[N / 2], rmu[N / 2], wt[N / 2], dsim[N / 2], dinv[N / 2];
  double y[N * N];  // P_l(mu_i) at [l * N + i]
};

// ConstTab from a host copy of the tab_* table layout
template <int N>
inline ConstTab<N> make_const_tab(const double* tab) {
  ConstTab<N> c;
  for (int k = 0; k < N / 2; ++k) {
    c.mu[k] = tab[tab_mu(N) + k];
    c.rmu[k] = 1.0 / c.mu[k];
    c.wt[k] = tab[tab_wt(N) + k];
    c.dsim[k] = tab[tab_dsim(N) + k];
    c.dinv[k] = tab[tab_dinv(N) + k];
  }
  for (int k = 0; k < N * N; ++k) c.y[k] = tab[tab_ylm(N) + k];
  return c;
}

// address of element e of task j in the lane-interleaved blocks
template <int NN>
__device__ __forceinline__ double* handoff_lane(double* bvp_rec, long long nt, long long j, int e) {
  using H = Handoff<NN>;
  const long long b = j >> 5;
  const long long left = nt - (b << 5);
  const int w = left < 32 ? (int)left : 32;
  return bvp_rec + b * 32 * H::HS + (long long)e * w + (j & 31);
}

// Round-robin pairing of NNP players in round r: (arr[a], arr[NNP-1-a]),
// arr[0] = 0, arr[j] = 1 + (j - 1 + r) mod (NNP - 1).
template <int NNP>
__device__ __forceinline__ int rr_player(int r, int j) {
  int x = j - 1 + r;  // < 2 (NNP - 1) for r < NNP - 1: one conditional subtract replaces the modulo
  if (x >= NNP - 1) x -= NNP - 1;
  return j == 0 ? 0 : 1 + x;
}

// Cholesky of the lower triangle of M (NN x NN, stride NS) into Lc; false if
// not SPD.  `flag` is team scratch; every thread leaves through a team
// barrier, so the caller may reuse it immediately.
template <int NN, int NS, int TEAM>
__device__ bool team_cholesky(const double* M, double* Lc, double* flag, int t) {
  for (int i = t; i < NN * NS; i += TEAM) Lc[i] = 0.0;
  if (t == 0) flag[0] = 0.0;
  team_sync<TEAM>();
  for (int j = 0; j < NN; ++j) {
    if (t == 0) {
      double d = M[j * NS + j];
      for (int k = 0; k < j; ++k) d -= Lc[j * NS + k] * Lc[j * NS + k];
      if (!(d > 0.0)) flag[0] = 1.0;
      else Lc[j * NS + j] = sqrt(d);
    }
    team_sync<TEAM>();
    const bool failed = flag[0] != 0.0;
    team_sync<TEAM>();
    if (failed) return false;
    const double ljj = Lc[j * NS + j];
    for (int i = t; i < NN; i += TEAM)
      if (i > j) {
        double s = M[i * NS + j];
        for (int k = 0; k < j; ++k) s -= Lc[i * NS + k] * Lc[j * NS + k];
        Lc[i * NS + j] = s / ljj;
      }
    team_sync<TEAM>();
  }
  return true;
}



// Right-looking Cholesky with row i held by thread i (sub-warp teams): column
// j's entries are broadcast by shuffles, no barriers.  Same contract as
// team_cholesky.
template <int NN, int NS, int TEAM>
__device__ bool team_cholesky_reg(const double* M, double* Lc, int t) {
  static_assert(TEAM <= 32, "shuffle Cholesky needs a sub-warp team");
  const unsigned msk = team_mask<TEAM>();
  double row[NN];
#pragma unroll
  for (int k = 0; k < NN; ++k) row[k] = (t < NN && k <= t) ? M[t * NS + k] : 0.0;
  bool ok = true;
#pragma unroll
  for (int j = 0; j < NN; ++j) {
    const double djj = __shfl_sync(msk, row[j], j, TEAM);
    if (!(djj > 0.0)) ok = false;
    const double ljj = ok ? sqrt(djj) : 1.0;
    const double lij = (t == j) ? ljj : ((t > j && t < NN) ? row[j] / ljj : 0.0);
    if (t < NN) Lc[t * NS + j] = (t >= j) ? lij : 0.0;
#pragma unroll
    for (int k = j + 1; k < NN; ++k) {
      const double lkj = __shfl_sync(msk, lij, k, TEAM);
      if (t >= k && t < NN) row[k] -= lij * lkj;
    }
  }
  if (t < NN)
    for (int k = t + 1; k < NN; ++k) Lc[t * NS + k] = 0.0;
  team_sync<TEAM>();
  return ok;
}

template <int NN, int NS, int TEAM>
__device__ __forceinline__ bool team_chol(const double* M, double* Lc, double* flag, int t) {
  if constexpr (TEAM <= 32) return team_cholesky_reg<NN, NS, TEAM>(M, Lc, t);
  else return team_cholesky<NN, NS, TEAM>(M, Lc, flag, t);
}

// Whether the Jacobi rotation of pair (p, q) is applied: |apq| above 1e-15 of
// sqrt|app aqq| (about 4.5 ulp).  With the quadratic convergence of cyclic
// Jacobi a threshold at this level rather than 1e-17 saves the last sweep of
// many tasks (one-thread eigensolver at 16 streams: 2.02 -> 1.82 ms per
// 20,000-band thermal step); an off-diagonal left at that level moves
// eigenvalues by its square and eigenvectors by it over the eigenvalue gap, far
// below the 1e-9 parity bound.
#ifndef DSP_JACOBI_TOL2
#define DSP_JACOBI_TOL2 1.0e-30
#endif
__device__ __forceinline__ bool jacobi_needed(double apq, double app, double aqq) {
  return fabs(apq) > 1e-300 && apq * apq > DSP_JACOBI_TOL2 * fabs(app * aqq);
}

// Jacobi rotation (Golub & Van Loan, Alg. 8.4.1) zeroing apq; tt = 0 when apq
// is negligible.  t = tan(theta) is the smaller root of t^2 + 2 th t - 1
// with th = d / e, d = aqq - app, e = 2 apq, written as
// t = sgn(th) |e| / (|d| + sqrt(d^2 + e^2)) (one square root, one division).
__device__ __forceinline__ void jacobi_rot(double apq, double app, double aqq, double& c, double& s,
                                           double& tt) {
  c = 1.0;
  s = 0.0;
  tt = 0.0;
  if (jacobi_needed(apq, app, aqq)) {
    const double d = aqq - app, e = 2.0 * apq;
    if (fabs(d) > 1e8 * fabs(e)) {
      tt = e / (2.0 * d);
      c = 1.0 - 0.5 * tt * tt;
    } else {
      const double num = d > 0.0 ? e : (d < 0.0 ? -e : fabs(e));  // sgn(th) |e|, sgn(0) = +1
      tt = num / (fabs(d) + sqrt(d * d + e * e));
      c = rsqrt(tt * tt + 1.0);
    }
    s = tt * c;
  }
}

// ---------------------------------------------------------------------------
// Length-NN vectors distributed one element per team thread (thread t < NN
// holds element t).  Sub-warp teams broadcast with shuffles; larger teams go
// through a shared scratch word.  Matrices are NN x NN, row stride NS.
// ---------------------------------------------------------------------------
template <int TEAM>
__device__ __forceinline__ double team_bcast(double v, int k, int t, double* scratch) {
  if constexpr (TEAM <= 32) {
    return __shfl_sync(team_mask<TEAM>(), v, k, TEAM);
  } else {
    if (t == k) scratch[0] = v;
    __syncthreads();
    const double r = scratch[0];
    __syncthreads();
    return r;
  }
}

// y = A x (trans = false) or A^T x (trans = true); part: 0 full, 1 lower, 2 upper
template <int NN, int NS, int TEAM>
__device__ __forceinline__ double team_matvec(const double* A, double x, bool trans, int part, int t,
                                              double* scratch) {
  double acc = 0.0;
  if constexpr (TEAM <= 32) {
#pragma unroll
    for (int k = 0; k < NN; ++k) {
      const double xk = __shfl_sync(team_mask<TEAM>(), x, k, TEAM);
      if (t < NN) {
        const int r = trans ? k : t, c = trans ? t : k;  // element A[r][c]
        const bool in = part == 0 || (part == 1 ? c <= r : c >= r);
        if (in) acc += A[r * NS + c] * xk;
      }
    }
  } else {
    if (t < NN) scratch[t] = x;
    __syncthreads();
    if (t < NN)
      for (int k = 0; k < NN; ++k) {
        const int r = trans ? k : t, c = trans ? t : k;
        const bool in = part == 0 || (part == 1 ? c <= r : c >= r);
        if (in) acc += A[r * NS + c] * scratch[k];
      }
    __syncthreads();
  }
  return acc;
}

// x <- L^{-1} x (forward) or L^{-T} x (backward), L lower triangular
template <int NN, int NS, int TEAM>
__device__ __forceinline__ double team_trsv(const double* Lm, double x, bool transposed, int t,
                                            double* scratch) {
  if (!transposed) {
    for (int k = 0; k < NN; ++k) {
      if (t == k) x = x / Lm[k * NS + k];
      const double xk = team_bcast<TEAM>(x, k, t, scratch);
      if (t > k && t < NN) x -= Lm[t * NS + k] * xk;
    }
  } else {
    for (int k = NN - 1; k >= 0; --k) {
      if (t == k) x = x / Lm[k * NS + k];
      const double xk = team_bcast<TEAM>(x, k, t, scratch);
      if (t < k) x -= Lm[k * NS + t] * xk;
    }
  }
  return x;
}

// Eigenvectors and sources of one layer at the user polar angles for mode m
// (interpEigenvec, DisortSolver.cpp:2468-2504; interpSource, :2506-2580):
//   W(l, c)   = 0.5 g'_l sum_jq P_l^m(mu_jq) w_jq G(row(jq), c)
//   GU(iu, c) = sum_l P_l^m(mu_u) W(l, c)
// with row(jq) = NN + jq for jq < NN, N - 1 - jq otherwise (the reference's
// reduced-eigenvector ordering); the beam and thermal sources likewise.
// Team thread c owns column c; the P_l^m columns of up to UCH user angles at a
// time sit beside W in the (now free) eigen work area.
template <int N>
__device__ void gen_user_angles(const FluxParams& p, int i, double* sm, const double* Y, const double* wt,
                                const double* gl, double* lrec, double fbeam, double ws, bool thermal,
                                int t) {
  using C = LCfg<N, true>;
  constexpr int NN = N / 2, TEAM = C::TEAM, UCH = C::UCH;
  const int m = p.g.m, numu = p.g.numu;
  double* W = sm + C::O_W;           // [N][N]
  double* U = W + N * N;             // [N][UCH]
  const double* ybm = sm + C::O_GX;  // P_l^m(-mu0) (written by the beam source)
  double* psi0 = sm + C::O_GX + N;
  double* p0 = psi0 + N;
  double* p1 = p0 + N;
  const double* G = lrec + lrec_G(N);
  const bool beam = fbeam > 0.0;
  team_sync<TEAM>();  // G and the particular solutions of this team are written
  if (t < N) {
    const int c = t;
    double gcol[N];
#pragma unroll
    for (int jq = 0; jq < N; ++jq) gcol[jq] = G[(jq < NN ? NN + jq : N - 1 - jq) * N + c];
    for (int l = 0; l < N; ++l) {
      double s = 0.0;
      if (l >= m) {
#pragma unroll
        for (int jq = 0; jq < N; ++jq) s += (Y[l * N + jq] * wt[jq]) * gcol[jq];
        s *= 0.5 * gl[l];
      }
      W[l * N + c] = s;
    }
    // source moments: psi0(l) = 0.5 g'_l sum_jq w_jq P_l^m(mu_jq) z(jq) with the
    // unordered beam solution z(jq) = zb[row(jq)], and the thermal z0 / z1 alike
    const int l = t;
    double sb = 0.0, s0 = 0.0, s1 = 0.0;
    if (l >= m) {
      for (int jq = 0; jq < N; ++jq) {
        const int r = jq < NN ? NN + jq : N - 1 - jq;
        const double yw = wt[jq] * Y[l * N + jq];
        if (beam) sb += yw * lrec[lrec_zb(N) + r];
        if (thermal) {
          s0 += yw * lrec[lrec_z0(N) + r];
          s1 += yw * lrec[lrec_z1(N) + r];
        }
      }
    }
    psi0[l] = 0.5 * gl[l] * sb;
    p0[l] = 0.5 * gl[l] * s0;
    p1[l] = 0.5 * gl[l] * s1;
  }
  team_sync<TEAM>();
  const double xr0 = lrec[lrec_xr(N)], xr1 = lrec[lrec_xr(N) + 1];
  const double fact = (m == 0 ? 1.0 : 2.0) * fbeam / (4.0 * 3.14159265358979323846);
  double* GU = lrec + glrec_gu(N);
  double* zbu = GU + numu * N;
  double* z0u = zbu + numu;
  double* z1u = z0u + numu;
  const double* umu = p.g.umu.row(i);
  for (int u0 = 0; u0 < numu; u0 += UCH) {
    const int nu = numu - u0 < UCH ? numu - u0 : UCH;
    for (int k = t; k < nu; k += TEAM) legendre_column(m, umu[u0 + k], N - 1, U + k, UCH);
    team_sync<TEAM>();
    if (t < N)
      for (int k = 0; k < nu; ++k) {
        double s = 0.0;
        for (int l = m; l < N; ++l) s += U[l * UCH + k] * W[l * N + t];
        GU[(u0 + k) * N + t] = s;
      }
    for (int k = t; k < nu; k += TEAM) {
      if (beam) {
        double s = 0.0;
        for (int l = m; l < N; ++l) s += U[l * UCH + k] * (psi0[l] + fact * gl[l] * ybm[l]);
        zbu[u0 + k] = s;
      }
      if (thermal) {
        double s0 = 0.0, s1 = 0.0;
        for (int l = m; l < N; ++l) {
          s0 += U[l * UCH + k] * p0[l];
          s1 += U[l * UCH + k] * p1[l];
        }
        z0u[u0 + k] = s0 + (1.0 - ws) * xr0;
        z1u[u0 + k] = s1 + (1.0 - ws) * xr1;
      }
    }
    team_sync<TEAM>();
  }
}

template <int N, bool GEN = false, bool JAC = false>
__global__ void __launch_bounds__(LCfg<N, GEN>::CTA, LCfg<N, GEN>::MINB) flux_layer_kernel(FluxParams p) {
  using C = LCfg<N, GEN>;
  constexpr int NN = C::NN, TEAM = C::TEAM, NNP = C::NNP, NPAIR = C::NPAIR, NS = C::NS, BPT = C::BPT;
  constexpr int BPA = NPAIR;  // blocks (a, b) per column pair b
  extern __shared__ double smem[];
  // CTA-level constant tables
  for (int k = threadIdx.x; k < C::TAB; k += blockDim.x) smem[k] = p.tables[k];
  __syncthreads();
  const double* mu = smem + tab_mu(N);
  const double* wt = smem + tab_wt(N);
  const double* dsim = smem + tab_dsim(N);
  const double* dinv = smem + tab_dinv(N);
  const double* Y = C::Y_GLOBAL ? p.tables + tab_ylm(N) : smem + tab_ylm(N);

  const int team = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
  const long long task = (long long)blockIdx.x * C::TPC + team;
  // i: status / input index; lc: layer; Lin: layers of the instance
  int i, lc, Lin;
  const double* rec;
  InstLayout il_gen;  // general solver: the layout of this instance
  const double* pml;
  if constexpr (GEN) {
    // general solver: ragged layers; task = chunk-local layer
    if (task >= p.g.lay_off[p.n]) return;
    const int ci = p.g.layer_inst[task];
    i = p.g.ids[ci];
    lc = (int)(task - p.g.lay_off[ci]);
    Lin = p.g.Ls[i];
    il_gen = InstLayout::make(Lin, N);
    rec = p.inst_rec + p.g.inst_off[ci];
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? Lin - 1 - lc : lc;
    pml = p.g.pmom + (p.g.in_off[i] + lin) * (long long)p.pc;
  } else {
    if (task >= (long long)p.n * p.L) return;
    i = (int)(task / p.L);
    lc = (int)(task % p.L);
    Lin = p.L;
    rec = p.inst_rec + (long long)i * p.il.stride;
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? p.L - 1 - lc : lc;
    pml = p.pmom.row(i) + (long long)lin * p.pc;
  }
  const InstLayout& il = GEN ? il_gen : p.il;
  if (p.status && p.status[i] == DSP_ERR_INVALID_INPUT) return;
  const int ncut = (int)rec[H_NCUT];
  if (lc >= ncut) return;  // layers below the absorption cut are never used
  if constexpr (GEN) {
    // modes past the instance's last one, or after its azimuthal series converged
    if (p.g.m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  }

  double* sm = smem + C::TAB + team * C::TEAM_SMEM;
  double* CC = sm + C::O_CC;
  double* gl = sm + C::O_GL;
  double* W = sm + C::O_W;
  double* AMB = W + 0 * C::MAT;
  double* APB = W + 1 * C::MAT;
  double* S0 = W + 2 * C::MAT;
  double* S1 = W + 3 * C::MAT;
  double* LC = W + 4 * C::MAT;
  double* V = sm + C::O_V;  // over the phase matrix when C::OVL (first written after alpha -/+ beta)
  double* EV = S0;  // eigenvectors of (a+b)(a-b); S0 is dead by then
  double* lam = sm + C::O_LAM;
  double* lamraw = sm + C::O_LAMR;
  double* rot = sm + C::O_ROT;
  double* bv = sm + C::O_B;
  double* zv = sm + C::O_Z;
  double* misc = sm + C::O_MISC;
  int* piv = reinterpret_cast<int*>(sm + C::O_PIV);

  DSP_PHASE_BEGIN
  const double ws = rec[il.ssa_s + lc];
  const double dts = rec[il.dtau_s + lc];
  // ---- scaled phase coefficients (disortSet, FluxSolver.cpp:336-386) ----
  {
    const int mode = (int)rec[il.mode + lc];
    const double f = rec[il.fsc + lc], sig = rec[il.sig + lc];
    for (int k = t; k < N; k += TEAM) {
      // the general solver normalises P_0 to 1 (DisortSolver.cpp:669)
      const double pk = (GEN && k == 0) ? 1.0 : pml[k];
      double g;
      if (mode == 0) g = (2.0 * k + 1.0) * ws * pk;
      else if (mode == 1) g = (2.0 * k + 1.0) * ws * (pk - f) / (1.0 - f);
      else {
        const double kd = (double)k;
        g = (2.0 * k + 1.0) * ws * (pk - f * exp(-kd * kd / (2.0 * sig))) / (1.0 - f);
      }
      gl[k] = g;
    }
  }
  team_sync<TEAM>();
  DSP_PHASE(0)
  // ---- phase matrix, unique half (FluxSolver.cpp:466-482) ---------------
  // thread t owns column jq = t; its Legendre column is held in registers
  if (t < N) {
    const int jq = t;
    double yj[N];
#pragma unroll
    for (int l = 0; l < N; ++l) yj[l] = Y[l * N + jq];
    const double wj = wt[jq];
    for (int iq = 0; iq < NN; ++iq) {
      double s = 0.0;
#pragma unroll
      for (int l = 0; l < N; ++l) s += (gl[l] * Y[l * N + iq]) * yj[l];
      CC[iq * N + jq] = (s * 0.5) * wj;
    }
  }
  team_sync<TEAM>();
  DSP_PHASE(1)
  // ---- alpha -/+ beta and the similarity transform (:485-514) ------------
  for (int it = t; it < NN * NN; it += TEAM) {
    const int iq = it / NN, jq = it % NN;
    const double inv_cmu = 1.0 / mu[iq];
    const double a = CC[iq * N + jq], b = CC[iq * N + NN + jq];
    double amb = inv_cmu * (a - b), apb = inv_cmu * (a + b);
    if (iq == jq) { amb -= inv_cmu; apb -= inv_cmu; }
    AMB[iq * NS + jq] = amb;
    APB[iq * NS + jq] = apb;
    S0[iq * NS + jq] = dsim[iq] * apb * dinv[jq];     // A_s
    S1[iq * NS + jq] = -dsim[iq] * amb * dinv[jq];    // -B_s
  }
  team_sync<TEAM>();
  // ---- Cholesky of -B_s, else of -A_s (:521-558) -------------------------
  bool primary = ws < 1.0 - 1e-12;
  if (primary) primary = team_chol<NN, NS, TEAM>(S1, LC, misc, t);
  if (!primary) {
    for (int it = t; it < NN * NN; it += TEAM) {
      const int r = it / NN, c = it % NN;
      V[r * NS + c] = -S0[r * NS + c];
    }
    team_sync<TEAM>();
    if (!team_chol<NN, NS, TEAM>(V, LC, misc, t)) {
      // -A_s not SPD either: try the primary factorisation regardless of omega'
      primary = team_chol<NN, NS, TEAM>(S1, LC, misc, t);
      if (!primary) {
        if (t == 0) set_status(p.status, i, DSP_ERR_EIGEN);
        return;
      }
    }
  }
  DSP_PHASE(2)
  // S = L^T M L with M = -A_s (primary) or -B_s (fallback); V used as scratch
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    double s = 0.0;
    if (primary)
      for (int k = 0; k < NN; ++k) s += -S0[r * NS + k] * LC[k * NS + c];
    else
      for (int k = 0; k < NN; ++k) s += S1[r * NS + k] * LC[k * NS + c];
    V[r * NS + c] = s;
  }
  team_sync<TEAM>();
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    double s = 0.0;
    for (int k = 0; k < NN; ++k) s += LC[k * NS + r] * V[k * NS + c];
    S0[r * NS + c] = s;
  }
  team_sync<TEAM>();
  // ---- cyclic Jacobi on S (symmetrised from its lower triangle) -----------
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    S1[r * NS + c] = (c > r) ? S0[c * NS + r] : S0[r * NS + c];
    V[r * NS + c] = (r == c) ? 1.0 : 0.0;
  }
  team_sync<TEAM>();
  DSP_PHASE(3)
  // In place: in a round every 2x2 block of S is read and written by its owner
  // only, and the diagonal blocks a rotation is computed from are written by
  // their owner after it has received that rotation.
  double* const Sc = S1;
  double* const Sn = S1;
  for (int sweep = 0; sweep < 20; ++sweep) {
    for (int r = 0; r < NNP - 1; ++r) {
      // rotation of pair a is computed by thread a; each thread then needs the
      // rotations of its block's two pairs only (blocks are assigned statically)
      double c = 1.0, sn = 0.0, tt = 0.0;
      if (t < NPAIR) {
        const int pp = rr_player<NNP>(r, t), qq = rr_player<NNP>(r, NNP - 1 - t);
        if (pp < NN && qq < NN) {
          jacobi_rot(Sc[pp * NS + qq], Sc[pp * NS + pp], Sc[qq * NS + qq], c, sn, tt);
        }
      }
      if constexpr (TEAM > 32) {
        if (t < NPAIR) {
          rot[3 * t] = c;
          rot[3 * t + 1] = sn;
          rot[3 * t + 2] = tt;
        }
        team_sync<TEAM>();
      }
#pragma unroll
      for (int k = 0; k < BPT; ++k) {
        const int blk = t + k * TEAM;
        const bool act = blk < NPAIR * NPAIR;
        const int a = act ? blk / NPAIR : 0, b = act ? blk % NPAIR : 0;  // NPAIR is a power of two or small
        double ca, sa, ta, cb, sb;
        if constexpr (TEAM <= 32) {
          const unsigned m = team_mask<TEAM>();
          ca = __shfl_sync(m, c, a, TEAM);
          sa = __shfl_sync(m, sn, a, TEAM);
          ta = __shfl_sync(m, tt, a, TEAM);
          cb = __shfl_sync(m, c, b, TEAM);
          sb = __shfl_sync(m, sn, b, TEAM);
        } else {
          ca = rot[3 * a]; sa = rot[3 * a + 1]; ta = rot[3 * a + 2];
          cb = rot[3 * b]; sb = rot[3 * b + 1];
        }
        if (!act) continue;
        const int pa = rr_player<NNP>(r, a), qa = rr_player<NNP>(r, NNP - 1 - a);
        const int pb = rr_player<NNP>(r, b), qb = rr_player<NNP>(r, NNP - 1 - b);
        const bool va = qa < NN && pa < NN, vb = qb < NN && pb < NN;
        if (a == b) {
          if (va) {
            const double apq = Sc[pa * NS + qa];
            Sn[pa * NS + pa] = Sc[pa * NS + pa] - ta * apq;
            Sn[qa * NS + qa] = Sc[qa * NS + qa] + ta * apq;
            const double off = (ta != 0.0) ? 0.0 : apq;
            Sn[pa * NS + qa] = off;
            Sn[qa * NS + pa] = off;
          } else {
            const int x = pa < NN ? pa : qa;
            if (x < NN) Sn[x * NS + x] = Sc[x * NS + x];
          }
        } else {
          // rows of pair a (rotated), columns of pair b (rotated); absent
          // (padding) indices act as the identity
          const int ri[2] = {pa, qa}, cj[2] = {pb, qb};
          double X[2][2];
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
              const int rr = ri[u], cc = cj[v];
              X[u][v] = (rr < NN && cc < NN) ? Sc[rr * NS + cc] : 0.0;
            }
          double Y2[2][2];
          if (va) {
#pragma unroll
            for (int v = 0; v < 2; ++v) {
              Y2[0][v] = ca * X[0][v] - sa * X[1][v];
              Y2[1][v] = sa * X[0][v] + ca * X[1][v];
            }
          } else {
#pragma unroll
            for (int v = 0; v < 2; ++v) { Y2[0][v] = X[0][v]; Y2[1][v] = X[1][v]; }
          }
          double Z2[2][2];
          if (vb) {
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              Z2[u][0] = cb * Y2[u][0] - sb * Y2[u][1];
              Z2[u][1] = sb * Y2[u][0] + cb * Y2[u][1];
            }
          } else {
#pragma unroll
            for (int u = 0; u < 2; ++u) { Z2[u][0] = Y2[u][0]; Z2[u][1] = Y2[u][1]; }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v) {
              const int rr = ri[u], cc = cj[v];
              if (rr < NN && cc < NN) Sn[rr * NS + cc] = Z2[u][v];
            }
        }
        // eigenvectors V <- V J for pair b: this thread's share of the rows
        if (vb) {
          const int rows_per = (NN + BPA - 1) / BPA;  // blocks sharing pair b split its rows
          const int r0 = a * rows_per;
#pragma unroll 4
          for (int row = r0; row < r0 + rows_per && row < NN; ++row) {
            const double vp = V[row * NS + pb], vq = V[row * NS + qb];
            V[row * NS + pb] = cb * vp - sb * vq;
            V[row * NS + qb] = sb * vp + cb * vq;
          }
        }
      }
      team_sync<TEAM>();
    }
    // stop when a further sweep would rotate no pair (the sweep that finds
    // nothing to do is not run)
    if (t == 0) misc[1] = 0.0;
    team_sync<TEAM>();
    for (int it = t; it < NN * NN; it += TEAM) {
      const int r = it / NN, c = it % NN;
      if (c > r && jacobi_needed(Sc[r * NS + c], Sc[r * NS + r], Sc[c * NS + c])) misc[1] = 1.0;
    }
    team_sync<TEAM>();
    const bool more = misc[1] != 0.0;
    team_sync<TEAM>();
    DSP_PHASE(6)
    if (!more) break;
  }
  DSP_PHASE(4)
  // ---- sort ascending; eigenvectors of (a+b)(a-b) ------------------------
  for (int k = t; k < NN; k += TEAM) {
    const double lk = Sc[k * NS + k];
    int rank = 0;
    for (int j = 0; j < NN; ++j) {
      const double lj = Sc[j * NS + j];
      if (lj < lk || (lj == lk && j < k)) ++rank;
    }
    lam[rank] = lk;
    piv[rank] = k;
  }
  team_sync<TEAM>();
  double* Wm = S1;  // sorted eigenvectors of S (columns), over the diagonalised S
  for (int it = t; it < NN * NN; it += TEAM) {
    const int row = it / NN, rank = it % NN;
    Wm[row * NS + rank] = V[row * NS + piv[rank]];
  }
  team_sync<TEAM>();
  // primary: evec = D^{-1} L^{-T} w ; fallback: evec = D^{-1} L' w
  for (int c = t; c < NN; c += TEAM) {
    if (primary) {
      for (int r = NN - 1; r >= 0; --r) {
        double s = Wm[r * NS + c];
        for (int k = r + 1; k < NN; ++k) s -= LC[k * NS + r] * EV[k * NS + c];
        EV[r * NS + c] = s / LC[r * NS + r];
      }
      for (int r = 0; r < NN; ++r) EV[r * NS + c] *= dinv[r];
    } else {
      for (int r = NN - 1; r >= 0; --r) {
        double s = 0.0;
        for (int k = 0; k <= r; ++k) s += LC[r * NS + k] * Wm[k * NS + c];
        EV[r * NS + c] = dinv[r] * s;
      }
    }
  }
  team_sync<TEAM>();
  // ---- k, G+/-  (FluxSolver.cpp:561-587) ---------------------------------
  double* lrec;
  if constexpr (GEN) lrec = p.layer_rec + task * p.g.lstride;
  else lrec = p.layer_rec + ((long long)i * p.L + lc) * lrec_stride(N);
  for (int k = t; k < NN; k += TEAM) {
    const double kr = sqrt(fabs(lam[k]));
    lamraw[k] = lam[k];
    lam[k] = kr;
    lrec[lrec_eig(N) + k + NN] = kr;
    lrec[lrec_eig(N) + NN - 1 - k] = -kr;
  }
  team_sync<TEAM>();
  for (int it = t; it < NN * NN; it += TEAM) {
    const int iq = it / NN, jq = it % NN;
    double s = 0.0;
    for (int k = 0; k < NN; ++k) s += AMB[iq * NS + k] * EV[k * NS + jq];
    const double gpplgm = s / lam[jq];
    const double gpmigm = EV[iq * NS + jq];
    double* G = lrec + lrec_G(N);
    G[(NN + iq) * N + NN + jq] = 0.5 * (gpplgm + gpmigm);
    G[(NN - iq - 1) * N + NN + jq] = 0.5 * (gpplgm - gpmigm);
    G[(NN + iq) * N + NN - jq - 1] = 0.5 * (-gpplgm + gpmigm);
    G[(NN - iq - 1) * N + NN - jq - 1] = 0.5 * (-gpplgm - gpmigm);
  }
  team_sync<TEAM>();
  DSP_PHASE(5)

  // ---- particular solutions in the eigen basis ------------------------------
  // The reference factors the N x N matrices I - C and I + diag(mu)/mu0 - C with
  // a partial-pivot LU (FluxSolver.cpp:634, :758).  With s = z+ + z-, d = z+ - z-
  // and M = diag(mu_1..mu_NN) these split into the NN x NN blocks
  //   I - P - Q = -M (a+b),   I - P + Q = -M (a-b),
  // whose inverses the eigensystem already provides:
  //   (a+b)^{-1} = D^{-1} A_s^{-1} D,  (a-b)^{-1} = D^{-1} B_s^{-1} D,
  //   primary  (-B_s = L L^T, L^T(-A_s)L = W Lam W^T):
  //     B_s^{-1} = -L^{-T} L^{-1},   A_s^{-1} = -L W Lam^{-1} W^T L^T;
  //   fallback (-A_s = L L^T, L^T(-B_s)L = W Lam W^T): the two roles swap.
  // The beam matrix reduces to (a-b)(a+b) - mu0^{-2} = D^{-1}(B_s A_s - mu0^{-2})D,
  // diagonal in the same basis: B_s A_s = L W Lam W^T L^{-1} (primary) or
  // L^{-T} W Lam W^T L^T (fallback); its singular points are the reference's
  // dithering condition |1 - mu0^2 k^2| ~ 0 (FluxSolver.cpp:610-618).
  double* scratch = zv;
  const double dt_ = (t < NN) ? dsim[t] : 1.0;
  const double di_ = (t < NN) ? dinv[t] : 1.0;
  const double mui = (t < NN) ? mu[t] : 1.0;
  const double lami = (t < NN) ? lamraw[t] : 1.0;
  // X1 x = -L^{-T} L^{-1} x ;  X2 x = -L W Lam^{-1} W^T L^T x   (shift: Lam -> Lam - shift)
  auto applyX1 = [&](double x) {
    x = team_trsv<NN, NS, TEAM>(LC, x, false, t, scratch);
    x = team_trsv<NN, NS, TEAM>(LC, x, true, t, scratch);
    return -x;
  };
  auto applyX2 = [&](double x) {
    x = team_matvec<NN, NS, TEAM>(LC, x, true, 1, t, scratch);   // L^T x
    x = team_matvec<NN, NS, TEAM>(Wm, x, true, 0, t, scratch);   // W^T
    x = x / lami;
    x = team_matvec<NN, NS, TEAM>(Wm, x, false, 0, t, scratch);  // W
    x = team_matvec<NN, NS, TEAM>(LC, x, false, 1, t, scratch);  // L
    return -x;
  };
  // (a+b)^{-1} y and (a-b)^{-1} y
  auto inv_apb = [&](double y) {
    const double x = dt_ * y;
    return di_ * (primary ? applyX2(x) : applyX1(x));
  };
  auto inv_amb = [&](double y) {
    const double x = dt_ * y;
    return di_ * (primary ? applyX1(x) : applyX2(x));
  };

  const double fbeam = rec[H_FBEAM];
  if (fbeam > 0.0) {
    // ---- beam (computeBeamSource, FluxSolver.cpp:595-643) -----------------
    // source coefficients zj in bv
    const double umu0 = rec[H_UMU0];
    const double* yb;
    if constexpr (GEN) {
      // P_l^m(-mu0) of this mode (DisortSolver.cpp:1334-1335); Y rows l < m are zero
      double* ybm = sm + C::O_GX;
      if (t == 0) legendre_column(p.g.m, -umu0, N - 1, ybm, 1);
      team_sync<TEAM>();
      yb = ybm;
    } else {
      yb = rec + il.yb;
    }
    // (2 - delta_m0) F0 sum_k g'_k P_k^m(mu_r) P_k^m(-mu0) / 4pi (DisortSolver.cpp:1361-1368)
    const double bfac = (GEN && p.g.m > 0) ? 2.0 * fbeam : fbeam;
    for (int r = t; r < N; r += TEAM) {
      double sacc = 0.0;
      for (int k = 0; k < N; ++k) sacc += gl[k] * Y[k * N + r] * yb[k];
      bv[r] = bfac * sacc / (4.0 * 3.14159265358979323846);
    }
    team_sync<TEAM>();
  }
  if (fbeam > 0.0 && GEN && (p.flags & DSP_FLAG_SPHERICAL_BEAM)) {
    // pseudo-spherical beam (general solver): the source coefficients zj go to
    // the particular-solution slot in its row order, where the user-angle
    // interpolation reads them (computeBeamSourceSpherical keeps the raw zj
    // for interpSource, DisortSolver.cpp:1524-1527); gen_sph_source_kernel
    // then replaces them with Z0
    if (t < NN) {
      lrec[lrec_zb(N) + NN + t] = bv[t];
      lrec[lrec_zb(N) + NN - t - 1] = bv[NN + t];
    }
    team_sync<TEAM>();
  } else if (fbeam > 0.0) {
    const double umu0 = rec[H_UMU0];
    double beam_mu = umu0;
    const double mu0sq = umu0 * umu0;
    const double dither = 1000.0 * 2.220446049250313e-16;
    bool dith = false;
    for (int k = 0; k < NN; ++k) {
      const double kk = lam[k];
      if (fabs(1.0 - mu0sq * kk * kk) < dither) dith = true;
    }
    if (dith) beam_mu = 0.999 * umu0;
    const double bp = (t < NN) ? bv[t] : 0.0, bm = (t < NN) ? bv[NN + t] : 0.0;
    const double m1 = (bp + bm) / mui;  // M^{-1} r1
    const double m2 = (bp - bm) / mui;  // M^{-1} r2
    // rhs = mu0^{-1} M^{-1} r2 + (a-b) M^{-1} r1
    double y = m2 / beam_mu + team_matvec<NN, NS, TEAM>(AMB, m1, false, 0, t, scratch);
    // s = -(D^{-1} (B_s A_s - mu0^{-2})^{-1} D) y
    const double shift = 1.0 / (beam_mu * beam_mu);
    double x = dt_ * y;
    if (primary) {
      x = team_trsv<NN, NS, TEAM>(LC, x, false, t, scratch);          // L^{-1}
      x = team_matvec<NN, NS, TEAM>(Wm, x, true, 0, t, scratch);       // W^T
      x = x / (lami - shift);
      x = team_matvec<NN, NS, TEAM>(Wm, x, false, 0, t, scratch);      // W
      x = team_matvec<NN, NS, TEAM>(LC, x, false, 1, t, scratch);      // L
    } else {
      x = team_matvec<NN, NS, TEAM>(LC, x, true, 1, t, scratch);       // L^T
      x = team_matvec<NN, NS, TEAM>(Wm, x, true, 0, t, scratch);       // W^T
      x = x / (lami - shift);
      x = team_matvec<NN, NS, TEAM>(Wm, x, false, 0, t, scratch);      // W
      x = team_trsv<NN, NS, TEAM>(LC, x, true, t, scratch);            // L^{-T}
    }
    const double sv = -di_ * x;
    // d = mu0 ((a+b) s + M^{-1} r1)
    const double dv = beam_mu * (team_matvec<NN, NS, TEAM>(APB, sv, false, 0, t, scratch) + m1);
    if (t < NN) {
      lrec[lrec_zb(N) + NN + t] = 0.5 * (sv + dv);      // z+ (quadrature index t)
      lrec[lrec_zb(N) + NN - t - 1] = 0.5 * (sv - dv);  // z- (quadrature index NN+t)
    }
    team_sync<TEAM>();
  }
  const bool thermal_src = (p.flags & DSP_FLAG_THERMAL) && (!GEN || p.g.m == 0);
  if (thermal_src) {
    // ---- thermal (computeIsotropicSource, FluxSolver.cpp:745-787) ---------
    // Z1 solves (I-C) z = (1-w') xr1 (isotropic: d1 = 0); Z0 solves
    // (I-C) z = (1-w') xr0 + mu Z1, i.e. r1 = 2(1-w') xr0, r2 = M s1.
    const double taus_top = rec[il.tau_s + lc];
    const double pk0 = rec[il.pkag + lc], pk1 = rec[il.pkag + lc + 1];
    double xr1 = 0.0;
    if (dts > 1e-4) xr1 = (pk1 - pk0) / dts;
    const double xr0 = pk0 - xr1 * taus_top;
    // omega' = 1: no thermal source; (a+b) is singular there, so skip it (uniform per team)
    const bool src = (1.0 - ws) != 0.0;
    const double u = src ? -inv_apb(1.0 / mui) : 0.0;  // -(a+b)^{-1} M^{-1} 1
    const double s1 = 2.0 * (1.0 - ws) * xr1 * u;
    const double s0 = 2.0 * (1.0 - ws) * xr0 * u;
    const double d0 = src ? -inv_amb(s1) : 0.0;        // -(a-b)^{-1} M^{-1} (M s1)
    if (t < NN) {
      lrec[lrec_z1(N) + NN + t] = 0.5 * s1;
      lrec[lrec_z1(N) + NN - t - 1] = 0.5 * s1;
      lrec[lrec_z0(N) + NN + t] = 0.5 * (s0 + d0);
      lrec[lrec_z0(N) + NN - t - 1] = 0.5 * (s0 - d0);
    }
    if (t == 0) {
      lrec[lrec_xr(N)] = xr0;
      lrec[lrec_xr(N) + 1] = xr1;
    }
    if constexpr (JAC) {
      // the source per unit intercept (P) and slope (Q) for the temperature
      // Jacobian: s0 = xr0 P, d0 = xr1 Q
      const double P = 2.0 * (1.0 - ws) * u;
      const double Q = src ? -inv_amb(P) : 0.0;
      if (t < NN) {
        p.jac_pq[task * jpq_stride(N) + t] = P;
        p.jac_pq[task * jpq_stride(N) + NN + t] = Q;
      }
    }
  }
  DSP_PHASE(7)
  if constexpr (GEN) {
    if (p.g.numu > 0) gen_user_angles<N>(p, i, sm, Y, wt, gl, lrec, rec[H_FBEAM], ws, thermal_src, t);
  }
  DSP_PHASE(8)
  DSP_PHASE_END
}


// The rotation of jacobi_rot from two reciprocal square roots, without branches
// or divisions (a sweep is then one scheduling region): with
// r = 1/sqrt(d^2 + e^2), cos 2theta = |d| r and sin 2theta = sgn(d) e r, so
// h = cos^2 theta = (1 + |d| r) / 2, g = 1/sqrt(h) = 1/cos theta,
// c = h g, s = sin 2theta g / 2 and t = tan theta = s g (the same angle as
// jacobi_rot's t = sgn(d) |e| / (|d| + sqrt(d^2 + e^2)); no cancellation for
// small angles).  A pair whose d^2 + e^2 is below 1e-280 is left unrotated:
// S's norm is at least its largest eigenvalue, far above that.
__device__ __forceinline__ void jacobi_rot_rsq(double apq, double app, double aqq, double& c, double& s,
                                               double& tt) {
  const double d = aqq - app, e = 2.0 * apq;
  const double q = fma(d, d, e * e);
  const bool rot = jacobi_needed(apq, app, aqq) && q > 1e-280;
  const double r = rsqrt(rot ? q : 1.0);
  const double num = d > 0.0 ? e : (d < 0.0 ? -e : fabs(e));  // sgn(d) e, sgn(0) = +1
  const double h = fma(0.5 * fabs(d), r, 0.5);
  const double g = rsqrt(h);
  const double sv = (0.5 * num * r) * g;
  c = rot ? h * g : 1.0;
  s = rot ? sv : 0.0;
  tt = rot ? sv * g : 0.0;
}

// ---------------------------------------------------------------------------
// Front of a split layer stage, one thread per layer task (the STAGE before the
// eigensolver): scaled phase coefficients (disortSet, FluxSolver.cpp:336-386),
// the phase sums, alpha -/+ beta in the symmetric form of the reference
// (FluxSolver.cpp:466-514), the Cholesky factorisation of -B_s, else of -A_s
// (:521-558), and S = L^T M L, written to the hand-off.  Every matrix is a
// packed symmetric NN x NN in registers; the tables are constant-bank operands.
// ---------------------------------------------------------------------------
// Cholesky of a packed lower triangle in place; false when a pivot is not
// positive (the factor is then not used).  The updates are subtracted in the
// order of the right-looking form and the column is divided by its pivot, as
// the reference's LLT does: at omega' = 1 one pivot is rounding noise around
// zero, and the factor's other entries should carry the same rounding.
template <int NN>
__device__ __forceinline__ bool chol_packed(double* A) {
  bool ok = true;
#pragma unroll
  for (int j = 0; j < NN; ++j) {
    double s = A[tri_idx(j, j)];
#pragma unroll
    for (int k = 0; k < j; ++k) s -= A[tri_idx(j, k)] * A[tri_idx(j, k)];
    ok = ok && s > 0.0;
    const double ljj = sqrt(ok ? s : 1.0);
    A[tri_idx(j, j)] = ljj;
#pragma unroll
    for (int i = j + 1; i < NN; ++i) {
      double t = A[tri_idx(i, j)];
#pragma unroll
      for (int k = 0; k < j; ++k) t -= A[tri_idx(i, k)] * A[tri_idx(j, k)];
      A[tri_idx(i, j)] = t / ljj;
    }
  }
  return ok;
}

template <int N>
__global__ void __launch_bounds__(128) flux_layer_front_kernel(FluxParams p, ConstTab<N> tc) {
  constexpr int NN = N / 2;
  using H = Handoff<NN>;
  constexpr int TRI = H::TRI;
  const long long nt = (long long)p.n * p.L;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nt) return;
  auto hp = [&](int e) { return handoff_lane<NN>(p.bvp_rec, nt, j, e); };
  const int i = (int)(j / p.L), lc = (int)(j % p.L);
  const double* rec = p.inst_rec + (long long)i * p.il.stride;
  const InstLayout& il = p.il;
  // the layer's inputs are requested before the test that may skip it
  const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? p.L - 1 - lc : lc;
  const double* pml = p.pmom.row(i) + (long long)lin * p.pc;
  double pmk[N];
#pragma unroll
  for (int k = 0; k < N; ++k) pmk[k] = pml[k];
  const double ws = rec[il.ssa_s + lc];
  const bool beam = rec[H_FBEAM] > 0.0;
  const int mode = (int)rec[il.mode + lc];
  const double f = rec[il.fsc + lc], sig = rec[il.sig + lc];
  // invalid instances and layers below the absorption cut are not solved
  if ((p.status && p.status[i] == DSP_ERR_INVALID_INPUT) || lc >= (int)rec[H_NCUT]) {
    *hp(H::S_FLAG) = 0.0;
    return;
  }
  // ---- phase sums O (odd orders) and E (even orders) ----------------------
  double O[TRI], E[TRI];
  {
    double gl[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double pk = pmk[k];
      double g;
      if (mode == 0) g = (2.0 * k + 1.0) * ws * pk;
      else if (mode == 1) g = (2.0 * k + 1.0) * ws * (pk - f) / (1.0 - f);
      else {
        const double kd = (double)k;
        g = (2.0 * k + 1.0) * ws * (pk - f * exp(-kd * kd / (2.0 * sig))) / (1.0 - f);
      }
      gl[k] = g;
    }
#pragma unroll
    for (int a = 0; a < NN; ++a) {
      double z[N];
#pragma unroll
      for (int l = 0; l < N; ++l) z[l] = gl[l] * tc.y[l * N + a];
#pragma unroll
      for (int b = 0; b <= a; ++b) {
        double se = 0.0, so = 0.0;
#pragma unroll
        for (int l = 0; l < N; l += 2) se += z[l] * tc.y[l * N + b];
#pragma unroll
        for (int l = 1; l < N; l += 2) so += z[l] * tc.y[l * N + b];
        E[tri_idx(a, b)] = se;
        O[tri_idx(a, b)] = so;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < TRI; ++e) {
    *hp(H::S_O + e) = O[e];
    if (beam) *hp(H::S_E + e) = E[e];
  }
  // -B_s = -D (a-b) D^{-1} and -A_s = -D (a+b) D^{-1} (packed lower; both symmetric)
  auto minus_s = [&](const double* P, double* X) {
#pragma unroll
    for (int r = 0; r < NN; ++r)
#pragma unroll
      for (int c = 0; c <= r; ++c) {
        const double a = (tc.wt[c] * P[tri_idx(r, c)]) * tc.rmu[r] - (r == c ? tc.rmu[r] : 0.0);
        X[tri_idx(r, c)] = -tc.dsim[r] * a * tc.dinv[c];
      }
  };
  // ---- Cholesky of -B_s, else of -A_s, else of -B_s regardless of omega' --
  double Lf[TRI];
  bool primary = ws < 1.0 - 1e-12;
  if (primary) {
    minus_s(O, Lf);
    primary = chol_packed<NN>(Lf);
  }
  if (!primary) {
    minus_s(E, Lf);
    if (!chol_packed<NN>(Lf)) {
      minus_s(O, Lf);
      primary = chol_packed<NN>(Lf);
      if (!primary) {
        set_status(p.status, i, DSP_ERR_EIGEN);
        *hp(H::S_FLAG) = 0.0;
        return;
      }
    }
  }
  // ---- S = L^T M L, M = -A_s (primary) or -B_s (fallback), by columns ----
  double M[TRI];
  minus_s(primary ? E : O, M);
#pragma unroll
  for (int c = 0; c < NN; ++c) {
    double t[NN];  // (M L)[:, c]; L[k][c] = 0 for k < c
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = c; k < NN; ++k) s += M[tri_idx(r, k)] * Lf[tri_idx(k, c)];
      t[r] = s;
    }
#pragma unroll
    for (int r = c; r < NN; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = r; k < NN; ++k) s += Lf[tri_idx(k, r)] * t[k];
      *hp(H::S_S + tri_idx(r, c)) = s;
    }
  }
#pragma unroll
  for (int e = 0; e < TRI; ++e) *hp(H::S_L + e) = Lf[e];
  *hp(H::S_FLAG) = primary ? 1.0 : 2.0;
}

// Rotation of the pair (p, q) applied to S (packed lower, both sides) and to the
// columns p, q of V; the same update as the team form's 2x2 blocks:
// column p' = c col p - s col q, column q' = s col p + c col q, and on the
// diagonal block a_pp - t a_pq, a_qq + t a_pq, a_pq -> 0.
template <int NN>
__device__ __forceinline__ void jacobi_apply(double* S, double* V, int p, int q, double c, double s,
                                             double t) {
  const double apq = S[tri_idx(p, q)];
#pragma unroll
  for (int k = 0; k < NN; ++k) {
    if (k == p || k == q) continue;
    const double x = S[tri_idx(k, p)], y = S[tri_idx(k, q)];
    S[tri_idx(k, p)] = c * x - s * y;
    S[tri_idx(k, q)] = s * x + c * y;
  }
  S[tri_idx(p, p)] -= t * apq;
  S[tri_idx(q, q)] += t * apq;
  S[tri_idx(p, q)] = (t != 0.0) ? 0.0 : apq;
#pragma unroll
  for (int k = 0; k < NN; ++k) {
    const double x = V[k * NN + p], y = V[k * NN + q];
    V[k * NN + p] = c * x - s * y;
    V[k * NN + q] = s * x + c * y;
  }
}

// The sweeps of the one-thread-per-task eigensolver on S (packed lower) and the
// eigenvector matrix V (row-major), every index a compile-time constant (rounds
// and pairs unrolled).  The sweeps, the round-robin pair order, the rotation
// angle (as jacobi_rot) and the stopping rule (a sweep is run while some pair
// still needs a rotation, at most 20) are those of the team form in
// flux_layer_kernel; a warp runs until its last active task has converged, and
// a converged task's rotations are the identity.  Called by all 32 lanes.
template <int NN>
__device__ __forceinline__ void jacobi_sweeps(double* S, double* V, bool act) {
  constexpr int NNP = NN + (NN & 1), NPAIR = NNP / 2;
  for (int sweep = 0; sweep < 20; ++sweep) {
#pragma unroll
    for (int r = 0; r < NNP - 1; ++r) {
      double c[NPAIR], s[NPAIR], tt[NPAIR];
#pragma unroll
      for (int a = 0; a < NPAIR; ++a) {
        const int pp = rr_player<NNP>(r, a), qq = rr_player<NNP>(r, NNP - 1 - a);
        c[a] = 1.0;
        s[a] = 0.0;
        tt[a] = 0.0;
        if (pp < NN && qq < NN)
          jacobi_rot_rsq(S[tri_idx(pp, qq)], S[tri_idx(pp, pp)], S[tri_idx(qq, qq)], c[a], s[a], tt[a]);
      }
#pragma unroll
      for (int a = 0; a < NPAIR; ++a) {
        const int pp = rr_player<NNP>(r, a), qq = rr_player<NNP>(r, NNP - 1 - a);
        if (pp < NN && qq < NN) jacobi_apply<NN>(S, V, pp, qq, c[a], s[a], tt[a]);
      }
    }
    bool more = false;
#pragma unroll
    for (int r = 1; r < NN; ++r)
#pragma unroll
      for (int q = 0; q < r; ++q)
        if (jacobi_needed(S[tri_idx(r, q)], S[tri_idx(r, r)], S[tri_idx(q, q)])) more = true;
    if (!__any_sync(0xffffffffu, act && more)) break;
  }
}

// Eigensolver of the split layer stage: one thread per layer task, S from the
// hand-off into registers, jacobi_sweeps, the diagonal and the eigenvectors
// back to the hand-off.  (Fusing it into the front kernel, S staying in
// registers, was slower: 4.30 against 4.03 ms for the layer stage of a
// 20,000-band thermal step.)
template <int NN>
__global__ void __launch_bounds__(128) flux_jacobi_kernel(FluxParams p) {
  using H = Handoff<NN>;
  constexpr int NNP = NN + (NN & 1), NPAIR = NNP / 2;
  const long long nt = (long long)p.n * p.L;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j - (threadIdx.x & 31) >= nt) return;  // whole warp past the end (warp-uniform)
  const bool in = j < nt;
  double* const flag = handoff_lane<NN>(p.bvp_rec, nt, in ? j : nt - 1, H::S_FLAG);
  const bool act = in && *flag != 0.0;
  double S[H::TRI], V[NN * NN];
#pragma unroll
  for (int e = 0; e < H::TRI; ++e) S[e] = act ? *handoff_lane<NN>(p.bvp_rec, nt, j, H::S_S + e) : 0.0;
#pragma unroll
  for (int e = 0; e < NN * NN; ++e) V[e] = (e / NN == e % NN) ? 1.0 : 0.0;
  jacobi_sweeps<NN>(S, V, act);
  if (!act) return;
#pragma unroll
  for (int k = 0; k < NN; ++k) *handoff_lane<NN>(p.bvp_rec, nt, j, H::S_D + k) = S[tri_idx(k, k)];
#pragma unroll
  for (int e = 0; e < NN * NN; ++e) *handoff_lane<NN>(p.bvp_rec, nt, j, H::S_V + e) = V[e];
}

// ---------------------------------------------------------------------------
// Back of a split layer stage, one thread per layer task: from the eigenpairs
// of S to the layer record (the STAGE 0 kernel's steps after its Jacobi loop:
// FluxSolver.cpp:561-587 for k and G+/-, :595-643 and :745-787 for the
// particular solutions, in the eigen basis described there).  NN x NN operands
// are held in registers with compile-time indices or read from the
// lane-interleaved hand-off, whose loads are coalesced across the warp; the
// Cholesky factor is read again by each phase that needs it (registers, not
// bandwidth, bound a one-thread task).  Eigenpairs stay in the eigensolver's
// order: the rank of each eigenvalue in the ascending order places its column
// of G and its k, and the sums over eigenpairs (W Lam^{-1} W^T) do not depend
// on the order.
// ---------------------------------------------------------------------------
template <int NN>
struct BackOps {
  const double* L;    // packed lower
  const double* rdg;  // 1 / L_kk
  // x <- L^{-1} x
  __device__ __forceinline__ void fwd(double* x) const {
#pragma unroll
    for (int k = 0; k < NN; ++k) {
      x[k] *= rdg[k];
#pragma unroll
      for (int r = k + 1; r < NN; ++r) x[r] -= L[tri_idx(r, k)] * x[k];
    }
  }
  // x <- L^{-T} x
  __device__ __forceinline__ void bwd(double* x) const {
#pragma unroll
    for (int k = NN - 1; k >= 0; --k) {
      x[k] *= rdg[k];
#pragma unroll
      for (int r = 0; r < k; ++r) x[r] -= L[tri_idx(k, r)] * x[k];
    }
  }
  // x <- L x
  __device__ __forceinline__ void lmul(double* x) const {
#pragma unroll
    for (int r = NN - 1; r >= 0; --r) {
      double s = 0.0;
#pragma unroll
      for (int c = 0; c <= r; ++c) s += L[tri_idx(r, c)] * x[c];
      x[r] = s;
    }
  }
  // x <- L^T x
  __device__ __forceinline__ void ltmul(double* x) const {
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = r; k < NN; ++k) s += L[tri_idx(k, r)] * x[k];
      x[r] = s;
    }
  }
};

// The warp's 32 tasks have consecutive layer records; a row of W doubles that
// each lane has put at stg[lane * RS + k] is written for every task of `ok`
// with consecutive lanes on consecutive doubles (32 / W tasks per store).
template <int RS>
__device__ __forceinline__ void warp_flush_rows(const double* stg, double* rec0, int rstride, int W, int off,
                                                unsigned ok, int lane) {
  __syncwarp();
  const int tpi = 32 / W;
  const int tl = lane / W, k = lane - tl * W;
  if (tl < tpi)
    for (int b = tl; b < 32; b += tpi)
      if ((ok >> b) & 1u) rec0[(long long)b * rstride + off + k] = stg[b * RS + k];
  __syncwarp();
}

template <int N, bool JAC = false>
__global__ void __launch_bounds__(128) flux_layer_back_kernel(FluxParams p, ConstTab<N> tc) {
  constexpr int NN = N / 2;
  constexpr int RS = N + 3;  // staging row stride: a row of N (+2 for xr after z1)
  constexpr int LS = lrec_stride(N);
  using H = Handoff<NN>;
  constexpr double PI = 3.14159265358979323846;
  __shared__ double stage[4][2][32 * RS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double* const stA = stage[wid][0];
  const double* const stB = stage[wid][1];
  double* const sA = stage[wid][0] + lane * RS;
  double* const sB = stage[wid][1] + lane * RS;
  const long long nt = (long long)p.n * p.L;
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long j0 = j - lane;
  if (j0 >= nt) return;  // whole warp past the end (warp-uniform)
  // lanes past the end or skipped by the front compute on a valid task's
  // addresses and write nothing (no early exit: the warp writes rows together)
  const long long jj = j < nt ? j : nt - 1;
  auto hv = [&](int e) { return *handoff_lane<NN>(p.bvp_rec, nt, jj, e); };
  // the hand-off operands of the eigenvector phase are all requested up front,
  // so that their latency overlaps the ordering of the eigenvalues
  double d[NN], L[H::TRI], rdg[NN], EV[NN][NN];  // EV[c][r]: column c
  const double flag = hv(H::S_FLAG);
#pragma unroll
  for (int k = 0; k < NN; ++k) d[k] = hv(H::S_D + k);
#pragma unroll
  for (int e = 0; e < H::TRI; ++e) L[e] = hv(H::S_L + e);
#pragma unroll
  for (int c = 0; c < NN; ++c)
#pragma unroll
    for (int r = 0; r < NN; ++r) EV[c][r] = hv(H::S_V + r * NN + c);
  const bool act = j < nt && flag != 0.0;  // skipped: cut layer, invalid input, no factorisation
  const unsigned okm = __ballot_sync(0xffffffffu, act);
  if (okm == 0u) return;  // warp-uniform
  const bool primary = flag == 1.0;
  const int i = (int)(jj / p.L), lc = (int)(jj % p.L);
  const double* rec = p.inst_rec + (long long)i * p.il.stride;
  const InstLayout& il = p.il;
  double* const rec0 = p.layer_rec + j0 * LS;

  // ---- ascending order of the eigenvalues; k = sqrt|lambda| ----------------
  double kr[NN], rk[NN];
  int rank[NN];
  {
#pragma unroll
    for (int k = 0; k < NN; ++k) {
      int r = 0;
#pragma unroll
      for (int q = 0; q < NN; ++q)
        if (d[q] < d[k] || (d[q] == d[k] && q < k)) ++r;
      rank[k] = r;
      kr[k] = sqrt(fabs(d[k]));
      rk[k] = 1.0 / kr[k];
      sA[NN + r] = kr[k];
      sA[NN - 1 - r] = -kr[k];
    }
  }
  warp_flush_rows<RS>(stA, rec0, LS, N, lrec_eig(N), okm, lane);
  auto load_L = [&]() {
#pragma unroll
    for (int e = 0; e < H::TRI; ++e) L[e] = hv(H::S_L + e);
#pragma unroll
    for (int k = 0; k < NN; ++k) rdg[k] = 1.0 / L[tri_idx(k, k)];
  };
  const BackOps<NN> ops{L, rdg};
  {
    // ---- eigenvectors of (a+b)(a-b): D^{-1} L^{-T} w (primary), D^{-1} L w --
#pragma unroll
    for (int k = 0; k < NN; ++k) rdg[k] = 1.0 / L[tri_idx(k, k)];
#pragma unroll
    for (int c = 0; c < NN; ++c) {
      if (primary) ops.bwd(EV[c]);
      else ops.lmul(EV[c]);
#pragma unroll
      for (int r = 0; r < NN; ++r) EV[c][r] *= tc.dinv[r];
    }
    // ---- G+/- (FluxSolver.cpp:575-587), two rows per step -------------------
    // row iq of O is loaded one step ahead
    double orow[NN];
#pragma unroll
    for (int k = 0; k < NN; ++k) orow[k] = hv(H::S_O + tri_idx(0, k));
#pragma unroll 1
    for (int iq = 0; iq < NN; ++iq) {
      // row iq of alpha - beta = M^{-1} (O W - I)
      double rm = 0.0, arow[NN];
#pragma unroll
      for (int k = 0; k < NN; ++k) rm = (k == iq) ? tc.rmu[k] : rm;
#pragma unroll
      for (int k = 0; k < NN; ++k) arow[k] = (tc.wt[k] * orow[k]) * rm - (k == iq ? rm : 0.0);
      const int iqn = iq + 1 < NN ? iq + 1 : iq;
#pragma unroll
      for (int k = 0; k < NN; ++k) orow[k] = hv(H::S_O + tri_idx(iqn, k));
      double* g0 = sA;  // row NN + iq
      double* g1 = sB;  // row NN - iq - 1
#pragma unroll
      for (int c = 0; c < NN; ++c) {
        double s = 0.0, gpmigm = 0.0;
#pragma unroll
        for (int k = 0; k < NN; ++k) {
          s += arow[k] * EV[c][k];
          gpmigm = (k == iq) ? EV[c][k] : gpmigm;
        }
        const double gpplgm = s * rk[c];
        const int jq = rank[c];
        g0[NN + jq] = 0.5 * (gpplgm + gpmigm);
        g1[NN + jq] = 0.5 * (gpplgm - gpmigm);
        g0[NN - jq - 1] = 0.5 * (-gpplgm + gpmigm);
        g1[NN - jq - 1] = 0.5 * (-gpplgm - gpmigm);
      }
      warp_flush_rows<RS>(stA, rec0, LS, N, lrec_G(N) + (NN + iq) * N, okm, lane);
      warp_flush_rows<RS>(stB, rec0, LS, N, lrec_G(N) + (NN - iq - 1) * N, okm, lane);
    }
  }
  // x <- V diag(1 / (d - shift)) V^T x, one eigenpair at a time
  auto vsolve = [&](double* x, double shift) {
    double acc[NN];
#pragma unroll
    for (int r = 0; r < NN; ++r) acc[r] = 0.0;
#pragma unroll 2
    for (int c = 0; c < NN; ++c) {
      double v[NN], s = 0.0;
#pragma unroll
      for (int r = 0; r < NN; ++r) {
        v[r] = hv(H::S_V + r * NN + c);
        s += v[r] * x[r];
      }
      const double coef = s / (hv(H::S_D + c) - shift);
#pragma unroll
      for (int r = 0; r < NN; ++r) acc[r] += coef * v[r];
    }
#pragma unroll
    for (int r = 0; r < NN; ++r) x[r] = acc[r];
  };
  // X1 x = -L^{-T} L^{-1} x ;  X2 x = -L W Lam^{-1} W^T L^T x
  auto applyX1 = [&](double* x) {
    ops.fwd(x);
    ops.bwd(x);
#pragma unroll
    for (int r = 0; r < NN; ++r) x[r] = -x[r];
  };
  auto applyX2 = [&](double* x) {
    ops.ltmul(x);
    vsolve(x, 0.0);
    ops.lmul(x);
#pragma unroll
    for (int r = 0; r < NN; ++r) x[r] = -x[r];
  };

  const double ws = rec[il.ssa_s + lc];
  const double dts = rec[il.dtau_s + lc];
  const double fbeam = rec[H_FBEAM];
  const unsigned beamm = __ballot_sync(0xffffffffu, act && fbeam > 0.0);
  if (beamm != 0u && fbeam > 0.0) {
    // ---- beam (computeBeamSource, FluxSolver.cpp:595-643) -------------------
    load_L();
    const double umu0 = rec[H_UMU0];
    double beam_mu = umu0;
    const double mu0sq = umu0 * umu0;
    const double dither = 1000.0 * 2.220446049250313e-16;
    bool dith = false;
#pragma unroll
    for (int k = 0; k < NN; ++k)
      if (fabs(1.0 - mu0sq * kr[k] * kr[k]) < dither) dith = true;
    if (dith) beam_mu = 0.999 * umu0;
    // scaled phase coefficients g'_k (disortSet, FluxSolver.cpp:336-386) times
    // P_k(-mu0), summed against P_k(+/-mu_r)
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? p.L - 1 - lc : lc;
    const double* pml = p.pmom.row(i) + (long long)lin * p.pc;
    const int mode = (int)rec[il.mode + lc];
    const double f = rec[il.fsc + lc], sig = rec[il.sig + lc];
    const double* yb = rec + il.yb;
    double sp[NN], sm[NN];
#pragma unroll
    for (int r = 0; r < NN; ++r) sp[r] = sm[r] = 0.0;
#pragma unroll 1
    for (int k = 0; k < N; ++k) {
      const double pk = pml[k];
      double g;
      if (mode == 0) g = (2.0 * k + 1.0) * ws * pk;
      else if (mode == 1) g = (2.0 * k + 1.0) * ws * (pk - f) / (1.0 - f);
      else {
        const double kd = (double)k;
        g = (2.0 * k + 1.0) * ws * (pk - f * exp(-kd * kd / (2.0 * sig))) / (1.0 - f);
      }
      const double gy = g * yb[k];
#pragma unroll
      for (int r = 0; r < NN; ++r) {
        sp[r] += gy * tc.y[k * N + r];
        sm[r] += gy * tc.y[k * N + NN + r];
      }
    }
    double m1[NN], y[NN];
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      const double bp = fbeam * sp[r] / (4.0 * PI), bm = fbeam * sm[r] / (4.0 * PI);
      m1[r] = (bp + bm) * tc.rmu[r];
      y[r] = (bp - bm) * tc.rmu[r];  // M^{-1} r2
    }
    // rhs = mu0^{-1} M^{-1} r2 + (a-b) M^{-1} r1, then D rhs
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NN; ++k)
        s += ((tc.wt[k] * hv(H::S_O + tri_idx(r, k))) * tc.rmu[r] - (k == r ? tc.rmu[r] : 0.0)) * m1[k];
      y[r] = tc.dsim[r] * (y[r] / beam_mu + s);
    }
    // s = -(D^{-1} (B_s A_s - mu0^{-2})^{-1} D) rhs
    const double shift = 1.0 / (beam_mu * beam_mu);
    if (primary) {
      ops.fwd(y);
      vsolve(y, shift);
      ops.lmul(y);
    } else {
      ops.ltmul(y);
      vsolve(y, shift);
      ops.bwd(y);
    }
#pragma unroll
    for (int r = 0; r < NN; ++r) y[r] = -tc.dinv[r] * y[r];
    // d = mu0 ((a+b) s + M^{-1} r1)
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < NN; ++k)
        s += ((tc.wt[k] * hv(H::S_E + tri_idx(r, k))) * tc.rmu[r] - (k == r ? tc.rmu[r] : 0.0)) * y[k];
      const double dv = beam_mu * (s + m1[r]);
      sA[NN + r] = 0.5 * (y[r] + dv);
      sA[NN - r - 1] = 0.5 * (y[r] - dv);
    }
  }
  if (beamm != 0u) warp_flush_rows<RS>(stA, rec0, LS, N, lrec_zb(N), beamm, lane);
  if (p.flags & DSP_FLAG_THERMAL) {
    // ---- thermal (computeIsotropicSource, FluxSolver.cpp:745-787) -----------
    load_L();
    const double taus_top = rec[il.tau_s + lc];
    const double pk0 = rec[il.pkag + lc], pk1 = rec[il.pkag + lc + 1];
    double xr1 = 0.0;
    if (dts > 1e-4) xr1 = (pk1 - pk0) / dts;
    const double xr0 = pk0 - xr1 * taus_top;
    // omega' = 1: no thermal source ((a+b) is singular there)
    const bool src = (1.0 - ws) != 0.0;
    double u[NN], dd[NN];
    // u = -(a+b)^{-1} M^{-1} 1 with (a+b)^{-1} y = D^{-1} X D y (X2 primary, X1 fallback)
#pragma unroll
    for (int r = 0; r < NN; ++r) u[r] = tc.dsim[r] * tc.rmu[r];
    if (src) {
      if (primary) applyX2(u);
      else applyX1(u);
    }
#pragma unroll
    for (int r = 0; r < NN; ++r) u[r] = src ? -tc.dinv[r] * u[r] : 0.0;
    const double c1 = 2.0 * (1.0 - ws) * xr1, c0 = 2.0 * (1.0 - ws) * xr0;
    // d0 = -(a-b)^{-1} s1 with (a-b)^{-1} y = D^{-1} X D y (X1 primary, X2 fallback)
#pragma unroll
    for (int r = 0; r < NN; ++r) dd[r] = tc.dsim[r] * (c1 * u[r]);
    if (src) {
      if (primary) applyX1(dd);
      else applyX2(dd);
    }
#pragma unroll
    for (int r = 0; r < NN; ++r) {
      const double s1 = c1 * u[r], s0 = c0 * u[r];
      const double d0 = src ? -tc.dinv[r] * dd[r] : 0.0;
      sB[NN + r] = 0.5 * s1;
      sB[NN - r - 1] = 0.5 * s1;
      sA[NN + r] = 0.5 * (s0 + d0);
      sA[NN - r - 1] = 0.5 * (s0 - d0);
    }
    sB[N] = xr0;  // xr0, xr1 follow z1 in the record
    sB[N + 1] = xr1;
    warp_flush_rows<RS>(stA, rec0, LS, N, lrec_z0(N), okm, lane);
    warp_flush_rows<RS>(stB, rec0, LS, N + 2, lrec_z1(N), okm, lane);
    if constexpr (JAC) {
      // the source per unit intercept (P) and slope (Q) for the temperature
      // Jacobian: s0 = xr0 P, d0 = xr1 Q
      const double cu = 2.0 * (1.0 - ws);
      double qq[NN];
#pragma unroll
      for (int r = 0; r < NN; ++r) qq[r] = tc.dsim[r] * (cu * u[r]);
      if (src) {
        if (primary) applyX1(qq);
        else applyX2(qq);
      }
      if (act) {
        double* pq = p.jac_pq + jj * jpq_stride(N);
#pragma unroll
        for (int r = 0; r < NN; ++r) {
          pq[r] = cu * u[r];
          pq[NN + r] = src ? -tc.dinv[r] * qq[r] : 0.0;
        }
      }
    }
  }
}

// Host side of the layer stage: launches (through `wrap(name, launch)`, which
// may time them) one layer kernel, or the three launches of a split stage;
// `host_tab` is a host copy of the tab_* tables of N.
template <int N, bool JAC = false>
inline void flux_layer_set_attrs() {
  using C = LCfg<N>;
  if constexpr (layer_split<N>())
    static_assert(Handoff<N / 2>::HS <= brec_stride(N), "the hand-off must fit in the boundary-value records");
  // the team kernel serves every N (N <= 16: when a schedule asks for it)
  cudaFuncSetAttribute(flux_layer_kernel<N, false, JAC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)C::smem_bytes());
}

// The layer stage of a flux chunk.  split: the three one-thread-per-task
// launches (N <= 16 only), with `cta` threads per CTA (64 or 128); otherwise
// the team kernel (shared-memory eigensolver, one team per layer task).
template <int N, bool JAC = false, class Wrap>
inline void flux_layer_launch(const FluxParams& p, const double* host_tab, cudaStream_t s, Wrap&& wrap,
                              bool split = layer_split<N>(), int cta = 128) {
  using C = LCfg<N>;
  const long long tasks = (long long)p.n * p.L;
  if constexpr (layer_split<N>()) {
    if (split) {
      const int b = cta == 64 ? 64 : 128;
      const ConstTab<N> tc = make_const_tab<N>(host_tab);
      const unsigned g = (unsigned)((tasks + b - 1) / b);
      wrap("flux_layer_kernel", [&] { flux_layer_front_kernel<N><<<g, b, 0, s>>>(p, tc); });
      wrap("flux_jacobi_kernel", [&] { flux_jacobi_kernel<N / 2><<<g, b, 0, s>>>(p); });
      wrap("flux_layer_kernel", [&] { flux_layer_back_kernel<N, JAC><<<g, b, 0, s>>>(p, tc); });
      return;
    }
  }
  const unsigned grid = (unsigned)((tasks + C::TPC - 1) / C::TPC);
  wrap("flux_layer_kernel", [&] { flux_layer_kernel<N, false, JAC><<<grid, C::CTA, C::smem_bytes(), s>>>(p); });
}

}  // namespace dsp
