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
#pragma once

#include "dsp_device.cuh"

namespace dsp {

template <int N>
struct LCfg {
  static constexpr int NN = N / 2;
  static constexpr int TEAM = pow2ceil(N) < 4 ? 4 : pow2ceil(N);
  static constexpr int CTA = TEAM >= 32 ? TEAM : 128;
  static constexpr int TPC = CTA / TEAM;
  static constexpr int NNP = NN + (NN & 1);
  static constexpr int NPAIR = NNP / 2;
  static constexpr int LDA = N + 1;  // padded row stride of N x N matrices
  // team shared-memory layout (doubles)
  static constexpr int O_C = 0;                    // C[N][LDA]
  static constexpr int O_A = O_C + N * LDA;        // A[N][LDA] (LU work)
  static constexpr int O_GL = O_A + N * LDA;       // gl[N]
  static constexpr int O_AMB = O_GL + N;           // NN x NN blocks
  static constexpr int O_APB = O_AMB + NN * NN;
  static constexpr int O_S0 = O_APB + NN * NN;
  static constexpr int O_S1 = O_S0 + NN * NN;
  static constexpr int O_V = O_S1 + NN * NN;
  static constexpr int O_LC = O_V + NN * NN;
  static constexpr int O_EV = O_LC + NN * NN;      // eigenvectors of (a+b)(a-b)
  static constexpr int O_LAM = O_EV + NN * NN;     // NN
  static constexpr int O_ROT = O_LAM + NN;         // c, s, t per pair: 3*NPAIR
  static constexpr int O_B = O_ROT + 3 * NPAIR;    // b[N]
  static constexpr int O_Z = O_B + N;              // z[N]
  static constexpr int O_MISC = O_Z + N;           // 8 slots: flags, reduction scratch
  static constexpr int O_PIV = O_MISC + 8;         // N ints (as N doubles)
  static constexpr int TEAM_SMEM = round4(O_PIV + N);
  // CTA-level tables: mu[N] wt[N] dsim[NN] dinv[NN] ylm[N*N]
  static constexpr int TAB = tab_size(N);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(TAB + TPC * TEAM_SMEM); }
};

// Round-robin pairing of NNP players in round r: (arr[a], arr[NNP-1-a]),
// arr[0] = 0, arr[j] = 1 + (j - 1 + r) mod (NNP - 1).
template <int NNP>
__device__ __forceinline__ int rr_player(int r, int j) {
  return j == 0 ? 0 : 1 + (j - 1 + r) % (NNP - 1);
}

// Partial-pivot LU of A (n x n, row stride LDA) in shared memory, the stand-in
// for Eigen::PartialPivLU (FluxSolver.cpp:634, :758).  Returns false on a zero pivot.
template <int N, int TEAM>
__device__ bool team_lu(double* A, int* piv, double* red, int t) {
  constexpr int LDA = N + 1;
  bool ok = true;
  for (int k = 0; k < N; ++k) {
    double v = -1.0;
    int idx = N;
    for (int r = t; r < N; r += TEAM)
      if (r >= k) {
        double a = fabs(A[r * LDA + k]);
        if (isnan(a)) a = __longlong_as_double(0x7ff0000000000000ll);  // NaN ranks as +inf: one total order
        if (a > v || (a == v && r < idx)) { v = a; idx = r; }
      }
    team_argmax<TEAM>(v, idx, red);
    if (idx >= N) idx = k;
    if (t == 0) piv[k] = idx;
    if (idx != k)
      for (int j = t; j < N; j += TEAM) {
        const double tmp = A[k * LDA + j];
        A[k * LDA + j] = A[idx * LDA + j];
        A[idx * LDA + j] = tmp;
      }
    team_sync<TEAM>();
    const double akk = A[k * LDA + k];
    if (akk == 0.0) { ok = false; continue; }
    for (int r = t; r < N; r += TEAM)
      if (r > k) {
        const double l = A[r * LDA + k] / akk;
        A[r * LDA + k] = l;
        for (int j = k + 1; j < N; ++j) A[r * LDA + j] -= l * A[k * LDA + j];
      }
    team_sync<TEAM>();
  }
  return ok;
}

// Solve with the factors of team_lu; b in shared memory, overwritten by x.
template <int N, int TEAM>
__device__ void team_lu_solve(const double* A, const int* piv, double* b, int t) {
  constexpr int LDA = N + 1;
  if (t == 0)
    for (int k = 0; k < N; ++k)
      if (piv[k] != k) {
        const double tmp = b[k];
        b[k] = b[piv[k]];
        b[piv[k]] = tmp;
      }
  team_sync<TEAM>();
  for (int k = 0; k < N - 1; ++k) {
    const double bk = b[k];
    for (int r = t; r < N; r += TEAM)
      if (r > k) b[r] -= A[r * LDA + k] * bk;
    team_sync<TEAM>();
  }
  for (int k = N - 1; k >= 0; --k) {
    if (t == 0) b[k] = b[k] / A[k * LDA + k];
    team_sync<TEAM>();
    const double bk = b[k];
    for (int r = t; r < N; r += TEAM)
      if (r < k) b[r] -= A[r * LDA + k] * bk;
    team_sync<TEAM>();
  }
}

// Cholesky of the lower triangle of M (NN x NN) into Lc; false if not SPD.
// `flag` is team scratch; every thread leaves through a team barrier, so the
// caller may reuse it immediately.
template <int NN, int TEAM>
__device__ bool team_cholesky(const double* M, double* Lc, double* flag, int t) {
  for (int i = t; i < NN * NN; i += TEAM) Lc[i] = 0.0;
  if (t == 0) flag[0] = 0.0;
  team_sync<TEAM>();
  for (int j = 0; j < NN; ++j) {
    if (t == 0) {
      double d = M[j * NN + j];
      for (int k = 0; k < j; ++k) d -= Lc[j * NN + k] * Lc[j * NN + k];
      if (!(d > 0.0)) flag[0] = 1.0;
      else Lc[j * NN + j] = sqrt(d);
    }
    team_sync<TEAM>();
    const bool failed = flag[0] != 0.0;
    team_sync<TEAM>();
    if (failed) return false;
    const double ljj = Lc[j * NN + j];
    for (int i = t; i < NN; i += TEAM)
      if (i > j) {
        double s = M[i * NN + j];
        for (int k = 0; k < j; ++k) s -= Lc[i * NN + k] * Lc[j * NN + k];
        Lc[i * NN + j] = s / ljj;
      }
    team_sync<TEAM>();
  }
  return true;
}

template <int N>
__global__ void __launch_bounds__(LCfg<N>::CTA) flux_layer_kernel(FluxParams p) {
  using C = LCfg<N>;
  constexpr int NN = C::NN, TEAM = C::TEAM, LDA = C::LDA, NNP = C::NNP, NPAIR = C::NPAIR;
  extern __shared__ double smem[];
  // CTA-level constant tables
  for (int k = threadIdx.x; k < C::TAB; k += blockDim.x) smem[k] = p.tables[k];
  __syncthreads();
  const double* mu = smem + tab_mu(N);
  const double* wt = smem + tab_wt(N);
  const double* dsim = smem + tab_dsim(N);
  const double* dinv = smem + tab_dinv(N);
  const double* Y = smem + tab_ylm(N);

  const int team = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
  const long long task = (long long)blockIdx.x * C::TPC + team;
  if (task >= (long long)p.n * p.L) return;
  const int i = (int)(task / p.L), lc = (int)(task % p.L);
  if (p.status && p.status[i] == DSP_ERR_INVALID_INPUT) return;
  const InstLayout& il = p.il;
  const double* rec = p.inst_rec + (long long)i * il.stride;
  const int ncut = (int)rec[H_NCUT];
  if (lc >= ncut) return;  // layers below the absorption cut are never used

  double* sm = smem + C::TAB + team * C::TEAM_SMEM;
  double* Cm = sm + C::O_C;
  double* A = sm + C::O_A;
  double* gl = sm + C::O_GL;
  double* AMB = sm + C::O_AMB;
  double* APB = sm + C::O_APB;
  double* S0 = sm + C::O_S0;
  double* S1 = sm + C::O_S1;
  double* V = sm + C::O_V;
  double* LC = sm + C::O_LC;
  double* EV = sm + C::O_EV;
  double* lam = sm + C::O_LAM;
  double* rot = sm + C::O_ROT;
  double* bv = sm + C::O_B;
  double* zv = sm + C::O_Z;
  double* misc = sm + C::O_MISC;
  int* piv = reinterpret_cast<int*>(sm + C::O_PIV);

  const double ws = rec[il.ssa_s + lc];
  const double dts = rec[il.dtau_s + lc];
  // ---- scaled phase coefficients (disortSet, FluxSolver.cpp:336-386) ----
  {
    const int mode = (int)rec[il.mode + lc];
    const double f = rec[il.fsc + lc], sig = rec[il.sig + lc];
    const int lin = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) ? p.L - 1 - lc : lc;
    const double* pml = p.pmom.row(i) + (long long)lin * p.pc;
    for (int k = t; k < N; k += TEAM) {
      const double pk = pml[k];
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
  // ---- phase matrix C (FluxSolver.cpp:466-482) ---------------------------
  for (int it = t; it < NN * N; it += TEAM) {
    const int iq = it / N, jq = it % N;
    double s = 0.0;
#pragma unroll 8
    for (int l = 0; l < N; ++l) s += (gl[l] * Y[l * N + iq]) * Y[l * N + jq];
    const double cc = (s * 0.5) * wt[jq];
    Cm[iq * LDA + jq] = cc;
    if (jq < NN) Cm[(NN + iq) * LDA + NN + jq] = cc;
    else Cm[(NN + iq) * LDA + jq - NN] = cc;
  }
  team_sync<TEAM>();
  // ---- alpha -/+ beta and the similarity transform (:485-514) ------------
  for (int it = t; it < NN * NN; it += TEAM) {
    const int iq = it / NN, jq = it % NN;
    const double inv_cmu = 1.0 / mu[iq];
    const double a = Cm[iq * LDA + jq], b = Cm[iq * LDA + NN + jq];
    double amb = inv_cmu * (a - b), apb = inv_cmu * (a + b);
    if (iq == jq) { amb -= inv_cmu; apb -= inv_cmu; }
    AMB[it] = amb;
    APB[it] = apb;
    S0[it] = dsim[iq] * apb * dinv[jq];     // A_s
    S1[it] = -dsim[iq] * amb * dinv[jq];    // -B_s
  }
  team_sync<TEAM>();
  // ---- Cholesky of -B_s, else of -A_s (:521-558) -------------------------
  bool primary = ws < 1.0 - 1e-12;
  if (primary) {
    primary = team_cholesky<NN, TEAM>(S1, LC, misc, t);
  }
  if (!primary) {
    // V <- -A_s (temporary), factor it
    for (int it = t; it < NN * NN; it += TEAM) V[it] = -S0[it];
    team_sync<TEAM>();
    if (!team_cholesky<NN, TEAM>(V, LC, misc, t)) {
      // -A_s not SPD either: try the primary factorisation regardless of omega'
      primary = team_cholesky<NN, TEAM>(S1, LC, misc, t);
      if (!primary) {
        if (t == 0) set_status(p.status, i, DSP_ERR_EIGEN);
        return;
      }
    }
  }
  // S = L^T M L with M = -A_s (primary) or -B_s (fallback); EV used as scratch
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    double s = 0.0;
    if (primary)
      for (int k = 0; k < NN; ++k) s += -S0[r * NN + k] * LC[k * NN + c];
    else
      for (int k = 0; k < NN; ++k) s += S1[r * NN + k] * LC[k * NN + c];
    EV[it] = s;
  }
  team_sync<TEAM>();
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    double s = 0.0;
    for (int k = 0; k < NN; ++k) s += LC[k * NN + r] * EV[k * NN + c];
    S0[it] = s;
    V[it] = (r == c) ? 1.0 : 0.0;
  }
  team_sync<TEAM>();
  // ---- cyclic Jacobi on S (symmetrise from the lower triangle first) ------
  for (int it = t; it < NN * NN; it += TEAM) {
    const int r = it / NN, c = it % NN;
    if (c > r) S1[it] = S0[c * NN + r];
    else S1[it] = S0[it];
  }
  team_sync<TEAM>();
  double* Sc = S1;
  double* Sn = S0;
  for (int sweep = 0; sweep < 20; ++sweep) {
    if (t == 0) misc[1] = 0.0;
    team_sync<TEAM>();
    for (int r = 0; r < NNP - 1; ++r) {
      for (int a = t; a < NPAIR; a += TEAM) {
        const int pp = rr_player<NNP>(r, a), qq = rr_player<NNP>(r, NNP - 1 - a);
        double c = 1.0, s = 0.0, tt = 0.0;
        if (pp < NN && qq < NN) {
          const double apq = Sc[pp * NN + qq], app = Sc[pp * NN + pp], aqq = Sc[qq * NN + qq];
          if (fabs(apq) > 1e-300 && fabs(apq) > 1.0e-17 * sqrt(fabs(app * aqq))) {
            const double th = (aqq - app) / (2.0 * apq);
            tt = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
            c = 1.0 / sqrt(tt * tt + 1.0);
            s = tt * c;
            misc[1] = 1.0;
          }
        }
        rot[3 * a] = c;
        rot[3 * a + 1] = s;
        rot[3 * a + 2] = tt;
      }
      team_sync<TEAM>();
      for (int blk = t; blk < NPAIR * NPAIR; blk += TEAM) {
        const int a = blk / NPAIR, b = blk % NPAIR;
        const int pa = rr_player<NNP>(r, a), qa = rr_player<NNP>(r, NNP - 1 - a);
        const int pb = rr_player<NNP>(r, b), qb = rr_player<NNP>(r, NNP - 1 - b);
        const double ca = rot[3 * a], sa = rot[3 * a + 1];
        const double cb = rot[3 * b], sb = rot[3 * b + 1];
        const bool va = qa < NN && pa < NN, vb = qb < NN && pb < NN;
        if (a == b) {
          if (va) {
            const double apq = Sc[pa * NN + qa];
            const double ta = rot[3 * a + 2];
            Sn[pa * NN + pa] = Sc[pa * NN + pa] - ta * apq;
            Sn[qa * NN + qa] = Sc[qa * NN + qa] + ta * apq;
            const double off = (ta != 0.0) ? 0.0 : apq;
            Sn[pa * NN + qa] = off;
            Sn[qa * NN + pa] = off;
          } else {
            const int x = pa < NN ? pa : qa;
            if (x < NN) Sn[x * NN + x] = Sc[x * NN + x];
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
              X[u][v] = (rr < NN && cc < NN) ? Sc[rr * NN + cc] : 0.0;
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
              if (rr < NN && cc < NN) Sn[rr * NN + cc] = Z2[u][v];
            }
        }
      }
      // eigenvectors V <- V J
      for (int u = t; u < NN * NPAIR; u += TEAM) {
        const int row = u / NPAIR, b = u % NPAIR;
        const int pb = rr_player<NNP>(r, b), qb = rr_player<NNP>(r, NNP - 1 - b);
        if (pb < NN && qb < NN) {
          const double cb = rot[3 * b], sb = rot[3 * b + 1];
          const double vp = V[row * NN + pb], vq = V[row * NN + qb];
          V[row * NN + pb] = cb * vp - sb * vq;
          V[row * NN + qb] = sb * vp + cb * vq;
        }
      }
      team_sync<TEAM>();
      double* tmp = Sc;
      Sc = Sn;
      Sn = tmp;
    }
    const bool rotated = misc[1] != 0.0;
    team_sync<TEAM>();
    if (!rotated) break;
  }
  // ---- sort ascending; eigenvectors of (a+b)(a-b) ------------------------
  for (int k = t; k < NN; k += TEAM) {
    const double lk = Sc[k * NN + k];
    int rank = 0;
    for (int j = 0; j < NN; ++j) {
      const double lj = Sc[j * NN + j];
      if (lj < lk || (lj == lk && j < k)) ++rank;
    }
    lam[rank] = lk;
    for (int row = 0; row < NN; ++row) Sn[row * NN + rank] = V[row * NN + k];
  }
  team_sync<TEAM>();
  // primary: evec = D^{-1} L^{-T} w ; fallback: evec = D^{-1} L' w
  for (int c = t; c < NN; c += TEAM) {
    if (primary) {
      for (int r = NN - 1; r >= 0; --r) {
        double s = Sn[r * NN + c];
        for (int k = r + 1; k < NN; ++k) s -= LC[k * NN + r] * EV[k * NN + c];
        EV[r * NN + c] = s / LC[r * NN + r];
      }
      for (int r = 0; r < NN; ++r) EV[r * NN + c] *= dinv[r];
    } else {
      for (int r = NN - 1; r >= 0; --r) {
        double s = 0.0;
        for (int k = 0; k <= r; ++k) s += LC[r * NN + k] * Sn[k * NN + c];
        EV[r * NN + c] = dinv[r] * s;
      }
    }
  }
  team_sync<TEAM>();
  // ---- k, G+/-  (FluxSolver.cpp:561-587) ---------------------------------
  double* lrec = p.layer_rec + ((long long)i * p.L + lc) * lrec_stride(N);
  for (int k = t; k < NN; k += TEAM) {
    const double kr = sqrt(fabs(lam[k]));
    lam[k] = kr;
    lrec[lrec_eig(N) + k + NN] = kr;
    lrec[lrec_eig(N) + NN - 1 - k] = -kr;
  }
  team_sync<TEAM>();
  for (int it = t; it < NN * NN; it += TEAM) {
    const int iq = it / NN, jq = it % NN;
    double s = 0.0;
    for (int k = 0; k < NN; ++k) s += AMB[iq * NN + k] * EV[k * NN + jq];
    const double gpplgm = s / lam[jq];
    const double gpmigm = EV[iq * NN + jq];
    double* G = lrec + lrec_G(N);
    G[(NN + iq) * N + NN + jq] = 0.5 * (gpplgm + gpmigm);
    G[(NN - iq - 1) * N + NN + jq] = 0.5 * (gpplgm - gpmigm);
    G[(NN + iq) * N + NN - jq - 1] = 0.5 * (-gpplgm + gpmigm);
    G[(NN - iq - 1) * N + NN - jq - 1] = 0.5 * (-gpplgm - gpmigm);
  }

  // ---- beam particular solution (FluxSolver.cpp:595-643) -----------------
  const double fbeam = rec[H_FBEAM];
  if (fbeam > 0.0) {
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
    const double* yb = rec + il.yb;
    for (int r = t; r < N; r += TEAM) {
      for (int j = 0; j < N; ++j) A[r * LDA + j] = -Cm[r * LDA + j];
      A[r * LDA + r] += 1.0 + mu[r] / beam_mu;
      double s = 0.0;
      for (int k = 0; k < N; ++k) s += gl[k] * Y[k * N + r] * yb[k];
      bv[r] = fbeam * s / (4.0 * 3.14159265358979323846);
    }
    team_sync<TEAM>();
    if (!team_lu<N, TEAM>(A, piv, misc + 2, t) && t == 0) set_status(p.status, i, DSP_ERR_SINGULAR);
    team_lu_solve<N, TEAM>(A, piv, bv, t);
    for (int iq = t; iq < NN; iq += TEAM) {
      lrec[lrec_zb(N) + NN + iq] = bv[iq];
      lrec[lrec_zb(N) + NN - iq - 1] = bv[iq + NN];
    }
    team_sync<TEAM>();
  }
  // ---- thermal particular solution (FluxSolver.cpp:745-787) --------------
  if (p.flags & DSP_FLAG_THERMAL) {
    const double taus_top = rec[il.tau_s + lc];
    const double pk0 = rec[il.pkag + lc], pk1 = rec[il.pkag + lc + 1];
    double xr1 = 0.0;
    if (dts > 1e-4) xr1 = (pk1 - pk0) / dts;
    const double xr0 = pk0 - xr1 * taus_top;
    for (int r = t; r < N; r += TEAM) {
      for (int j = 0; j < N; ++j) A[r * LDA + j] = -Cm[r * LDA + j];
      A[r * LDA + r] += 1.0;
      zv[r] = (1.0 - ws) * xr1;
    }
    team_sync<TEAM>();
    if (!team_lu<N, TEAM>(A, piv, misc + 2, t) && t == 0) set_status(p.status, i, DSP_ERR_SINGULAR);
    team_lu_solve<N, TEAM>(A, piv, zv, t);
    for (int r = t; r < N; r += TEAM) bv[r] = (1.0 - ws) * xr0 + mu[r] * zv[r];
    team_sync<TEAM>();
    team_lu_solve<N, TEAM>(A, piv, bv, t);
    for (int iq = t; iq < NN; iq += TEAM) {
      lrec[lrec_z0(N) + NN + iq] = bv[iq];
      lrec[lrec_z0(N) + NN - iq - 1] = bv[iq + NN];
      lrec[lrec_z1(N) + NN + iq] = zv[iq];
      lrec[lrec_z1(N) + NN - iq - 1] = zv[iq + NN];
    }
    if (t == 0) {
      lrec[lrec_xr(N)] = xr0;
      lrec[lrec_xr(N) + 1] = xr1;
    }
  }
}

}  // namespace dsp
