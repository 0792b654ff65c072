// flux_bvp_tile.cuh — boundary-value problem and fluxes for N = 32 and 64, one
// CTA per instance with the elimination panel tiled over the CTA's registers.
//
// Replaces setMatrix (FluxSolver.cpp:838-959), solve0 (:966-1131, the LINPACK
// band LU of BandSolver.hpp:29-172) and computeFluxes (:1138-1287), and their
// DisortSolver counterparts (DisortSolver.cpp:1153-1317, 1669-1920, 1980-2124).
//
// Same staircase elimination as flux_bvp_reg.cuh: the band system's rows are
// NN top-boundary rows, N continuity rows per interface and NN bottom rows; for
// the N columns of x_l the candidate pivot rows are the NN rows carried from
// the previous interface plus the N new ones -- the rows LINPACK's band pivot
// search sees -- so the elimination runs on a PR = 3NN row panel with columns
// [x_l block | x_{l+1} block] and a right-hand side.  Panel slots keep their
// rows from layer to layer; the two column blocks swap roles each layer.
//
// Tiling: thread (cg, rg) holds the slots k * RG + rg (k < RPT) restricted to
// the panel columns cg * CPT .. cg * CPT + CPT - 1, and the right-hand side of
// its slots (every column group keeps its own copy and updates it the same way).
// The RG threads of a column group form a half-warp.  A pivot step is
//   A. the half-warp owning column c finds the pivot (arg-max of |a| over the
//      candidate slots, ties to the lower slot, a NaN ranking as +inf), and
//      writes the multipliers of its candidate rows;            barrier
//   B. the threads holding the pivot row stage it in shared memory (it becomes
//      row c of U);                                              barrier
//   C. every thread updates its candidate rows: a += m * pivot row.
// After N steps the pivot rows [U | V | d] and the pivot reciprocals go to the
// layer's elimination record; the upward sweep solves U_l x_l = d_l - V_l x_{l+1}
// layer by layer and evaluates the fluxes (or, for the general solver, stores
// the solution coefficients).
#pragma once

#include "dsp_device.cuh"

namespace dsp {

template <int N>
struct TCfg {
  static constexpr int NN = N / 2;
  static constexpr int PR = 3 * NN;       // panel row slots
  static constexpr int RG = 16;           // row groups: a column group is a half-warp
  static constexpr int RPT = PR / RG;     // slots per thread
  static constexpr int CPT = N >= 64 ? 4 : 8;  // panel columns per thread
  static constexpr int CG = 2 * N / CPT;  // column groups
  static constexpr int CTA = RG * CG;
  static constexpr int TPC = 1;           // instances per CTA
  // resident CTAs per SM the register budget is sized for (128 registers per thread)
  static constexpr int MINB = 65536 / (CTA * 128);
  static constexpr int NW = (PR + 31) / 32;  // words of a slot mask
  static constexpr int LDU = 2 * N + 2;   // staged pivot row: both blocks, rhs, pad
  static constexpr int RL = 2 * N + 1;    // row of the layer's elimination record: [U | V | rhs]
  // shared memory (doubles)
  static constexpr int O_TAB = 0;              // mu[N], wt[N]
  static constexpr int O_U = 2 * N;            // U rows in pivot order [N][LDU]
  static constexpr int O_R = O_U + N * LDU;    // right-hand side of the upward solve [N]
  static constexpr int O_M = O_R + N;          // multipliers, two buffers [2][PR]
  static constexpr int O_X = O_M + 2 * PR;     // x ping-pong [2][N]
  static constexpr int O_EC = O_X + 2 * N;     // [N]
  static constexpr int O_I = O_EC + N;         // intensities [N]
  static constexpr int O_E = O_I + N;          // exp(eig * dtau) of layers l, l + 1 [2][NN]
  static constexpr int O_RD = O_E + 2 * NN;    // 1 / pivot of U row c [N]
  static constexpr int O_MISC = O_RD + N;      // [8]
  static constexpr int O_INT = O_MISC + 8;     // ints: pivot slot [2], pivslot[N], singular flag
  static constexpr int SMEM = round4(O_INT + (N + 4) / 2 + 1);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)SMEM; }
  static_assert(PR % RG == 0 && N % CPT == 0, "tile shape");
  static_assert(CTA <= 1024, "CTA size");
};

template <int NW>
struct TMask {
  uint32_t w[NW];
  __device__ __forceinline__ bool test(int s) const { return (w[s >> 5] >> (s & 31)) & 1u; }
  __device__ __forceinline__ void set(int s) { w[s >> 5] |= 1u << (s & 31); }
  __device__ __forceinline__ void reset(int s) { w[s >> 5] &= ~(1u << (s & 31)); }
  // number of set bits below slot s
  __device__ __forceinline__ int rank(int s) const {
    int r = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      if ((k << 5) + 32 <= s) r += __popc(w[k]);
      else if ((k << 5) < s) r += __popc(w[k] & ((1u << (s & 31)) - 1u));
    }
    return r;
  }
};

// One instance (chunk slot `slot`) on the whole CTA; the constant tables are in
// shared memory already.
template <int N, bool GEN, bool JAC, bool SPH>
__device__ __forceinline__ void bvp_tile_instance(const FluxParams& p, const int slot) {
  using C = TCfg<N>;
  constexpr int NN = C::NN, PR = C::PR, RG = C::RG, RPT = C::RPT, CPT = C::CPT, NW = C::NW;
  constexpr int LDU = C::LDU, RL = C::RL;
  constexpr double PI = 3.14159265358979323846;
  constexpr int TEAM = C::CTA;
  extern __shared__ double smem[];
  const int t = threadIdx.x;
  const int cg = t / RG, rg = t % RG;
  const unsigned half = 0xffffu << (threadIdx.x & 16u);  // this thread's half-warp
  const double* mu = smem + C::O_TAB;
  const double* wt = smem + C::O_TAB + N;
  double* U = smem + C::O_U;
  double* Rv = smem + C::O_R;
  double* mltb = smem + C::O_M;
  double* X = smem + C::O_X;
  double* ec = smem + C::O_EC;
  double* Iv = smem + C::O_I;
  double* E = smem + C::O_E;
  double* rdg = smem + C::O_RD;
  int* ints = reinterpret_cast<int*>(smem + C::O_INT);
  int* psb = ints;           // pivot slot, two buffers
  int* pivslot = ints + 2;   // [N]
  int* sflag = ints + 2 + N; // singular column seen

  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  int i, L, NT;
  const double* rec;
  InstLayout il_gen;
  const double* lrec0;
  double* brec0;
  double* cc0 = nullptr;
  long long lstride;
  if constexpr (GEN) {
    i = p.g.ids[slot];
    L = p.g.Ls[i];
    NT = p.g.user_tau ? p.g.user_tau : L + 1;
    il_gen = InstLayout::make(L, N);
    rec = p.inst_rec + p.g.inst_off[slot];
    lstride = p.g.lstride;
    lrec0 = p.layer_rec + p.g.lay_off[slot] * lstride;
    brec0 = p.bvp_rec + p.g.lay_off[slot] * brec_stride(N);
    cc0 = p.g.cc + p.g.lay_off[slot] * N;
  } else {
    i = slot;
    L = p.L;
    NT = L + 1;
    rec = p.inst_rec + (long long)i * p.il.stride;
    lstride = lrec_stride(N);
    lrec0 = p.layer_rec + (long long)i * L * lstride;
    brec0 = p.bvp_rec + (long long)i * L * brec_stride(N);
  }
  const InstLayout& il = GEN ? il_gen : p.il;
  const int mode_m = GEN ? p.g.m : 0;
  auto oidx = [&](int lev) {
    if constexpr (GEN) return (long long)i * p.g.ntau_out + (ifb ? NT - 1 - lev : lev);
    else return (long long)i * NT + (ifb ? L - lev : lev);
  };
  double* const* outp = GEN ? p.g.out_flux : p.out;
  const int st0 = p.status ? p.status[i] : 0;
  if (st0 == DSP_ERR_INVALID_INPUT || st0 == DSP_ERR_EIGEN) {
    const double qnan = __longlong_as_double(0x7ff8000000000000ll);
    if (mode_m == 0)
      for (int lev = t; lev < NT; lev += TEAM)
        for (int f = 0; f < 8; ++f) outp[f][oidx(lev)] = qnan;
    return;
  }
  if constexpr (GEN) {
    if (mode_m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  }
  DSP_PHASE_BEGIN
  const int ncut = (int)rec[H_NCUT];
  const bool lyrcut = rec[H_LYRCUT] != 0.0;
  // modes m > 0 carry the beam only (DisortSolver.cpp:1246-1250, 1693-1748)
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0 && mode_m == 0;
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double fbeam = rec[H_FBEAM], umu0 = rec[H_UMU0];
  const double alb = mode_m == 0 ? rec[H_ALB] : 0.0;
  // bidirectional surface (general solver): this mode's table, row r =
  // [beam | diffuse streams | emissivity]; it couples at every mode
  const double* sft = nullptr;
  if constexpr (GEN)
    if (p.g.brdf) sft = p.g.brdf + (long long)slot * brdf_stride(N, p.g.numu);
  const bool beam = fbeam > 0.0;
  const double* taus = rec + il.tau_s;
  const double* btr = rec + il.btr;
  const double* dtau_s = rec + il.dtau_s;
  auto LR = [&](int l) { return lrec0 + (long long)l * lstride; };
  // pseudo-spherical beam: layer l's record [Z1 | xba | ch], and its particular
  // solution exp(-xba tau) (Z0 + Z1 tau) at stream iq (solve0, FluxSolver.cpp:1001-1090)
  // (general solver: one record per layer task of the chunk)
  const long long sph0 = GEN ? (long long)p.g.lay_off[slot] : (long long)i * L;
  auto SR = [&](int l) { return p.sph + (sph0 + l) * sph_stride(N); };
  auto zsph = [&](int l, int iq, double tau) {
    const double* sr = SR(l);
    return exp(-sr[sph_xba(N)] * tau) * (__ldg(LR(l) + lrec_zb(N) + iq) + sr[iq] * tau);
  };

  // this thread's tile
  double a[RPT][CPT], rh[RPT];
  const int col0 = cg * CPT;                // first panel column of the thread
  const int myblk = col0 >= N ? 1 : 0;      // column block of the thread
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    rh[k] = 0.0;
#pragma unroll
    for (int j = 0; j < CPT; ++j) a[k][j] = 0.0;
  }
  if (t == 0) sflag[0] = 0;

  // ------------------------------------------------------------------ forward
  TMask<NW> carried;
#pragma unroll
  for (int w = 0; w < NW; ++w) carried.w[w] = 0u;
  for (int s = 0; s < NN; ++s) carried.set(s);  // the top boundary rows
  if (t < NN) E[t] = exp(LR(0)[lrec_eig(N) + t] * dtau_s[0]);
  __syncthreads();
  {
    // top boundary rows in slots 0..NN-1 (setMatrix :890-907, solve0 :978-990)
    const double* l0 = LR(0);
    const double ptop = mode_m == 0 ? rec[H_PTOP] : 0.0, fisot = mode_m == 0 ? rec[H_FISOT] : 0.0;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int s = k * RG + rg;
      if (s < NN) {
        const int jq = NN - 1 - s;
        if (myblk == 0)
#pragma unroll
          for (int j = 0; j < CPT; ++j) {
            const int iq = col0 + j;
            const double g = __ldg(l0 + lrec_G(N) + jq * N + iq);
            a[k][j] = (iq < NN) ? g * E[iq] : g;
          }
        double sum = 0.0;
        if (beam) sum -= __ldg(l0 + lrec_zb(N) + jq);
        if (thermal) sum -= __ldg(l0 + lrec_z0(N) + jq);
        rh[k] = sum + fisot + ptop;
      }
    }
  }

  for (int l = 0; l < ncut; ++l) {
    const bool last = (l == ncut - 1);
    const int cbk = l & 1;  // current column block
    const double* lr = LR(l);
    const double* Ecur = E + (l & 1) * NN;
    double* Enext = E + ((l & 1) ^ 1) * NN;
    if (!last && t < NN) Enext[t] = exp(LR(l + 1)[lrec_eig(N) + t] * dtau_s[l + 1]);
    __syncthreads();
    // carried rows: their next block starts empty (it held the eliminated block)
    const bool in_next = myblk != cbk;
    TMask<NW> freem;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const int lo = w << 5;
      const uint32_t all = (PR - lo >= 32) ? 0xffffffffu : ((1u << (PR - lo)) - 1u);
      freem.w[w] = all & ~carried.w[w];
    }
    const int nnew = last ? NN : N;
    TMask<NW> cand = carried;
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
      const int s = k * RG + rg;
      if (carried.test(s)) {
        if (in_next)
#pragma unroll
          for (int j = 0; j < CPT; ++j) a[k][j] = 0.0;
      } else {
        const int rk = freem.rank(s);
        if (rk < nnew) {
          // new row rk in slot s
          if (!last) {
            // continuity row jq of interface (l, l+1) (setMatrix :852-887, solve0 :1080-1104)
            const int jq = rk;
            const double* ln = LR(l + 1);
            if (!in_next) {
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int iq = col0 - cbk * N + j;
                const double g = __ldg(lr + lrec_G(N) + jq * N + iq);
                a[k][j] = (iq < NN) ? g : g * Ecur[N - 1 - iq];
              }
            } else {
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int iq = col0 - (cbk ^ 1) * N + j;
                const double h = __ldg(ln + lrec_G(N) + jq * N + iq);
                a[k][j] = (iq < NN) ? -h * Enext[iq] : -h;
              }
            }
            const double T = btr[l + 1], tau = taus[l + 1];
            double sum = 0.0;
            if (beam) {
              if constexpr (SPH) {
                sum += zsph(l + 1, jq, tau);
                sum -= zsph(l, jq, tau);
              } else {
                sum += __ldg(ln + lrec_zb(N) + jq) * T;
                sum -= __ldg(lr + lrec_zb(N) + jq) * T;
              }
            }
            if (thermal) {
              sum += __ldg(ln + lrec_z0(N) + jq) - __ldg(lr + lrec_z0(N) + jq);
              sum += (__ldg(ln + lrec_z1(N) + jq) - __ldg(lr + lrec_z1(N) + jq)) * tau;
            }
            rh[k] = sum;
          } else {
            // bottom boundary row (setMatrix :909-958, solve0 :993-1076)
            const int rb = rk, jq = NN + rb;
            const bool plain = lyrcut || dlbc;
            const double* Gl = lr + lrec_G(N);
            const double* srow = sft ? sft + rb * brdf_row(N) : nullptr;
            const double cpl = mode_m == 0 ? 2.0 : 1.0;  // 1 + delta_m0
            if (!in_next) {
#pragma unroll
              for (int j = 0; j < CPT; ++j) {
                const int iq = col0 - cbk * N + j;
                double base = __ldg(Gl + jq * N + iq);
                if (!plain) {
                  double refl = 0.0;
                  if (srow)
                    for (int kk = 0; kk < NN; ++kk)
                      refl += wt[kk] * mu[kk] * srow[1 + kk] * __ldg(Gl + (NN - 1 - kk) * N + iq);
                  else
                    for (int kk = 0; kk < NN; ++kk) refl += wt[kk] * mu[kk] * alb * __ldg(Gl + (NN - 1 - kk) * N + iq);
                  base = base - cpl * refl;
                }
                a[k][j] = (iq < NN) ? base : base * Ecur[N - 1 - iq];
              }
            } else {
#pragma unroll
              for (int j = 0; j < CPT; ++j) a[k][j] = 0.0;
            }
            const double T = btr[ncut], tau = taus[ncut];
            const double pbot = mode_m == 0 ? rec[H_PBOT] : 0.0, pbotd = mode_m == 0 ? rec[H_PBOTD] : 0.0;
            const double fisob = mode_m == 0 ? rec[H_FISOB] : 0.0;
            double sum = 0.0;
            if (dlbc) {
              if (beam) sum -= SPH ? zsph(l, NN + rb, tau) : __ldg(lr + lrec_zb(N) + NN + rb) * T;
              if (thermal) {
                sum -= __ldg(lr + lrec_z0(N) + NN + rb);
                sum -= __ldg(lr + lrec_z1(N) + NN + rb) * tau;
              }
              sum += pbot + mu[rb] * pbotd;
            } else {
              if (!lyrcut) {
                double refl = 0.0;
                for (int jj = 0; jj < NN; ++jj) {
                  double ps = 0.0;
                  if (beam) ps += SPH ? zsph(l, NN - 1 - jj, tau) : __ldg(lr + lrec_zb(N) + NN - 1 - jj) * T;
                  if (thermal)
                    ps += __ldg(lr + lrec_z0(N) + NN - 1 - jj) + __ldg(lr + lrec_z1(N) + NN - 1 - jj) * tau;
                  refl += wt[jj] * mu[jj] * (srow ? srow[1 + jj] : alb) * ps;
                }
                sum += cpl * refl;
              }
              if (beam) {
                sum -= SPH ? zsph(l, NN + rb, tau) : __ldg(lr + lrec_zb(N) + NN + rb) * T;
                if (!lyrcut) sum += (srow ? srow[0] : alb) * umu0 * fbeam * T / PI;
              }
              if (thermal) {
                sum -= __ldg(lr + lrec_z0(N) + NN + rb);
                sum -= __ldg(lr + lrec_z1(N) + NN + rb) * tau;
              }
              sum += fisob;
              if (thermal) sum += (srow ? srow[NN + 1] : 1.0 - alb) * pbot;
            }
            rh[k] = sum;
          }
        }
      }
    }
    // candidates: carried rows and the new rows (identical in every thread)
#pragma unroll
    for (int s = 0; s < PR; ++s)
      if (!carried.test(s) && freem.rank(s) < nnew) cand.set(s);
    DSP_PHASE(10)

    // ---- eliminate the N columns of x_l (sgbfa steps) ----------------------
    const int cgo0 = cbk * (N / CPT);  // first column group of the current block
    // temperature Jacobian: this layer's multipliers and pivot slots
    double* const jrow = !JAC ? nullptr
        : p.jac_rec + ((GEN ? (long long)p.g.lay_off[slot] : (long long)i * L) + l) * jrec_stride(N);
#pragma unroll 1
    for (int cb8 = 0; cb8 < N / CPT; ++cb8) {
      const int cgo = cgo0 + cb8;  // column group owning the next CPT pivot columns
#pragma unroll
      for (int jo = 0; jo < CPT; ++jo) {
        const int c = cb8 * CPT + jo;
        double* mlt = mltb + (c & 1) * PR;
        // A. pivot search and multipliers, in the owning half-warp
        if (cg == cgo) {
          double best = -1.0, bestv = 0.0;
          int bs = PR;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const int s = k * RG + rg;
            if (cand.test(s)) {
              double v = fabs(a[k][jo]);
              if (isnan(v)) v = __longlong_as_double(0x7ff0000000000000ll);  // NaN ranks as +inf
              if (v > best) {  // slots of a thread ascend with k: ties keep the lower slot
                best = v;
                bs = s;
                bestv = a[k][jo];
              }
            }
          }
#pragma unroll
          for (int off = RG / 2; off > 0; off >>= 1) {
            const double ob = __shfl_xor_sync(half, best, off, RG);
            const int os = __shfl_xor_sync(half, bs, off, RG);
            if (ob > best || (ob == best && os < bs)) {
              best = ob;
              bs = os;
            }
          }
          const int ps = bs;
          const double pv = __shfl_sync(half, bestv, ps < PR ? ps % RG : 0, RG);
          const bool sing = ps >= PR || pv == 0.0;  // LINPACK skips a zero pivot (BandSolver.hpp:76-78)
          const double tinv = sing ? 0.0 : -1.0 / pv;
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const int s = k * RG + rg;
            if (cand.test(s) && s != ps) mlt[s] = a[k][jo] * tinv;
          }
          if (rg == 0) {
            psb[c & 1] = sing ? -1 - (ps < PR ? ps : 0) : ps;
            pivslot[c] = ps < PR ? ps : 0;
            rdg[c] = -tinv;
            if (sing) sflag[0] = 1;
          }
        }
        __syncthreads();
        // B. the pivot row becomes row c of U
        const int pcode = psb[c & 1];
        const bool sing = pcode < 0;
        const int ps = sing ? -1 - pcode : pcode;
        if constexpr (JAC) {
          if (t < PR) jrow[c * PR + t] = (!sing && cand.test(t) && t != ps) ? mlt[t] : 0.0;
          if (t == 0) jrow[N * PR + c] = (double)ps;
        }
        if (rg == ps % RG) {
          const int kp = ps / RG;
#pragma unroll
          for (int k = 0; k < RPT; ++k)
            if (k == kp) {
#pragma unroll
              for (int j = 0; j < CPT; ++j) U[c * LDU + col0 + j] = a[k][j];
              if (cg == 0) U[c * LDU + 2 * N] = rh[k];
            }
        }
        cand.reset(ps);
        __syncthreads();
        // C. rank-1 update of the candidate rows (the columns before the pivot
        // column are finished and skipped)
        if (!sing) {
          const bool cols_live = myblk != cbk || col0 + CPT - 1 > cbk * N + c;
          double prow[CPT];
          if (cols_live)
#pragma unroll
            for (int j = 0; j < CPT; ++j) prow[j] = U[c * LDU + col0 + j];
          const double prhs = U[c * LDU + 2 * N];
#pragma unroll
          for (int k = 0; k < RPT; ++k) {
            const int s = k * RG + rg;
            if (cand.test(s)) {
              const double m = mlt[s];
              if (cols_live)
#pragma unroll
                for (int j = 0; j < CPT; ++j) a[k][j] += m * prow[j];
              rh[k] += m * prhs;
            }
          }
        }
      }
    }
    __syncthreads();
    DSP_PHASE(11)

    // ---- the layer's elimination record ------------------------------------
    // Row c of U (the pivot row of column c): [x_l block | x_{l+1} block | rhs],
    // blocks in x order, then 1 / pivot; the upward sweep solves
    // U_l x_l = rhs_l - V_l x_{l+1} with it.
    {
      const int cb = cbk * N, nb = (cbk ^ 1) * N;
      double* br = brec0 + (long long)l * brec_stride(N);
      for (int idx = t; idx < N * RL; idx += TEAM) {
        const int c = idx / RL, col = idx % RL;
        const int src = col < N ? cb + col : (col < 2 * N ? nb + (col - N) : 2 * N);
        br[idx] = U[c * LDU + src];
      }
      for (int c = t; c < N; c += TEAM) br[N * RL + c] = rdg[c];
    }
    // the pivot rows are done; the others are carried into the next layer
    carried = cand;
    __syncthreads();
    DSP_PHASE(12)
  }
  if (sflag[0] && t == 0) set_status(p.status, i, DSP_ERR_SINGULAR);

  // ----------------------------------------------------------------- backward
  bool nonfinite = false;
  // fluxes at output level lu of layer l (computeFluxes, FluxSolver.cpp:1138-1287;
  // DisortSolver.cpp:1980-2124): utaupr scaled depth, utau unscaled depth
  auto eval_level = [&](int l, const double* x, int lu, double utaupr, double utau) {
    const double* lr = LR(l);
    const double* eig = lr + lrec_eig(N);
    const double* Gl = lr + lrec_G(N);
    for (int j = t; j < N; j += TEAM) {
      const double d = (j < NN) ? (utaupr - taus[l + 1]) : (utaupr - taus[l]);
      ec[j] = x[j] * exp(-eig[j] * d);
    }
    __syncthreads();
    // pseudo-spherical: the Chapman factor of the layer replaces mu0
    // (computeFluxes, FluxSolver.cpp:1184-1188, 1216-1219)
    const double ch = SPH && beam ? SR(l)[sph_ch(N)] : 0.0;
    const double fact = beam ? (SPH ? exp(-utaupr / ch) : exp(-utaupr / umu0)) : 0.0;
    for (int r = t; r < N; r += TEAM) {
      double s = 0.0;
      for (int j = 0; j < N; ++j) s += Gl[r * N + j] * ec[j];
      if (beam) s += SPH ? zsph(l, r, utaupr) : lr[lrec_zb(N) + r] * fact;
      if (thermal) s += lr[lrec_z0(N) + r] + lr[lrec_z1(N) + r] * utaupr;
      Iv[r] = s;
    }
    __syncthreads();
    if (t == 0) {
      double dirint = 0.0, fldir = 0.0, fdir = 0.0;
      if (beam) {
        dirint = fbeam * fact;
        fldir = umu0 * fbeam * fact;
        fdir = SPH ? fabs(umu0) * fbeam * exp(-utau / ch) : umu0 * fbeam * exp(-utau / umu0);
      }
      double ua = 0.0, uad = 0.0, uau = 0.0, fldn = 0.0, fup = 0.0;
      for (int iq = 0; iq < NN; ++iq) {
        const int cw = NN - iq - 1;
        ua += wt[cw] * Iv[iq];
        uad += wt[cw] * Iv[iq];
        fldn += wt[cw] * Iv[iq] * mu[cw];
      }
      for (int iq = NN; iq < N; ++iq) {
        const int cw = iq - NN;
        ua += wt[cw] * Iv[iq];
        uau += wt[cw] * Iv[iq];
        fup += wt[cw] * Iv[iq] * mu[cw];
      }
      fup *= 2.0 * PI;
      fldn *= 2.0 * PI;
      const double fdn = (fldn + fldir) - fdir;
      ua = (2.0 * PI * ua + dirint) / (4.0 * PI);
      const double uaso = dirint / (4.0 * PI);
      uad = (2.0 * PI * uad) / (4.0 * PI);
      uau = (2.0 * PI * uau) / (4.0 * PI);
      double plsorc = 0.0;
      if (thermal) plsorc = lr[lrec_xr(N)] + lr[lrec_xr(N) + 1] * utaupr;
      const int lin = ifb ? L - 1 - l : l;
      const double w0 = GEN ? p.g.ssa[p.g.in_off[i] + lin] : p.ssa(i, lin);
      const double dfdt = (1.0 - w0) * 4.0 * PI * (ua - plsorc);
      const double o[8] = {fdir, fdn, fup, dfdt, ua, uad, uau, uaso};
      for (int f = 0; f < 8; ++f) {
        outp[f][oidx(lu)] = o[f];
        if (!isfinite(o[f])) nonfinite = true;
      }
    }
    __syncthreads();
  };
  const double* utau_l = GEN ? rec + GenLayout::make(L, N, NT).utau : nullptr;
  const double* utaus_l = GEN ? rec + GenLayout::make(L, N, NT).utaus : nullptr;
  const double* lyr_l = GEN ? rec + GenLayout::make(L, N, NT).lyr : nullptr;
  if constexpr (!GEN) {
    // levels below the cut carry zeros (computeFluxes :1151-1163)
    for (int lev = ncut + 1 + t; lev <= L; lev += TEAM)
      for (int f = 0; f < 8; ++f) p.out[f][oidx(lev)] = 0.0;
  } else {
    if (mode_m == 0)
      for (int lu = t; lu < NT; lu += TEAM)
        if ((int)lyr_l[lu] > ncut - 1)
          for (int f = 0; f < 8; ++f) outp[f][oidx(lu)] = 0.0;
  }
  constexpr int TPR = TEAM / N;  // threads per row of the matrix-vector product
  static_assert(TPR >= 1 && (TPR & (TPR - 1)) == 0 && TPR <= 32, "row groups within a warp");
  for (int l = ncut - 1; l >= 0; --l) {
    double* x = X + (l & 1) * N;
    // stage the layer's record (U rows in RL-strided rows, then 1 / pivot)
    {
      const double* br = brec0 + (long long)l * brec_stride(N);
      for (int idx = t; idx < N * RL + N; idx += TEAM) U[idx] = br[idx];
    }
    __syncthreads();
    // rhs - V x_{l+1} (x_{l+1} = 0 below the last layer)
    {
      const int c = t / TPR, r = t % TPR;
      const double* xn = X + ((l & 1) ^ 1) * N;
      double s = 0.0;
      if (l < ncut - 1)
        for (int n = r; n < N; n += TPR) s += U[c * RL + N + n] * xn[n];
#pragma unroll
      for (int off = TPR / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off, TPR);
      if (r == 0) Rv[c] = U[c * RL + 2 * N] - s;
    }
    __syncthreads();
    // U x_l = r: column-oriented back substitution in one warp, rows t and t + 32
    if (t < 32) {
      const double* rdiag = U + N * RL;
      double r0 = Rv[t], r1 = (N > 32) ? Rv[(t + 32) % N] : 0.0;
#pragma unroll 4
      for (int c = N - 1; c >= 0; --c) {
        const double u0 = U[t * RL + c];
        const double u1 = (N > 32) ? U[((t + 32) % N) * RL + c] : 0.0;
        const double mine = (c < 32) ? r0 : r1;
        const double xc = __shfl_sync(0xffffffffu, mine * rdiag[c], c & 31);
        if (t == (c & 31)) x[c] = xc;
        if (t < c) r0 -= u0 * xc;
        if (N > 32 && t + 32 < c) r1 -= u1 * xc;
      }
    }
    __syncthreads();
    DSP_PHASE(13)
    if constexpr (GEN) {
      for (int c = t; c < N; c += TEAM) cc0[(long long)l * N + c] = x[c];
      if (mode_m == 0)
        for (int lu = 0; lu < NT; ++lu)
          if ((int)lyr_l[lu] == l) eval_level(l, x, lu, utaus_l[lu], utau_l[lu]);
    } else {
      eval_level(l, x, l + 1, taus[l + 1], rec[il.tauc + l + 1]);
      if (l == 0) eval_level(0, x, 0, taus[0], rec[il.tauc]);
    }
    DSP_PHASE(14)
  }
  DSP_PHASE_END
  if (nonfinite && t == 0) set_status(p.status, i, DSP_ERR_NONFINITE);
}

// One CTA per instance, in chunk-slot order.
template <int N, bool GEN = false, bool JAC = false, bool SPH = false>
__global__ void __launch_bounds__(TCfg<N>::CTA, TCfg<N>::MINB) flux_bvp_tile_kernel(FluxParams p) {
  using C = TCfg<N>;
  extern __shared__ double smem[];
  for (int k = threadIdx.x; k < 2 * N; k += C::CTA) smem[C::O_TAB + k] = p.tables[k];
  __syncthreads();
  if ((int)blockIdx.x >= p.n) return;
  bvp_tile_instance<N, GEN, JAC, SPH>(p, blockIdx.x);
}

// Persistent form (general solver): a resident grid whose CTAs take chunk slots
// from the size-class-ordered queue `order` through the counter `head`.
template <int N, bool JAC = false, bool SPH = false>
__global__ void __launch_bounds__(TCfg<N>::CTA, TCfg<N>::MINB)
    gen_bvp_tile_persistent_kernel(FluxParams p, const int* order, int* head) {
  using C = TCfg<N>;
  extern __shared__ double smem[];
  __shared__ int task;
  for (int k = threadIdx.x; k < 2 * N; k += C::CTA) smem[C::O_TAB + k] = p.tables[k];
  for (;;) {
    if (threadIdx.x == 0) task = atomicAdd(head, 1);
    __syncthreads();  // the task, and (first trip) the tables, are visible
    const int k = task;
    if (k >= p.n) break;
    bvp_tile_instance<N, true, JAC, SPH>(p, order[k]);
    __syncthreads();  // every thread is done with the instance before `task` changes
  }
}

}  // namespace dsp
