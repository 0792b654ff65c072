// flux_bvp.cuh — boundary-value problem and fluxes, one team per instance.
//
// Replaces setMatrix (FluxSolver.cpp:838-959), solve0 (:966-1131, the LINPACK
// band LU of BandSolver.hpp:29-172) and computeFluxes (:1138-1287).
//
// The reference stores the (N*ncut)^2 system in LINPACK band form (lda = 9NN-2)
// and factors it with partial pivoting (ml = mu = 3NN-1).  Its rows are a
// staircase: NN top-boundary rows on x_0, N continuity rows on (x_l, x_{l+1})
// per interface, NN bottom rows on x_{ncut-1}.  For the N columns of x_l the
// rows with non-zeros that are not yet pivot rows are exactly NN carried rows
// plus the N rows of interface (l, l+1) -- the same candidate set the band
// pivot search sees -- so the elimination is done on a 3NN x (2N+1) panel held
// in shared memory: pivot = largest |a| among candidates, multipliers
// a * (-1/pivot) and row updates as in sgbfa, the right-hand side carried along
// as sgbsl's forward sweep.  After the N pivots of a layer the pivot rows give
// U_l x_l + V_l x_{l+1} = c_l; the team stores W_l = U_l^{-1} V_l (transposed)
// and d_l = U_l^{-1} c_l in an L2-resident workspace and keeps the NN remaining
// rows as the next layer's carried rows.  Back substitution then runs bottom-up,
// x_l = d_l - W_l x_{l+1}, and each x_l immediately yields the fluxes at the
// layer's bottom level (and at the top level for layer 0).
#pragma once

#include "dsp_device.cuh"

namespace dsp {

// Bitmask over the panel's row slots, kept identical in every thread of a team.
template <int PR>
struct SlotMask {
  static constexpr int W = (PR + 31) / 32;
  uint32_t w[W];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int k = 0; k < W; ++k) w[k] = 0u;
  }
  __device__ __forceinline__ void set(int s) { w[s >> 5] |= 1u << (s & 31); }
  __device__ __forceinline__ void reset(int s) { w[s >> 5] &= ~(1u << (s & 31)); }
  __device__ __forceinline__ bool test(int s) const { return (w[s >> 5] >> (s & 31)) & 1u; }
};

template <int N>
struct BCfg {
  static constexpr int NN = N / 2;
  static constexpr int TEAM = pow2ceil(2 * N) < 8 ? 8 : pow2ceil(2 * N);
  static constexpr int CTA = TEAM >= 32 ? TEAM : 32;
  static constexpr int TPC = CTA / TEAM;
  static constexpr int PR = 3 * NN;       // panel row slots
  static constexpr int LDP = 2 * N + 1;   // two column blocks + rhs (odd stride)
  static constexpr int RHS = 2 * N;
  static constexpr int O_P = 0;
  static constexpr int O_M = O_P + PR * LDP;  // multipliers [PR]
  static constexpr int O_X = O_M + PR;        // x ping-pong [2][N]
  static constexpr int O_EC = O_X + 2 * N;    // [N]
  static constexpr int O_I = O_EC + N;        // intensities [N]
  static constexpr int O_E = O_I + N;         // exp(eig*dtau) of layer l and l+1 [2][NN]
  static constexpr int O_MISC = O_E + 2 * NN; // 8
  static constexpr int O_ST = O_MISC + 8;     // int state[PR], pivslot[N], freeslot[PR]
  static constexpr int TEAM_SMEM = round4(O_ST + (2 * PR + N + 1) / 2 + 1);
  static constexpr int TAB = tab_size(N);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(TAB + TPC * TEAM_SMEM); }
  // resident CTAs per SM the register allocation must allow (<= 168 registers for 32-thread CTAs)
  static constexpr int MINB = TEAM >= 128 ? 1 : (TEAM >= 64 ? 4 : 12);
};

template <int N, bool GEN = false>
__global__ void __launch_bounds__(BCfg<N>::CTA, BCfg<N>::MINB) flux_bvp_kernel(FluxParams p) {
  using C = BCfg<N>;
  constexpr int NN = C::NN, TEAM = C::TEAM, PR = C::PR, LDP = C::LDP, RHS = C::RHS;
  constexpr double PI = 3.14159265358979323846;
  extern __shared__ double smem[];
  for (int k = threadIdx.x; k < C::TAB; k += blockDim.x) smem[k] = p.tables[k];
  __syncthreads();
  const double* mu = smem + tab_mu(N);
  const double* wt = smem + tab_wt(N);

  const int team = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
  const int slot = blockIdx.x * C::TPC + team;
  if (slot >= p.n) return;
  // index_from_bottom: outputs are reversed (IndexConversion.hpp:60-116)
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  // i: status / input / output index, L: layers, NT: output levels
  int i, L, NT;
  const double* rec;
  InstLayout il_gen;  // general solver: the layout of this instance
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
  const int ncut = (int)rec[H_NCUT];
  const bool lyrcut = rec[H_LYRCUT] != 0.0;
  // modes m > 0 carry the beam only: no thermal or isotropic sources and no
  // Lambertian coupling (DisortSolver.cpp:1246-1250, 1693-1748)
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0 && mode_m == 0;
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double fbeam = rec[H_FBEAM], umu0 = rec[H_UMU0];
  const double alb = mode_m == 0 ? rec[H_ALB] : 0.0;
  const bool beam = fbeam > 0.0;
  const double* taus = rec + il.tau_s;
  const double* btr = rec + il.btr;
  const double* dtau_s = rec + il.dtau_s;

  double* sm = smem + C::TAB + team * C::TEAM_SMEM;
  double* P = sm + C::O_P;
  double* mlt = sm + C::O_M;
  double* X = sm + C::O_X;
  double* ec = sm + C::O_EC;
  double* Iv = sm + C::O_I;
  double* E = sm + C::O_E;
  double* misc = sm + C::O_MISC;
  int* state = reinterpret_cast<int*>(sm + C::O_ST);
  int* pivslot = state + PR;
  int* freeslot = pivslot + N;

  auto LR = [&](int l) { return lrec0 + (long long)l * lstride; };
  bool singular = false;

  DSP_PHASE_BEGIN
  // ------------------------------------------------------------------ forward
  for (int s = t; s < PR; s += TEAM) state[s] = 0;
  for (int m = t; m < NN; m += TEAM) {
    const double* l0 = LR(0);
    E[m] = exp(l0[lrec_eig(N) + m] * dtau_s[0]);
  }
  team_sync<TEAM>();
  // top boundary rows into slots 0..NN-1 (setMatrix :890-907, solve0 :978-990)
  {
    const double* l0 = LR(0);
    const double* G0 = l0 + lrec_G(N);
    const double ptop = mode_m == 0 ? rec[H_PTOP] : 0.0, fisot = mode_m == 0 ? rec[H_FISOT] : 0.0;
    for (int it = t; it < NN * (2 * N + 1); it += TEAM) {
      const int r = it / (2 * N + 1), col = it % (2 * N + 1);
      const int jq = NN - 1 - r;
      double v;
      if (col < N) v = (col < NN) ? G0[jq * N + col] * E[col] : G0[jq * N + col];
      else if (col < 2 * N) v = 0.0;
      else {
        double s = 0.0;
        if (beam) s -= l0[lrec_zb(N) + jq];
        if (thermal) s -= l0[lrec_z0(N) + jq];
        s += fisot + ptop;
        v = s;
      }
      P[r * LDP + col] = v;
    }
    for (int r = t; r < NN; r += TEAM) state[r] = 1;
  }
  team_sync<TEAM>();

  for (int l = 0; l < ncut; ++l) {
    const int cb = (l & 1) * N, nb = ((l & 1) ^ 1) * N;
    const bool last = (l == ncut - 1);
    const double* lr = LR(l);
    const double* Gl = lr + lrec_G(N);
    const double* Ecur = E + (l & 1) * NN;
    double* Enext = E + ((l & 1) ^ 1) * NN;
    // free slots list (slots not carried), carried rows lose their stale block
    if (t == 0) {
      int nf = 0;
      for (int s = 0; s < PR; ++s) {
        if (state[s] == 2) state[s] = 0;
        if (state[s] == 0) freeslot[nf++] = s;
      }
    }
    if (!last) {
      const double* ln = LR(l + 1);
      for (int m = t; m < NN; m += TEAM) Enext[m] = exp(ln[lrec_eig(N) + m] * dtau_s[l + 1]);
    }
    team_sync<TEAM>();
    if (l > 0)
      for (int it = t; it < PR * N; it += TEAM) {
        const int s = it / N, c = it % N;
        if (state[s] == 1) P[s * LDP + nb + c] = 0.0;
      }
    if (!last) {
      // continuity rows of interface (l, l+1) (setMatrix :852-887, solve0 :1080-1104).
      // All global reads of an item batch are issued before any shared-memory store.
      const double* ln = LR(l + 1);
      const double* Gn = ln + lrec_G(N);
      const double T = btr[l + 1], tau = taus[l + 1];
      constexpr int ITEMS = N * (2 * N + 1);
      constexpr int PER = (ITEMS + TEAM - 1) / TEAM;
      double val[PER];
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int it = t + k * TEAM;
        if (it < ITEMS) {
          const int jq = it / (2 * N + 1), col = it % (2 * N + 1);
          if (col < N) {
            const int iq = col;
            const double g = __ldg(Gl + jq * N + iq);
            val[k] = (iq < NN) ? g : g * Ecur[N - 1 - iq];
          } else if (col < 2 * N) {
            const int iq = col - N;
            const double g = __ldg(Gn + jq * N + iq);
            val[k] = (iq < NN) ? -g * Enext[iq] : -g;
          } else {
            double sum = 0.0;
            if (beam) {
              sum += __ldg(ln + lrec_zb(N) + jq) * T;
              sum -= __ldg(lr + lrec_zb(N) + jq) * T;
            }
            if (thermal) {
              sum += __ldg(ln + lrec_z0(N) + jq) - __ldg(lr + lrec_z0(N) + jq);
              sum += (__ldg(ln + lrec_z1(N) + jq) - __ldg(lr + lrec_z1(N) + jq)) * tau;
            }
            val[k] = sum;
          }
        }
      }
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int it = t + k * TEAM;
        if (it < ITEMS) {
          const int jq = it / (2 * N + 1), col = it % (2 * N + 1);
          const int sl = freeslot[jq];
          const int pc = (col < N) ? cb + col : (col < 2 * N) ? nb + (col - N) : RHS;
          P[sl * LDP + pc] = val[k];
        }
      }
      for (int jq = t; jq < N; jq += TEAM) state[freeslot[jq]] = 1;
    } else {
      // bottom boundary rows (setMatrix :909-958, solve0 :993-1076)
      const bool plain = lyrcut || dlbc;
      const double T = btr[ncut], tau = taus[ncut];
      const double pbot = mode_m == 0 ? rec[H_PBOT] : 0.0, pbotd = mode_m == 0 ? rec[H_PBOTD] : 0.0;
      const double fisob = mode_m == 0 ? rec[H_FISOB] : 0.0;
      for (int it = t; it < NN * (2 * N + 1); it += TEAM) {
        const int rb = it / (2 * N + 1), col = it % (2 * N + 1);
        const int jq = NN + rb;
        const int s = freeslot[rb];
        if (col < N) {
          const int iq = col;
          double base = Gl[jq * N + iq];
          if (!plain) {
            double refl = 0.0;
            for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * alb * Gl[(NN - 1 - k) * N + iq];
            base = Gl[jq * N + iq] - 2.0 * refl;
          }
          P[s * LDP + cb + iq] = (iq < NN) ? base : base * Ecur[N - 1 - iq];
        } else if (col < 2 * N) {
          P[s * LDP + nb + (col - N)] = 0.0;
        } else {
          double sum = 0.0;
          if (dlbc) {
            if (beam) sum -= lr[lrec_zb(N) + NN + rb] * T;
            if (thermal) {
              sum -= lr[lrec_z0(N) + NN + rb];
              sum -= lr[lrec_z1(N) + NN + rb] * tau;
            }
            sum += pbot + mu[rb] * pbotd;
          } else {
            if (!lyrcut) {
              double refl = 0.0;
              for (int jj = 0; jj < NN; ++jj) {
                double ps = 0.0;
                if (beam) ps += lr[lrec_zb(N) + NN - 1 - jj] * T;
                if (thermal) ps += lr[lrec_z0(N) + NN - 1 - jj] + lr[lrec_z1(N) + NN - 1 - jj] * tau;
                refl += wt[jj] * mu[jj] * alb * ps;
              }
              sum += 2.0 * refl;
            }
            if (beam) {
              sum -= lr[lrec_zb(N) + NN + rb] * T;
              if (!lyrcut) sum += alb * umu0 * fbeam * T / PI;
            }
            if (thermal) {
              sum -= lr[lrec_z0(N) + NN + rb];
              sum -= lr[lrec_z1(N) + NN + rb] * tau;
            }
            sum += fisob;
            if (thermal) sum += (1.0 - alb) * pbot;
          }
          P[s * LDP + RHS] = sum;
        }
      }
      for (int rb = t; rb < NN; rb += TEAM) state[freeslot[rb]] = 1;
    }
    team_sync<TEAM>();
    DSP_PHASE(10)

    // ---- eliminate the N columns of x_l (sgbfa steps) ----------------------
    // Candidate rows form a bitmask that every thread tracks identically.
    SlotMask<PR> cand;
    cand.clear();
    for (int sl = 0; sl < PR; ++sl)
      if (state[sl] == 1) cand.set(sl);
    const int ncols_next = last ? 0 : N;
    for (int c = 0; c < N; ++c) {
      const int col = cb + c;
      double v = -1.0;
      int idx = PR;
      for (int sl = t; sl < PR; sl += TEAM)
        if (cand.test(sl)) {
          double a = fabs(P[sl * LDP + col]);
          if (isnan(a)) a = __longlong_as_double(0x7ff0000000000000ll);  // NaN ranks as +inf: one total order
          if (a > v || (a == v && sl < idx)) { v = a; idx = sl; }
        }
      team_argmax<TEAM>(v, idx, misc);
      const int ps = idx;
      if (ps >= PR) {  // no candidate row (cannot happen for a well-formed system)
        singular = true;
        if (t == 0) pivslot[c] = 0;
        continue;
      }
      cand.reset(ps);
      if (t == 0) {
        state[ps] = 2;
        pivslot[c] = ps;
      }
      const double pv = P[ps * LDP + col];
      if (pv == 0.0) {  // LINPACK skips a zero pivot column (BandSolver.hpp:76-78)
        singular = true;
        team_sync<TEAM>();
        continue;
      }
      const double tinv = -1.0 / pv;
      // one column per thread: col+1 .. end of block, the next block (unless last), rhs
      const int ncur = N - 1 - c;
      const int ntot = ncur + ncols_next + 1;
      if (t < ntot) {
        const int j = (t < ncur) ? col + 1 + t : (t < ncur + ncols_next) ? nb + (t - ncur) : RHS;
        const double pj = P[ps * LDP + j];
        if (pj != 0.0) {
          // slots in chunks of 16: all loads of a chunk are issued before its FMAs
          constexpr int CH = PR < 16 ? PR : 16;
#pragma unroll
          for (int base = 0; base < PR; base += CH) {
            double m[CH], a[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k) {
              const int sl = base + k;
              if (sl < PR && cand.test(sl)) {
                m[k] = P[sl * LDP + col];
                a[k] = P[sl * LDP + j];
              }
            }
#pragma unroll
            for (int k = 0; k < CH; ++k) {
              const int sl = base + k;
              if (sl < PR && cand.test(sl)) P[sl * LDP + j] = a[k] + (m[k] * tinv) * pj;
            }
          }
        }
      }
      team_sync<TEAM>();
    }

    DSP_PHASE(11)
    if (!last) {
      // W_l = U^{-1} V (stored transposed), d_l = U^{-1} c: one column per thread,
      // column-oriented back substitution held in registers
      double* br = brec0 + (long long)l * brec_stride(N);
      if (t <= N) {
        const int colj = (t < N) ? nb + t : RHS;
        double r[N];
#pragma unroll
        for (int c = 0; c < N; ++c) r[c] = P[pivslot[c] * LDP + colj];
#pragma unroll
        for (int c = N - 1; c >= 0; --c) {
          const double x = r[c] / P[pivslot[c] * LDP + cb + c];
          r[c] = x;
#pragma unroll
          for (int c2 = 0; c2 < c; ++c2) r[c2] -= P[pivslot[c2] * LDP + cb + c] * x;
        }
        double* dst = (t < N) ? br + t * N : br + N * N;
#pragma unroll
        for (int c = 0; c < N; ++c) dst[c] = r[c];
      }
      team_sync<TEAM>();
    } else {
      // x_{ncut-1} = U^{-1} rhs (sgbsl back substitution)
      double* x = X + (l & 1) * N;
      if (t == 0) {
        int ps[N];
        double r[N];
#pragma unroll
        for (int c = 0; c < N; ++c) ps[c] = pivslot[c];
#pragma unroll
        for (int c = 0; c < N; ++c) r[c] = P[ps[c] * LDP + RHS];
#pragma unroll
        for (int c = N - 1; c >= 0; --c) {
          const double xv = r[c] / P[ps[c] * LDP + cb + c];
          r[c] = xv;
#pragma unroll
          for (int c2 = 0; c2 < c; ++c2) r[c2] -= P[ps[c2] * LDP + cb + c] * xv;
        }
#pragma unroll
        for (int c = 0; c < N; ++c) x[c] = r[c];
      }
      team_sync<TEAM>();
    }
    DSP_PHASE(12)
  }
  if (singular && t == 0) set_status(p.status, i, DSP_ERR_SINGULAR);

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
    team_sync<TEAM>();
    const double fact = beam ? exp(-utaupr / umu0) : 0.0;
    for (int r = t; r < N; r += TEAM) {
      double s = 0.0;
      for (int j = 0; j < N; ++j) s += Gl[r * N + j] * ec[j];
      if (beam) s += lr[lrec_zb(N) + r] * fact;
      if (thermal) s += lr[lrec_z0(N) + r] + lr[lrec_z1(N) + r] * utaupr;
      Iv[r] = s;
    }
    team_sync<TEAM>();
    if (t == 0) {
      double dirint = 0.0, fldir = 0.0, fdir = 0.0;
      if (beam) {
        dirint = fbeam * fact;
        fldir = umu0 * fbeam * fact;
        fdir = umu0 * fbeam * exp(-utau / umu0);
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
    team_sync<TEAM>();
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
  for (int l = ncut - 1; l >= 0; --l) {
    double* x = X + (l & 1) * N;
    if (l < ncut - 1) {
      const double* xn = X + ((l & 1) ^ 1) * N;
      const double* br = brec0 + (long long)l * brec_stride(N);
      for (int c = t; c < N; c += TEAM) {
        double s = br[N * N + c];
        for (int n = 0; n < N; ++n) s -= br[n * N + c] * xn[n];
        x[c] = s;
      }
      team_sync<TEAM>();
    }
    DSP_PHASE(13)
    if constexpr (GEN) {
      for (int c = t; c < N; c += TEAM) cc0[(long long)l * N + c] = x[c];
      if (mode_m == 0)
        for (int lu = 0; lu < NT; ++lu)
          if ((int)lyr_l[lu] == l) eval_level(l, x, lu, utaus_l[lu], utau_l[lu]);
    } else {
      // outputs at the bottom level of layer l, and at the top for l == 0
      eval_level(l, x, l + 1, taus[l + 1], rec[il.tauc + l + 1]);
      if (l == 0) eval_level(0, x, 0, taus[0], rec[il.tauc]);
    }
    DSP_PHASE(14)
  }
  if (nonfinite && t == 0) set_status(p.status, i, DSP_ERR_NONFINITE);
}

}  // namespace dsp
