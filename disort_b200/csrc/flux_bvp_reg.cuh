// flux_bvp_reg.cuh — boundary-value problem and fluxes for N <= 16 with the
// elimination panel held in registers (one panel row per thread).
//
// Same algorithm as flux_bvp_tile.cuh (the staircase form of the LINPACK band LU,
// setMatrix/solve0/computeFluxes of FluxSolver.cpp:838-1287), mapped so that
// the sgbfa row operations are register FMAs:
//  - slot thread s holds its row's x_l columns as cur[N]; the row's x_{l+1}
//    columns and right-hand side go to shared memory once the layer's new rows
//    are in the panel, and carried rows take theirs back as cur between layers;
//  - the pivot of column c is an arg-max of |cur[c]| over candidate slots
//    (warp reductions of the bit patterns for a full-warp team, shuffles
//    otherwise); only the pivot row and its negated reciprocal are broadcast
//    through shared memory;
//  - free slots (last layer's pivot rows) receive the new continuity rows in
//    slot order, each thread finding its row index by a popcount;
//  - a pivot step updates the x_l columns only (the multipliers replace the
//    pivot column's entries); the x_{l+1} columns and the right-hand side of
//    the panel follow after the layer's N steps, one lane per column: a unit
//    lower-triangular solve for the pivot rows, then the carried rows, each
//    element with the same FMA sequence as inside the steps;
//  - the N pivot rows of a layer, [U | V | c] with U x_l + V x_{l+1} = c, go
//    to the layer's elimination record as they are; going back up, x_l is the
//    solution of U x_l = c - V x_{l+1}, a 16-step triangular solve across the
//    lanes (one row each) instead of a back substitution over N + 1 columns on
//    the way down;
//  - the layer records (and, going back up, the elimination records) are
//    brought into a shared-memory ring with cp.async one layer ahead of their
//    use, so the work on a layer hides the memory latency of the next one.
#pragma once

#include "dsp_device.cuh"

namespace dsp {

#ifndef DSP_BVP_REGS
#define DSP_BVP_REGS 128
#endif

// record element read (records are staged in shared memory)
__device__ __forceinline__ double ld_rec(const double* q) { return *q; }

template <int N>
struct RCfg {
  static constexpr int NN = N / 2;
  static constexpr int PR = 3 * NN;
  static constexpr int TEAM = pow2ceil(PR) < 8 ? 8 : pow2ceil(PR);
  static constexpr int CTA = TEAM >= 32 ? TEAM : 32;
  static constexpr int TPC = CTA / TEAM;
  // team shared memory (doubles)
  static constexpr int BL = N + 2;                 // pivot-step buffer: cur[c+1..N-1] | rhs | -1/pivot
  static constexpr int O_BUF = 0;                  // 2 x pivot-step buffer
  static constexpr int O_XV = O_BUF + 2 * BL;      // x ping-pong [2][N]
  static constexpr int O_EC = O_XV + 2 * N;    // [N]
  static constexpr int O_I = O_EC + N;         // intensities [N]
  static constexpr int O_E = O_I + N;          // exp(eig*dtau) of layers l, l+1 [2][NN]
  static constexpr int O_MISC = O_E + 2 * NN;  // 8
  static constexpr int O_PIV = O_MISC + 8;     // int pivot slot per column [N]
  // record ring: 3 layer records going down; 2 x (layer record + W record) going up
  static constexpr int RS = lrec_stride(N);
  static constexpr int BS = brec_stride(N);
  static constexpr int RL = 2 * N + 2;  // record row: U[N] | V[N] | c | 1/pivot
  // A layer record in the ring keeps its layout except that the rows of G are
  // GS doubles apart: GS = 2 mod 4 (and even, for the 16-byte copies), so that
  // lanes reading one row each of G hit different shared-memory banks (row
  // stride N would put them all on one bank).
  static constexpr int GS = (N + 2) % 4 == 2 ? N + 2 : N + 4;
  static constexpr int SEIG = N * GS, SZB = SEIG + N, SZ0 = SZB + N, SZ1 = SZ0 + N, SXR = SZ1 + N;
  static constexpr int RSP = round4(SXR + 2);
  static_assert(RS - N * N == round4(N * N + 4 * N + 2) - N * N, "layer record: G then eig, zb, z0, z1, xr");
  static constexpr int O_RING = round4(O_PIV + N / 2 + 1);
  // Going down: 3 layer records, then the panel rows' right-hand blocks
  // [x_{l+1} columns | rhs] by slot (PR rows of R0S doubles, odd so that a lane
  // per row writing one column spreads over the banks); the multipliers of the
  // layer's pivot steps go to the free slot of the layer's own record (packed:
  // pivot row k's k multipliers at k(k-1)/2, carried row r's N at N(N-1)/2 + rN).
  // Going up: 2 layer records and 1 elimination record.
  static constexpr int R0S = N + 1;
  static constexpr int O_R0 = 3 * RSP;
  static constexpr int ML_CARRIED = N * (N - 1) / 2;
  static_assert(ML_CARRIED + (PR - N) * N <= RSP, "multipliers fit a layer record's ring slot");
  static constexpr int RING = imax(3 * RSP + PR * R0S, 2 * RSP + BS);
  static constexpr int TEAM_SMEM = round4(O_RING + RING);
  static constexpr int TAB = 2 * N;  // mu and wt of the constant tables
  // register budget per thread: 128 keeps 16 single-warp CTAs resident per SM
  static constexpr int MINB = 65536 / (CTA * DSP_BVP_REGS);
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(TAB + TPC * TEAM_SMEM); }
  // 16 resident CTAs (one per warp of the register budget) fit 228 KB with 1 KB reserved each
  static_assert(N != 16 || 16 * (smem_bytes() + 1024) <= 228 * 1024, "16 CTAs per SM at 16 streams");
};

// One instance (chunk slot `slot`) on this thread's team; the CTA's constant
// tables are in shared memory already.
template <int N, bool GEN, bool JAC, bool SPH>
__device__ __forceinline__ void bvp_reg_instance(const FluxParams& p, const int slot) {
  using C = RCfg<N>;
  constexpr int NN = C::NN, TEAM = C::TEAM, PR = C::PR;
  constexpr double PI = 3.14159265358979323846;
  static_assert(PR <= 32 && TEAM <= 32, "register panel needs one warp");
  extern __shared__ double smem[];
  const double* mu = smem + tab_mu(N);
  const double* wt = smem + tab_wt(N);

  const int team = threadIdx.x / TEAM, t = threadIdx.x % TEAM;
  const unsigned msk = team_mask<TEAM>();
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
  const int m = GEN ? p.g.m : 0;
  auto oidx = [&](int lev) {
    if constexpr (GEN) return (long long)i * p.g.ntau_out + (ifb ? NT - 1 - lev : lev);
    else return (long long)i * NT + (ifb ? L - lev : lev);
  };
  double* const* outp = GEN ? p.g.out_flux : p.out;
  const int st0 = p.status ? p.status[i] : 0;
  if (st0 == DSP_ERR_INVALID_INPUT || st0 == DSP_ERR_EIGEN) {
    const double qnan = __longlong_as_double(0x7ff8000000000000ll);
    if (m == 0)
      for (int lev = t; lev < NT; lev += TEAM)
        for (int f = 0; f < 8; ++f) outp[f][oidx(lev)] = qnan;
    return;
  }
  if constexpr (GEN) {
    if (m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  }
  DSP_PHASE_BEGIN
  const int ncut = (int)rec[H_NCUT];
  const bool lyrcut = rec[H_LYRCUT] != 0.0;
  // modes m > 0 carry the beam only: no thermal or isotropic sources and no
  // Lambertian coupling (DisortSolver.cpp:1246-1250, 1693-1748)
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0 && m == 0;
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double fbeam = rec[H_FBEAM], umu0 = rec[H_UMU0];
  const double alb = m == 0 ? rec[H_ALB] : 0.0;
  // bidirectional surface (general solver): this mode's table, row r =
  // [beam | diffuse streams | emissivity]; it couples at every mode
  const double* sft = nullptr;
  if constexpr (GEN)
    if (p.g.brdf) sft = p.g.brdf + (long long)slot * brdf_stride(N, p.g.numu);
  const double fisot = m == 0 ? rec[H_FISOT] : 0.0, ptop = m == 0 ? rec[H_PTOP] : 0.0;
  const double fisob = m == 0 ? rec[H_FISOB] : 0.0, pbot = m == 0 ? rec[H_PBOT] : 0.0;
  const double pbotd = m == 0 ? rec[H_PBOTD] : 0.0;
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
  auto zsph = [&](const double* lrl, int l, int iq, double tau) {
    const double* sr = SR(l);
    return exp(-sr[sph_xba(N)] * tau) * (ld_rec(lrl + C::SZB + iq) + sr[iq] * tau);
  };

  double* sm = smem + C::TAB + team * C::TEAM_SMEM;
  double* bufs = sm + C::O_BUF;
  double* XV = sm + C::O_XV;
  double* ec = sm + C::O_EC;
  double* Iv = sm + C::O_I;
  double* E = sm + C::O_E;
  int* pivslot = reinterpret_cast<int*>(sm + C::O_PIV);
  constexpr int RS = C::RS, BS = C::BS;
  double* ring = sm + C::O_RING;
  constexpr int RSP = C::RSP, GS = C::GS;
  auto RF = [&](int l) { return ring + (l % 3) * RSP; };  // going down: layer l's record
  auto RB = [&](int l) { return ring + (l & 1) * RSP; };  // going up: layer records
  double* const EB = ring + 2 * RSP;                      // going up: the elimination record
  // a layer record into a ring slot, G's rows GS apart
  auto copy_lrec = [&](double* dst, const double* src) {
    team_copy_rows_async<TEAM>(dst, GS, src, N, N, N, t);
    team_copy_async<TEAM>(dst + C::SEIG, src + N * N, RS - N * N, t);
  };

  double cur[N], nxt[N], rhs = 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) { cur[k] = 0.0; nxt[k] = 0.0; }
  bool singular = false;

  // ------------------------------------------------------------------ forward
  copy_lrec(RF(0), LR(0));
  cp_async_commit();
  if (ncut > 1) copy_lrec(RF(1), LR(1));
  cp_async_commit();
  cp_async_wait<1>();
  __syncwarp(msk);
  if (t < NN) E[t] = exp(RF(0)[C::SEIG + t] * dtau_s[0]);
  __syncwarp(msk);
  // top boundary rows in slots 0..NN-1 (setMatrix :890-907, solve0 :978-990)
  if (t < NN) {
    const double* l0 = RF(0);
    const int jq = NN - 1 - t;
#pragma unroll
    for (int iq = 0; iq < N; ++iq) {
      const double g = ld_rec(l0 + jq * GS + iq);
      cur[iq] = (iq < NN) ? g * E[iq] : g;
    }
    double s = 0.0;
    if (beam) s -= ld_rec(l0 + C::SZB + jq);
    if (thermal) s -= ld_rec(l0 + C::SZ0 + jq);
    s += fisot + ptop;
    rhs = s;
  }
  unsigned carried = (1u << NN) - 1u;  // slots holding carried (un-pivoted) rows

  double rdiag = 0.0;  // 1 / pivot of this thread's pivot row
  // per-layer scalars of the instance record, loaded one layer ahead
  double dts_n = ncut > 1 ? dtau_s[1] : 0.0, btr_n = btr[1], tau_n = taus[1];
  for (int l = 0; l < ncut; ++l) {
    const bool last = (l == ncut - 1);
    const double dts1 = dts_n, btr1 = btr_n, tau1 = tau_n;  // values at l + 1
    if (l + 2 <= ncut) {
      dts_n = (l + 2 < ncut) ? dtau_s[l + 2] : 0.0;
      btr_n = btr[l + 2];
      tau_n = taus[l + 2];
    }
    // record l+2 starts loading into the slot of record l-1; record l+1 is waited for
    if (l + 2 < ncut) copy_lrec(RF(l + 2), LR(l + 2));
    cp_async_commit();
    cp_async_wait<1>();
    __syncwarp(msk);
    const double* lr = RF(l);
    const double* Ecur = E + (l & 1) * NN;
    double* Enext = E + ((l & 1) ^ 1) * NN;
    if (!last && t < NN) Enext[t] = exp(RF(l + 1)[C::SEIG + t] * dts1);
    __syncwarp(msk);
    // new rows into the free slots, in slot order
    const unsigned freem = ((PR == 32) ? 0xffffffffu : ((1u << PR) - 1u)) & ~carried;
    const bool isfree = t < PR && ((freem >> t) & 1u);
    const int rank = __popc(freem & ((1u << t) - 1u));
    const int nnew = last ? NN : N;
    const bool fresh = isfree && rank < nnew;
    if (fresh) {
      if (!last) {
        // continuity row jq of interface (l, l+1) (setMatrix :852-887, solve0 :1080-1104)
        const int jq = rank;
        const double* ln = RF(l + 1);
        const double* Gl = lr + jq * GS;
        const double* Gn = ln + jq * GS;
#pragma unroll
        for (int iq = 0; iq < N; ++iq) {
          const double g = ld_rec(Gl + iq);
          cur[iq] = (iq < NN) ? g : g * Ecur[N - 1 - iq];
          const double h = ld_rec(Gn + iq);
          nxt[iq] = (iq < NN) ? -h * Enext[iq] : -h;
        }
        const double T = btr1, tau = tau1;
        double sum = 0.0;
        if (beam) {
          if constexpr (SPH) {
            sum += zsph(ln, l + 1, jq, tau);
            sum -= zsph(lr, l, jq, tau);
          } else {
            sum += ld_rec(ln + C::SZB + jq) * T;
            sum -= ld_rec(lr + C::SZB + jq) * T;
          }
        }
        if (thermal) {
          sum += ld_rec(ln + C::SZ0 + jq) - ld_rec(lr + C::SZ0 + jq);
          sum += (ld_rec(ln + C::SZ1 + jq) - ld_rec(lr + C::SZ1 + jq)) * tau;
        }
        rhs = sum;
      } else {
        // bottom boundary row (setMatrix :909-958, solve0 :993-1076)
        const int rb = rank, jq = NN + rb;
        const bool plain = lyrcut || dlbc;
        const double* Gl = lr;
        const double* srow = sft ? sft + rb * brdf_row(N) : nullptr;
        const double cpl = m == 0 ? 2.0 : 1.0;  // 1 + delta_m0
#pragma unroll
        for (int iq = 0; iq < N; ++iq) {
          double base = ld_rec(Gl + jq * GS + iq);
          if (!plain) {
            double refl = 0.0;
            if (srow)
              for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * srow[1 + k] * ld_rec(Gl + (NN - 1 - k) * GS + iq);
            else
              for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * alb * ld_rec(Gl + (NN - 1 - k) * GS + iq);
            base = base - cpl * refl;
          }
          cur[iq] = (iq < NN) ? base : base * Ecur[N - 1 - iq];
          nxt[iq] = 0.0;
        }
        const double T = btr1, tau = tau1;
        double sum = 0.0;
        if (dlbc) {
          if (beam) sum -= SPH ? zsph(lr, l, NN + rb, tau) : ld_rec(lr + C::SZB + NN + rb) * T;
          if (thermal) {
            sum -= ld_rec(lr + C::SZ0 + NN + rb);
            sum -= ld_rec(lr + C::SZ1 + NN + rb) * tau;
          }
          sum += pbot + mu[rb] * pbotd;
        } else {
          if (!lyrcut) {
            double refl = 0.0;
            for (int jj = 0; jj < NN; ++jj) {
              double ps = 0.0;
              if (beam) ps += SPH ? zsph(lr, l, NN - 1 - jj, tau) : ld_rec(lr + C::SZB + NN - 1 - jj) * T;
              if (thermal) ps += ld_rec(lr + C::SZ0 + NN - 1 - jj) + ld_rec(lr + C::SZ1 + NN - 1 - jj) * tau;
              refl += wt[jj] * mu[jj] * (srow ? srow[1 + jj] : alb) * ps;
            }
            sum += cpl * refl;
          }
          if (beam) {
            sum -= SPH ? zsph(lr, l, NN + rb, tau) : ld_rec(lr + C::SZB + NN + rb) * T;
            if (!lyrcut) sum += (srow ? srow[0] : alb) * umu0 * fbeam * T / PI;
          }
          if (thermal) {
            sum -= ld_rec(lr + C::SZ0 + NN + rb);
            sum -= ld_rec(lr + C::SZ1 + NN + rb) * tau;
          }
          sum += fisob;
          if (thermal) sum += (srow ? srow[NN + 1] : 1.0 - alb) * pbot;
        }
        rhs = sum;
      }
    }
    // slots receiving a new row: this team's bits of the ballot of `fresh`
    const unsigned newm = (__ballot_sync(msk, fresh) >> (threadIdx.x & 31u & ~(unsigned)(TEAM - 1))) &
                          (TEAM == 32 ? 0xffffffffu : ((1u << TEAM) - 1u));
    unsigned cand = carried | newm;
    // the panel rows' right-hand blocks [x_{l+1} columns | rhs] wait in shared
    // memory for the column phase (carried rows have no x_{l+1} entries)
    double* R0 = ring + C::O_R0;
    if (!last && t < PR) {
#pragma unroll
      for (int j = 0; j < N; ++j) R0[t * C::R0S + j] = fresh ? nxt[j] : 0.0;
      R0[t * C::R0S + N] = rhs;
    }
    DSP_PHASE(20)

    // ---- eliminate the N columns of x_l (sgbfa steps) ----------------------
    // Each pivot step updates the x_l columns only; the multiplier of every
    // candidate row replaces its entry in the pivot column (LINPACK keeps L
    // there too).  The x_{l+1} columns and the right-hand side are brought up to
    // date afterwards, column by column (below), with the same FMA sequence per
    // element as the row operations of the steps; the last layer, with no
    // x_{l+1} columns, updates its right-hand side within the steps.
    int myc = -1;  // pivot column of this thread's row, if it becomes a pivot row
    // temperature Jacobian: this layer's multipliers and pivot slots
    double* const jrow = !JAC ? nullptr
        : p.jac_rec + ((GEN ? (long long)p.g.lay_off[slot] : (long long)i * L) + l) * jrec_stride(N);
#pragma unroll
    for (int c = 0; c < N; ++c) {
      const bool isc = t < PR && ((cand >> t) & 1u);
      // every lane's reciprocal, branch-free, issued alongside the search: the
      // pivot lane's is ready when the search ends
      const double rc = -rcp_newton(cur[c]);
      double a = fabs(cur[c]);
      if (isnan(a)) a = __longlong_as_double(0x7ff0000000000000ll);  // NaN ranks as +inf: one total order
      int idx;
      bool zero_piv;
      if constexpr (TEAM == 32) {
        idx = warp_argmax_nonneg(a, isc, zero_piv);
      } else {
        double v = isc ? a : -1.0;
        idx = isc ? t : PR;
        team_argmax<TEAM>(v, idx, nullptr);
        zero_piv = v == 0.0;
      }
      DSP_PHASE(27)
      const int ps = idx < PR ? idx : 0;
      cand &= ~(1u << ps);
      if (t == ps) myc = c;
      if (t == 0) pivslot[c] = ps;
      if (idx >= PR || zero_piv) {  // LINPACK skips a zero pivot column (BandSolver.hpp:76-78)
        singular = true;
        if constexpr (JAC) {
          if (t < PR) jrow[c * PR + t] = 0.0;
          if (t == 0) jrow[N * PR + c] = (double)ps;
        }
        continue;
      }
      double* buf = bufs + (c & 1) * C::BL;  // alternate buffers: no barrier after the update
      if (t == ps) {
        rdiag = -rc;
#pragma unroll
        for (int j = c + 1; j < N; ++j) buf[j] = cur[j];
        if (last) buf[N] = rhs;
        buf[N + 1] = rc;
      }
      __syncwarp(msk);
      const double tinv = buf[N + 1];
      const double* pv = buf;
      const double prhs = buf[N];
      DSP_PHASE(28)
      if constexpr (JAC) {
        if (t < PR) jrow[c * PR + t] = ((cand >> t) & 1u) ? cur[c] * tinv : 0.0;
        if (t == 0) jrow[N * PR + c] = (double)ps;
      }
      if ((cand >> t) & 1u) {
        const double m = cur[c] * tinv;
#pragma unroll
        for (int j = c + 1; j < N; ++j) cur[j] = fma(m, pv[j], cur[j]);
        cur[c] = m;
        if (last) rhs = fma(m, prhs, rhs);
      }
    }
    DSP_PHASE(21)

    if (JAC && last && myc >= 0) {
      // the Jacobian's upward solve also needs the last layer's pivot rows
      double* row = brec0 + (long long)l * BS + myc * C::RL;
#pragma unroll
      for (int j = 0; j < N; ++j) {
        row[j] = cur[j];
        row[N + j] = 0.0;
      }
      row[2 * N] = rhs;
      row[2 * N + 1] = rdiag;
    }
    if (!last) {
      // ---- the right-hand block [x_{l+1} columns | rhs] --------------------
      // Pivot row k (slot p_k): R_k = R0[p_k] + sum_{k' < k} m[p_k][k'] R_k', a
      // unit lower-triangular solve; carried row s: R0[s] + sum_k m[s][k] R_k.
      // One lane per column (N + 1 lanes), the panel rows' initial right-hand
      // blocks and multipliers in shared memory.
      double* ML = RF(l);  // the layer's record is used up
      double* brow = brec0 + (long long)l * BS;
      __syncwarp(msk);  // every read of the record's slot is done
      if (t < PR) {
        if (myc >= 0) {
          // pivot row of column myc: its multipliers, and [U | . | . | 1/pivot] of
          // the elimination record (row myc)
          double* mk = ML + myc * (myc - 1) / 2;
#pragma unroll
          for (int k = 0; k < N - 1; ++k)
            if (k < myc) mk[k] = cur[k];
          double* row = brow + myc * C::RL;
#pragma unroll
          for (int j = 0; j < N; j += 2) *reinterpret_cast<double2*>(row + j) = make_double2(cur[j], cur[j + 1]);
          row[2 * N + 1] = rdiag;
        } else {
          double* mk = ML + C::ML_CARRIED + __popc(cand & ((1u << t) - 1u)) * N;
#pragma unroll
          for (int k = 0; k < N; ++k) mk[k] = cur[k];
        }
      }
      __syncwarp(msk);
      DSP_PHASE(29)
      if (t <= N) {
        // A zero-pivot step left its candidates' multiplier slots at +-0, so
        // its terms add nothing: no test per term.
        double r[N];
#pragma unroll
        for (int k = 0; k < N; ++k) r[k] = R0[pivslot[k] * C::R0S + t];
        // right-looking: once R_kk is final it enters every later pivot row
        // (each row still takes its terms in step order)
#pragma unroll
        for (int kk = 0; kk < N - 1; ++kk)
#pragma unroll
          for (int k = kk + 1; k < N; ++k) r[k] = fma(ML[k * (k - 1) / 2 + kk], r[kk], r[k]);
        // V and c of the pivot rows (columns N + t of the record rows)
#pragma unroll
        for (int k = 0; k < N; ++k) brow[k * C::RL + N + t] = r[k];
        // the NN carried rows, CQ at a time interleaved
        constexpr int NC = PR - N, CQ = NC < 4 ? NC : 4;
        unsigned cm = cand;
#pragma unroll
        for (int q0 = 0; q0 < NC; q0 += CQ) {
          int sl[CQ];
          double acc[CQ];
#pragma unroll
          for (int q = 0; q < CQ; ++q) {
            if (q0 + q < NC) {  // the last group may be partial
              sl[q] = cm ? __ffs(cm) - 1 : 0;
              cm &= cm - 1u;
              acc[q] = R0[sl[q] * C::R0S + t];
            }
          }
#pragma unroll
          for (int k = 0; k < N; ++k)
#pragma unroll
            for (int q = 0; q < CQ; ++q)
              if (q0 + q < NC) acc[q] = fma(ML[C::ML_CARRIED + (q0 + q) * N + k], r[k], acc[q]);
#pragma unroll
          for (int q = 0; q < CQ; ++q)
            if (q0 + q < NC) R0[sl[q] * C::R0S + t] = acc[q];
        }
      }
      __syncwarp(msk);
      // carried rows become the next layer's current block; the other lanes'
      // rows are replaced or unused, so cur is not live across the column phase
      {
        const bool keep = t < PR && ((cand >> t) & 1u);
        const double* rr = R0 + (keep ? t : 0) * C::R0S;
#pragma unroll
        for (int k = 0; k < N; ++k) {
          const double v = rr[k];
          cur[k] = keep ? v : 0.0;
        }
        rhs = keep ? rr[N] : 0.0;
      }
      carried = cand;
      __syncwarp(msk);
    } else {
      // x_{ncut-1} = U^{-1} rhs (sgbsl back substitution)
      double* x = XV + (l & 1) * N;
#pragma unroll
      for (int c = N - 1; c >= 0; --c) {
        if (myc == c) {
          const double xv = rhs / cur[c];
          rhs = xv;
          x[c] = xv;
        }
        __syncwarp(msk);
        if (myc >= 0 && myc < c) rhs -= cur[c] * x[c];
      }
      __syncwarp(msk);
    }
    DSP_PHASE(22)
  }
  if (singular && t == 0) set_status(p.status, i, DSP_ERR_SINGULAR);
  cp_async_wait<0>();
  __syncwarp(msk);

  // ----------------------------------------------------------------- backward
  bool nonfinite = false;
  const double rumu0 = beam ? 1.0 / umu0 : 0.0;
  auto ssa_of = [&](int l) {
    const int lin = ifb ? L - 1 - l : l;
    return GEN ? p.g.ssa[p.g.in_off[i] + lin] : p.ssa(i, lin);
  };
  // fluxes at output level lu of layer l (computeFluxes, FluxSolver.cpp:1138-1287;
  // DisortSolver.cpp:1980-2124): utaupr scaled depth, utau unscaled depth
  // tau_top, tau_bot: scaled depths of the layer's top and bottom; w0: its
  // single-scattering albedo (loaded ahead by the caller)
  auto eval_level = [&](int l, const double* x, int lu, double utaupr, double utau, double tau_top,
                        double tau_bot, double w0) {
    const double* lr = RB(l);
    const double* eig = lr + C::SEIG;
    const double* Gl = lr;
    if (t < N) {
      const double d = (t < NN) ? (utaupr - tau_bot) : (utaupr - tau_top);
      ec[t] = x[t] * exp(-eig[t] * d);
    }
    __syncwarp(msk);
    // pseudo-spherical: the Chapman factor of the layer replaces mu0
    // (computeFluxes, FluxSolver.cpp:1184-1188, 1216-1219)
    const double ch = SPH && beam ? SR(l)[sph_ch(N)] : 0.0;
    const double fact = beam ? (SPH ? exp(-utaupr / ch) : exp(-utaupr * rumu0)) : 0.0;
    double s = 0.0;
    if (t < N) {
#pragma unroll
      for (int j = 0; j < N; ++j) s += ld_rec(Gl + t * GS + j) * ec[j];
      if (beam) s += SPH ? zsph(lr, l, t, utaupr) : ld_rec(lr + C::SZB + t) * fact;
      if (thermal) s += ld_rec(lr + C::SZ0 + t) + ld_rec(lr + C::SZ1 + t) * utaupr;
    }
    // the quadrature sums over the streams' intensities: at 16 streams as
    // reductions over lanes 0-7 (downward streams) and 8-15 (upward), else by
    // lane 0 from shared memory
    double ua = 0.0, uad = 0.0, uau = 0.0, fldn = 0.0, fup = 0.0;
    if constexpr (TEAM == 32 && NN == 8) {
      const int cw = t < NN ? NN - t - 1 : t - NN;
      double a = t < N ? wt[cw < NN ? cw : 0] * s : 0.0;
      double b = t < N ? a * mu[cw < NN ? cw : 0] : 0.0;
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) {
        a += __shfl_xor_sync(msk, a, off);
        b += __shfl_xor_sync(msk, b, off);
      }
      const double a8 = __shfl_sync(msk, a, 8), b8 = __shfl_sync(msk, b, 8);
      uad = a;
      fldn = b;
      uau = a8;
      fup = b8;
      ua = uad + uau;
    } else {
      if (t < N) Iv[t] = s;
      __syncwarp(msk);
      if (t == 0) {
        double iv[N];
#pragma unroll
        for (int k = 0; k < N; ++k) iv[k] = Iv[k];
#pragma unroll
        for (int iq = 0; iq < NN; ++iq) {
          const int cw = NN - iq - 1;
          ua += wt[cw] * iv[iq];
          uad += wt[cw] * iv[iq];
          fldn += wt[cw] * iv[iq] * mu[cw];
        }
#pragma unroll
        for (int iq = NN; iq < N; ++iq) {
          const int cw = iq - NN;
          ua += wt[cw] * iv[iq];
          uau += wt[cw] * iv[iq];
          fup += wt[cw] * iv[iq] * mu[cw];
        }
      }
    }
    if (t == 0) {
      double dirint = 0.0, fldir = 0.0, fdir = 0.0;
      if (beam) {
        dirint = fbeam * fact;
        fldir = umu0 * fbeam * fact;
        fdir = SPH ? fabs(umu0) * fbeam * exp(-utau / ch) : umu0 * fbeam * exp(-utau * rumu0);
      }
      fup *= 2.0 * PI;
      fldn *= 2.0 * PI;
      const double fdn = (fldn + fldir) - fdir;
      constexpr double R4PI = 1.0 / (4.0 * PI);
      ua = (2.0 * PI * ua + dirint) * R4PI;
      const double uaso = dirint * R4PI;
      uad = (2.0 * PI * uad) * R4PI;
      uau = (2.0 * PI * uau) * R4PI;
      double plsorc = 0.0;
      if (thermal) plsorc = lr[C::SXR] + lr[C::SXR + 1] * utaupr;
      const double dfdt = (1.0 - w0) * 4.0 * PI * (ua - plsorc);
      const double o[8] = {fdir, fdn, fup, dfdt, ua, uad, uau, uaso};
#pragma unroll
      for (int f = 0; f < 8; ++f) {
        outp[f][oidx(lu)] = o[f];
        if (!isfinite(o[f])) nonfinite = true;
      }
    }
    __syncwarp(msk);
  };
  const double* utau_l = GEN ? rec + GenLayout::make(L, N, NT).utau : nullptr;
  const double* utaus_l = GEN ? rec + GenLayout::make(L, N, NT).utaus : nullptr;
  const double* lyr_l = GEN ? rec + GenLayout::make(L, N, NT).lyr : nullptr;
  if constexpr (!GEN) {
    for (int lev = ncut + 1 + t; lev <= L; lev += TEAM)
      for (int f = 0; f < 8; ++f) p.out[f][oidx(lev)] = 0.0;
  } else {
    // levels below the absorption cut stay zero (DisortSolver.cpp:1998-2009)
    if (m == 0)
      for (int lu = t; lu < NT; lu += TEAM)
        if ((int)lyr_l[lu] > ncut - 1)
          for (int f = 0; f < 8; ++f) outp[f][oidx(lu)] = 0.0;
  }
  copy_lrec(RB(ncut - 1), LR(ncut - 1));
  cp_async_commit();
  // per-layer scalars of layer l, loaded one layer ahead
  double tau_top = taus[ncut - 1], tau_bot = taus[ncut], tauc_bot = GEN ? 0.0 : rec[il.tauc + ncut];
  double w0 = ssa_of(ncut - 1);
  for (int l = ncut - 1; l >= 0; --l) {
    const double tau_top_n = l > 0 ? taus[l - 1] : 0.0, w0_n = l > 0 ? ssa_of(l - 1) : 0.0;
    const double tauc_top = GEN ? 0.0 : rec[il.tauc + l];
    cp_async_wait<0>();
    __syncwarp(msk);
    DSP_PHASE(24)
    double* x = XV + (l & 1) * N;
    if (l < ncut - 1) {
      // U x_l = c - V x_{l+1}: lane t holds row t; column c's unknown is
      // formed by lane c and broadcast, the rows above it are updated
      const double* xn = XV + ((l & 1) ^ 1) * N;
      const double* row = EB + (t < N ? t : 0) * C::RL;
      double r = 0.0, rd = 0.0;
      if (t < N) {
        r = row[2 * N];
#pragma unroll
        for (int n = 0; n < N; ++n) r -= row[N + n] * xn[n];
        rd = row[2 * N + 1];
      }
#pragma unroll
      for (int c = N - 1; c >= 0; --c) {
        const double xc = __shfl_sync(msk, r * rd, c, TEAM);
        if (t == c) x[c] = xc;
        if (t < c) r -= row[c] * xc;
      }
      __syncwarp(msk);
    }
    DSP_PHASE(25)
    // the records of layer l-1 start loading (the elimination record is used
    // up; the layer-record slot held layer l+1)
    if (l > 0) {
      copy_lrec(RB(l - 1), LR(l - 1));
      team_copy_async<TEAM>(EB, brec0 + (long long)(l - 1) * BS, BS, t);
    }
    cp_async_commit();
    DSP_PHASE(26)
    if constexpr (GEN) {
      if (t < N) cc0[(long long)l * N + t] = x[t];
      if (m == 0)
        for (int lu = 0; lu < NT; ++lu)
          if ((int)lyr_l[lu] == l) eval_level(l, x, lu, utaus_l[lu], utau_l[lu], tau_top, tau_bot, w0);
    } else {
      eval_level(l, x, l + 1, tau_bot, tauc_bot, tau_top, tau_bot, w0);
      if (l == 0) eval_level(0, x, 0, tau_top, tauc_top, tau_top, tau_bot, w0);
    }
    tau_bot = tau_top;
    tau_top = tau_top_n;
    tauc_bot = tauc_top;
    w0 = w0_n;
    DSP_PHASE(23)
  }
  DSP_PHASE_END
  if (nonfinite && t == 0) set_status(p.status, i, DSP_ERR_NONFINITE);
}

// One team (a warp or part of one) per instance, in chunk-slot order.
template <int N, bool GEN = false, bool JAC = false, bool SPH = false>
__global__ void __launch_bounds__(RCfg<N>::CTA, RCfg<N>::MINB) flux_bvp_reg_kernel(FluxParams p) {
  using C = RCfg<N>;
  extern __shared__ double smem[];
  for (int k = threadIdx.x; k < C::TAB; k += blockDim.x) smem[k] = p.tables[k];
  __syncthreads();
  const int slot = blockIdx.x * C::TPC + threadIdx.x / C::TEAM;
  if (slot >= p.n) return;
  bvp_reg_instance<N, GEN, JAC, SPH>(p, slot);
}

// Persistent form (general solver): a resident grid whose teams take chunk
// slots from a work queue -- `order`, the chunk's slots by descending layer
// count (the size classes), consumed through the counter `head` -- so that
// the longest instances start first and the tail of the launch is short.
template <int N, bool JAC = false, bool SPH = false>
__global__ void __launch_bounds__(RCfg<N>::CTA, RCfg<N>::MINB)
    gen_bvp_reg_persistent_kernel(FluxParams p, const int* order, int* head) {
  using C = RCfg<N>;
  constexpr int TEAM = C::TEAM;
  extern __shared__ double smem[];
  for (int k = threadIdx.x; k < C::TAB; k += blockDim.x) smem[k] = p.tables[k];
  __syncthreads();
  const int t = threadIdx.x % TEAM;
  const unsigned msk = team_mask<TEAM>();
  for (;;) {
    int k = 0;
    if (t == 0) k = atomicAdd(head, 1);
    k = __shfl_sync(msk, k, 0, TEAM);
    if (k >= p.n) break;
    bvp_reg_instance<N, true, JAC, SPH>(p, order[k]);
    __syncwarp(msk);  // the team's shared memory serves the next instance
  }
}

}  // namespace dsp
