// flux_jac.cuh — temperature Jacobians of the flux path (compute_temperature_jacobian).
//
// Replaces computeThermalJacobian (FluxSolver.cpp:1294-1497) and the derivative
// sources of computeIsotropicSource (:786-829).  The reference solves
// A dC = dB_k with the band LU that solve0 left, for every level-Planck degree
// of freedom k = 0..L and the surface, then propagates dC through the flux
// formulas and chains with dB/dT.
//
// Here the boundary-value kernels, in their Jacobian form, record the
// elimination itself: per layer and pivot column the multiplier applied to
// every panel slot and the pivot slot (jrec_stride), next to the pivot rows
// [U | V | c] they always keep.  flux_jac_kernel replays that elimination on
// the L + 2 right-hand sides of the Jacobian, one CTA per instance and one
// thread per degree of freedom:
//  - going down, each thread keeps the right-hand side value of every panel
//    slot of its column in shared memory; new rows enter the free slots in slot
//    order exactly as in the elimination, pivot rows leave with their value
//    (row c's right-hand side, stored per layer), and every pivot adds
//    multiplier x pivot value to the other slots;
//  - going up, U_l x_l = c_l - V_l x_{l+1} per column, and at each level the
//    six outputs of the column (homogeneous part G (x o e) plus the derivative
//    of the thermal particular solution), times dB/dT of its temperature.
// The derivative sources come from the layer stage's P and Q (jpq_stride):
// Z1 = xr1 P / 2 and Z0 = (xr0 P +/- xr1 Q) / 2, so a layer's source derivative
// with respect to its top / bottom level Planck value is P, Q weighted by the
// derivatives of its intercept xr0 and slope xr1 (FluxSolver.cpp:789-806).
#pragma once

#include "dsp_device.cuh"
#include "flux_setup.cuh"

namespace dsp {

// planckFunctionDeriv2 (Planck.cpp:171-214): dB/dT, with the closed form of the
// derivative of the band integral, 4 B / T minus the boundary terms of the
// integration limits, and the single-wavenumber form when lo == hi.
static __device__ double planck_deriv2(double lo, double hi, double T, const PlanckConsts& pk) {
  constexpr double C2 = 1.438786;
  if (T < 0.0 || hi < lo || lo < 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  if (T < 1.e-4) return 0.0;
  auto fk = [](double v) {  // v^3 / (e^v - 1), v^2 near 0
    if (v < 1.e-6) return v * v;
    const double em = exp(-v);
    return v * v * v * em / (1.0 - em);
  };
  if (hi == lo) {
    const double x = C2 * hi / T;
    const double em = exp(-x);
    const double b = pk.c1 * hi * hi * hi * em / (1.0 - em);
    return b * (x / T) / (1.0 - em);
  }
  const double v0 = C2 * lo / T, v1 = C2 * hi / T;
  const double B = planck2(lo, hi, T, pk);
  const double boundary = pk.sigdpi * pk.conc * T * T * T * (v1 * fk(v1) - v0 * fk(v0));
  return 4.0 * B / T - boundary;
}

template <int N>
struct JCfg {
  static constexpr int NN = N / 2;
  static constexpr int PR = 3 * NN;  // panel slots
  static constexpr int KB = 64;      // degrees of freedom per pass (threads per CTA)
  // shared memory (doubles): slot values [PR][KB] going down, x_l and x_{l+1}
  // [2][N][KB] going up (the same area), exp factors of one level [N]
  static constexpr int O_R = 0;
  static constexpr int R_SIZE = (PR > 2 * N ? PR : 2 * N) * KB;
  static constexpr int O_EX = O_R + R_SIZE;
  static constexpr int O_TAB = O_EX + N;  // mu[N], wt[N]
  static constexpr int SMEM = O_TAB + 2 * N;
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)SMEM; }
  static constexpr int NW = (PR + 31) / 32;
};

// GEN: the general path (mode 0 of a ragged chunk): outputs at the instance's
// output depths (user optical depths or the levels), rows of ndof_out columns.
template <int N, bool GEN = false>
__global__ void __launch_bounds__(64) flux_jac_kernel(FluxParams p, JacView jv) {
  using C = JCfg<N>;
  constexpr int NN = C::NN, PR = C::PR, KB = C::KB, NW = C::NW;
  constexpr double PI = 3.14159265358979323846;
  extern __shared__ double smem[];
  double* Rv = smem + C::O_R;
  double* ex = smem + C::O_EX;
  double* mu = smem + C::O_TAB;
  double* wt = smem + C::O_TAB + N;
  const int tid = threadIdx.x;
  for (int k = tid; k < 2 * N; k += KB) smem[C::O_TAB + k] = p.tables[k];  // tab_mu, tab_wt
  __syncthreads();
  const int slot = blockIdx.x;  // chunk-local instance
  if (slot >= p.n) return;
  // i: batch index; L: layers; NT: output depths; cvs: column stride of cv
  int i, L, NT;
  const double *rec, *lrec0, *brec0, *jrec0, *pq0;
  double* cv0;
  InstLayout il_gen;
  long long lstride;
  const int cvs = jv.ndof;
  if constexpr (GEN) {
    i = p.g.ids[slot];
    L = p.g.Ls[i];
    NT = p.g.user_tau ? p.g.user_tau : L + 1;
    il_gen = InstLayout::make(L, N);
    rec = p.inst_rec + p.g.inst_off[slot];
    const long long l0 = p.g.lay_off[slot];
    lstride = p.g.lstride;
    lrec0 = p.layer_rec + l0 * lstride;
    brec0 = p.bvp_rec + l0 * brec_stride(N);
    jrec0 = p.jac_rec + l0 * jrec_stride(N);
    pq0 = p.jac_pq + l0 * jpq_stride(N);
    cv0 = jv.cv + l0 * N * cvs;
  } else {
    i = slot;
    L = p.L;
    NT = L + 1;
    rec = p.inst_rec + (long long)i * p.il.stride;
    lstride = lrec_stride(N);
    lrec0 = p.layer_rec + (long long)i * L * lstride;
    brec0 = p.bvp_rec + (long long)i * L * brec_stride(N);
    jrec0 = p.jac_rec + (long long)i * L * jrec_stride(N);
    pq0 = p.jac_pq + (long long)i * L * jpq_stride(N);
    cv0 = jv.cv + (long long)i * L * N * cvs;
  }
  const InstLayout& il = GEN ? il_gen : p.il;
  const int ndof = L + 2;
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  auto store = [&](int f, int lu, int k, double v) {
    const int row = ifb ? NT - 1 - lu : lu;
    const int col = (ifb && k <= L) ? L - k : k;
    if constexpr (GEN) jv.out[f][((long long)i * p.g.ntau_out + row) * jv.ndof_out + col] = v;
    else jv.out[f][((long long)i * NT + row) * ndof + col] = v;
  };
  const int st = p.status ? p.status[i] : 0;
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0;
  if (st == DSP_ERR_INVALID_INPUT || st == DSP_ERR_EIGEN || !thermal) {
    // invalid instances: NaN like their fluxes; no thermal emission: zero
    const double v = thermal ? __longlong_as_double(0x7ff8000000000000ll) : 0.0;
    for (long long e = tid; e < (long long)NT * ndof; e += KB) {
      const int lu = (int)(e / ndof), k = (int)(e % ndof);
      for (int f = 0; f < 6; ++f) store(f, lu, k, v);
    }
    return;
  }
  const double* taus = rec + il.tau_s;
  const double* dtau_s = rec + il.dtau_s;
  // output depth lu: its layer and scaled depth (general path: the user depths)
  const GenLayout gl_ = GenLayout::make(L, N, NT);
  auto out_layer = [&](int lu) { return GEN ? (int)rec[gl_.lyr + lu] : (lu == 0 ? 0 : lu - 1); };
  auto out_taus = [&](int lu) { return GEN ? rec[gl_.utaus + lu] : taus[lu]; };
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double alb = rec[H_ALB];
  // bidirectional surface (general solver): mode 0's table, row r =
  // [beam | diffuse streams | emissivity]
  const double* sft = nullptr;
  if constexpr (GEN)
    if (p.g.brdf) sft = p.g.brdf + (long long)blockIdx.x * brdf_stride(N, p.g.numu);
  const double wlo = p.wlo(i), whi = p.whi(i);
  const double* temp_in = GEN ? p.g.temp + p.g.in_off[i] + i : p.temp.row(i);
  const double dtau_last = dtau_s[L - 1];
  // row width and 1/pivot position of the elimination record (flux_bvp_reg /
  // flux_bvp_tile layouts)
  constexpr int RL = N <= 16 ? 2 * N + 2 : 2 * N + 1;
  auto rdiag = [&](const double* br, int c) { return N <= 16 ? br[c * RL + 2 * N + 1] : br[N * RL + c]; };

  for (int k0 = 0; k0 < ndof; k0 += KB) {
    const int k = k0 + tid;
    const bool act = k < ndof;
    // derivative coefficients of layer lc's intercept (a0) and slope (a1) with
    // respect to degree of freedom k (FluxSolver.cpp:792-800)
    auto coef = [&](int lc, double& a0, double& a1) {
      a0 = 0.0;
      a1 = 0.0;
      if (k != lc && k != lc + 1) return;
      const double dts = dtau_s[lc], tc = taus[lc];
      double d1t = 0.0, d1b = 0.0;
      if (dts > 1e-4) {
        d1t = -1.0 / dts;
        d1b = 1.0 / dts;
      }
      if (k == lc) {
        a0 += 1.0 - d1t * tc;
        a1 += d1t;
      }
      if (k == lc + 1) {
        a0 += -d1b * tc;
        a1 += d1b;
      }
    };
    // derivative of the thermal source of layer lc at stream iq: z0 and z1 parts
    auto dz = [&](int lc, int iq, double a0, double a1, double& d0, double& d1) {
      if (a0 == 0.0 && a1 == 0.0) {
        d0 = 0.0;
        d1 = 0.0;
        return;
      }
      const double* pq = pq0 + (long long)lc * jpq_stride(N);
      const bool upper = iq >= NN;
      const int r = upper ? iq - NN : NN - 1 - iq;
      const double P = pq[r], Q = pq[NN + r];
      d1 = 0.5 * (a1 * P);
      d0 = upper ? 0.5 * (a0 * P + a1 * Q) : 0.5 * (a0 * P - a1 * Q);
    };

    // ---- down: replay the elimination on this column's right-hand side ----
    double* R = Rv + tid;  // slot s at R[s * KB]
    for (int s = 0; s < PR; ++s) R[s * KB] = 0.0;
    uint32_t carried[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) carried[w] = 0u;
    for (int s = 0; s < NN; ++s) carried[s >> 5] |= 1u << (s & 31);
    {
      // top boundary rows, slot s = row NN-1-s of the source (solve0 :978-990)
      double a0, a1;
      coef(0, a0, a1);
      for (int s = 0; s < NN; ++s) {
        double d0, d1;
        dz(0, NN - 1 - s, a0, a1, d0, d1);
        R[s * KB] = -d0;
      }
    }
    for (int l = 0; l < L; ++l) {
      const bool last = l == L - 1;
      const int nnew = last ? NN : N;
      double b0, b1, n0 = 0.0, n1 = 0.0;
      coef(l, b0, b1);
      if (!last) coef(l + 1, n0, n1);
      uint32_t cand[NW];
      int rank = 0;
      for (int s = 0; s < PR; ++s) {
        const bool isc = (carried[s >> 5] >> (s & 31)) & 1u;
        if (isc || rank >= nnew) continue;
        // new row `rank` in slot s
        double v;
        if (!last) {
          // continuity row jq of interface (l, l+1) (solve0 :1080-1104)
          const int jq = rank;
          double dl0, dl1, dn0, dn1;
          dz(l, jq, b0, b1, dl0, dl1);
          dz(l + 1, jq, n0, n1, dn0, dn1);
          v = dn0 - dl0 + (dn1 - dl1) * taus[l + 1];
        } else {
          // bottom boundary row rb (FluxSolver.cpp:1437-1461, 1477-1492)
          const int rb = rank;
          const double tb = taus[L];
          if (k == L + 1) {  // the surface temperature
            if (dlbc) {
              v = 1.0;
              if (dtau_last > 0.0) v += mu[rb] * (1.0 / dtau_last);
            } else {
              v = sft ? sft[rb * brdf_row(N) + NN + 1] : 1.0 - alb;
            }
          } else {
            double d0, d1;
            dz(l, NN + rb, b0, b1, d0, d1);
            if (dlbc) {
              v = -d0 - d1 * tb;
              if (k == L - 1 && dtau_last > 0.0) v += mu[rb] * (-1.0 / dtau_last);
            } else {
              double refl = 0.0;
              for (int jq = 0; jq < NN; ++jq) {
                double e0, e1;
                dz(l, NN - 1 - jq, b0, b1, e0, e1);
                refl += wt[jq] * mu[jq] * (sft ? sft[rb * brdf_row(N) + 1 + jq] : alb) * (e0 + e1 * tb);
              }
              v = 2.0 * refl;
              v -= d0 + d1 * tb;
            }
          }
        }
        R[s * KB] = v;
        carried[s >> 5] |= 1u << (s & 31);  // now a candidate
        ++rank;
      }
#pragma unroll
      for (int w = 0; w < NW; ++w) cand[w] = carried[w];
      const double* jr = jrec0 + (long long)l * jrec_stride(N);
      double* cvl = cv0 + (long long)l * N * cvs;
      for (int c = 0; c < N; ++c) {
        int ps = (int)jr[N * PR + c];
        ps = ps < 0 ? 0 : (ps >= PR ? PR - 1 : ps);  // a record slot always, whatever was stored
        const double rp = R[ps * KB];
        if (act) cvl[c * cvs + k] = rp;
        cand[ps >> 5] &= ~(1u << (ps & 31));
        const double* m = jr + c * PR;
        for (int s = 0; s < PR; ++s) R[s * KB] += m[s] * rp;
      }
#pragma unroll
      for (int w = 0; w < NW; ++w) carried[w] = cand[w];
    }
    __syncthreads();  // R's area becomes X

    // ---- up: U_l x_l = c_l - V_l x_{l+1}, outputs level by level ----------
    double* X = Rv + tid;  // x of parity b at X[(b * N + j) * KB]
    for (int j = 0; j < N; ++j) X[(N + j) * KB] = 0.0;
    double chain_lev = 0.0;
    if (act) {
      if (k <= L) chain_lev = planck_deriv2(wlo, whi, temp_in[ifb ? L - k : k], p.pk);
      else chain_lev = planck_deriv2(wlo, whi, p.tbot(i), p.pk);
    }
    for (int l = L - 1; l >= 0; --l) {
      const int b = l & 1;
      double* x = X + b * N * KB;
      const double* xn = X + (b ^ 1) * N * KB;
      const double* br = brec0 + (long long)l * brec_stride(N);
      const double* cvl = cv0 + (long long)l * N * cvs;
      for (int c = N - 1; c >= 0; --c) {
        double s = act ? cvl[c * cvs + k] : 0.0;
        const double* row = br + c * RL;
        for (int j = c + 1; j < N; ++j) s -= row[j] * x[j * KB];
        if (l < L - 1)
          for (int j = 0; j < N; ++j) s -= row[N + j] * xn[j * KB];
        x[c * KB] = s * rdiag(br, c);
      }
      // outputs at the depths of layer l (flux path: its bottom level, and the
      // top for l = 0)
      const double* lr = lrec0 + (long long)l * lstride;
      const double* eig = lr + lrec_eig(N);
      const double* G = lr + lrec_G(N);
      double a0, a1;
      coef(l, a0, a1);
      const int lin = ifb ? L - 1 - l : l;
      const double w0 = GEN ? p.g.ssa[p.g.in_off[i] + lin] : p.ssa(i, lin);
      const int npass = GEN ? NT : (l == 0 ? 2 : 1);
      for (int pass = 0; pass < npass; ++pass) {
        const int lu = GEN ? pass : (pass == 0 ? l + 1 : 0);
        if (GEN && out_layer(lu) != l) continue;  // uniform over the CTA
        const double utaupr = out_taus(lu);
        __syncthreads();
        for (int j = tid; j < N; j += KB) {
          const double d = (j < NN) ? (utaupr - taus[l + 1]) : (utaupr - taus[l]);
          ex[j] = exp(-eig[j] * d);
        }
        __syncthreads();
        double dmi = 0.0, dmidn = 0.0, dmiup = 0.0, dfdn = 0.0, dfup = 0.0;
        for (int iq = 0; iq < N; ++iq) {
          double v = 0.0;
          for (int j = 0; j < N; ++j) v += G[iq * N + j] * (x[j * KB] * ex[j]);
          double d0, d1;
          dz(l, iq, a0, a1, d0, d1);
          v += d0 + d1 * utaupr;
          if (iq < NN) {
            const int c = NN - iq - 1;
            dmi += wt[c] * v;
            dmidn += wt[c] * v;
            dfdn += wt[c] * v * mu[c];
          } else {
            const int c = iq - NN;
            dmi += wt[c] * v;
            dmiup += wt[c] * v;
            dfup += wt[c] * v * mu[c];
          }
        }
        if (act) {
          dfup *= 2.0 * PI;
          dfdn *= 2.0 * PI;
          const double dmi_t = (2.0 * PI * dmi) / (4.0 * PI);
          const double dmi_d = (2.0 * PI * dmidn) / (4.0 * PI);
          const double dmi_u = (2.0 * PI * dmiup) / (4.0 * PI);
          const double dpls = a0 + a1 * utaupr;
          const double dfdiv = (1.0 - w0) * 4.0 * PI * (dmi_t - dpls);
          store(0, lu, k, chain_lev * dfup);
          store(1, lu, k, chain_lev * dfdn);
          store(2, lu, k, chain_lev * dmi_t);
          store(3, lu, k, chain_lev * dmi_d);
          store(4, lu, k, chain_lev * dmi_u);
          store(5, lu, k, chain_lev * dfdiv);
        }
      }
    }
    __syncthreads();  // X's area is the next pass's R
  }
}

}  // namespace dsp
