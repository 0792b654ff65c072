// flux_oracle.hpp — CPU restatement of DisortFluxSolver<NStr>::solve
// (src/FluxSolver.cpp:23-1287 of DisORT++), plane-parallel geometry, Lambertian
// surface, thermal emission, delta-M / delta-M+ and the absorption layer cut.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into the product.
#pragma once

#include <vector>

#include "../include/dsp.h"
#include "oracle_common.hpp"

namespace oracle {

// One instance of a flux solve, already flattened (the reference's
// DisortFluxConfig after applyOverrides, python_bindings.cpp:73-82).
struct FluxInstance {
  int num_layers = 0, num_streams = 0, num_phase_func_moments = 0;
  int pmom_count = 0;  // stride of pmom per layer
  bool thermal = false, delta_m_plus = false, diffusion_lower_bc = false, index_from_bottom = false;
  bool temperature_jac = false;  // compute_temperature_jacobian
  bool spherical = false;        // use_spherical_beam
  double bottom_radius = 0;
  const double* level_altitudes = nullptr;  // [L+1] (spherical only)
  double wavenumber_low = 0, wavenumber_high = 0;
  double surface_albedo = 0, emissivity_top = 1, direct_beam_flux = 0, direct_beam_mu = 0.5;
  double isotropic_flux_top = 0, isotropic_flux_bottom = 0, temperature_top = 0, temperature_bottom = 0;
  const double* delta_tau = nullptr;  // [L]
  const double* ssa = nullptr;        // [L]
  const double* pmom = nullptr;       // [L][pmom_count]
  const double* temperature = nullptr;  // [L+1]
};

struct FluxOutput {  // each [L+1]
  double *fdir, *fdn, *fup, *dfdt, *uavg, *uavgdn, *uavgup, *uavgso;
  // temperature Jacobians (FluxResult *_temperature_jac), each [L+1][L+2] or null:
  // flux_up, flux_down, mean_intensity, mean_intensity_down, mean_intensity_up,
  // flux_divergence
  double* jac[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

// DisortFluxConfig::validate (DisortFluxConfig.cpp:43-143) for the fields the
// batch carries.  Returns DSP_OK or DSP_ERR_INVALID_INPUT.
inline int validate_flux_instance(const FluxInstance& c) {
  const int L = c.num_layers, N = c.num_streams;
  if (L <= 0) return DSP_ERR_INVALID_INPUT;
  if (N < 4 || N % 2 != 0) return DSP_ERR_INVALID_INPUT;
  if (c.num_phase_func_moments < 0) return DSP_ERR_INVALID_INPUT;
  const int nmom_needed = std::max(c.num_phase_func_moments, N) + 1;
  if (c.pmom_count < nmom_needed) return DSP_ERR_INVALID_INPUT;
  for (int lc = 0; lc < L; ++lc) {
    if (c.delta_tau[lc] < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.ssa[lc] < 0.0 || c.ssa[lc] > 1.0) return DSP_ERR_INVALID_INPUT;
  }
  if (c.diffusion_lower_bc && !c.thermal) return DSP_ERR_INVALID_INPUT;
  if (c.direct_beam_flux < 0.0) return DSP_ERR_INVALID_INPUT;
  if (c.direct_beam_flux > 0.0 && (c.direct_beam_mu <= 0.0 || c.direct_beam_mu > 1.0)) return DSP_ERR_INVALID_INPUT;
  if (c.surface_albedo < 0.0 || c.surface_albedo > 1.0) return DSP_ERR_INVALID_INPUT;
  if (c.thermal) {
    if (c.temperature == nullptr) return DSP_ERR_INVALID_INPUT;
    for (int lev = 0; lev <= L; ++lev)
      if (c.temperature[lev] < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.wavenumber_low < 0.0 || c.wavenumber_low > c.wavenumber_high) return DSP_ERR_INVALID_INPUT;
    if (c.temperature_top < 0.0 || c.temperature_bottom < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.emissivity_top < 0.0 || c.emissivity_top > 1.0) return DSP_ERR_INVALID_INPUT;
  }
  if (c.spherical && (c.bottom_radius <= 0.0 || c.level_altitudes == nullptr)) return DSP_ERR_INVALID_INPUT;
  if (c.delta_m_plus && c.num_phase_func_moments < N + 1) return DSP_ERR_INVALID_INPUT;
  return DSP_OK;
}

// LINPACK sgbfa / sgbsl band LU (BandSolver.hpp:29-172), restated.
// abd column-major with leading dimension lda = 2*ml+mu+1; 1-based pivots.
inline bool band_factor(double* abd, int lda, int n, int ml, int mu, int* ipvt) {
  bool ok = true;
  const int m0 = ml + mu, m1 = m0 + 1;
  {
    const int j1 = std::min(n, m1) - 1;
    for (int j = mu + 2; j <= j1; ++j) {
      const int i0 = m1 + 1 - j;
      const int nzero = ml - i0 + 1;
      if (nzero > 0) std::memset(abd + (i0 - 1) + (j - 1) * lda, 0, nzero * sizeof(double));
    }
  }
  int jz = std::min(n, m1) - 1;
  int ju = 0;
  for (int k = 1; k <= n - 1; ++k) {
    jz++;
    if (jz <= n && ml > 0) std::memset(abd + (jz - 1) * lda, 0, ml * sizeof(double));
    const int lm = std::min(ml, n - k);
    double* col_k = abd + (k - 1) * lda;
    int l_off = 0;
    double smax = std::abs(col_k[m0]);
    for (int i = 1; i <= lm; ++i) {
      const double x = std::abs(col_k[m0 + i]);
      if (x > smax) { smax = x; l_off = i; }
    }
    const int l = m1 + l_off;
    ipvt[k - 1] = l + k - m1;
    if (col_k[m0 + l_off] == 0.0) { ok = false; continue; }
    if (l_off != 0) std::swap(col_k[m0 + l_off], col_k[m0]);
    const double t = -1.0 / col_k[m0];
    for (int i = 0; i < lm; ++i) col_k[m0 + 1 + i] *= t;
    ju = std::min(std::max(ju, mu + ipvt[k - 1]), n);
    int ll = l, mm = m1;
    const double* src = col_k + m0 + 1;
    for (int j = k + 1; j <= ju; ++j) {
      ll--; mm--;
      double* col_j = abd + (j - 1) * lda;
      const int ll0 = ll - 1, mm0 = mm - 1;
      const double tj = col_j[ll0];
      if (ll0 != mm0) { col_j[ll0] = col_j[mm0]; col_j[mm0] = tj; }
      if (tj != 0.0)
        for (int i = 0; i < lm; ++i) col_j[mm0 + 1 + i] += tj * src[i];
    }
  }
  ipvt[n - 1] = n;
  if (abd[(n - 1) * lda + m0] == 0.0) ok = false;
  return ok;
}

inline void band_solve(const double* abd, int lda, int n, int ml, int mu, const int* ipvt, double* b) {
  const int m0 = mu + ml;
  if (ml > 0) {
    for (int k = 1; k <= n - 1; ++k) {
      const int lm = std::min(ml, n - k);
      const int l = ipvt[k - 1];
      const double t = b[l - 1];
      if (l != k) { b[l - 1] = b[k - 1]; b[k - 1] = t; }
      const double* mults = abd + (k - 1) * lda + m0 + 1;
      for (int i = 0; i < lm; ++i) b[k + i] += t * mults[i];
    }
  }
  const int m1 = m0 + 1;
  for (int kb = 1; kb <= n; ++kb) {
    const int k = n + 1 - kb;
    const double* col_k = abd + (k - 1) * lda;
    b[k - 1] /= col_k[m0];
    const int lm = std::min(k, m1) - 1;
    if (lm > 0) {
      const double t = -b[k - 1];
      const double* src = col_k + m0 - lm;
      double* dst = b + k - 1 - lm;
      for (int i = 0; i < lm; ++i) dst[i] += t * src[i];
    }
  }
}

// Symmetric reduction of the layer eigenproblem shared by the flux and general
// solvers (FluxSolver.cpp:508-566, DisortSolver.cpp:1023-1140):
// given alpha-beta (amb) and alpha+beta (apb), NN x NN row-major, and the
// similarity vector D, fill evec (NN x NN, eigenvectors of (a+b)(a-b) as
// columns) and kred (NN, sqrt|lambda|).  `spd_allowed` is false when the
// reference takes its general-eigensolver branch (omega' >= 1 - 1e-12); the
// oracle then uses the equivalent factorisation of -A_s instead.
// Returns DSP_OK or DSP_ERR_EIGEN.
inline int layer_eigen(int nn, const double* amb, const double* apb, const double* dsim, const double* dinv,
                       bool spd_allowed, double* evec, double* kred) {
  constexpr int M = 32;
  double As[M * M], nBs[M * M], L[M * M], T[M * M], S[M * M], W[M * M], lam[M];
  for (int i = 0; i < nn; ++i)
    for (int j = 0; j < nn; ++j) {
      As[i * M + j] = dsim[i] * apb[i * nn + j] * dinv[j];
      nBs[i * M + j] = -dsim[i] * amb[i * nn + j] * dinv[j];
    }
  bool spd = spd_allowed && cholesky_lower(nBs, nn, M, L);
  if (spd) {
    // S = L^T (-A_s) L  (FluxSolver.cpp:530-534)
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) {
        double s = 0.0;
        for (int k = 0; k < nn; ++k) s += -As[i * M + k] * L[k * M + j];
        T[i * M + j] = s;
      }
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) {
        double s = 0.0;
        for (int k = 0; k < nn; ++k) s += L[k * M + i] * T[k * M + j];
        S[i * M + j] = s;
      }
    sym_eigen(S, nn, M, lam, W);
    // u = D^{-1} L^{-T} w   (FluxSolver.cpp:539-546)
    for (int c = 0; c < nn; ++c) {
      double v[M];
      for (int i = nn - 1; i >= 0; --i) {
        double s = W[i * M + c];
        for (int k = i + 1; k < nn; ++k) s -= L[k * M + i] * v[k];
        v[i] = s / L[i * M + i];
      }
      for (int j = 0; j < nn; ++j) evec[j * nn + c] = dinv[j] * v[j];
    }
  } else {
    // -A_s = L' L'^T, S' = L'^T (-B_s) L', u = D^{-1} L' w: the same eigenpairs
    // as the reference's general EigenSolver on (a+b)(a-b) (FluxSolver.cpp:547-558).
    double nAs[M * M];
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) nAs[i * M + j] = -As[i * M + j];
    if (!cholesky_lower(nAs, nn, M, L)) {
      if (!cholesky_lower(nBs, nn, M, L)) return DSP_ERR_EIGEN;
      // -B_s is SPD after all: use the primary path
      return layer_eigen(nn, amb, apb, dsim, dinv, true, evec, kred);
    }
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) {
        double s = 0.0;
        for (int k = 0; k < nn; ++k) s += nBs[i * M + k] * L[k * M + j];
        T[i * M + j] = s;
      }
    for (int i = 0; i < nn; ++i)
      for (int j = 0; j < nn; ++j) {
        double s = 0.0;
        for (int k = 0; k < nn; ++k) s += L[k * M + i] * T[k * M + j];
        S[i * M + j] = s;
      }
    sym_eigen(S, nn, M, lam, W);
    for (int c = 0; c < nn; ++c)
      for (int j = 0; j < nn; ++j) {
        double s = 0.0;
        for (int k = 0; k <= j; ++k) s += L[j * M + k] * W[k * M + c];
        evec[j * nn + c] = dinv[j] * s;
      }
  }
  for (int i = 0; i < nn; ++i) kred[i] = std::sqrt(std::abs(lam[i]));
  return DSP_OK;
}

// The Chapman function of the pseudo-spherical beam (chapmanImpl,
// FluxSolver.cpp:1503-1566): the slant optical depth from the top to a point
// a fraction tau_frac from the bottom of layer lc (1-based) along the beam
// through a spherical shell atmosphere of level altitudes zd[0..L] (top down)
// above radius r, with dtau_lyr the layers' optical depths.
inline double chapman(int lc, double tau_frac, const double* zd, const double* dtau_lyr, int num_layers, double r,
                      double direct_beam_mu) {
  const double DEG = M_PI / 180.0;
  const double zenang = std::acos(direct_beam_mu) * 180.0 / M_PI;
  const double zenrad = zenang * DEG;
  auto ZD = [&](int j) { return zd[j]; };
  auto DT = [&](int j) { return dtau_lyr[j - 1]; };
  const double xp = r + ZD(lc) + (ZD(lc - 1) - ZD(lc)) * tau_frac;
  const double xpsinz = xp * std::sin(zenrad);
  if (zenang > 90.0 && xpsinz < r) return 1.0e+20;
  int id = lc;
  if (zenang > 90.0)
    for (int j = lc; j <= num_layers; ++j)
      if (xpsinz < (ZD(j - 1) + r) && xpsinz >= (ZD(j) + r)) id = j;
  double sum = 0.0;
  for (int j = 1; j <= id; ++j) {
    double fact = 1.0, fact2 = 1.0;
    if (j > lc) fact = 2.0;
    else if (j == lc && lc == id && zenang > 90.0) fact2 = -1.0;
    const double rj = r + ZD(j - 1);
    double rjp1 = r + ZD(j);
    if (j == lc && id == lc) rjp1 = xp;
    const double dhj = ZD(j - 1) - ZD(j);
    double dsj;
    if (id > lc && j == id) dsj = std::sqrt(rj * rj - xpsinz * xpsinz);
    else dsj = std::sqrt(rj * rj - xpsinz * xpsinz) - fact2 * std::sqrt(rjp1 * rjp1 - xpsinz * xpsinz);
    sum += DT(j) * fact * dsj / dhj;
  }
  if (id > lc) {
    const double dhj = ZD(lc - 1) - ZD(lc);
    const double dsj = std::sqrt(xp * xp - xpsinz * xpsinz) - std::sqrt((ZD(lc) + r) * (ZD(lc) + r) - xpsinz * xpsinz);
    sum += DT(lc) * dsj / dhj;
  }
  return sum;
}

// ---------------------------------------------------------------------------
// The flux solver.  One object per thread, reused across instances, like the
// reference spectral loop (python_bindings.cpp:170-190).
// ---------------------------------------------------------------------------
class FluxOracle {
 public:
  int solve(const FluxInstance& cfg_in, const FluxOutput& out);

 private:
  void thermal_jacobian(const FluxInstance& cfg, const FluxOutput& out, int lda, int nc, int ncd);
  int N = 0, NN = 0, L = 0, ncut = 0;
  bool lyrcut = false, deltam = false, deltam_plus = false;
  // quadrature (FluxSolver.cpp:257-290, 442-445)
  std::vector<double> mu, wt, dsim, dinv, ylm;  // ylm[(N+1) x N]
  std::vector<double> dtau_s, tau_s, ssa_s, gl;  // gl[L][N]
  std::vector<double> beam_tr;                  // [L+1]
  // pseudo-spherical beam: Chapman factor per layer, the slope of the beam
  // particular solution and its attenuation (FluxSolver.cpp:391-419, 650-738)
  std::vector<double> chap, zbs1, xba;
  std::vector<double> rev_zalt;
  std::vector<double> kk, G, C;                 // kk[L][N], G[L][N][N], C[L][N][N]
  std::vector<double> zb, z0, z1, xr0, xr1;     // particular solutions
  // derivatives of the thermal source w.r.t. the layer's top / bottom level
  // Planck values (computeIsotropicSource, FluxSolver.cpp:786-829)
  std::vector<double> dz0t, dz0b, dz1t, dz1b, dxr0t, dxr0b, dxr1t, dxr1b;
  std::vector<double> jb, jll;  // Jacobian right-hand side and its reordered solution
  std::vector<double> band, rhs, cc;            // BVP
  std::vector<int> ipvt;
  double planck_top = 0, planck_bottom = 0, planck_bottom_deriv = 0;
  // reversed copies for index_from_bottom
  std::vector<double> rev_dtau, rev_ssa, rev_pmom, rev_temp;
};

inline int FluxOracle::solve(const FluxInstance& cfg_in, const FluxOutput& out) {
  FluxInstance cfg = cfg_in;
  L = cfg.num_layers;
  N = cfg.num_streams;
  NN = N / 2;
  const int nlev = L + 1;
  auto fill_nan = [&]() {
    for (int i = 0; i < nlev; ++i) {
      out.fdir[i] = out.fdn[i] = out.fup[i] = out.dfdt[i] = std::nan("");
      out.uavg[i] = out.uavgdn[i] = out.uavgup[i] = out.uavgso[i] = std::nan("");
    }
    if (out.jac[0])
      for (double* J : out.jac) std::fill(J, J + (size_t)nlev * (L + 2), std::nan(""));
  };
  if (L <= 0 || N < 4 || N % 2 != 0 || N > 64) { if (L > 0) fill_nan(); return DSP_ERR_INVALID_INPUT; }
  // index_from_bottom: reverse layer/level inputs (IndexConversion.hpp:42-52)
  if (cfg.index_from_bottom) {
    rev_dtau.assign(cfg.delta_tau, cfg.delta_tau + L);
    rev_ssa.assign(cfg.ssa, cfg.ssa + L);
    std::reverse(rev_dtau.begin(), rev_dtau.end());
    std::reverse(rev_ssa.begin(), rev_ssa.end());
    rev_pmom.resize((size_t)L * cfg.pmom_count);
    for (int lc = 0; lc < L; ++lc)
      std::memcpy(&rev_pmom[(size_t)lc * cfg.pmom_count], cfg.pmom + (size_t)(L - 1 - lc) * cfg.pmom_count,
                  sizeof(double) * cfg.pmom_count);
    cfg.delta_tau = rev_dtau.data();
    cfg.ssa = rev_ssa.data();
    cfg.pmom = rev_pmom.data();
    if (cfg.temperature) {
      rev_temp.assign(cfg.temperature, cfg.temperature + L + 1);
      std::reverse(rev_temp.begin(), rev_temp.end());
      cfg.temperature = rev_temp.data();
    }
    if (cfg.level_altitudes) {
      rev_zalt.assign(cfg.level_altitudes, cfg.level_altitudes + L + 1);
      std::reverse(rev_zalt.begin(), rev_zalt.end());
      cfg.level_altitudes = rev_zalt.data();
    }
  }
  int st = validate_flux_instance(cfg);
  if (st != DSP_OK) { fill_nan(); return st; }
  const int pc = cfg.pmom_count;
  auto PM = [&](int k, int lc) { return cfg.pmom[(size_t)lc * pc + k]; };

  // delta-M decisions (FluxSolver.cpp:56-81)
  deltam = false;
  for (int lc = 0; lc < L; ++lc)
    if (PM(N, lc) != 0.0) { deltam = true; break; }
  deltam_plus = cfg.delta_m_plus;
  if (deltam_plus) {
    for (int lc = 0; lc < L; ++lc) {
      const double pm = PM(N, lc), pm1 = PM(N + 1, lc);
      if (pm < 1e-4 || pm1 < 0.7 * pm) { deltam_plus = false; break; }
    }
    if (deltam_plus) deltam = false;
  }

  mu.assign(N, 0); wt.assign(N, 0); dsim.assign(NN, 0); dinv.assign(NN, 0);
  ylm.assign((size_t)(N + 1) * N, 0);
  dtau_s.assign(L, 0); tau_s.assign(L + 1, 0); ssa_s.assign(L, 0); gl.assign((size_t)L * N, 0);
  beam_tr.assign(L + 1, 0.0);

  // disortSet (FluxSolver.cpp:309-452)
  {
    const double abscut = 10.0;
    std::vector<double> tauc(L + 1);
    tauc[0] = 0.0;
    for (int lc = 0; lc < L; ++lc) tauc[lc + 1] = tauc[lc] + cfg.delta_tau[lc];
    tau_s[0] = 0.0;
    double abstau = 0.0;
    ncut = L;
    for (int lc = 0; lc < L; ++lc) {
      if (abstau < abscut) ncut = lc + 1;
      abstau += (1.0 - cfg.ssa[lc]) * cfg.delta_tau[lc];
      const double w0 = cfg.ssa[lc], dt = cfg.delta_tau[lc];
      if (!deltam && !deltam_plus) {
        ssa_s[lc] = w0;
        dtau_s[lc] = dt;
        tau_s[lc + 1] = tauc[lc + 1];
        for (int k = 0; k < N; ++k) gl[(size_t)lc * N + k] = (2.0 * k + 1.0) * ssa_s[lc] * PM(k, lc);
      } else if (!deltam_plus || PM(N - 1, lc) == PM(N, lc)) {
        const double f = PM(N, lc);
        ssa_s[lc] = w0 * (1.0 - f) / (1.0 - f * w0);
        dtau_s[lc] = (1.0 - f * w0) * dt;
        tau_s[lc + 1] = tau_s[lc] + dtau_s[lc];
        for (int k = 0; k < N; ++k) gl[(size_t)lc * N + k] = (2.0 * k + 1.0) * ssa_s[lc] * (PM(k, lc) - f) / (1.0 - f);
      } else {
        const double pm = PM(N, lc), pm1 = PM(N + 1, lc);
        if (pm == pm1) {
          const double f = pm;
          ssa_s[lc] = w0 * (1.0 - f) / (1.0 - f * w0);
          dtau_s[lc] = (1.0 - f * w0) * dt;
          tau_s[lc + 1] = tau_s[lc] + dtau_s[lc];
          for (int k = 0; k < N; ++k) gl[(size_t)lc * N + k] = (2.0 * k + 1.0) * ssa_s[lc] * (PM(k, lc) - f) / (1.0 - f);
        } else {
          const double M = static_cast<double>(N);
          const double sigma_sq = ((M + 1.0) * (M + 1.0) - M * M) / (std::log(pm * pm) - std::log(pm1 * pm1));
          const double c = std::exp(M * M / (2.0 * sigma_sq));
          const double f = c * pm;
          ssa_s[lc] = w0 * (1.0 - f) / (1.0 - f * w0);
          dtau_s[lc] = (1.0 - f * w0) * dt;
          tau_s[lc + 1] = tau_s[lc] + dtau_s[lc];
          for (int k = 0; k < N; ++k) {
            const double kd = static_cast<double>(k);
            gl[(size_t)lc * N + k] = (2.0 * k + 1.0) * ssa_s[lc] * (PM(k, lc) - f * std::exp(-kd * kd / (2.0 * sigma_sq))) / (1.0 - f);
          }
        }
      }
    }
    // Beam transmission for lc < ncut of the absorption loop (FluxSolver.cpp:391-412).
    // Entries past that cut are left at zero, as on a freshly constructed solver.
    chap.assign(L, 0.0);
    if (cfg.direct_beam_flux > 0.0) {
      beam_tr[0] = 1.0;
      if (cfg.spherical) {
        // Chapman factors on the scaled depths (FluxSolver.cpp:396-415)
        for (int lc = 0; lc < ncut; ++lc) {
          const double taup_mid = tau_s[lc] + dtau_s[lc] / 2.0;
          const double chtau_mid = chapman(lc + 1, 0.5, cfg.level_altitudes, dtau_s.data(), L, cfg.bottom_radius,
                                           cfg.direct_beam_mu);
          chap[lc] = taup_mid / chtau_mid;
          const double chtau = chapman(lc + 1, 0.0, cfg.level_altitudes, dtau_s.data(), L, cfg.bottom_radius,
                                       cfg.direct_beam_mu);
          beam_tr[lc + 1] = std::exp(-chtau);
        }
      } else {
        for (int lc = 0; lc < ncut; ++lc) {
          chap[lc] = cfg.direct_beam_mu;
          beam_tr[lc + 1] = std::exp(-tau_s[lc + 1] / cfg.direct_beam_mu);
        }
      }
    }
    lyrcut = (abstau >= abscut && !cfg.thermal && L > 1);
    if (!lyrcut) ncut = L;
    if (!gauss_quadrature(NN, mu.data(), wt.data())) { fill_nan(); return DSP_ERR_EIGEN; }
    for (int iq = 0; iq < NN; ++iq) {
      dsim[iq] = std::sqrt(wt[iq] * mu[iq]);
      dinv[iq] = 1.0 / dsim[iq];
    }
  }

  // Planck at the boundaries (FluxSolver.cpp:101-122)
  planck_top = planck_bottom = planck_bottom_deriv = 0.0;
  if (cfg.thermal) {
    planck_top = planck_function2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature_top) * cfg.emissivity_top;
    planck_bottom = planck_function2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature_bottom);
    if (cfg.diffusion_lower_bc) {
      const double B_layer = planck_function2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature[L - 1]);
      if (dtau_s[L - 1] > 0.0) planck_bottom_deriv = (planck_bottom - B_layer) / dtau_s[L - 1];
    }
  }
  // Legendre at the quadrature angles (FluxSolver.cpp:126)
  legendre_flat(N, 0, N, N - 1, mu.data(), ylm.data());
  auto Y = [&](int l, int i) { return ylm[(size_t)l * N + i]; };

  // Per-layer eigensystem (solveEigen, FluxSolver.cpp:459-588)
  kk.assign((size_t)L * N, 0); G.assign((size_t)L * N * N, 0); C.assign((size_t)L * N * N, 0);
  std::vector<double> cc_top((size_t)NN * N), amb(NN * NN), apb(NN * NN), evec(NN * NN), kred(NN), gpg(NN * NN);
  for (int lc = 0; lc < L; ++lc) {
    const double* g = &gl[(size_t)lc * N];
    for (int iq = 0; iq < NN; ++iq)
      for (int jq = 0; jq < N; ++jq) {
        double s = 0.0;
        for (int l = 0; l < N; ++l) s += (g[l] * Y(l, iq)) * Y(l, jq);
        cc_top[iq * N + jq] = (s * 0.5) * wt[jq];
      }
    double* Cl = &C[(size_t)lc * N * N];
    for (int iq = 0; iq < NN; ++iq)
      for (int jq = 0; jq < N; ++jq) Cl[iq * N + jq] = cc_top[iq * N + jq];
    for (int iq = 0; iq < NN; ++iq)
      for (int jq = 0; jq < NN; ++jq) {
        Cl[(NN + iq) * N + jq] = cc_top[iq * N + NN + jq];
        Cl[(NN + iq) * N + NN + jq] = cc_top[iq * N + jq];
      }
    for (int iq = 0; iq < NN; ++iq) {
      const double inv_cmu = 1.0 / mu[iq];
      for (int jq = 0; jq < NN; ++jq) {
        amb[iq * NN + jq] = inv_cmu * (cc_top[iq * N + jq] - cc_top[iq * N + NN + jq]);
        apb[iq * NN + jq] = inv_cmu * (cc_top[iq * N + jq] + cc_top[iq * N + NN + jq]);
      }
      amb[iq * NN + iq] -= inv_cmu;
      apb[iq * NN + iq] -= inv_cmu;
    }
    const bool spd_allowed = ssa_s[lc] < 1.0 - 1e-12;
    st = layer_eigen(NN, amb.data(), apb.data(), dsim.data(), dinv.data(), spd_allowed, evec.data(), kred.data());
    if (st != DSP_OK) { fill_nan(); return st; }
    double* kl = &kk[(size_t)lc * N];
    for (int iq = 0; iq < NN; ++iq) {
      kl[iq + NN] = kred[iq];
      kl[NN - 1 - iq] = -kred[iq];
    }
    // (G+ + G-) = (a-b) evec / k  (FluxSolver.cpp:570-571)
    for (int i = 0; i < NN; ++i)
      for (int j = 0; j < NN; ++j) {
        double s = 0.0;
        for (int k = 0; k < NN; ++k) s += amb[i * NN + k] * evec[k * NN + j];
        gpg[i * NN + j] = s / kred[j];
      }
    double* Gl = &G[(size_t)lc * N * N];
    for (int jq = 0; jq < NN; ++jq)
      for (int iq = 0; iq < NN; ++iq) {
        double gpplgm = gpg[iq * NN + jq];
        const double gpmigm = evec[iq * NN + jq];
        Gl[(NN + iq) * N + NN + jq] = 0.5 * (gpplgm + gpmigm);
        Gl[(NN - iq - 1) * N + NN + jq] = 0.5 * (gpplgm - gpmigm);
        gpplgm *= -1.0;
        Gl[(NN + iq) * N + NN - jq - 1] = 0.5 * (gpplgm + gpmigm);
        Gl[(NN - iq - 1) * N + NN - jq - 1] = 0.5 * (gpplgm - gpmigm);
      }
  }

  // Beam particular solution (computeBeamSource, FluxSolver.cpp:595-643)
  zb.assign((size_t)L * N, 0.0);
  zbs1.assign((size_t)L * N, 0.0);
  xba.assign(L, 0.0);
  std::vector<double> A((size_t)N * N), x(N);
  std::vector<int> piv(N);
  if (cfg.direct_beam_flux > 0.0 && cfg.spherical) {
    // pseudo-spherical source (computeBeamSourceSpherical, FluxSolver.cpp:650-738):
    // Z(tau) = exp(-xba tau) (Z0 + Z1 tau) with xba = 1 / Chapman factor
    std::vector<double> yb(N + 1), zj(N), xb0(N), xb1(N), z1v(N), z0v(N);
    const double umu0 = -cfg.direct_beam_mu;
    legendre_flat(1, 0, 1, N - 1, &umu0, yb.data());
    const double big = std::sqrt(std::numeric_limits<double>::max()) / 1.0e10;
    for (int lc = 0; lc < ncut; ++lc) {
      for (int iq = 0; iq < N; ++iq) {
        double sum = 0.0;
        for (int k = 0; k < N; ++k) sum += gl[(size_t)lc * N + k] * Y(k, iq) * yb[k];
        zj[iq] = cfg.direct_beam_flux * sum / (4.0 * M_PI);
      }
      const double q0a = beam_tr[lc], q2a = beam_tr[lc + 1];
      double xb = 1.0 / chap[lc];
      if (std::abs(xb) > big && tau_s[lc + 1] > 1.0) xb = 0.0;
      if (std::abs(xb * tau_s[lc + 1]) > std::log(big)) xb = 0.0;
      if (std::abs(xb) > 1.0e-5)
        for (int iq = 0; iq < NN; ++iq)
          if (std::abs((std::abs(xb) - 1.0 / mu[iq]) / xb) < 0.05) {
            xb *= 1.001;
            break;
          }
      const double deltat = tau_s[lc + 1] - tau_s[lc];
      for (int iq = 0; iq < N; ++iq) {
        const double q0 = q0a * zj[iq], q2 = q2a * zj[iq];
        xb1[iq] = (q2 * std::exp(xb * tau_s[lc + 1]) - q0 * std::exp(xb * tau_s[lc])) / deltat;
        xb0[iq] = q0 * std::exp(xb * tau_s[lc]) - xb1[iq] * tau_s[lc];
      }
      const double* Cl = &C[(size_t)lc * N * N];
      auto build = [&]() {
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
        for (int iq = 0; iq < N; ++iq) A[iq * N + iq] += 1.0 + xb * mu[iq];
      };
      build();
      // dither when near-singular: 1 / Frobenius norm of the system (FluxSolver.cpp:707-718)
      double fro = 0.0;
      for (int e = 0; e < N * N; ++e) fro += A[e] * A[e];
      const double rcond_approx = 1.0 / std::sqrt(fro);
      if (rcond_approx < 1.0e-4) {
        if (xb == 0.0) xb = 5.0e-9;
        xb *= 1.00000005;
        build();
      }
      xba[lc] = xb;
      lu_factor(A.data(), N, N, piv.data());
      for (int iq = 0; iq < N; ++iq) z1v[iq] = xb1[iq];
      lu_solve(A.data(), N, N, piv.data(), z1v.data());
      for (int iq = 0; iq < N; ++iq) z0v[iq] = xb0[iq] + mu[iq] * z1v[iq];
      lu_solve(A.data(), N, N, piv.data(), z0v.data());
      for (int iq = 0; iq < NN; ++iq) {
        zb[(size_t)lc * N + NN + iq] = z0v[iq];
        zb[(size_t)lc * N + NN - 1 - iq] = z0v[iq + NN];
        zbs1[(size_t)lc * N + NN + iq] = z1v[iq];
        zbs1[(size_t)lc * N + NN - 1 - iq] = z1v[iq + NN];
      }
    }
  } else if (cfg.direct_beam_flux > 0.0) {
    std::vector<double> yb(N + 1);
    const double umu0 = -cfg.direct_beam_mu;
    legendre_flat(1, 0, 1, N - 1, &umu0, yb.data());
    const double dither = 1000.0 * std::numeric_limits<double>::epsilon();
    for (int lc = 0; lc < L; ++lc) {
      double beam_mu = cfg.direct_beam_mu;
      const double mu0sq = cfg.direct_beam_mu * cfg.direct_beam_mu;
      for (int iq = 0; iq < NN; ++iq) {
        const double k = kk[(size_t)lc * N + iq + NN];
        if (std::abs(1.0 - mu0sq * k * k) < dither) { beam_mu = 0.999 * cfg.direct_beam_mu; break; }
      }
      const double* Cl = &C[(size_t)lc * N * N];
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
      for (int i = 0; i < N; ++i) A[i * N + i] += 1.0 + mu[i] / beam_mu;
      for (int iq = 0; iq < N; ++iq) {
        double s = 0.0;
        for (int k = 0; k < N; ++k) s += gl[(size_t)lc * N + k] * Y(k, iq) * yb[k];
        x[iq] = cfg.direct_beam_flux * s / (4.0 * M_PI);
      }
      lu_factor(A.data(), N, N, piv.data());
      lu_solve(A.data(), N, N, piv.data(), x.data());
      for (int iq = 0; iq < NN; ++iq) {
        zb[(size_t)lc * N + NN + iq] = x[iq];
        zb[(size_t)lc * N + NN - iq - 1] = x[iq + NN];
      }
    }
  }

  // Thermal particular solution (computeIsotropicSource, FluxSolver.cpp:745-831)
  z0.assign((size_t)L * N, 0.0); z1.assign((size_t)L * N, 0.0); xr0.assign(L, 0.0); xr1.assign(L, 0.0);
  const bool want_jac = cfg.temperature_jac && cfg.thermal && out.jac[0];
  if (want_jac) {
    for (auto* v : {&dz0t, &dz0b, &dz1t, &dz1b}) v->assign((size_t)L * N, 0.0);
    for (auto* v : {&dxr0t, &dxr0b, &dxr1t, &dxr1b}) v->assign(L, 0.0);
  }
  if (cfg.thermal) {
    std::vector<double> pkag(L + 1), b(N), zz1(N);
    for (int lev = 0; lev <= L; ++lev)
      pkag[lev] = planck_function2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature[lev]);
    for (int lc = 0; lc < L; ++lc) {
      const double* Cl = &C[(size_t)lc * N * N];
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
      for (int i = 0; i < N; ++i) A[i * N + i] += 1.0;
      lu_factor(A.data(), N, N, piv.data());
      double r1 = 0.0;
      if (dtau_s[lc] > 1e-4) r1 = (pkag[lc + 1] - pkag[lc]) / dtau_s[lc];
      const double r0 = pkag[lc] - r1 * tau_s[lc];
      xr0[lc] = r0;
      xr1[lc] = r1;
      for (int i = 0; i < N; ++i) zz1[i] = (1.0 - ssa_s[lc]) * r1;
      lu_solve(A.data(), N, N, piv.data(), zz1.data());
      for (int i = 0; i < N; ++i) b[i] = (1.0 - ssa_s[lc]) * r0 + mu[i] * zz1[i];
      lu_solve(A.data(), N, N, piv.data(), b.data());
      for (int iq = 0; iq < NN; ++iq) {
        z0[(size_t)lc * N + NN + iq] = b[iq];
        z0[(size_t)lc * N + NN - iq - 1] = b[iq + NN];
        z1[(size_t)lc * N + NN + iq] = zz1[iq];
        z1[(size_t)lc * N + NN - iq - 1] = zz1[iq + NN];
      }
      if (want_jac) {
        // d/d(pkag[lc]) and d/d(pkag[lc+1]) with the same factorisation
        // (FluxSolver.cpp:789-829)
        const double omm = 1.0 - ssa_s[lc], tc = tau_s[lc];
        double d1t = 0.0, d1b = 0.0;
        if (dtau_s[lc] > 1e-4) {
          d1t = -1.0 / dtau_s[lc];
          d1b = 1.0 / dtau_s[lc];
        }
        const double d0t = 1.0 - d1t * tc, d0b = -d1b * tc;
        dxr0t[lc] = d0t; dxr0b[lc] = d0b; dxr1t[lc] = d1t; dxr1b[lc] = d1b;
        for (int side = 0; side < 2; ++side) {
          const double d1 = side ? d1b : d1t, d0 = side ? d0b : d0t;
          for (int i = 0; i < N; ++i) zz1[i] = omm * d1;
          lu_solve(A.data(), N, N, piv.data(), zz1.data());
          for (int i = 0; i < N; ++i) b[i] = omm * d0 + mu[i] * zz1[i];
          lu_solve(A.data(), N, N, piv.data(), b.data());
          std::vector<double>& D0 = side ? dz0b : dz0t;
          std::vector<double>& D1 = side ? dz1b : dz1t;
          for (int iq = 0; iq < NN; ++iq) {
            D0[(size_t)lc * N + NN + iq] = b[iq];
            D0[(size_t)lc * N + NN - iq - 1] = b[iq + NN];
            D1[(size_t)lc * N + NN + iq] = zz1[iq];
            D1[(size_t)lc * N + NN - iq - 1] = zz1[iq + NN];
          }
        }
      }
    }
  }

  // setMatrix (FluxSolver.cpp:838-959): LINPACK band storage, lda = 9NN-2
  const int ncd = 3 * NN - 1;
  const int lda = 3 * ncd + 1;
  const int nshift = lda - 2 * N + 1;
  const int ncol_tot = N * L;
  band.assign((size_t)lda * ncol_tot, 0.0);
  auto BM = [&](int r, int c) -> double& { return band[(size_t)c * lda + r]; };
  auto Gv = [&](int lc, int r, int c) { return G[(size_t)lc * N * N + r * N + c]; };
  auto Kv = [&](int lc, int i) { return kk[(size_t)lc * N + i]; };
  int ncol = 0;
  std::vector<double> e(N);
  for (int lc = 0; lc < ncut; ++lc) {
    for (int iq = 0; iq < N; ++iq) e[iq] = 0.0;
    for (int iq = 0; iq < NN; ++iq) e[iq] = std::exp(Kv(lc, iq) * dtau_s[lc]);
    int jcol = 0;
    for (int iq = 0; iq < NN; ++iq) {
      int irow = nshift - jcol - 1;
      for (int jq = 0; jq < N; ++jq) {
        if (irow + N >= 0 && irow + N < lda && ncol < ncol_tot) BM(irow + N, ncol) = Gv(lc, jq, iq);
        if (irow >= 0 && irow < lda && ncol < ncol_tot) BM(irow, ncol) = -Gv(lc, jq, iq) * e[iq];
        irow++;
      }
      ncol++; jcol++;
    }
    for (int iq = NN; iq < N; ++iq) {
      int irow = nshift - jcol - 1;
      for (int jq = 0; jq < N; ++jq) {
        if (irow + N < lda) BM(irow + N, ncol) = Gv(lc, jq, iq) * e[N - iq - 1];
        BM(irow, ncol) = -Gv(lc, jq, iq);
        irow++;
      }
      ncol++; jcol++;
    }
  }
  {
    int jcol = 0;
    for (int iq = 0; iq < NN; ++iq) {
      const double expa = std::exp(Kv(0, iq) * tau_s[1]);
      int irow = nshift - jcol + NN - 1;
      for (int jq = NN - 1; jq >= 0; --jq) { BM(irow, jcol) = Gv(0, jq, iq) * expa; irow++; }
      jcol++;
    }
    for (int iq = NN; iq < N; ++iq) {
      int irow = nshift - jcol + NN - 1;
      for (int jq = NN - 1; jq >= 0; --jq) { BM(irow, jcol) = Gv(0, jq, iq); irow++; }
      jcol++;
    }
    int nncol = ncol - N - 1;
    jcol = 0;
    const int lb = ncut - 1;
    const bool plain_bottom = lyrcut || cfg.diffusion_lower_bc;
    for (int iq = 0; iq < NN; ++iq) {
      nncol++;
      int irow = nshift - jcol + N - 1;
      for (int jq = NN; jq < N; ++jq) {
        if (plain_bottom) BM(irow, nncol) = Gv(lb, jq, iq);
        else {
          double refl = 0.0;
          for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * cfg.surface_albedo * Gv(lb, NN - 1 - k, iq);
          BM(irow, nncol) = Gv(lb, jq, iq) - 2.0 * refl;
        }
        irow++;
      }
      jcol++;
    }
    for (int iq = NN; iq < N; ++iq) {
      nncol++;
      int irow = nshift - jcol + N - 1;
      const double expa = std::exp(Kv(lb, N - iq - 1) * dtau_s[lb]);
      for (int jq = NN; jq < N; ++jq) {
        if (plain_bottom) BM(irow, nncol) = Gv(lb, jq, iq) * expa;
        else {
          double refl = 0.0;
          for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * cfg.surface_albedo * Gv(lb, NN - 1 - k, iq);
          BM(irow, nncol) = (Gv(lb, jq, iq) - 2.0 * refl) * expa;
        }
        irow++;
      }
      jcol++;
    }
  }

  // solve0 (FluxSolver.cpp:966-1131)
  const int nc = N * ncut;
  rhs.assign(nc, 0.0);
  const bool beam = cfg.direct_beam_flux > 0.0;
  auto ZB = [&](int lc, int i) { return zb[(size_t)lc * N + i]; };
  // the beam particular solution of layer lc at scaled depth tau: plane-parallel
  // zb(lc) T (T the transmission at that level), pseudo-spherical
  // exp(-xba tau) (zb + zbs1 tau) (solve0, FluxSolver.cpp:1001-1090)
  const bool sph = cfg.spherical;
  auto ZBT = [&](int lc, int i, double tau, double T) {
    if (sph) return std::exp(-xba[lc] * tau) * (zb[(size_t)lc * N + i] + zbs1[(size_t)lc * N + i] * tau);
    return ZB(lc, i) * T;
  };
  auto Z0 = [&](int lc, int i) { return z0[(size_t)lc * N + i]; };
  auto Z1 = [&](int lc, int i) { return z1[(size_t)lc * N + i]; };
  for (int iq = 0; iq < NN; ++iq) {
    double s = 0.0;
    if (beam) s -= ZB(0, NN - iq - 1);
    if (cfg.thermal) s -= Z0(0, NN - iq - 1);
    s += cfg.isotropic_flux_top + planck_top;
    rhs[iq] = s;
  }
  const int lb = ncut - 1;
  if (cfg.diffusion_lower_bc) {
    for (int iq = 0; iq < NN; ++iq) {
      double s = 0.0;
      if (beam) s -= ZBT(lb, NN + iq, tau_s[ncut], beam_tr[ncut]);
      if (cfg.thermal) { s -= Z0(lb, NN + iq); s -= Z1(lb, NN + iq) * tau_s[ncut]; }
      s += planck_bottom + mu[iq] * planck_bottom_deriv;
      rhs[nc - NN + iq] = s;
    }
  } else {
    for (int iq = 0; iq < NN; ++iq) {
      double s = 0.0;
      if (!lyrcut) {
        double refl = 0.0;
        for (int jq = 0; jq < NN; ++jq) {
          double ps = 0.0;
          if (beam) ps += ZBT(lb, NN - 1 - jq, tau_s[ncut], beam_tr[ncut]);
          if (cfg.thermal) ps += Z0(lb, NN - 1 - jq) + Z1(lb, NN - 1 - jq) * tau_s[ncut];
          refl += wt[jq] * mu[jq] * cfg.surface_albedo * ps;
        }
        s += 2.0 * refl;
      }
      if (beam) {
        s -= ZBT(lb, NN + iq, tau_s[ncut], beam_tr[ncut]);
        if (!lyrcut) s += cfg.surface_albedo * cfg.direct_beam_mu * cfg.direct_beam_flux * beam_tr[ncut] / M_PI;
      }
      if (cfg.thermal) { s -= Z0(lb, NN + iq); s -= Z1(lb, NN + iq) * tau_s[ncut]; }
      s += cfg.isotropic_flux_bottom;
      if (cfg.thermal) s += (1.0 - cfg.surface_albedo) * planck_bottom;
      rhs[nc - NN + iq] = s;
    }
  }
  for (int lc = 1; lc < ncut; ++lc) {
    const int ipnt = lc * N - NN;
    for (int iq = 0; iq < N; ++iq) {
      double s = 0.0;
      if (beam) { s += ZBT(lc, iq, tau_s[lc], beam_tr[lc]); s -= ZBT(lc - 1, iq, tau_s[lc], beam_tr[lc]); }
      if (cfg.thermal) {
        s += Z0(lc, iq) - Z0(lc - 1, iq);
        s += (Z1(lc, iq) - Z1(lc - 1, iq)) * tau_s[lc];
      }
      rhs[ipnt + iq] = s;
    }
  }
  ipvt.assign(nc, 0);
  const bool nonsing = band_factor(band.data(), lda, nc, ncd, ncd, ipvt.data());
  band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), rhs.data());
  cc.assign((size_t)N * L, 0.0);
  for (int lc = 0; lc < ncut; ++lc) {
    const int ipnt = (lc + 1) * N - NN - 1;
    for (int iq = 0; iq < NN; ++iq) {
      const int b_idx = ipnt - iq;
      if (b_idx >= 0 && b_idx < nc) cc[(size_t)lc * N + NN - iq - 1] = rhs[b_idx];
    }
    for (int iq = 0; iq < NN; ++iq) {
      const int b_idx = ipnt + iq + 1;
      if (b_idx >= 0 && b_idx < nc) cc[(size_t)lc * N + NN + iq] = rhs[b_idx];
    }
  }

  // computeFluxes (FluxSolver.cpp:1138-1287)
  double tauc_lu = 0.0;
  std::vector<double> ec(N), inten(N);
  for (int lu = 0; lu <= L; ++lu) {
    int lyu = (lu == 0) ? 0 : lu - 1;
    if (lyrcut && lyu > ncut - 1) {
      out.fdir[lu] = out.fdn[lu] = out.fup[lu] = out.dfdt[lu] = 0.0;
      out.uavg[lu] = out.uavgdn[lu] = out.uavgup[lu] = out.uavgso[lu] = 0.0;
      continue;
    }
    if (lyu >= ncut) lyu = ncut - 1;
    const double utaupr = tau_s[lu];
    double fact = 0.0, dirint = 0.0, fldir = 0.0, fdir = 0.0;
    if (beam) {
      if (sph) {  // FluxSolver.cpp:1184-1188
        const double ch = chap[lyu];
        fact = std::exp(-utaupr / ch);
        fdir = std::abs(cfg.direct_beam_mu) * cfg.direct_beam_flux * std::exp(-tauc_lu / ch);
      } else {
        fact = std::exp(-utaupr / cfg.direct_beam_mu);
        fdir = cfg.direct_beam_mu * cfg.direct_beam_flux * std::exp(-tauc_lu / cfg.direct_beam_mu);
      }
      dirint = cfg.direct_beam_flux * fact;
      fldir = cfg.direct_beam_mu * cfg.direct_beam_flux * fact;
    }
    const double tau_bot = tau_s[lyu + 1], tau_top = tau_s[lyu];
    for (int jq = 0; jq < NN; ++jq) ec[jq] = cc[(size_t)lyu * N + jq] * std::exp(-Kv(lyu, jq) * (utaupr - tau_bot));
    for (int jq = NN; jq < N; ++jq) ec[jq] = cc[(size_t)lyu * N + jq] * std::exp(-Kv(lyu, jq) * (utaupr - tau_top));
    for (int i = 0; i < N; ++i) {
      double s = 0.0;
      for (int j = 0; j < N; ++j) s += Gv(lyu, i, j) * ec[j];
      inten[i] = s;
    }
    if (beam) {
      if (sph) {
        const double be = std::exp(-xba[lyu] * utaupr);
        for (int i = 0; i < N; ++i) inten[i] += be * (ZB(lyu, i) + zbs1[(size_t)lyu * N + i] * utaupr);
      } else {
        for (int i = 0; i < N; ++i) inten[i] += ZB(lyu, i) * fact;
      }
    }
    if (cfg.thermal)
      for (int i = 0; i < N; ++i) inten[i] += Z0(lyu, i) + Z1(lyu, i) * utaupr;
    double ua = 0.0, uad = 0.0, uau = 0.0, fldn = 0.0, fup = 0.0;
    for (int iq = 0; iq < NN; ++iq) {
      const int c = NN - iq - 1;
      ua += wt[c] * inten[iq];
      uad += wt[c] * inten[iq];
      fldn += wt[c] * inten[iq] * mu[c];
    }
    for (int iq = NN; iq < N; ++iq) {
      const int c = iq - NN;
      ua += wt[c] * inten[iq];
      uau += wt[c] * inten[iq];
      fup += wt[c] * inten[iq] * mu[c];
    }
    fup *= 2.0 * M_PI;
    fldn *= 2.0 * M_PI;
    const double fdntot = fldn + fldir;
    const double fdn = fdntot - fdir;
    ua = (2.0 * M_PI * ua + dirint) / (4.0 * M_PI);
    const double uaso = dirint / (4.0 * M_PI);
    uad = (2.0 * M_PI * uad) / (4.0 * M_PI);
    uau = (2.0 * M_PI * uau) / (4.0 * M_PI);
    double plsorc = 0.0;
    if (cfg.thermal) plsorc = xr0[lyu] + xr1[lyu] * utaupr;
    const double dfdt = (1.0 - cfg.ssa[lyu]) * 4.0 * M_PI * (ua - plsorc);
    out.fdir[lu] = fdir; out.fdn[lu] = fdn; out.fup[lu] = fup; out.dfdt[lu] = dfdt;
    out.uavg[lu] = ua; out.uavgdn[lu] = uad; out.uavgup[lu] = uau; out.uavgso[lu] = uaso;
    if (lu < L) tauc_lu += cfg.delta_tau[lu];
  }
  if (out.jac[0]) {
    const int ndof = L + 2;
    for (double* J : out.jac) std::fill(J, J + (size_t)nlev * ndof, 0.0);
    if (want_jac) thermal_jacobian(cfg, out, lda, nc, ncd);
  }
  if (cfg.index_from_bottom) {
    for (double* a : {out.fdir, out.fdn, out.fup, out.dfdt, out.uavg, out.uavgdn, out.uavgup, out.uavgso})
      std::reverse(a, a + nlev);
    // Jacobian rows reversed like the fluxes; level columns reversed, the
    // surface column kept last (IndexConversion.hpp:55-68)
    if (out.jac[0]) {
      const int ndof = L + 2;
      for (double* J : out.jac) {
        for (int r = 0; r < nlev / 2; ++r)
          std::swap_ranges(J + (size_t)r * ndof, J + (size_t)(r + 1) * ndof, J + (size_t)(L - r) * ndof);
        for (int r = 0; r < nlev; ++r) std::reverse(J + (size_t)r * ndof, J + (size_t)r * ndof + L + 1);
      }
    }
  }
  return nonsing ? DSP_OK : DSP_ERR_SINGULAR;
}

// computeThermalJacobian (FluxSolver.cpp:1294-1497): dC = A^{-1} dB for every
// level-Planck degree of freedom k = 0..L and the surface (column L+1), with the
// band LU left by solve0, propagated to the six outputs per level and chained
// with dB/dT (planckFunctionDeriv2).  Fills out.jac (top-down indexing).
inline void FluxOracle::thermal_jacobian(const FluxInstance& cfg, const FluxOutput& out, int lda, int nc,
                                         int ncd) {
  const int ndof = L + 2, surf = L + 1;
  auto at = [&](const std::vector<double>& v, int lc, int iq) { return v[(size_t)lc * N + iq]; };
  auto dz0 = [&](int lc, int iq, int k) {
    double r = 0.0;
    if (k == lc) r += at(dz0t, lc, iq);
    if (k == lc + 1) r += at(dz0b, lc, iq);
    return r;
  };
  auto dz1 = [&](int lc, int iq, int k) {
    double r = 0.0;
    if (k == lc) r += at(dz1t, lc, iq);
    if (k == lc + 1) r += at(dz1b, lc, iq);
    return r;
  };
  auto dintc = [&](int lc, int k) {
    double r = 0.0;
    if (k == lc) r += dxr0t[lc];
    if (k == lc + 1) r += dxr0b[lc];
    return r;
  };
  auto dslp = [&](int lc, int k) {
    double r = 0.0;
    if (k == lc) r += dxr1t[lc];
    if (k == lc + 1) r += dxr1b[lc];
    return r;
  };
  const double dtau_last = dtau_s[L - 1];
  const double tauc_bot = tau_s[ncut];
  jb.assign(nc, 0.0);
  jll.assign((size_t)N * L, 0.0);
  std::vector<double> dexp(N), dval(N);
  auto reorder = [&]() {
    std::fill(jll.begin(), jll.end(), 0.0);
    for (int lc = 0; lc < ncut; ++lc) {
      const int ipnt = (lc + 1) * N - NN - 1;
      for (int iq = 0; iq < NN; ++iq) {
        const int b_idx = ipnt - iq;
        if (b_idx >= 0 && b_idx < nc) jll[(size_t)lc * N + NN - iq - 1] = jb[b_idx];
      }
      for (int iq = 0; iq < NN; ++iq) {
        const int b_idx = ipnt + iq + 1;
        if (b_idx >= 0 && b_idx < nc) jll[(size_t)lc * N + NN + iq] = jb[b_idx];
      }
    }
  };
  auto propagate = [&](int k, int col, double chain) {
    for (int lu = 0; lu <= L; ++lu) {
      int lyu = (lu == 0) ? 0 : lu - 1;
      if (lyrcut && lyu > ncut - 1) continue;
      if (lyu >= ncut) lyu = ncut - 1;
      const double utaupr = tau_s[lu];
      const double tb = tau_s[lyu + 1], tt = tau_s[lyu];
      for (int jq = 0; jq < NN; ++jq) dexp[jq] = jll[(size_t)lyu * N + jq] * std::exp(-kk[(size_t)lyu * N + jq] * (utaupr - tb));
      for (int jq = NN; jq < N; ++jq) dexp[jq] = jll[(size_t)lyu * N + jq] * std::exp(-kk[(size_t)lyu * N + jq] * (utaupr - tt));
      for (int i = 0; i < N; ++i) {
        double sacc = 0.0;
        for (int j = 0; j < N; ++j) sacc += G[(size_t)lyu * N * N + i * N + j] * dexp[j];
        dval[i] = sacc;
      }
      if (k >= 0)
        for (int iq = 0; iq < N; ++iq) dval[iq] += dz0(lyu, iq, k) + dz1(lyu, iq, k) * utaupr;
      double dmi = 0.0, dmidn = 0.0, dmiup = 0.0, dfdn = 0.0, dfup = 0.0;
      for (int iq = 0; iq < NN; ++iq) {
        const int c = NN - iq - 1;
        const double v = dval[iq], w = wt[c];
        dmi += w * v; dmidn += w * v; dfdn += w * v * mu[c];
      }
      for (int iq = NN; iq < N; ++iq) {
        const int c = iq - NN;
        const double v = dval[iq], w = wt[c];
        dmi += w * v; dmiup += w * v; dfup += w * v * mu[c];
      }
      dfup *= 2.0 * M_PI;
      dfdn *= 2.0 * M_PI;
      const double dmi_t = (2.0 * M_PI * dmi) / (4.0 * M_PI);
      const double dmi_d = (2.0 * M_PI * dmidn) / (4.0 * M_PI);
      const double dmi_u = (2.0 * M_PI * dmiup) / (4.0 * M_PI);
      double dpls = 0.0;
      if (k >= 0) dpls = dintc(lyu, k) + dslp(lyu, k) * utaupr;
      const double dfdiv = (1.0 - cfg.ssa[lyu]) * 4.0 * M_PI * (dmi_t - dpls);
      const size_t o = (size_t)lu * ndof + col;
      out.jac[0][o] = chain * dfup;
      out.jac[1][o] = chain * dfdn;
      out.jac[2][o] = chain * dmi_t;
      out.jac[3][o] = chain * dmi_d;
      out.jac[4][o] = chain * dmi_u;
      out.jac[5][o] = chain * dfdiv;
    }
  };
  const double alb = cfg.surface_albedo;
  for (int k = 0; k <= L; ++k) {
    std::fill(jb.begin(), jb.end(), 0.0);
    for (int iq = 0; iq < NN; ++iq) jb[iq] = -dz0(0, NN - 1 - iq, k);
    if (cfg.diffusion_lower_bc) {
      for (int iq = 0; iq < NN; ++iq) {
        double sacc = -dz0(ncut - 1, NN + iq, k) - dz1(ncut - 1, NN + iq, k) * tauc_bot;
        if (k == L - 1 && dtau_last > 0.0) sacc += mu[iq] * (-1.0 / dtau_last);
        jb[nc - NN + iq] = sacc;
      }
    } else {
      for (int iq = 0; iq < NN; ++iq) {
        double sacc = 0.0;
        if (!lyrcut) {
          double refl = 0.0;
          for (int jq = 0; jq < NN; ++jq) {
            const double ps = dz0(ncut - 1, NN - 1 - jq, k) + dz1(ncut - 1, NN - 1 - jq, k) * tauc_bot;
            refl += wt[jq] * mu[jq] * alb * ps;
          }
          sacc += 2.0 * refl;
        }
        sacc -= dz0(ncut - 1, NN + iq, k) + dz1(ncut - 1, NN + iq, k) * tauc_bot;
        jb[nc - NN + iq] = sacc;
      }
    }
    for (int lc = 1; lc < ncut; ++lc) {
      const int ipnt = lc * N - NN;
      const double tc = tau_s[lc];
      for (int iq = 0; iq < N; ++iq)
        jb[ipnt + iq] = dz0(lc, iq, k) - dz0(lc - 1, iq, k) + (dz1(lc, iq, k) - dz1(lc - 1, iq, k)) * tc;
    }
    band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), jb.data());
    reorder();
    propagate(k, k, planck_function_deriv2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature[k]));
  }
  // surface degree of freedom: the emission (1 - albedo) B(T_bottom), or the
  // diffusion boundary's B and its gradient
  std::fill(jb.begin(), jb.end(), 0.0);
  for (int iq = 0; iq < NN; ++iq) {
    double sacc;
    if (cfg.diffusion_lower_bc) {
      sacc = 1.0;
      if (dtau_last > 0.0) sacc += mu[iq] * (1.0 / dtau_last);
    } else {
      sacc = 1.0 - alb;  // Lambertian emissivity (FluxSolver.cpp:147-154)
    }
    jb[nc - NN + iq] = sacc;
  }
  band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), jb.data());
  reorder();
  propagate(-1, surf, planck_function_deriv2(cfg.wavenumber_low, cfg.wavenumber_high, cfg.temperature_bottom));
}

}  // namespace oracle
