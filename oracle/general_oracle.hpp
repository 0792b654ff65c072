// general_oracle.hpp — CPU restatement of DisortSolver::solve
// (src/DisortSolver.cpp:21-399 of DisORT++) for plane-parallel geometry and a
// Lambertian or bidirectional (BRDF) surface, without intensity corrections: delta-M / delta-M+,
// Fourier azimuth modes, fluxes at user optical depths and intensities at user
// polar angles and azimuths.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Never linked into the product.
#pragma once

#include <vector>

#include "flux_oracle.hpp"

namespace oracle {

struct GeneralInstance {
  int L = 0, N = 0, nmom = 0, pc = 0;
  bool thermal = false, dmplus = false, dlbc = false, ifb = false;
  bool user_tau = false, user_mu = false, only_fluxes = false;
  bool temperature_jac = false;  // compute_temperature_jacobian
  bool spherical = false;        // use_spherical_beam
  double radius = 0.0;           // bottom_radius
  const double* zalt = nullptr;  // level_altitudes [L+1] (spherical only)
  double accur = 0.0;
  bool special = false;          // ibcnd = Special: albedo and transmissivity of the medium
  bool corr = false;             // intensity_corr_buras
  bool corr_be = false;          // ... with the Buras-Emde method (tabulated phase function)
  int nangles = 0;               // num_phase_func_angles
  const double* mup = nullptr;   // mu_phase_function [nangles], increasing
  const double* phasef = nullptr;  // phase_function [L][nangles]
  int brdf = 0;                  // 0: Lambertian; else the BrdfType (RPV 1, CoxMunk 2, Ambrals 3, Hapke 4)
  const double* bp = nullptr;    // its parameters (SurfaceTables, oracle_common.hpp)
  double wlo = 0, whi = 0, alb = 0, emis = 1, fbeam = 0, umu0 = 0.5, phi0 = 0, fisot = 0, fisob = 0, ttop = 0, tbot = 0;
  const double *dtau = nullptr, *ssa = nullptr, *pmom = nullptr, *temp = nullptr;
  int ntau = 0, numu = 0, nphi = 0;
  const double *utau = nullptr, *umu = nullptr, *phi = nullptr;
};

struct GeneralOutput {
  double* flux[8];   // [ntau_out]
  double* intensity; // [ntau_out][numu_out][nphi]
  double* iavg;      // [ntau_out][numu_out]
  int ntau_out = 0, numu_out = 0;
  // temperature Jacobians (DisortResult *_temperature_jac), each [ntau_out][jac_stride]
  // or null: flux_up, flux_down, mean_intensity, _down, _up, flux_divergence
  double* jac[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int jac_stride = 0;
  // ibcnd = Special: albedo_medium, transmissivity_medium [numu_half] and the
  // spherical albedo and transmissivity [1] each
  double* albtrans[4] = {nullptr, nullptr, nullptr, nullptr};
};

// DisortConfig::validate (DisortConfig.cpp:72-249) for the fields carried here,
// in the reference's order and with its comparisons (a NaN passes where the
// reference's test lets it pass).
inline int validate_general(const GeneralInstance& c) {
  if (c.L <= 0 || c.N < 4 || c.N % 2 != 0 || c.nmom < 0) return DSP_ERR_INVALID_INPUT;
  if (c.pc < std::max(c.nmom, c.N) + 1) return DSP_ERR_INVALID_INPUT;
  for (int lc = 0; lc < c.L; ++lc) {
    if (c.dtau[lc] < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.ssa[lc] < 0.0 || c.ssa[lc] > 1.0) return DSP_ERR_INVALID_INPUT;
  }
  if (c.thermal) {
    if (!c.temp) return DSP_ERR_INVALID_INPUT;
    for (int lev = 0; lev <= c.L; ++lev)
      if (c.temp[lev] < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.wlo < 0.0 || c.whi < c.wlo) return DSP_ERR_INVALID_INPUT;
  }
  if (c.dlbc && !c.thermal) return DSP_ERR_INVALID_INPUT;
  if (c.dlbc && c.brdf != BRDF_LAMBERT) return DSP_ERR_INVALID_INPUT;  // DisortConfig.cpp:144-146
  if (c.fbeam < 0.0) return DSP_ERR_INVALID_INPUT;
  if ((c.umu0 <= 0.0 || c.umu0 > 1.0) && c.fbeam > 0.0) return DSP_ERR_INVALID_INPUT;
  if (c.brdf == BRDF_LAMBERT && (c.alb < 0.0 || c.alb > 1.0)) return DSP_ERR_INVALID_INPUT;
  if (c.user_mu) {
    if (c.numu <= 0 || !c.umu) return DSP_ERR_INVALID_INPUT;
    for (int iu = 0; iu < c.numu; ++iu) {
      if (std::abs(c.umu[iu]) > 1.0) return DSP_ERR_INVALID_INPUT;
      if (iu > 0 && c.umu[iu] <= c.umu[iu - 1]) return DSP_ERR_INVALID_INPUT;
    }
  }
  if (!c.only_fluxes && !c.special) {  // DisortConfig.cpp:200
    if (c.nphi <= 0 || !c.phi) return DSP_ERR_INVALID_INPUT;
    for (int j = 0; j < c.nphi; ++j)
      if (c.phi[j] < 0.0 || c.phi[j] > 360.0) return DSP_ERR_INVALID_INPUT;
  }
  if (c.spherical && (c.radius <= 0.0 || !c.zalt)) return DSP_ERR_INVALID_INPUT;
  if (c.dmplus && c.nmom < c.N + 1) return DSP_ERR_INVALID_INPUT;
  if (c.accur < 0.0) return DSP_ERR_INVALID_INPUT;
  if (c.thermal) {
    if (c.wlo < 0.0 || c.whi <= c.wlo) return DSP_ERR_INVALID_INPUT;
    if (c.ttop < 0.0 || c.tbot < 0.0) return DSP_ERR_INVALID_INPUT;
    if (c.emis < 0.0 || c.emis > 1.0) return DSP_ERR_INVALID_INPUT;
  }
  // boundary of the C ABI: user optical depths must be given when requested
  if (c.user_tau && (c.ntau <= 0 || !c.utau)) return DSP_ERR_INVALID_INPUT;
  return DSP_OK;
}

// xiFunc (DisortSolver.cpp:3274-3285), eq. STWL (72)
inline double nt_xi(double umu1, double umu2, double tau) {
  const double x1 = (umu2 - umu1) / (umu2 * umu1);
  const double exp1 = std::exp(-tau / umu1);
  if (x1 != 0.0) return ((tau * x1 - 1.0) * std::exp(-tau / umu2) + exp1) / (x1 * x1 * umu1 * umu2);
  return tau * tau * exp1 / (2.0 * umu1 * umu2);
}

// singleScat (DisortSolver.cpp:3287-3328): the single-scattered intensity of
// the beam at scaled depth tau_user, eqs. STWL (65b,d,e).  phase, omega are
// 1-based over layers; tau is the cumulative scaled depth at the levels.
inline double nt_single_scat(double dither, int layru, int nl, const double* phase, const double* omega,
                             const double* tau, double umu, double umu0, double tau_user, double fbeam) {
  const double four_pi = 4.0 * M_PI;
  double ans = 0.0, exp0 = std::exp(-tau_user / umu0);
  if (std::abs(umu + umu0) <= dither) {
    for (int lyr = 1; lyr <= layru - 1; ++lyr) ans += omega[lyr] * phase[lyr] * (tau[lyr] - tau[lyr - 1]);
    return fbeam / (four_pi * umu0) * exp0 * (ans + omega[layru] * phase[layru] * (tau_user - tau[layru - 1]));
  }
  if (umu > 0.0) {
    for (int lyr = layru; lyr <= nl; ++lyr) {
      const double exp1 = std::exp(-((tau[lyr] - tau_user) / umu + tau[lyr] / umu0));
      ans += omega[lyr] * phase[lyr] * (exp0 - exp1);
      exp0 = exp1;
    }
  } else {
    for (int lyr = layru; lyr >= 1; --lyr) {
      const double exp1 = std::exp(-((tau[lyr - 1] - tau_user) / umu + tau[lyr - 1] / umu0));
      ans += omega[lyr] * phase[lyr] * (exp0 - exp1);
      exp0 = exp1;
    }
  }
  return ans * fbeam / (four_pi * (1.0 + umu / umu0));
}

// applyIntensityCorrection (DisortSolver.cpp:3403-3530) with secondaryScat
// (:3330-3401): Nakajima-Tanaka TMS (exact single scattering in place of the
// delta-M one) and IMS (secondary scattering in the aureole of the beam).
// pm: unscaled moments [L][pc] (moment 0 = 1); I3(lu, iu, j) the intensities.
template <class Acc>
inline void nakajima_tanaka(const GeneralInstance& c, int ncut, bool lyrcut, int numu, int nphi, int ntau,
                            const std::vector<double>& umu, const std::vector<double>& utau,
                            const std::vector<double>& utaus, const std::vector<int>& lyr,
                            const std::vector<double>& tauc, const std::vector<double>& taus,
                            const std::vector<double>& fsc, const std::vector<double>& ws,
                            const std::vector<double>& pm, Acc&& I3) {
  const int N = c.N, nmom = c.nmom, pc = c.pc;
  auto PM = [&](int k, int lc) { return pm[(size_t)lc * pc + k]; };
  const double dither = 100.0 * std::numeric_limits<double>::epsilon();
  const double dtheta = 10.0, deg = std::acos(-1.0) / 180.0, tiny = 1.0e-4;
  std::vector<double> phasa(ncut + 1), phasm(ncut + 1), phast(ncut + 1), ssa1(ncut + 1), opr1(ncut + 1);
  for (int lc = 1; lc <= ncut; ++lc) {
    ssa1[lc] = c.ssa[lc - 1];
    opr1[lc] = ws[lc - 1];
  }
  // secondaryScat: the IMS term of eq. STWL (A.13) at output depth lu
  auto secondary = [&](int iu, int lu, double ctheta, int layru) {
    const double ut = utau[lu];
    double dtau = ut - tauc[layru];
    double wbar = c.ssa[layru] * dtau;
    double fbar = fsc[layru] * wbar;
    double stau = dtau;
    for (int l = 0; l < layru; ++l) {
      wbar += c.dtau[l] * c.ssa[l];
      fbar += c.dtau[l] * c.ssa[l] * fsc[l];
      stau += c.dtau[l];
    }
    if (wbar <= tiny || fbar <= tiny || stau <= tiny || c.fbeam <= tiny) return 0.0;
    fbar /= wbar;
    wbar /= stau;
    double pspike = 1.0, gbar = 1.0, plm1 = 1.0, plm2 = 0.0;
    for (int k = 1; k <= N - 1; ++k) {
      const double pl = ((2 * k - 1) * ctheta * plm1 - (k - 1) * plm2) / k;
      plm2 = plm1;
      plm1 = pl;
      pspike += gbar * (2.0 - gbar) * (double)(2 * k + 1) * pl;
    }
    for (int k = N; k <= nmom; ++k) {
      const double pl = ((2 * k - 1) * ctheta * plm1 - (k - 1) * plm2) / k;
      plm2 = plm1;
      plm1 = pl;
      dtau = ut - tauc[layru];
      gbar = PM(k, layru) * c.ssa[layru] * dtau;
      for (int l = 0; l < layru; ++l) gbar += PM(k, l) * c.ssa[l] * c.dtau[l];
      const double tmp = fbar * wbar * stau;
      gbar = tmp <= tiny ? 0.0 : gbar / tmp;
      pspike += gbar * (2.0 - gbar) * (double)(2 * k + 1) * pl;
    }
    const double umu0p = c.umu0 / (1.0 - fbar * wbar);
    return c.fbeam / (4.0 * M_PI) * (fbar * wbar) * (fbar * wbar) / (1.0 - fbar * wbar) * pspike *
           nt_xi(-umu[iu], umu0p, ut);
  };
  for (int iu = 0; iu < numu; ++iu) {
    double theta0 = 0.0, thetap = 0.0;
    if (umu[iu] < 0.0) {
      theta0 = std::acos(-c.umu0) / deg;
      thetap = std::acos(umu[iu]) / deg;
    }
    for (int jp = 0; jp < nphi; ++jp) {
      const double phirad = (c.phi[jp] - c.phi0) * deg;
      const double ctheta =
          -c.umu0 * umu[iu] + std::sqrt((1.0 - c.umu0 * c.umu0) * (1.0 - umu[iu] * umu[iu])) * std::cos(phirad);
      for (int lc = 1; lc <= ncut; ++lc) phasa[lc] = phasm[lc] = 1.0;
      double plm1 = 1.0, plm2 = 0.0;
      for (int k = 1; k <= nmom; ++k) {
        const double pl = ((2 * k - 1) * ctheta * plm1 - (k - 1) * plm2) / k;
        plm2 = plm1;
        plm1 = pl;
        for (int lc = 1; lc <= ncut; ++lc) phasa[lc] += (double)(2 * k + 1) * pl * PM(k, lc - 1);
        if (k <= N - 1)
          for (int lc = 1; lc <= ncut; ++lc) {
            const double fl = fsc[lc - 1];
            phasm[lc] += (double)(2 * k + 1) * pl * (PM(k, lc - 1) - fl) / (1.0 - fl);
          }
      }
      for (int lc = 1; lc <= ncut; ++lc) phast[lc] = phasa[lc] / (1.0 - fsc[lc - 1] * c.ssa[lc - 1]);
      for (int lu = 0; lu < ntau; ++lu) {
        if (lyrcut && lyr[lu] >= ncut) continue;
        const double exact = nt_single_scat(dither, lyr[lu] + 1, ncut, phast.data(), ssa1.data(), taus.data(),
                                            umu[iu], c.umu0, utaus[lu], c.fbeam);
        const double scaled = nt_single_scat(dither, lyr[lu] + 1, ncut, phasm.data(), opr1.data(), taus.data(),
                                             umu[iu], c.umu0, utaus[lu], c.fbeam);
        I3(lu, iu, jp) += exact - scaled;
      }
      if (umu[iu] < 0.0 && std::abs(theta0 - thetap) <= dtheta) {
        const int ltau = utau[0] <= dither ? 1 : 0;
        for (int lu = ltau; lu < ntau; ++lu) {
          if (lyrcut && lyr[lu] >= ncut) continue;
          I3(lu, iu, jp) -= secondary(iu, lu, ctheta, lyr[lu]);
        }
      }
    }
  }
}

// locate (Utils.hpp:27-64): j with xx[j] <= x < xx[j+1] by bisection, 0 at
// xx[0] and below, n-2 at xx[n-1]
inline int be_locate(const double* xx, int n, double x) {
  if (n <= 0) return -1;
  if (n == 1) return 0;
  const bool inc = xx[1] > xx[0];
  int jl = 0, ju = n;
  while (ju - jl > 1) {
    const int jm = (ju + jl) >> 1;
    if ((x >= xx[jm] && inc) || (x <= xx[jm] && !inc)) jl = jm;
    else ju = jm;
  }
  if (x == xx[0]) return 0;
  if (x == xx[n - 1]) return n - 2;
  return jl;
}

// calcPhaseSquared (DisortSolver.cpp:3932-4023): the azimuthal integral of
// P''(mu_1) P''(theta_12) over the grid mu_eq equidistant in |P''|; arrays of
// output depth lu: p2[nangles], mueq[nf], neg[nf]
inline double be_phase_squared(int na, const double* mup, const double* p2, double ctheta, int nf,
                               const double* mueq, const int* neg, double norm) {
  double pspike2 = 0.0;
  const double st = std::sqrt(1.0 - ctheta * ctheta);
  for (int j = 0; j < nf; ++j) {
    const double me = mueq[j];
    double phint;
    if (ctheta == 1.0 || me == 1.0) {
      const int i2 = be_locate(mup, na, me * ctheta);
      phint = M_PI * (p2[i2] + (me * ctheta - mup[i2]) / (mup[i2 + 1] - mup[i2]) * (p2[i2 + 1] - p2[i2]));
      if (ctheta == 1.0) phint /= 2.0;
    } else {
      phint = 0.0;
      const double sm = std::sqrt(1.0 - me * me);
      double mumin = ctheta * me - st * sm, mumax = ctheta * me + st * sm;
      bool cutting = false;
      if (me < mumax) {
        mumax = me;
        cutting = true;
      }
      if (mumin < mumax) {
        const int imin = be_locate(mup, na, mumin), imax = be_locate(mup, na, mumax);
        int k = imin;
        double D = (p2[k + 1] - p2[k]) / (mup[k + 1] - mup[k]);
        double C = p2[k] - mup[k] * D;
        phint += (D * ctheta * me + C) * M_PI / 2.0;
        for (k = imin + 1; k <= imax; ++k) {
          const double Dp = (p2[k + 1] - p2[k]) / (mup[k + 1] - mup[k]);
          const double Cp = p2[k] - mup[k] * Dp;
          phint += (Dp - D) * std::sqrt(1.0 - ctheta * ctheta - me * me + 2.0 * ctheta * me * mup[k] - mup[k] * mup[k]) +
                   ((Dp - D) * ctheta * me + Cp - C) * std::asin((ctheta * me - mup[k]) / (sm * st));
          D = Dp;
          C = Cp;
        }
        if (cutting)
          phint += -D * std::sqrt(1.0 - ctheta * ctheta + 2.0 * me * me * (ctheta - 1.0)) -
                   (D * ctheta * me + C) * std::asin((ctheta - 1.0) * me / (sm * st));
        else
          phint += (D * ctheta * me + C) * M_PI / 2.0;
      }
    }
    const double w = (j == 0 || j == nf - 1) ? 0.5 : 1.0;
    pspike2 += (neg[j] ? -w : w) * phint;
  }
  return pspike2 * norm;
}

// applyNewIntensityCorrection (DisortSolver.cpp:3532-3749) with
// prepDoubleScatIntegr (:3812-3876) and newSecondaryScat (:3878-3930): the
// Buras-Emde correction, TMS from the tabulated phase function and IMS from
// the residual phase function P'' of the truncated peak and its square.
template <class Acc>
inline void buras_emde(const GeneralInstance& c, int ncut, bool lyrcut, int numu, int nphi, int ntau,
                       const std::vector<double>& umu, const std::vector<double>& utau,
                       const std::vector<double>& utaus, const std::vector<int>& lyr,
                       const std::vector<double>& tauc, const std::vector<double>& taus,
                       const std::vector<double>& fsc, const std::vector<double>& ws,
                       const std::vector<double>& pm, Acc&& I3) {
  const int N = c.N, L = c.L, na = c.nangles, pc = c.pc, nf = 100;
  auto PM = [&](int k, int lc) { return pm[(size_t)lc * pc + k]; };
  auto PF = [&](int lc, int it) { return c.phasef[(size_t)lc * na + it]; };
  const double* mup = c.mup;
  const double dither = 100.0 * std::numeric_limits<double>::epsilon();
  const double dtheta = 10.0, tiny = 1.0e-4, deg = M_PI / 180.0;
  bool need2 = false;
  for (int iu = 0; iu < numu; ++iu)
    if (umu[iu] < 0.0 && std::fabs(std::acos(-c.umu0) / deg - std::acos(umu[iu]) / deg) <= dtheta) need2 = true;
  std::vector<double> p2((size_t)na * ntau, 0.0), mueq, normp;
  std::vector<int> negp;
  auto P2 = [&](int it, int lu) -> double& { return p2[(size_t)lu * na + it]; };
  if (need2) {
    mueq.assign((size_t)nf * ntau, 0.0);
    negp.assign((size_t)nf * ntau, 0);
    normp.assign(ntau, 0.0);
    std::vector<double> phasr(L);
    for (int it = 0; it < na; ++it) {
      const double ct = mup[it];
      for (int lc = 0; lc < L; ++lc) phasr[lc] = 1.0 - fsc[lc];
      double plm1 = 1.0, plm2 = 0.0;
      for (int k = 1; k <= N - 1; ++k) {
        const double pl = ((2 * k - 1) * ct * plm1 - (k - 1) * plm2) / k;
        plm2 = plm1;
        plm1 = pl;
        for (int lc = 0; lc < L; ++lc) phasr[lc] += (2 * k + 1) * pl * (PM(k, lc) - fsc[lc]);
      }
      for (int lu = 0; lu < ntau; ++lu) {
        double v = 0.0;
        const int ll = lyr[lu];
        for (int l = 0; l < ll; ++l) v += (PF(l, it) - phasr[l]) * c.ssa[l] * c.dtau[l];
        v += (PF(ll, it) - phasr[ll]) * c.ssa[ll] * (utau[lu] - tauc[ll]);
        P2(it, lu) = v;
      }
    }
    for (int lu = 0; lu < ntau; ++lu) {
      const int ll = lyr[lu];
      double fbar = fsc[ll] * c.ssa[ll] * (utau[lu] - tauc[ll]);
      for (int l = 0; l < ll; ++l) fbar += c.ssa[l] * c.dtau[l] * fsc[l];
      if (fbar <= tiny || c.fbeam <= tiny) {
        for (int it = 0; it < na; ++it) P2(it, lu) = 0.0;
      } else {
        fbar = 1.0 / fbar;
        for (int it = 0; it < na; ++it) P2(it, lu) *= fbar;
      }
      double f2 = 0.0;
      for (int it = 1; it < na; ++it) f2 += (mup[it] - mup[it - 1]) * 0.5 * (P2(it, lu) + P2(it - 1, lu));
      if (f2 != 0.0) {
        const double norm = 2.0 / f2;
        for (int it = 0; it < na; ++it) P2(it, lu) *= norm;
      }
    }
    // prepDoubleScatIntegr
    std::vector<double> fabs2(na);
    for (int lu = 0; lu < ntau; ++lu) {
      double* me = &mueq[(size_t)lu * nf];
      int* ng = &negp[(size_t)lu * nf];
      fabs2[0] = 0.0;
      for (int it = 1; it < na; ++it)
        fabs2[it] = fabs2[it - 1] + (mup[it] - mup[it - 1]) * 0.5 * (std::fabs(P2(it, lu)) + std::fabs(P2(it - 1, lu)));
      double f = 0.0;
      const double df = fabs2[na - 1] / (nf - 1);
      me[0] = -1.0;
      ng[0] = P2(0, lu) > 0.0 ? 0 : 1;
      int it = 0;
      for (int q = 1; q < nf - 1; ++q) {
        f += df;
        while (fabs2[it + 1] < f) ++it;
        me[q] = mup[it] + (f - fabs2[it]) / (fabs2[it + 1] - fabs2[it]) * (mup[it + 1] - mup[it]);
        if (P2(it, lu) > 0.0 && P2(it + 1, lu) > 0.0) ng[q] = 0;
        else if (P2(it, lu) < 0.0 && P2(it + 1, lu) < 0.0) ng[q] = 1;
        else {
          const double val = P2(it, lu) + (f - fabs2[it]) / (fabs2[it + 1] - fabs2[it]) * (P2(it + 1, lu) - P2(it, lu));
          ng[q] = val > 0.0 ? 0 : 1;
        }
      }
      me[nf - 1] = 1.0;
      ng[nf - 1] = P2(na - 1, lu) > 0.0 ? 0 : 1;
      normp[lu] = fabs2[na - 1] / ((nf - 1) * M_PI);
    }
  }
  std::vector<double> phasm(ncut + 1), phast(ncut + 1), ssa1(ncut + 1), opr1(ncut + 1);
  for (int lc = 1; lc <= ncut; ++lc) {
    ssa1[lc] = c.ssa[lc - 1];
    opr1[lc] = ws[lc - 1];
  }
  for (int iu = 0; iu < numu; ++iu) {
    double theta0 = 0.0, thetap = 0.0;
    if (umu[iu] < 0.0) {
      theta0 = std::acos(-c.umu0) / deg;
      thetap = std::acos(umu[iu]) / deg;
    }
    for (int jp = 0; jp < nphi; ++jp) {
      const double phirad = (c.phi[jp] - c.phi0) * deg;
      const double ctheta =
          -c.umu0 * umu[iu] + std::sqrt((1.0 - c.umu0 * c.umu0) * (1.0 - umu[iu] * umu[iu])) * std::cos(phirad);
      for (int lc = 1; lc <= ncut; ++lc) phasm[lc] = 1.0;
      const int it = be_locate(mup, na, ctheta);
      for (int lc = 1; lc <= ncut; ++lc) {
        const double phasa = PF(lc - 1, it) + (ctheta - mup[it]) / (mup[it + 1] - mup[it]) * (PF(lc - 1, it + 1) - PF(lc - 1, it));
        phast[lc] = phasa / (1.0 - fsc[lc - 1] * c.ssa[lc - 1]);
      }
      double plm1 = 1.0, plm2 = 0.0;
      for (int k = 1; k <= N - 1; ++k) {
        const double pl = ((2 * k - 1) * ctheta * plm1 - (k - 1) * plm2) / k;
        plm2 = plm1;
        plm1 = pl;
        for (int lc = 1; lc <= ncut; ++lc)
          phasm[lc] += (2.0 * k + 1) * pl * (PM(k, lc - 1) - fsc[lc - 1]) / (1.0 - fsc[lc - 1]);
      }
      for (int lu = 0; lu < ntau; ++lu) {
        if (lyrcut && lyr[lu] >= ncut) continue;
        const double exact = nt_single_scat(dither, lyr[lu] + 1, ncut, phast.data(), ssa1.data(), taus.data(),
                                            umu[iu], c.umu0, utaus[lu], c.fbeam);
        const double scaled = nt_single_scat(dither, lyr[lu] + 1, ncut, phasm.data(), opr1.data(), taus.data(),
                                             umu[iu], c.umu0, utaus[lu], c.fbeam);
        I3(lu, iu, jp) += exact - scaled;
      }
      if (umu[iu] < 0.0 && std::abs(theta0 - thetap) <= dtheta) {
        const int ltau = utau[0] <= dither ? 1 : 0;
        for (int lu = ltau; lu < ntau; ++lu) {
          if (lyrcut && lyr[lu] >= ncut) continue;
          // newSecondaryScat
          const int layru = lyr[lu];
          const double ut = utau[lu];
          double dt = ut - tauc[layru];
          double wbar = c.ssa[layru] * dt, fbar = fsc[layru] * wbar, stau = dt;
          for (int l = 0; l < layru; ++l) {
            wbar += c.dtau[l] * c.ssa[l];
            fbar += c.dtau[l] * c.ssa[l] * fsc[l];
            stau += c.dtau[l];
          }
          if (wbar <= tiny || fbar <= tiny || stau <= tiny || c.fbeam <= tiny) continue;
          fbar /= wbar;
          wbar /= stau;
          const double ps1 = P2(it, lu) + (ctheta - mup[it]) / (mup[it + 1] - mup[it]) * (P2(it + 1, lu) - P2(it, lu));
          const double ps2 = be_phase_squared(na, mup, &p2[(size_t)lu * na], ctheta, nf, &mueq[(size_t)lu * nf],
                                              &negp[(size_t)lu * nf], normp[lu]);
          const double pspike = 2.0 * ps1 - ps2;
          const double umu0p = c.umu0 / (1.0 - fbar * wbar);
          I3(lu, iu, jp) -= c.fbeam / (4.0 * M_PI) * (fbar * wbar) * (fbar * wbar) / (1.0 - fbar * wbar) * pspike *
                            nt_xi(-umu[iu], umu0p, ut);
        }
      }
    }
  }
}

class GeneralOracle {
 public:
  int solve(const GeneralInstance& in, const GeneralOutput& out);
};

inline int GeneralOracle::solve(const GeneralInstance& cin, const GeneralOutput& out) {
  GeneralInstance c = cin;
  const int L = c.L, N = c.N, NN = N / 2;
  std::vector<double> rdt, rss, rpm, rtp, rut, rza, rpf;
  if (c.ifb) {  // reverseInputArrays (IndexConversion.hpp:16-40)
    rdt.assign(c.dtau, c.dtau + L);
    rss.assign(c.ssa, c.ssa + L);
    std::reverse(rdt.begin(), rdt.end());
    std::reverse(rss.begin(), rss.end());
    rpm.resize((size_t)L * c.pc);
    for (int lc = 0; lc < L; ++lc)
      std::memcpy(&rpm[(size_t)lc * c.pc], c.pmom + (size_t)(L - 1 - lc) * c.pc, sizeof(double) * c.pc);
    c.dtau = rdt.data();
    c.ssa = rss.data();
    c.pmom = rpm.data();
    if (c.phasef && c.nangles > 0) {
      rpf.resize((size_t)L * c.nangles);
      for (int lc = 0; lc < L; ++lc)
        std::memcpy(&rpf[(size_t)lc * c.nangles], c.phasef + (size_t)(L - 1 - lc) * c.nangles,
                    sizeof(double) * c.nangles);
      c.phasef = rpf.data();
    }
    if (c.temp) {
      rtp.assign(c.temp, c.temp + L + 1);
      std::reverse(rtp.begin(), rtp.end());
      c.temp = rtp.data();
    }
    if (c.zalt) {
      rza.assign(c.zalt, c.zalt + L + 1);
      std::reverse(rza.begin(), rza.end());
      c.zalt = rza.data();
    }
    if (c.user_tau && c.utau && c.ntau > 0) {
      // the column total and the converted depths rounded to double at every
      // step, as the reference computes them: the extended-precision build
      // would otherwise turn a user depth equal to the total into a tiny
      // negative depth above the top of the column
      volatile double total = 0.0;
      for (int lc = 0; lc < L; ++lc) total = total + c.dtau[lc];
      rut.assign(c.utau, c.utau + c.ntau);
      for (auto& t : rut) {
        volatile double v = total - t;
        t = v;
      }
      std::reverse(rut.begin(), rut.end());
      c.utau = rut.data();
    }
  }
  if (int st = validate_general(c)) return st;
  // ibcnd = Special (computeAlbTrans, DisortSolver.cpp:4025-4163): isotropic
  // illumination of unit intensity from the top (and the bottom), no other
  // source, a black surface in the boundary-value problem; the user angles
  // become [-mu reversed | +mu] (DisortSolver.cpp:52-58, 852-865)
  const double special_alb = c.alb;
  std::vector<double> sp_umu;
  if (c.special) {
    c.fbeam = 0.0;
    c.thermal = false;
    c.spherical = false;
    c.fisot = 1.0;
    c.fisob = 0.0;
    c.alb = 0.0;
    c.brdf = BRDF_LAMBERT;
    c.corr = false;
    c.user_tau = false;
    c.only_fluxes = false;
    c.temperature_jac = false;
    if (c.user_mu) {
      sp_umu.resize(2 * c.numu);
      for (int iu = 0; iu < c.numu; ++iu) {
        sp_umu[c.numu + iu] = c.umu[iu];
        sp_umu[iu] = -c.umu[c.numu - 1 - iu];
      }
      c.umu = sp_umu.data();
      c.numu *= 2;
    }
  }
  const int ntau = c.user_tau ? c.ntau : L + 1;
  const bool do_int = (!c.only_fluxes && c.user_mu) || c.special;
  const int numu = (c.user_mu && !c.only_fluxes) ? c.numu : N;
  const int nphi = c.nphi;
  const int pc = c.pc;
  // pmom with P_0 = 1 (the reference sets it, DisortSolver.cpp:669)
  std::vector<double> pm(c.pmom, c.pmom + (size_t)L * pc);
  for (int lc = 0; lc < L; ++lc) pm[(size_t)lc * pc] = 1.0;
  auto PM = [&](int k, int lc) { return pm[(size_t)lc * pc + k]; };

  // delta-M decisions (DisortSolver.cpp:72-112)
  bool deltam = false;
  for (int lc = 0; lc < L; ++lc)
    if (PM(N, lc) != 0.0) { deltam = true; break; }
  const bool needdm = deltam;
  bool dmplus = c.dmplus;
  if (dmplus) {
    for (int lc = 0; lc < L; ++lc) {
      const double a = PM(N, lc), b = PM(N + 1, lc);
      if (a < 1e-4 || b < 0.7 * a) { dmplus = false; break; }
    }
    deltam = dmplus ? false : needdm;
  }

  // disortSet (DisortSolver.cpp:641-866)
  std::vector<double> tauc(L + 1), taus(L + 1), dts(L), ws(L), fsc(L), gl((size_t)L * N), btr(L + 1, 0.0);
  tauc[0] = 0.0;
  for (int lc = 0; lc < L; ++lc) tauc[lc + 1] = tauc[lc] + c.dtau[lc];
  std::vector<double> utau(ntau);
  if (c.user_tau) for (int k = 0; k < ntau; ++k) utau[k] = c.utau[k];
  else for (int k = 0; k < ntau; ++k) utau[k] = tauc[k];
  taus[0] = 0.0;
  double abstau = 0.0;
  int ncut = L;
  for (int lc = 0; lc < L; ++lc) {
    if (abstau < 10.0) ncut = lc + 1;
    abstau += (1.0 - c.ssa[lc]) * c.dtau[lc];
    const double w0 = c.ssa[lc], dt = c.dtau[lc];
    double f;
    double* g = &gl[(size_t)lc * N];
    if (!deltam && !dmplus) {
      ws[lc] = w0; dts[lc] = dt; taus[lc + 1] = tauc[lc + 1];
      for (int k = 0; k < N; ++k) g[k] = (2.0 * k + 1.0) * ws[lc] * PM(k, lc);
      f = 0.0;
    } else if (!dmplus || PM(N - 1, lc) == PM(N, lc) || PM(N, lc) == PM(N + 1, lc)) {
      f = PM(N, lc);
      ws[lc] = w0 * (1.0 - f) / (1.0 - f * w0);
      dts[lc] = (1.0 - f * w0) * dt;
      taus[lc + 1] = taus[lc] + dts[lc];
      for (int k = 0; k < N; ++k) g[k] = (2.0 * k + 1.0) * ws[lc] * (PM(k, lc) - f) / (1.0 - f);
    } else {
      const double a = PM(N, lc), b = PM(N + 1, lc);
      const double M = N;
      const double sig = ((M + 1.0) * (M + 1.0) - M * M) / (std::log(a * a) - std::log(b * b));
      const double cc = std::exp(M * M / (2.0 * sig));
      f = cc * a;
      ws[lc] = w0 * (1.0 - f) / (1.0 - f * w0);
      dts[lc] = (1.0 - f * w0) * dt;
      taus[lc + 1] = taus[lc] + dts[lc];
      for (int k = 0; k < N; ++k) {
        const double kd = k;
        g[k] = (2.0 * k + 1.0) * ws[lc] * (PM(k, lc) - f * std::exp(-kd * kd / (2.0 * sig))) / (1.0 - f);
      }
    }
    fsc[lc] = f;
  }
  // Chapman factor per layer (the pseudo-spherical beam, DisortSolver.cpp:740-782)
  std::vector<double> chap(L, 0.0);
  if (c.fbeam > 0.0) {
    btr[0] = 1.0;
    if (c.spherical) {
      for (int lc = 0; lc < ncut; ++lc) {
        const double taup_mid = taus[lc] + dts[lc] / 2.0;
        const double chtau_mid = chapman(lc + 1, 0.5, c.zalt, dts.data(), L, c.radius, c.umu0);
        chap[lc] = taup_mid / chtau_mid;
        btr[lc + 1] = std::exp(-chapman(lc + 1, 0.0, c.zalt, dts.data(), L, c.radius, c.umu0));
      }
    } else {
      for (int lc = 0; lc < ncut; ++lc) {
        chap[lc] = c.umu0;
        btr[lc + 1] = std::exp(-taus[lc + 1] / c.umu0);
      }
    }
  }
  const bool lyrcut = !c.special && (abstau >= 10.0 && !c.thermal && L > 1);  // computeAlbTrans: no cut
  if (!lyrcut) ncut = L;
  std::vector<double> utaus(ntau);
  std::vector<int> lyr(ntau);
  for (int lu = 0; lu < ntau; ++lu) {
    int lc;
    for (lc = 0; lc < L - 1; ++lc)
      if (utau[lu] >= tauc[lc] && utau[lu] <= tauc[lc + 1]) break;
    utaus[lu] = utau[lu];
    if (deltam || dmplus) utaus[lu] = taus[lc] + (1.0 - c.ssa[lc] * fsc[lc]) * (utau[lu] - tauc[lc]);
    lyr[lu] = lc;
  }
  std::vector<double> mu(N), wt(N), dsim(NN), dinv(NN);
  if (!gauss_quadrature(NN, mu.data(), wt.data())) return DSP_ERR_EIGEN;
  for (int iq = 0; iq < NN; ++iq) {
    dsim[iq] = std::sqrt(wt[iq] * mu[iq]);
    dinv[iq] = 1.0 / dsim[iq];
  }
  std::vector<double> umu(numu);
  if (c.user_mu && !c.only_fluxes) for (int iu = 0; iu < numu; ++iu) umu[iu] = c.umu[iu];
  else {
    for (int iu = 0; iu < NN; ++iu) umu[iu] = -mu[NN - 1 - iu];
    for (int iu = NN; iu < N; ++iu) umu[iu] = mu[iu - NN];
  }

  double ptop = 0, pbot = 0, pbotd = 0;
  if (c.thermal) {
    ptop = planck_function2(c.wlo, c.whi, c.ttop) * c.emis;
    pbot = planck_function2(c.wlo, c.whi, c.tbot);
    if (c.dlbc) {
      const double bl = planck_function2(c.wlo, c.whi, c.temp[L - 1]);
      if (dts[L - 1] > 0.0) pbotd = (pbot - bl) / dts[L - 1];
    }
  }

  // naz (DisortSolver.cpp:218-234); the reference's 1-based mu_user lookups
  // are read here only where the index exists
  int naz = N - 1;
  {
    auto um = [&](int k) { return (k < numu) ? umu[k] : 0.0; };
    const bool indep = (c.fbeam == 0.0) || (std::abs(1.0 - c.umu0) < 1.e-5) || c.only_fluxes ||
                       (numu == 1 && std::abs(1.0 - um(1)) < 1.e-5) || (numu == 1 && std::abs(1.0 + um(1)) < 1.e-5) ||
                       (numu == 2 && std::abs(1.0 + um(1)) < 1.e-5 && std::abs(1.0 - um(2)) < 1.e-5);
    if (indep) naz = 0;
  }

  // outputs start at zero
  for (int f = 0; f < 8; ++f) for (int lu = 0; lu < out.ntau_out; ++lu) out.flux[f][lu] = 0.0;
  if (out.intensity)
    for (size_t k = 0; k < (size_t)out.ntau_out * out.numu_out * nphi; ++k) out.intensity[k] = 0.0;
  if (out.iavg)
    for (size_t k = 0; k < (size_t)out.ntau_out * out.numu_out; ++k) out.iavg[k] = 0.0;
  auto I3 = [&](int lu, int iu, int j) -> double& {
    return out.intensity[((size_t)lu * out.numu_out + iu) * nphi + j];
  };

  // persistent Legendre tables (the m > 0 recurrence reads row m-1 of the previous mode)
  std::vector<double> ylq((size_t)(N + 1) * N, 0.0), ylu((size_t)(N + 1) * std::max(numu, 1), 0.0), ylb(N + 1, 0.0);
  std::vector<double> kk((size_t)L * N), G((size_t)L * N * N), C((size_t)L * N * N), zb((size_t)L * N),
      zbraw((size_t)L * N), z0((size_t)L * N, 0.0), z1((size_t)L * N, 0.0), xr0(L, 0.0), xr1(L, 0.0),
      GU((size_t)L * numu * N), zbu((size_t)L * numu, 0.0), z0u((size_t)L * numu, 0.0), z1u((size_t)L * numu, 0.0),
      cc((size_t)N * L), Im((size_t)ntau * numu);
  std::vector<double> cc_top((size_t)NN * N), amb(NN * NN), apb(NN * NN), evec(NN * NN), kred(NN), gpg(NN * NN);
  std::vector<double> A((size_t)N * N), xv(N), bvec(N);
  std::vector<double> zbs1((size_t)L * N, 0.0), xba(L, 0.0);  // pseudo-spherical beam source
  std::vector<int> piv(N);
  int kconv = 0;
  int status = DSP_OK;
  // temperature Jacobian: derivative sources of the thermal particular solution
  // with respect to each layer's top / bottom level Planck value
  const bool want_jac = c.temperature_jac && c.thermal && out.jac[0];
  std::vector<double> dz0t, dz0b, dz1t, dz1b, dxr0t, dxr0b, dxr1t, dxr1b;
  if (want_jac) {
    for (auto* v : {&dz0t, &dz0b, &dz1t, &dz1b}) v->assign((size_t)L * N, 0.0);
    for (auto* v : {&dxr0t, &dxr0b, &dxr1t, &dxr1b}) v->assign(L, 0.0);
  }
  if (out.jac[0])
    for (double* J : out.jac) std::fill(J, J + (size_t)ntau * out.jac_stride, 0.0);

  // surface reflectance and emissivity of each mode (computeSurfaceBidir)
  SurfaceTables sfc;
  sfc.init(NN, do_int ? numu : 0);
  std::vector<double> brdf_beam_u((size_t)numu * N, 0.0);
  const bool lamb = c.brdf == BRDF_LAMBERT;
  for (int m = 0; m <= naz; ++m) {
    const double d0 = (m == 0) ? 1.0 : 0.0;
    sfc.fill(c.brdf, c.bp, c.alb, m, mu.data(), umu.data(), do_int, c.fbeam, c.umu0);
    // the beam's surface coefficient of each mode at the user angles, for the
    // BRDF intensity correction (DisortSolver.cpp:306-313)
    if (!lamb && do_int && c.fbeam > 0.0)
      for (int iu = 0; iu < numu; ++iu) brdf_beam_u[(size_t)iu * N + m] = sfc.RU(iu, 0);
    legendre_flat(N, m, N, N - 1, mu.data(), ylq.data());
    auto Yq = [&](int l, int i) { return ylq[(size_t)l * N + i]; };
    if (do_int) legendre_flat(numu, m, numu, N - 1, umu.data(), ylu.data());
    auto Yu = [&](int l, int iu) { return ylu[(size_t)l * numu + iu]; };

    // solveEigen + interpEigenvec per layer (DisortSolver.cpp:872-1140, 2468-2504)
    for (int lc = 0; lc < L; ++lc) {
      const double* g = &gl[(size_t)lc * N];
      for (int iq = 0; iq < NN; ++iq)
        for (int jq = 0; jq < N; ++jq) {
          double s = 0.0;
          for (int l = m; l < N; ++l) s += (Yq(l, iq) * g[l]) * Yq(l, jq);
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
        const double inv = 1.0 / mu[iq];
        for (int jq = 0; jq < NN; ++jq) {
          amb[iq * NN + jq] = inv * (cc_top[iq * N + jq] - cc_top[iq * N + NN + jq]);
          apb[iq * NN + jq] = inv * (cc_top[iq * N + jq] + cc_top[iq * N + NN + jq]);
        }
        amb[iq * NN + iq] -= inv;
        apb[iq * NN + iq] -= inv;
      }
      if (int st = layer_eigen(NN, amb.data(), apb.data(), dsim.data(), dinv.data(), ws[lc] < 1.0 - 1e-12,
                               evec.data(), kred.data()))
        return st;
      double* kl = &kk[(size_t)lc * N];
      for (int iq = 0; iq < NN; ++iq) {
        kl[iq + NN] = kred[iq];
        kl[NN - 1 - iq] = -kred[iq];
      }
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
      if (do_int) {
        // GU(iu, c) = sum_l Yu(l,iu) 0.5 gl(l) sum_jq Yq(l,jq) w(jq) G(row(jq), c)
        auto row = [&](int jq) { return jq < NN ? NN + jq : N - 1 - jq; };
        std::vector<double> Wl((size_t)N * N, 0.0);
        for (int l = m; l < N; ++l)
          for (int col = 0; col < N; ++col) {
            double s = 0.0;
            for (int jq = 0; jq < N; ++jq) s += (Yq(l, jq) * wt[jq]) * Gl[row(jq) * N + col];
            Wl[(size_t)l * N + col] = s * (0.5 * g[l]);
          }
        for (int iu = 0; iu < numu; ++iu)
          for (int col = 0; col < N; ++col) {
            double s = 0.0;
            for (int l = m; l < N; ++l) s += Yu(l, iu) * Wl[(size_t)l * N + col];
            GU[((size_t)lc * numu + iu) * N + col] = s;
          }
      }
    }
    // pseudo-spherical beam source of mode m (computeBeamSourceSpherical,
    // DisortSolver.cpp:1396-1530): Z(tau) = exp(-xba tau) (Z0 + Z1 tau); the
    // user-angle interpolation then reads the source coefficients zj themselves
    if (c.fbeam > 0.0 && c.spherical) {
      const double umu0n = -c.umu0;
      legendre_flat(1, m, 1, N - 1, &umu0n, ylb.data());
      const double big = std::sqrt(std::numeric_limits<double>::max()) / 1.0e10;
      std::vector<double> zj(N), xb0(N), xb1(N), z1v(N);
      for (int lc = 0; lc < L; ++lc) {
        for (int iq = 0; iq < N; ++iq) {
          double s = 0.0;
          for (int k = m; k < N; ++k) s += gl[(size_t)lc * N + k] * Yq(k, iq) * ylb[k];
          zj[iq] = (2.0 - d0) * c.fbeam * s / (4.0 * M_PI);
        }
        const double q0a = btr[lc], q2a = btr[lc + 1];
        double xb = 1.0 / chap[lc];
        if (std::abs(xb) > big && taus[lc + 1] > 1.0) xb = 0.0;
        if (std::abs(xb * taus[lc + 1]) > std::log(big)) xb = 0.0;
        if (std::abs(xb) > 1.0e-5)
          for (int iq = 0; iq < NN; ++iq)
            if (std::abs((std::abs(xb) - 1.0 / mu[iq]) / xb) < 0.05) {
              xb *= 1.001;
              break;
            }
        const double deltat = taus[lc + 1] - taus[lc];
        for (int iq = 0; iq < N; ++iq) {
          const double q0 = q0a * zj[iq], q2 = q2a * zj[iq];
          xb1[iq] = (q2 * std::exp(xb * taus[lc + 1]) - q0 * std::exp(xb * taus[lc])) / deltat;
          xb0[iq] = q0 * std::exp(xb * taus[lc]) - xb1[iq] * taus[lc];
        }
        const double* Cl = &C[(size_t)lc * N * N];
        auto build = [&]() {
          for (int i = 0; i < N; ++i)
            for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
          for (int iq = 0; iq < N; ++iq) A[iq * N + iq] += 1.0 + xb * mu[iq];
        };
        build();
        double fro = 0.0;
        for (int e = 0; e < N * N; ++e) fro += A[e] * A[e];
        if (1.0 / std::sqrt(fro) < 1.0e-4) {
          if (xb == 0.0) xb = 5.0e-9;
          xb *= 1.00000005;
          build();
        }
        xba[lc] = xb;
        lu_factor(A.data(), N, N, piv.data());
        for (int iq = 0; iq < N; ++iq) z1v[iq] = xb1[iq];
        lu_solve(A.data(), N, N, piv.data(), z1v.data());
        for (int iq = 0; iq < N; ++iq) xv[iq] = xb0[iq] + mu[iq] * z1v[iq];
        lu_solve(A.data(), N, N, piv.data(), xv.data());
        for (int iq = 0; iq < N; ++iq) zbraw[(size_t)lc * N + iq] = zj[iq];
        for (int iq = 0; iq < NN; ++iq) {
          zb[(size_t)lc * N + NN + iq] = xv[iq];
          zb[(size_t)lc * N + NN - iq - 1] = xv[iq + NN];
          zbs1[(size_t)lc * N + NN + iq] = z1v[iq];
          zbs1[(size_t)lc * N + NN - iq - 1] = z1v[iq + NN];
        }
      }
    }
    // beam particular solution (DisortSolver.cpp:1319-1395)
    if (c.fbeam > 0.0 && !c.spherical) {
      const double umu0n = -c.umu0;
      legendre_flat(1, m, 1, N - 1, &umu0n, ylb.data());
      const double dither = 1000.0 * std::numeric_limits<double>::epsilon();
      for (int lc = 0; lc < L; ++lc) {
        double beam_mu = c.umu0;
        const double mu0sq = c.umu0 * c.umu0;
        for (int iq = 0; iq < NN; ++iq) {
          const double k = kk[(size_t)lc * N + iq + NN];
          if (std::abs(1.0 - mu0sq * k * k) < dither) { beam_mu = 0.999 * c.umu0; break; }
        }
        const double* Cl = &C[(size_t)lc * N * N];
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
        for (int i = 0; i < N; ++i) A[i * N + i] += 1.0 + mu[i] / beam_mu;
        for (int iq = 0; iq < N; ++iq) {
          double s = 0.0;
          for (int k = m; k < N; ++k) s += gl[(size_t)lc * N + k] * Yq(k, iq) * ylb[k];
          xv[iq] = (2.0 - d0) * c.fbeam * s / (4.0 * M_PI);
        }
        lu_factor(A.data(), N, N, piv.data());
        lu_solve(A.data(), N, N, piv.data(), xv.data());
        for (int iq = 0; iq < N; ++iq) zbraw[(size_t)lc * N + iq] = xv[iq];
        for (int iq = 0; iq < NN; ++iq) {
          zb[(size_t)lc * N + NN + iq] = xv[iq];
          zb[(size_t)lc * N + NN - iq - 1] = xv[iq + NN];
        }
      }
    }
    // thermal particular solution, mode 0 (DisortSolver.cpp:1533-1648)
    if (c.thermal && m == 0) {
      std::vector<double> pkag(L + 1), zz1(N);
      for (int lev = 0; lev <= L; ++lev) pkag[lev] = planck_function2(c.wlo, c.whi, c.temp[lev]);
      for (int lc = 0; lc < L; ++lc) {
        const double* Cl = &C[(size_t)lc * N * N];
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j) A[i * N + j] = -Cl[i * N + j];
        for (int i = 0; i < N; ++i) A[i * N + i] += 1.0;
        lu_factor(A.data(), N, N, piv.data());
        double r1 = 0.0;
        if (dts[lc] > 1e-4) r1 = (pkag[lc + 1] - pkag[lc]) / dts[lc];
        const double r0 = pkag[lc] - r1 * taus[lc];
        xr0[lc] = r0;
        xr1[lc] = r1;
        for (int i = 0; i < N; ++i) zz1[i] = (1.0 - ws[lc]) * r1;
        lu_solve(A.data(), N, N, piv.data(), zz1.data());
        for (int i = 0; i < N; ++i) bvec[i] = (1.0 - ws[lc]) * r0 + mu[i] * zz1[i];
        lu_solve(A.data(), N, N, piv.data(), bvec.data());
        for (int iq = 0; iq < NN; ++iq) {
          z0[(size_t)lc * N + NN + iq] = bvec[iq];
          z0[(size_t)lc * N + NN - iq - 1] = bvec[iq + NN];
          z1[(size_t)lc * N + NN + iq] = zz1[iq];
          z1[(size_t)lc * N + NN - iq - 1] = zz1[iq + NN];
        }
        if (want_jac) {
          // d/d(pkag[lc]) and d/d(pkag[lc+1]) with the same factorisation
          // (DisortSolver.cpp:1588-1640)
          const double omm = 1.0 - ws[lc], tc = taus[lc];
          double d1t = 0.0, d1b = 0.0;
          if (dts[lc] > 1e-4) {
            d1t = -1.0 / dts[lc];
            d1b = 1.0 / dts[lc];
          }
          const double d0t = 1.0 - d1t * tc, d0b = -d1b * tc;
          dxr0t[lc] = d0t; dxr0b[lc] = d0b; dxr1t[lc] = d1t; dxr1b[lc] = d1b;
          for (int side = 0; side < 2; ++side) {
            const double d1 = side ? d1b : d1t, d0 = side ? d0b : d0t;
            for (int i = 0; i < N; ++i) zz1[i] = omm * d1;
            lu_solve(A.data(), N, N, piv.data(), zz1.data());
            for (int i = 0; i < N; ++i) bvec[i] = omm * d0 + mu[i] * zz1[i];
            lu_solve(A.data(), N, N, piv.data(), bvec.data());
            std::vector<double>& D0 = side ? dz0b : dz0t;
            std::vector<double>& D1 = side ? dz1b : dz1t;
            for (int iq = 0; iq < NN; ++iq) {
              D0[(size_t)lc * N + NN + iq] = bvec[iq];
              D0[(size_t)lc * N + NN - iq - 1] = bvec[iq + NN];
              D1[(size_t)lc * N + NN + iq] = zz1[iq];
              D1[(size_t)lc * N + NN - iq - 1] = zz1[iq + NN];
            }
          }
        }
      }
    }
    // interpSource (DisortSolver.cpp:2506-2580)
    if (do_int) {
      for (int lc = 0; lc < L; ++lc) {
        const double* g = &gl[(size_t)lc * N];
        if (c.fbeam > 0.0) {
          std::vector<double> psi0(N, 0.0);
          for (int l = m; l < N; ++l) {
            double ps = 0.0;
            for (int jq = 0; jq < N; ++jq) ps += wt[jq] * Yq(l, jq) * zbraw[(size_t)lc * N + jq];
            psi0[l] = 0.5 * g[l] * ps;
          }
          const double fact = (2.0 - d0) * c.fbeam / (4.0 * M_PI);
          for (int iu = 0; iu < numu; ++iu) {
            double s = 0.0;
            for (int l = m; l < N; ++l) s += Yu(l, iu) * (psi0[l] + fact * g[l] * ylb[l]);
            zbu[(size_t)lc * numu + iu] = s;
          }
        }
        if (c.thermal && m == 0) {
          std::vector<double> p0(N, 0.0), p1(N, 0.0);
          for (int l = m; l < N; ++l) {
            double s0 = 0.0, s1 = 0.0;
            for (int jq = 0; jq < N; ++jq) {
              const int r = jq < NN ? NN + jq : N - 1 - jq;
              s0 += wt[jq] * Yq(l, jq) * z0[(size_t)lc * N + r];
              s1 += wt[jq] * Yq(l, jq) * z1[(size_t)lc * N + r];
            }
            p0[l] = 0.5 * g[l] * s0;
            p1[l] = 0.5 * g[l] * s1;
          }
          for (int iu = 0; iu < numu; ++iu) {
            double s0 = 0.0, s1 = 0.0;
            for (int l = m; l < N; ++l) {
              s0 += Yu(l, iu) * p0[l];
              s1 += Yu(l, iu) * p1[l];
            }
            z0u[(size_t)lc * numu + iu] = s0 + (1.0 - ws[lc]) * xr0[lc];
            z1u[(size_t)lc * numu + iu] = s1 + (1.0 - ws[lc]) * xr1[lc];
          }
        }
      }
    }
    // setMatrix (DisortSolver.cpp:1153-1317): surface coupling at every mode of a
    // BRDF, at mode 0 only for a Lambertian surface
    const int ncd = 3 * NN - 1, lda = 3 * ncd + 1, nshift = lda - 2 * N + 1;
    std::vector<double> band((size_t)lda * N * L, 0.0);
    auto BM = [&](int r, int col) -> double& { return band[(size_t)col * lda + r]; };
    auto Gv = [&](int lc, int r, int col) { return G[(size_t)lc * N * N + r * N + col]; };
    int ncol = 0;
    std::vector<double> e(N, 0.0);
    for (int lc = 0; lc < ncut; ++lc) {
      for (int iq = 0; iq < NN; ++iq) e[iq] = std::exp(kk[(size_t)lc * N + iq] * dts[lc]);
      int jcol = 0;
      for (int iq = 0; iq < NN; ++iq) {
        int irow = nshift - jcol - 1;
        for (int jq = 0; jq < N; ++jq) {
          if (irow + N >= 0 && irow + N < lda) BM(irow + N, ncol) = Gv(lc, jq, iq);
          if (irow >= 0 && irow < lda) BM(irow, ncol) = -Gv(lc, jq, iq) * e[iq];
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
        const double expa = std::exp(kk[iq] * taus[1]);
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
      const bool plain = lyrcut || c.dlbc || (lamb && d0 == 0.0);
      for (int iq = 0; iq < NN; ++iq) {
        nncol++;
        int irow = nshift - jcol + N - 1;
        for (int jq = NN; jq < N; ++jq) {
          if (plain) BM(irow, nncol) = Gv(lb, jq, iq);
          else {
            double refl = 0.0;
            for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * sfc.RQ(jq - NN, k + 1) * Gv(lb, NN - 1 - k, iq);
            BM(irow, nncol) = Gv(lb, jq, iq) - (1.0 + d0) * refl;
          }
          irow++;
        }
        jcol++;
      }
      for (int iq = NN; iq < N; ++iq) {
        nncol++;
        int irow = nshift - jcol + N - 1;
        const double expa = e[N - iq - 1];
        for (int jq = NN; jq < N; ++jq) {
          if (plain) BM(irow, nncol) = Gv(lb, jq, iq) * expa;
          else {
            double refl = 0.0;
            for (int k = 0; k < NN; ++k) refl += wt[k] * mu[k] * sfc.RQ(jq - NN, k + 1) * Gv(lb, NN - 1 - k, iq);
            BM(irow, nncol) = (Gv(lb, jq, iq) - (1.0 + d0) * refl) * expa;
          }
          irow++;
        }
        jcol++;
      }
    }
    // solve0 (DisortSolver.cpp:1669-1974)
    const int nc = N * ncut;
    std::vector<double> b(nc, 0.0);
    const int lb = ncut - 1;
    auto ZB = [&](int lc, int i) { return zb[(size_t)lc * N + i]; };
    auto Z0 = [&](int lc, int i) { return z0[(size_t)lc * N + i]; };
    auto Z1 = [&](int lc, int i) { return z1[(size_t)lc * N + i]; };
    const bool beam = c.fbeam > 0.0;
    // the beam particular solution of layer lc at scaled depth tau (T: the
    // transmission there); pseudo-spherical: exp(-xba tau) (Z0 + Z1 tau)
    // (DisortSolver.cpp:1722-1760, 1800-1905)
    auto ZBT = [&](int lc, int i, double tau, double T) {
      if (c.spherical) return std::exp(-xba[lc] * tau) * (ZB(lc, i) + zbs1[(size_t)lc * N + i] * tau);
      return ZB(lc, i) * T;
    };
    if (m > 0) {
      if (beam) {
        for (int iq = 0; iq < NN; ++iq) b[iq] = -ZB(0, NN - 1 - iq);
        for (int iq = 0; iq < NN; ++iq) {
          if (lyrcut || lamb) {
            b[nc - NN + iq] = -ZBT(lb, NN + iq, taus[ncut], btr[ncut]);
          } else {  // BRDF reflection of the diffuse and direct beam (DisortSolver.cpp:1729-1741)
            double s = 0.0;
            for (int jq = 0; jq < NN; ++jq)
              s += wt[jq] * mu[jq] * sfc.RQ(iq, jq + 1) * ZB(lb, NN - 1 - jq) * btr[ncut];
            b[nc - NN + iq] = s + (sfc.RQ(iq, 0) * c.umu0 * c.fbeam / M_PI - ZB(lb, NN + iq)) * btr[ncut];
          }
        }
        for (int lc = 1; lc < ncut; ++lc)
          for (int iq = 0; iq < N; ++iq)
            b[lc * N - NN + iq] = c.spherical ? ZBT(lc, iq, taus[lc], 0.0) - ZBT(lc - 1, iq, taus[lc], 0.0)
                                              : (ZB(lc, iq) - ZB(lc - 1, iq)) * btr[lc];
      }
    } else {
      for (int iq = 0; iq < NN; ++iq) {
        double s = 0.0;
        if (beam) s -= ZB(0, NN - iq - 1);
        if (c.thermal) s -= Z0(0, NN - iq - 1);
        s += c.fisot + ptop;
        b[iq] = s;
      }
      if (c.dlbc) {
        for (int iq = 0; iq < NN; ++iq) {
          double s = 0.0;
          if (beam) s -= ZBT(lb, NN + iq, taus[ncut], btr[ncut]);
          if (c.thermal) { s -= Z0(lb, NN + iq); s -= Z1(lb, NN + iq) * taus[ncut]; }
          s += pbot + mu[iq] * pbotd;
          b[nc - NN + iq] = s;
        }
      } else {
        for (int iq = 0; iq < NN; ++iq) {
          double s = 0.0;
          if (!lyrcut) {
            double refl = 0.0;
            for (int jq = 0; jq < NN; ++jq) {
              double ps = 0.0;
              if (beam) ps += ZBT(lb, NN - 1 - jq, taus[ncut], btr[ncut]);
              if (c.thermal) ps += Z0(lb, NN - 1 - jq) + Z1(lb, NN - 1 - jq) * taus[ncut];
              refl += wt[jq] * mu[jq] * sfc.RQ(iq, jq + 1) * ps;
            }
            s += 2.0 * refl;
          }
          if (beam) {
            s -= ZBT(lb, NN + iq, taus[ncut], btr[ncut]);
            if (!lyrcut) s += sfc.RQ(iq, 0) * c.umu0 * c.fbeam * btr[ncut] / M_PI;
          }
          if (c.thermal) { s -= Z0(lb, NN + iq); s -= Z1(lb, NN + iq) * taus[ncut]; }
          s += c.fisob;
          if (c.thermal) s += sfc.eq[iq] * pbot;
          b[nc - NN + iq] = s;
        }
      }
      for (int lc = 1; lc < ncut; ++lc)
        for (int iq = 0; iq < N; ++iq) {
          double s = 0.0;
          if (beam) { s += ZBT(lc, iq, taus[lc], btr[lc]); s -= ZBT(lc - 1, iq, taus[lc], btr[lc]); }
          if (c.thermal) {
            s += Z0(lc, iq) - Z0(lc - 1, iq);
            s += (Z1(lc, iq) - Z1(lc - 1, iq)) * taus[lc];
          }
          b[lc * N - NN + iq] = s;
        }
    }
    std::vector<int> ipvt(nc);
    if (!band_factor(band.data(), lda, nc, ncd, ncd, ipvt.data())) status = DSP_ERR_SINGULAR;
    if (c.special) {
      // solve1 (DisortSolver.cpp:4165-4220) for the top and the bottom
      // illumination, albTransIntensity (:4222-4293) at the top and the bottom
      // for the half of the angles leaving the medium there, albTransSpherical
      // (:4295-4358)
      const int half = numu / 2;
      auto solve1 = [&](bool top, std::vector<double>& x) {
        x.assign(nc, 0.0);
        for (int q = 0; q < NN; ++q) x[top ? q : nc - NN + q] = c.fisot;
        band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), x.data());
      };
      auto intensity = [&](const std::vector<double>& x, int iu, bool top) {
        const double ut = top ? 0.0 : taus[L], sgn = top ? 1.0 : -1.0, um = umu[iu];
        double pal = 0.0;
        std::vector<double> wk(NN);
        for (int lc = 0; lc < L; ++lc) {
          const double dtau = taus[lc + 1] - taus[lc];
          const double e1 = std::exp((ut - taus[lc]) / um), e2 = std::exp((ut - taus[lc + 1]) / um);
          for (int iq = 0; iq < NN; ++iq) {
            const double k = kk[(size_t)lc * N + iq];
            wk[iq] = std::exp(k * dtau);
            const double den = 1.0 + um * k;
            const double expn = std::abs(den) < 0.0001 ? dtau / um * e2 : (e1 * wk[iq] - e2) * sgn / den;
            pal += GU[((size_t)lc * numu + iu) * N + iq] * x[(size_t)lc * N + iq] * expn;
          }
          for (int iq = NN; iq < N; ++iq) {
            const double den = 1.0 + um * kk[(size_t)lc * N + iq];
            const double expn = std::abs(den) < 0.0001 ? -dtau / um * e1 : (e1 - e2 * wk[N - 1 - iq]) * sgn / den;
            pal += GU[((size_t)lc * numu + iu) * N + iq] * x[(size_t)lc * N + iq] * expn;
          }
        }
        return pal;
      };
      std::vector<double> xt, xb;
      solve1(true, xt);
      double* alb_out = out.albtrans[0];
      double* trn_out = out.albtrans[1];
      for (int iu = 0; iu < half; ++iu) alb_out[iu] = intensity(xt, iu + half, true);
      if (L == 1) {
        for (int iu = 0; iu < half; ++iu)
          trn_out[iu] = intensity(xt, half - 1 - iu, false) + std::exp(-taus[L] / umu[iu + half]);
      } else {
        solve1(false, xb);
        for (int iu = 0; iu < half; ++iu)
          trn_out[iu] = intensity(xb, iu + half, true) + std::exp(-taus[L] / umu[iu + half]);
      }
      out.albtrans[2][0] = 0.0;
      out.albtrans[3][0] = 0.0;
      if (special_alb > 0.0) {
        const std::vector<double>& x = L == 1 ? xt : xb;
        double up = 0.0, dn = 0.0;
        for (int iq = NN; iq < N; ++iq) {
          double z = 0.0;
          for (int jq = 0; jq < NN; ++jq) z += Gv(0, iq, jq) * x[jq] * std::exp(kk[jq] * (taus[1] - taus[0]));
          for (int jq = NN; jq < N; ++jq) z += Gv(0, iq, jq) * x[jq];
          up += wt[iq - NN] * mu[iq - NN] * z;
        }
        const int ll = L - 1;
        for (int iq = 0; iq < NN; ++iq) {
          double z = 0.0;
          for (int jq = 0; jq < NN; ++jq) z += Gv(ll, iq, jq) * x[(size_t)ll * N + jq];
          for (int jq = NN; jq < N; ++jq)
            z += Gv(ll, iq, jq) * x[(size_t)ll * N + jq] * std::exp(-kk[(size_t)ll * N + jq] * (taus[L] - taus[L - 1]));
          dn += wt[NN - 1 - iq] * mu[NN - 1 - iq] * z;
        }
        up *= 2.0;
        dn *= 2.0;
        const double sphalb = L == 1 ? up : dn, sphtrn = L == 1 ? dn : up;
        const double corr = special_alb / (1.0 - special_alb * sphalb);
        for (int iu = 0; iu < half; ++iu) {
          alb_out[iu] += corr * sphtrn * trn_out[iu];
          trn_out[iu] += corr * sphalb * trn_out[iu];
        }
        out.albtrans[2][0] = sphalb;
        out.albtrans[3][0] = sphtrn;
      }
      return status;
    }
    band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), b.data());
    std::fill(cc.begin(), cc.end(), 0.0);
    for (int k = 0; k < nc; ++k) cc[k] = b[k];  // the reference's reorder is the identity
    auto CCv = [&](int lc, int i) { return cc[(size_t)lc * N + i]; };

    // computeFluxes (DisortSolver.cpp:1980-2124), mode 0
    if (m == 0) {
      for (int lu = 0; lu < ntau; ++lu) {
        const int y = lyr[lu];
        if (lyrcut && y > ncut - 1) continue;  // zeros
        const double u = utaus[lu];
        double fact = 0, dirint = 0, fldir = 0, fdir = 0;
        if (beam) {
          if (c.spherical) {  // DisortSolver.cpp:2022-2025
            fact = std::exp(-u / chap[y]);
            fdir = std::abs(c.umu0) * c.fbeam * std::exp(-utau[lu] / chap[y]);
          } else {
            fact = std::exp(-u / c.umu0);
            fdir = c.umu0 * c.fbeam * std::exp(-utau[lu] / c.umu0);
          }
          dirint = c.fbeam * fact;
          fldir = c.umu0 * c.fbeam * fact;
        }
        std::vector<double> ec(N), in(N);
        for (int jq = 0; jq < NN; ++jq) ec[jq] = CCv(y, jq) * std::exp(-kk[(size_t)y * N + jq] * (u - taus[y + 1]));
        for (int jq = NN; jq < N; ++jq) ec[jq] = CCv(y, jq) * std::exp(-kk[(size_t)y * N + jq] * (u - taus[y]));
        for (int i = 0; i < N; ++i) {
          double s = 0.0;
          for (int j = 0; j < N; ++j) s += Gv(y, i, j) * ec[j];
          in[i] = s;
        }
        if (beam) {
          if (c.spherical) {
            const double be = std::exp(-xba[y] * u);
            for (int i = 0; i < N; ++i) in[i] += be * (ZB(y, i) + zbs1[(size_t)y * N + i] * u);
          } else {
            for (int i = 0; i < N; ++i) in[i] += ZB(y, i) * fact;
          }
        }
        if (c.thermal) for (int i = 0; i < N; ++i) in[i] += Z0(y, i) + Z1(y, i) * u;
        double ua = 0, uad = 0, uau = 0, fldn = 0, fup = 0;
        for (int iq = 0; iq < NN; ++iq) {
          const int cw = NN - iq - 1;
          ua += wt[cw] * in[iq]; uad += wt[cw] * in[iq]; fldn += wt[cw] * in[iq] * mu[cw];
        }
        for (int iq = NN; iq < N; ++iq) {
          const int cw = iq - NN;
          ua += wt[cw] * in[iq]; uau += wt[cw] * in[iq]; fup += wt[cw] * in[iq] * mu[cw];
        }
        fup *= 2.0 * M_PI;
        fldn *= 2.0 * M_PI;
        const double fdn = (fldn + fldir) - fdir;
        ua = (2.0 * M_PI * ua + dirint) / (4.0 * M_PI);
        const double uaso = dirint / (4.0 * M_PI);
        uad = (2.0 * M_PI * uad) / (4.0 * M_PI);
        uau = (2.0 * M_PI * uau) / (4.0 * M_PI);
        double pls = 0.0;
        if (c.thermal) pls = xr0[y] + xr1[y] * u;
        const double dfdt = (1.0 - c.ssa[y]) * 4.0 * M_PI * (ua - pls);
        const double o[8] = {fdir, fdn, fup, dfdt, ua, uad, uau, uaso};
        for (int f = 0; f < 8; ++f) out.flux[f][lu] = o[f];
      }
      // computeThermalJacobian (DisortSolver.cpp:2130-2358): dC = A^{-1} dB with
      // the mode-0 band LU, for every level Planck value and the surface, at
      // the output optical depths, chained with dB/dT
      if (want_jac) {
        auto pick = [&](const std::vector<double>& v, int lc, int iq) { return v[(size_t)lc * N + iq]; };
        auto dz0 = [&](int lc, int iq, int k) {
          return (k == lc ? pick(dz0t, lc, iq) : 0.0) + (k == lc + 1 ? pick(dz0b, lc, iq) : 0.0);
        };
        auto dz1 = [&](int lc, int iq, int k) {
          return (k == lc ? pick(dz1t, lc, iq) : 0.0) + (k == lc + 1 ? pick(dz1b, lc, iq) : 0.0);
        };
        auto dint = [&](int lc, int k) { return (k == lc ? dxr0t[lc] : 0.0) + (k == lc + 1 ? dxr0b[lc] : 0.0); };
        auto dslp = [&](int lc, int k) { return (k == lc ? dxr1t[lc] : 0.0) + (k == lc + 1 ? dxr1b[lc] : 0.0); };
        const double dtau_last = dts[L - 1], tauc_bot = taus[ncut];
        std::vector<double> jb(nc), dexp(N), dval(N);
        auto propagate = [&](int k, int col, double chain) {
          for (int lu = 0; lu < ntau; ++lu) {
            const int y = lyr[lu];
            if (lyrcut && y > ncut - 1) continue;
            const double u = utaus[lu];
            for (int jq = 0; jq < NN; ++jq) dexp[jq] = jb[(size_t)y * N + jq] * std::exp(-kk[(size_t)y * N + jq] * (u - taus[y + 1]));
            for (int jq = NN; jq < N; ++jq) dexp[jq] = jb[(size_t)y * N + jq] * std::exp(-kk[(size_t)y * N + jq] * (u - taus[y]));
            for (int i = 0; i < N; ++i) {
              double sacc = 0.0;
              for (int j = 0; j < N; ++j) sacc += Gv(y, i, j) * dexp[j];
              dval[i] = sacc;
            }
            if (k >= 0)
              for (int i = 0; i < N; ++i) dval[i] += dz0(y, i, k) + dz1(y, i, k) * u;
            double dmi = 0, dmidn = 0, dmiup = 0, dfdn = 0, dfup = 0;
            for (int iq = 0; iq < NN; ++iq) {
              const int cw = NN - iq - 1;
              dmi += wt[cw] * dval[iq]; dmidn += wt[cw] * dval[iq]; dfdn += wt[cw] * dval[iq] * mu[cw];
            }
            for (int iq = NN; iq < N; ++iq) {
              const int cw = iq - NN;
              dmi += wt[cw] * dval[iq]; dmiup += wt[cw] * dval[iq]; dfup += wt[cw] * dval[iq] * mu[cw];
            }
            dfup *= 2.0 * M_PI;
            dfdn *= 2.0 * M_PI;
            const double dmt = (2.0 * M_PI * dmi) / (4.0 * M_PI);
            const double dmd = (2.0 * M_PI * dmidn) / (4.0 * M_PI);
            const double dmu = (2.0 * M_PI * dmiup) / (4.0 * M_PI);
            const double dpls = k >= 0 ? dint(y, k) + dslp(y, k) * u : 0.0;
            const double dfdiv = (1.0 - c.ssa[y]) * 4.0 * M_PI * (dmt - dpls);
            const double v[6] = {dfup, dfdn, dmt, dmd, dmu, dfdiv};
            for (int f = 0; f < 6; ++f) out.jac[f][(size_t)lu * out.jac_stride + col] = chain * v[f];
          }
        };
        for (int k = 0; k <= L + 1; ++k) {
          const bool surf = k == L + 1;
          std::fill(jb.begin(), jb.end(), 0.0);
          if (!surf)
            for (int iq = 0; iq < NN; ++iq) jb[iq] = -dz0(0, NN - 1 - iq, k);
          for (int iq = 0; iq < NN; ++iq) {
            double sacc = 0.0;
            if (surf) {
              if (c.dlbc) {
                sacc = 1.0;
                if (dtau_last > 0.0) sacc += mu[iq] * (1.0 / dtau_last);
              } else {
                sacc = sfc.eq[iq];  // surface emissivity
              }
            } else if (c.dlbc) {
              sacc = -dz0(ncut - 1, NN + iq, k) - dz1(ncut - 1, NN + iq, k) * tauc_bot;
              if (k == L - 1 && dtau_last > 0.0) sacc += mu[iq] * (-1.0 / dtau_last);
            } else {
              if (!lyrcut) {
                double refl = 0.0;
                for (int jq = 0; jq < NN; ++jq)
                  refl += wt[jq] * mu[jq] * sfc.RQ(iq, jq + 1) * (dz0(ncut - 1, NN - 1 - jq, k) + dz1(ncut - 1, NN - 1 - jq, k) * tauc_bot);
                sacc += 2.0 * refl;
              }
              sacc -= dz0(ncut - 1, NN + iq, k) + dz1(ncut - 1, NN + iq, k) * tauc_bot;
            }
            jb[nc - NN + iq] = sacc;
          }
          if (!surf)
            for (int lc = 1; lc < ncut; ++lc)
              for (int iq = 0; iq < N; ++iq)
                jb[lc * N - NN + iq] = dz0(lc, iq, k) - dz0(lc - 1, iq, k) + (dz1(lc, iq, k) - dz1(lc - 1, iq, k)) * taus[lc];
          band_solve(band.data(), lda, nc, ncd, ncd, ipvt.data(), jb.data());
          const double T = surf ? c.tbot : c.temp[k];
          propagate(surf ? -1 : k, k, planck_function_deriv2(c.wlo, c.whi, T));
        }
      }
    }

    // computeUserIntensities (DisortSolver.cpp:2938-3268)
    if (do_int) {
      for (int lc = 0; lc < ncut; ++lc)
        for (int iq = 0; iq < N; ++iq)
          for (int iu = 0; iu < numu; ++iu) GU[((size_t)lc * numu + iu) * N + iq] *= CCv(lc, iq);
      auto gu = [&](int lc, int iu, int iq) { return GU[((size_t)lc * numu + iu) * N + iq]; };
      std::vector<double> wk(NN), wkc(NN), wkb(NN);
      for (int lu = 0; lu < ntau; ++lu) {
        double exp0 = 0.0;
        if (beam) exp0 = std::exp(-utaus[lu] / c.umu0);
        const int y = lyr[lu];
        for (int iu = 0; iu < numu; ++iu) {
          const double um = umu[iu];
          double& Iout = Im[(size_t)lu * numu + iu];
          if (lyrcut && y >= ncut) { Iout = 0.0; continue; }
          const bool neg = um < 0.0;
          int ls, le;
          double sgn;
          if (neg) { ls = 0; le = y - 1; sgn = -1.0; }
          else { ls = y + 1; le = ncut - 1; sgn = 1.0; }
          double palint = 0.0, plkint = 0.0;
          for (int lc = ls; lc <= le; ++lc) {
            const double dt = dts[lc];
            const double e1 = std::exp((utaus[lu] - taus[lc]) / um);
            const double e2 = std::exp((utaus[lu] - taus[lc + 1]) / um);
            if (c.thermal && m == 0) {
              const double f0n = sgn * (e1 - e2);
              const double f1n = sgn * ((taus[lc] + um) * e1 - (taus[lc + 1] + um) * e2);
              plkint += z0u[(size_t)lc * numu + iu] * f0n + z1u[(size_t)lc * numu + iu] * f1n;
            }
            if (beam) {
              const double den = 1.0 + um / c.umu0;
              double expn;
              if (std::abs(den) < 0.0001) expn = (dt / c.umu0) * exp0;
              else expn = (e1 * btr[lc] - e2 * btr[lc + 1]) * sgn / den;
              palint += zbu[(size_t)lc * numu + iu] * expn;
            }
            for (int iq = 0; iq < NN; ++iq) {
              const double kq = kk[(size_t)lc * N + iq];
              wk[iq] = std::exp(kq * dt);
              const double den = 1.0 + um * kq;
              double expn;
              if (std::abs(den) < 0.0001) expn = (dt / um) * e2;
              else expn = sgn * (e1 * wk[iq] - e2) / den;
              palint += gu(lc, iu, iq) * expn;
            }
            for (int iq = NN; iq < N; ++iq) {
              const double den = 1.0 + um * kk[(size_t)lc * N + iq];
              double expn;
              if (std::abs(den) < 0.0001) expn = -(dt / um) * e1;
              else expn = sgn * (e1 - e2 * wk[N - 1 - iq]) / den;
              palint += gu(lc, iu, iq) * expn;
            }
          }
          const double dt1 = utaus[lu] - taus[y], dt2 = utaus[lu] - taus[y + 1];
          if ((std::abs(dt1) >= 1e-6 || !neg) && (std::abs(dt2) >= 1e-6 || neg)) {
            double e1c = 0.0, e2c = 0.0;
            if (neg) e1c = std::exp(dt1 / um);
            else e2c = std::exp(dt2 / um);
            if (beam) {
              const double den = 1.0 + um / c.umu0;
              double expn;
              if (std::abs(den) < 0.0001) expn = (dt1 / c.umu0) * exp0;
              else if (neg) expn = (exp0 - btr[y] * e1c) / den;
              else expn = (exp0 - btr[y + 1] * e2c) / den;
              palint += zbu[(size_t)y * numu + iu] * expn;
            }
            const double dty = dts[y];
            for (int iq = 0; iq < NN; ++iq) {
              const double kq = kk[(size_t)y * N + iq];
              const double den = 1.0 + um * kq;
              double expn;
              if (std::abs(den) < 0.0001) expn = -dt2 / um * e2c;
              else if (neg) expn = (std::exp(-kq * dt2) - std::exp(kq * dty) * e1c) / den;
              else expn = (std::exp(-kq * dt2) - e2c) / den;
              wkc[iq] = std::exp(kq * dty);
              palint += gu(y, iu, iq) * expn;
            }
            for (int iq = NN; iq < N; ++iq) {
              const double kq = kk[(size_t)y * N + iq];
              const double den = 1.0 + um * kq;
              double expn;
              if (std::abs(den) < 0.0001) expn = -(dt1 / um) * e1c;
              else if (neg) expn = (std::exp(-kq * dt1) - e1c) / den;
              else expn = (std::exp(-kq * dt1) - std::exp(-kq * dty) * e2c) / den;
              palint += gu(y, iu, iq) * expn;
            }
            if (c.thermal && m == 0) {
              double expn, fact;
              if (neg) { expn = e1c; fact = taus[y] + um; }
              else { expn = e2c; fact = taus[y + 1] + um; }
              const double f0n = 1.0 - expn;
              const double f1n = utaus[lu] + um - fact * expn;
              plkint += z0u[(size_t)y * numu + iu] * f0n + z1u[(size_t)y * numu + iu] * f1n;
            }
          }
          double bndint = 0.0;
          if (neg && m == 0) {
            bndint = (c.fisot + ptop) * std::exp(utaus[lu] / um);
          } else if (!neg) {
            if (c.dlbc) {
              if (lyrcut || m > 0) { Iout = palint + plkint; continue; }
              bndint = (pbot + um * pbotd) * std::exp((utaus[lu] - taus[L]) / um);
            } else if (lyrcut || (lamb && m > 0)) {
              Iout = palint + plkint;
              continue;
            } else {
              // surface at user angles (DisortSolver.cpp:3170-3220; tables set for mu > 0 only)
              for (int jq = NN; jq < N; ++jq) wkb[jq - NN] = std::exp(-kk[(size_t)(L - 1) * N + jq] * dts[L - 1]);
              double bnddfu = 0.0;
              for (int iq = NN - 1; iq >= 0; --iq) {
                double dfu = 0.0;
                for (int jq = 0; jq < NN; ++jq) dfu += Gv(L - 1, iq, jq) * CCv(L - 1, jq);
                for (int jq = NN; jq < N; ++jq) dfu += Gv(L - 1, iq, jq) * CCv(L - 1, jq) * wkb[jq - NN];
                if (beam) dfu += ZB(L - 1, iq) * btr[L];
                dfu += d0 * (Z0(L - 1, iq) + Z1(L - 1, iq) * taus[L]);
                bnddfu += (1.0 + d0) * sfc.RU(iu, NN - iq) * mu[NN - iq - 1] * wt[NN - iq - 1] * dfu;
              }
              const double bnddir = c.umu0 * c.fbeam / M_PI * sfc.RU(iu, 0) * btr[L];
              bndint = (bnddfu + bnddir + d0 * sfc.eu[iu] * pbot + c.fisob) * std::exp((utaus[lu] - taus[L]) / um);
            }
          }
          Iout = palint + plkint + bndint;
        }
      }
      if (m == 0) {
        for (int lu = 0; lu < ntau; ++lu)
          for (int iu = 0; iu < numu; ++iu) {
            const double v = Im[(size_t)lu * numu + iu];
            out.iavg[(size_t)lu * out.numu_out + iu] = v;
            for (int j = 0; j < nphi; ++j) I3(lu, iu, j) = v;
          }
      } else {
        double maxc = 0.0;
        for (int j = 0; j < nphi; ++j) {
          const double phirad = (c.phi[j] - c.phi0) * M_PI / 180.0;
          const double cosphi = std::cos(static_cast<double>(m) * phirad);
          for (int lu = 0; lu < ntau; ++lu)
            for (int iu = 0; iu < numu; ++iu) {
              const double az = Im[(size_t)lu * numu + iu] * cosphi;
              I3(lu, iu, j) += az;
              const double uu = std::abs(I3(lu, iu, j));
              double ratio;
              if (uu == 0.0) ratio = 1.0 + std::abs(az);
              else if (std::abs(az) == 0.0) ratio = 0.0;
              else ratio = std::abs(az) / uu;
              maxc = std::max(maxc, ratio);
            }
        }
        if (c.accur > 0.0) {
          if (maxc <= c.accur) ++kconv;
          if (kconv >= 2) break;
        }
      }
    }
  }
  // ---- intensity corrections, after the mode loop (DisortSolver.cpp:352-392) ----
  if (do_int && c.corr && c.fbeam > 0.0) {
    bool scat_yes = false;
    for (int lc = 0; lc < L; ++lc)
      if (c.ssa[lc] > 0.0) scat_yes = true;
    if (deltam && scat_yes) {
      if (c.corr_be)
        buras_emde(c, ncut, lyrcut, numu, nphi, ntau, umu, utau, utaus, lyr, tauc, taus, fsc, ws, pm, I3);
      else
        nakajima_tanaka(c, ncut, lyrcut, numu, nphi, ntau, umu, utau, utaus, lyr, tauc, taus, fsc, ws, pm, I3);
    }
    if (!dmplus && !lamb) {
      // applyBrdfIntensityCorrection (DisortSolver.cpp:3751-3810): the exact
      // reflectance of the beam against its Fourier sum over the modes run
      for (int iu = 0; iu < numu; ++iu) {
        const double u = umu[iu];
        if (u <= 0.0) continue;
        for (int j = 0; j < nphi; ++j) {
          const double dphi = (c.phi[j] - c.phi0) * (M_PI / 180.0);
          const double exact = brdf_value(c.brdf, c.bp, u, c.umu0, dphi);
          if (exact < 0.0) continue;
          double approx = 0.0;
          for (int m = 0; m < N; ++m) approx += brdf_beam_u[(size_t)iu * N + m] * std::cos(static_cast<double>(m) * dphi);
          const double drho = exact - approx;
          if (std::abs(drho) < 1e-15) continue;
          const double to_bottom = std::exp(-taus[ncut] / c.umu0);
          for (int lu = 0; lu < ntau; ++lu) {
            if (lyrcut && lyr[lu] >= ncut) continue;
            I3(lu, iu, j) += c.umu0 * c.fbeam * drho * to_bottom * std::exp((utaus[lu] - taus[ncut]) / u);
          }
        }
      }
    }
  }
  if (c.ifb) {  // reverseOutputArrays (IndexConversion.hpp:60-80): the level axis
    for (int f = 0; f < 8; ++f) std::reverse(out.flux[f], out.flux[f] + ntau);
    if (out.jac[0]) {  // rows reversed; level columns reversed, the surface column kept last
      const size_t js = out.jac_stride;
      for (double* J : out.jac) {
        for (int a = 0, z = ntau - 1; a < z; ++a, --z)
          std::swap_ranges(J + a * js, J + a * js + L + 2, J + z * js);
        for (int r = 0; r < ntau; ++r) std::reverse(J + r * js, J + r * js + L + 1);
      }
    }
    if (do_int) {
      const size_t row3 = (size_t)out.numu_out * nphi, row2 = out.numu_out;
      for (int a = 0, z = ntau - 1; a < z; ++a, --z) {
        for (size_t k = 0; k < row3; ++k) std::swap(out.intensity[a * row3 + k], out.intensity[z * row3 + k]);
        for (size_t k = 0; k < row2; ++k) std::swap(out.iavg[a * row2 + k], out.iavg[z * row2 + k]);
      }
    }
  }
  return status;
}

}  // namespace oracle
