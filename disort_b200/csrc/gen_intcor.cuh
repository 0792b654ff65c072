// gen_intcor.cuh — the intensity corrections DisortSolver applies after its
// azimuth-mode loop (DisortSolver.cpp:352-392):
//  - Nakajima-Tanaka (applyIntensityCorrection, :3403-3530): the delta-M
//    single-scattered beam is replaced by the exact one (TMS, eq. STWL 68 with
//    singleScat :3287-3328) and, in the aureole of the beam, the secondary
//    scattering of the truncated forward peak is removed (IMS, secondaryScat
//    :3330-3401, xiFunc :3274-3285);
//  - Buras-Emde (applyNewIntensityCorrection, :3532-3749) instead, with a
//    tabulated phase function: the exact single scattering interpolates the
//    table, the secondary scattering uses the residual phase function P'' of the
//    truncated peak (prepDoubleScatIntegr :3812-3876, newSecondaryScat
//    :3878-3930, calcPhaseSquared :3932-4023), whose tables are built per
//    output depth first;
//  - over a BRDF surface, the reflected beam is corrected by the difference of
//    the exact reflectance and its Fourier sum over the modes that ran
//    (applyBrdfIntensityCorrection, :3751-3810).
// One CTA per chunk slot; a thread per (user angle, azimuth, output depth)
// element computes both corrections for its element, evaluating each layer's
// phase functions on the fly from the unscaled moments.  Fluxes and azimuthal
// averages are not touched.
#pragma once

#include "dsp_device.cuh"
#include "gen_brdf.cuh"

namespace dsp {

// xi of eq. STWL (72)
__device__ inline double intcor_xi(double umu1, double umu2, double tau) {
  const double x1 = (umu2 - umu1) / (umu2 * umu1);
  const double e1 = exp(-tau / umu1);
  if (x1 != 0.0) return ((tau * x1 - 1.0) * exp(-tau / umu2) + e1) / (x1 * x1 * umu1 * umu2);
  return tau * tau * e1 / (2.0 * umu1 * umu2);
}

// locate (Utils.hpp:27-64): j with xx[j] <= x < xx[j+1] by bisection, 0 at
// xx[0] and below, n-2 at xx[n-1]
__device__ inline int intcor_locate(const double* xx, int n, double x) {
  if (n <= 1) return 0;
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

// calcPhaseSquared: the azimuthal integral of P''(mu_1) P''(theta_12) over the
// grid mu_eq of one output depth (p2[na], mueq[nf], neg[nf] as 0 / 1)
__device__ inline double intcor_phase_squared(int na, const double* mup, const double* p2, double ct,
                                              const double* mueq, const double* neg, double norm) {
  const double PI_ = 3.14159265358979323846;
  double acc = 0.0;
  const double st = sqrt(1.0 - ct * ct);
  for (int j = 0; j < BE_NF; ++j) {
    const double me = mueq[j];
    double phint;
    if (ct == 1.0 || me == 1.0) {
      const int i2 = intcor_locate(mup, na, me * ct);
      phint = PI_ * (p2[i2] + (me * ct - mup[i2]) / (mup[i2 + 1] - mup[i2]) * (p2[i2 + 1] - p2[i2]));
      if (ct == 1.0) phint /= 2.0;
    } else {
      phint = 0.0;
      const double sm = sqrt(1.0 - me * me);
      double lo = ct * me - st * sm, hi = ct * me + st * sm;
      bool cut = false;
      if (me < hi) {
        hi = me;
        cut = true;
      }
      if (lo < hi) {
        const int imin = intcor_locate(mup, na, lo), imax = intcor_locate(mup, na, hi);
        double D = (p2[imin + 1] - p2[imin]) / (mup[imin + 1] - mup[imin]);
        double C = p2[imin] - mup[imin] * D;
        phint += (D * ct * me + C) * PI_ / 2.0;
        for (int k = imin + 1; k <= imax; ++k) {
          const double Dp = (p2[k + 1] - p2[k]) / (mup[k + 1] - mup[k]);
          const double Cp = p2[k] - mup[k] * Dp;
          phint += (Dp - D) * sqrt(1.0 - ct * ct - me * me + 2.0 * ct * me * mup[k] - mup[k] * mup[k]) +
                   ((Dp - D) * ct * me + Cp - C) * asin((ct * me - mup[k]) / (sm * st));
          D = Dp;
          C = Cp;
        }
        if (cut)
          phint += -D * sqrt(1.0 - ct * ct + 2.0 * me * me * (ct - 1.0)) -
                   (D * ct * me + C) * asin((ct - 1.0) * me / (sm * st));
        else
          phint += (D * ct * me + C) * PI_ / 2.0;
      }
    }
    const double w = (j == 0 || j == BE_NF - 1) ? 0.5 : 1.0;
    acc += (neg[j] != 0.0 ? -w : w) * phint;
  }
  return acc * norm;
}

template <int N>
__global__ void __launch_bounds__(128) gen_intcor_kernel(FluxParams p) {
  const int slot = blockIdx.x;
  if (slot >= p.n) return;
  const GenView& g = p.g;
  const int i = g.ids[slot];
  const int st0 = p.status ? p.status[i] : 0;
  if (st0 == DSP_ERR_INVALID_INPUT || st0 == DSP_ERR_EIGEN) return;
  const int L = g.Ls[i];
  const int NT = g.user_tau ? g.user_tau : L + 1;
  const double* rec = p.inst_rec + g.inst_off[slot];
  const double fbeam = rec[H_FBEAM], umu0 = rec[H_UMU0];
  if (!(fbeam > 0.0)) return;
  const GenLayout gly = GenLayout::make(L, N, NT);
  const InstLayout& il = gly.il;
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  const long long base = g.in_off[i];
  const int pc = p.pc, nmom = g.nmoms[i];
  auto lay = [&](int lc) { return base + (ifb ? L - 1 - lc : lc); };
  auto ssa_at = [&](int lc) { return g.ssa[lay(lc)]; };
  auto dtau_at = [&](int lc) { return g.dtau[lay(lc)]; };
  auto mom = [&](int lc) { return g.pmom + lay(lc) * (long long)pc; };
  // scattering anywhere in the column (scat_yes_, DisortSolver.cpp:72-78)
  int scat = 0;
  for (int lc = threadIdx.x; lc < L; lc += blockDim.x) scat |= ssa_at(lc) > 0.0;
  scat = __syncthreads_or(scat);
  const bool nt = rec[H_DELTAM] != 0.0 && scat;
  const bool reflect = g.brdf != nullptr && rec[H_DMPLUS] == 0.0;
  if (!nt && !reflect) return;

  const int ncut = (int)rec[H_NCUT];
  const bool lyrcut = rec[H_LYRCUT] != 0.0;
  const double* taus = rec + il.tau_s;  // scaled depths of the levels
  const double* tauc = rec + il.tauc;   // unscaled depths of the levels
  const double* fsc = rec + il.fsc;
  const double* ssa_s = rec + il.ssa_s;
  const double* utau = rec + gly.utau;
  const double* utaus = rec + gly.utaus;
  const double* lyr = rec + gly.lyr;
  const double* um = g.umu.row(i);
  const double* ph = g.phi.row(i);
  const double phi0 = g.phi0(i);
  const int numu = g.numu, nphi = g.nphi;
  const double PI_ = 3.14159265358979323846, deg = PI_ / 180.0;
  const double dither = 100.0 * 2.220446049250313e-16, tiny = 1.0e-4;
  const double* tab = reflect ? g.brdf + (long long)slot * brdf_stride(N, numu) : nullptr;
  // Buras-Emde: the tabulated phase function, and P'' tables where an angle
  // lies in the aureole
  const bool be = nt && (p.flags & DSP_GFLAG_INTENSITY_CORR_BE) != 0;
  const int na = g.nangles;
  const double* mup = be ? g.mup.row(i) : nullptr;
  auto ptab = [&](int lc) { return g.phasef + lay(lc) * (long long)na; };
  double* bt = be ? g.becor + (long long)slot * g.becor_ld : nullptr;
  double* p2t = bt;                                  // [NT][na]
  double* meq = be ? bt + (long long)NT * na : nullptr;  // [NT][nf]
  double* neg = be ? meq + (long long)NT * BE_NF : nullptr;  // [NT][nf]
  double* nrm = be ? neg + (long long)NT * BE_NF : nullptr;  // [NT]
  bool need2 = false;
  if (be)
    for (int iu = 0; iu < numu; ++iu)
      if (um[iu] < 0.0 && fabs(acos(-umu0) / deg - acos(um[iu]) / deg) <= 10.0) need2 = true;
  if (need2) {
    // P''(mu_it) at every output depth: the tabulated phase function minus its
    // truncated Legendre sum, averaged over the scattering above the depth
    for (int e = threadIdx.x; e < na * NT; e += blockDim.x) {
      const int it = e % na, lu = e / na;
      const double ct = mup[it];
      const int ll = (int)lyr[lu];
      double v = 0.0;
      for (int l = 0; l <= ll; ++l) {
        const double* m = mom(l);
        const double f = fsc[l];
        double pr = 1.0 - f, p1 = 1.0, p2 = 0.0;
        for (int k = 1; k <= N - 1; ++k) {
          const double pl = ((2 * k - 1) * ct * p1 - (k - 1) * p2) / k;
          p2 = p1;
          p1 = pl;
          pr += (2 * k + 1) * pl * (m[k] - f);
        }
        const double w = l < ll ? dtau_at(l) : utau[lu] - tauc[ll];
        v += (ptab(l)[it] - pr) * ssa_at(l) * w;
      }
      p2t[(long long)lu * na + it] = v;
    }
    __syncthreads();
    // normalisation and the grid equidistant in the integral of |P''|, one
    // thread per depth
    for (int lu = threadIdx.x; lu < NT; lu += blockDim.x) {
      double* q = p2t + (long long)lu * na;
      const int ll = (int)lyr[lu];
      double fbar = fsc[ll] * ssa_at(ll) * (utau[lu] - tauc[ll]);
      for (int l = 0; l < ll; ++l) fbar += ssa_at(l) * dtau_at(l) * fsc[l];
      if (fbar <= tiny || fbeam <= tiny) {
        for (int it = 0; it < na; ++it) q[it] = 0.0;
      } else {
        fbar = 1.0 / fbar;
        for (int it = 0; it < na; ++it) q[it] *= fbar;
      }
      double f2 = 0.0;
      for (int it = 1; it < na; ++it) f2 += (mup[it] - mup[it - 1]) * 0.5 * (q[it] + q[it - 1]);
      if (f2 != 0.0) {
        const double s2 = 2.0 / f2;
        for (int it = 0; it < na; ++it) q[it] *= s2;
      }
      // cumulative integral of |P''|, written over the grid's slots until used
      double* me = meq + (long long)lu * BE_NF;
      double* ng = neg + (long long)lu * BE_NF;
      double total = 0.0;
      for (int it = 1; it < na; ++it) total += (mup[it] - mup[it - 1]) * 0.5 * (fabs(q[it]) + fabs(q[it - 1]));
      const double df = total / (BE_NF - 1);
      double fprev = 0.0, fcur = (mup[1] - mup[0]) * 0.5 * (fabs(q[1]) + fabs(q[0]));  // F at it, it+1
      int it = 0;
      double f = 0.0;
      for (int k = 1; k < BE_NF - 1; ++k) {
        f += df;
        while (fcur < f && it + 2 < na) {
          ++it;
          fprev = fcur;
          fcur = fprev + (mup[it + 1] - mup[it]) * 0.5 * (fabs(q[it + 1]) + fabs(q[it]));
        }
        me[k] = mup[it] + (f - fprev) / (fcur - fprev) * (mup[it + 1] - mup[it]);
        if (q[it] > 0.0 && q[it + 1] > 0.0) ng[k] = 0.0;
        else if (q[it] < 0.0 && q[it + 1] < 0.0) ng[k] = 1.0;
        else ng[k] = (q[it] + (f - fprev) / (fcur - fprev) * (q[it + 1] - q[it])) > 0.0 ? 0.0 : 1.0;
      }
      me[0] = -1.0;
      ng[0] = q[0] > 0.0 ? 0.0 : 1.0;
      me[BE_NF - 1] = 1.0;
      ng[BE_NF - 1] = q[na - 1] > 0.0 ? 0.0 : 1.0;
      nrm[lu] = total / ((BE_NF - 1) * PI_);
    }
    __syncthreads();
  }

  for (int e = threadIdx.x; e < numu * nphi * NT; e += blockDim.x) {
    const int lu = e % NT, jp = (e / NT) % nphi, iu = e / (NT * nphi);
    const int y = (int)lyr[lu];
    if (lyrcut && y >= ncut) continue;
    const double u = um[iu];
    const double dphi = (ph[jp] - phi0) * deg;
    double corr = 0.0;
    if (nt) {
      const double ct = -umu0 * u + sqrt((1.0 - umu0 * umu0) * (1.0 - u * u)) * cos(dphi);
      // layer lc's exact (TMS) and delta-M phase functions at scattering cosine ct
      // Buras-Emde: the table's interval holding ct
      const int itc = be ? intcor_locate(mup, na, ct) : 0;
      auto phases = [&](int lc, double& exact, double& scaled) {
        const double* m = mom(lc);
        const double f = fsc[lc];
        double a = 1.0, b = 1.0, p1 = 1.0, p2 = 0.0;
        const int kmax = be ? N - 1 : nmom;
        for (int k = 1; k <= kmax; ++k) {
          const double pl = ((2 * k - 1) * ct * p1 - (k - 1) * p2) / k;
          p2 = p1;
          p1 = pl;
          if (!be) a += (double)(2 * k + 1) * pl * m[k];
          if (k <= N - 1) b += (double)(2 * k + 1) * pl * (m[k] - f) / (1.0 - f);
        }
        if (be) {
          const double* pt = ptab(lc);
          a = pt[itc] + (ct - mup[itc]) / (mup[itc + 1] - mup[itc]) * (pt[itc + 1] - pt[itc]);
        }
        exact = a / (1.0 - f * ssa_at(lc));
        scaled = b;
      };
      // singleScat of both phase functions along the same layers (1-based lyr)
      const int layru = y + 1;
      const double tu = utaus[lu];
      double sx = 0.0, ss = 0.0, exp0 = exp(-tu / umu0);
      double px, ps;
      if (fabs(u + umu0) <= dither) {
        for (int l = 1; l <= layru - 1; ++l) {
          phases(l - 1, px, ps);
          sx += ssa_at(l - 1) * px * (taus[l] - taus[l - 1]);
          ss += ssa_s[l - 1] * ps * (taus[l] - taus[l - 1]);
        }
        phases(layru - 1, px, ps);
        const double fac = fbeam / (4.0 * PI_ * umu0) * exp0;
        sx = fac * (sx + ssa_at(layru - 1) * px * (tu - taus[layru - 1]));
        ss = fac * (ss + ssa_s[layru - 1] * ps * (tu - taus[layru - 1]));
      } else {
        if (u > 0.0) {
          for (int l = layru; l <= ncut; ++l) {
            const double e1 = exp(-((taus[l] - tu) / u + taus[l] / umu0));
            phases(l - 1, px, ps);
            sx += ssa_at(l - 1) * px * (exp0 - e1);
            ss += ssa_s[l - 1] * ps * (exp0 - e1);
            exp0 = e1;
          }
        } else {
          for (int l = layru; l >= 1; --l) {
            const double e1 = exp(-((taus[l - 1] - tu) / u + taus[l - 1] / umu0));
            phases(l - 1, px, ps);
            sx += ssa_at(l - 1) * px * (exp0 - e1);
            ss += ssa_s[l - 1] * ps * (exp0 - e1);
            exp0 = e1;
          }
        }
        const double fac = fbeam / (4.0 * PI_ * (1.0 + u / umu0));
        sx *= fac;
        ss *= fac;
      }
      corr += sx - ss;
      // IMS: downward angles within 10 degrees of the beam, below the top
      if (u < 0.0 && fabs(acos(-umu0) / deg - acos(u) / deg) <= 10.0 && !(lu == 0 && utau[0] <= dither)) {
        const double ut = utau[lu];
        double dt = ut - tauc[y];
        double wbar = ssa_at(y) * dt, fbar = fsc[y] * wbar, stau = dt;
        for (int l = 0; l < y; ++l) {
          wbar += dtau_at(l) * ssa_at(l);
          fbar += dtau_at(l) * ssa_at(l) * fsc[l];
          stau += dtau_at(l);
        }
        if (be && wbar > tiny && fbar > tiny && stau > tiny && fbeam > tiny) {
          fbar /= wbar;
          wbar /= stau;
          const double* q = p2t + (long long)lu * na;
          const double ps1 = q[itc] + (ct - mup[itc]) / (mup[itc + 1] - mup[itc]) * (q[itc + 1] - q[itc]);
          const double ps2 = intcor_phase_squared(na, mup, q, ct, meq + (long long)lu * BE_NF,
                                                  neg + (long long)lu * BE_NF, nrm[lu]);
          const double fw = fbar * wbar;
          const double umu0p = umu0 / (1.0 - fw);
          corr -= fbeam / (4.0 * PI_) * fw * fw / (1.0 - fw) * (2.0 * ps1 - ps2) * intcor_xi(-u, umu0p, ut);
        } else if (!be && wbar > tiny && fbar > tiny && stau > tiny && fbeam > tiny) {
          fbar /= wbar;
          wbar /= stau;
          double pspike = 1.0, p1 = 1.0, p2 = 0.0;
          for (int k = 1; k <= N - 1; ++k) {
            const double pl = ((2 * k - 1) * ct * p1 - (k - 1) * p2) / k;
            p2 = p1;
            p1 = pl;
            pspike += (double)(2 * k + 1) * pl;  // gbar = 1 below the truncation
          }
          const double fw = fbar * wbar;
          for (int k = N; k <= nmom; ++k) {
            const double pl = ((2 * k - 1) * ct * p1 - (k - 1) * p2) / k;
            p2 = p1;
            p1 = pl;
            double gbar = mom(y)[k] * ssa_at(y) * (ut - tauc[y]);
            for (int l = 0; l < y; ++l) gbar += mom(l)[k] * ssa_at(l) * dtau_at(l);
            const double tmp = fw * stau;
            gbar = tmp <= tiny ? 0.0 : gbar / tmp;
            pspike += gbar * (2.0 - gbar) * (double)(2 * k + 1) * pl;
          }
          const double umu0p = umu0 / (1.0 - fw);
          corr -= fbeam / (4.0 * PI_) * fw * fw / (1.0 - fw) * pspike * intcor_xi(-u, umu0p, ut);
        }
      }
    }
    if (reflect && u > 0.0) {
      const double exact = brdf_eval(g.brdf_type, g.brdf_par.row(i), u, umu0, dphi);
      if (exact >= 0.0) {
        const double* modes = tab + brdf_beam_modes(N, numu) + iu * N;
        double approx = 0.0;
        for (int m = 0; m < N; ++m) approx += modes[m] * cos(static_cast<double>(m) * dphi);
        const double drho = exact - approx;
        if (fabs(drho) >= 1e-15)
          corr += umu0 * fbeam * drho * exp(-taus[ncut] / umu0) * exp((utaus[lu] - taus[ncut]) / u);
      }
    }
    const long long row = (long long)i * g.ntau_out + (ifb ? NT - 1 - lu : lu);
    g.out_int[(row * g.numu_out + iu) * nphi + jp] += corr;
  }
}

}  // namespace dsp
