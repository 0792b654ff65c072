// gen_intcor.cuh — the intensity corrections DisortSolver applies after its
// azimuth-mode loop (DisortSolver.cpp:352-392):
//  - Nakajima-Tanaka (applyIntensityCorrection, :3403-3530): the delta-M
//    single-scattered beam is replaced by the exact one (TMS, eq. STWL 68 with
//    singleScat :3287-3328) and, in the aureole of the beam, the secondary
//    scattering of the truncated forward peak is removed (IMS, secondaryScat
//    :3330-3401, xiFunc :3274-3285);
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
      auto phases = [&](int lc, double& exact, double& scaled) {
        const double* m = mom(lc);
        const double f = fsc[lc];
        double a = 1.0, b = 1.0, p1 = 1.0, p2 = 0.0;
        for (int k = 1; k <= nmom; ++k) {
          const double pl = ((2 * k - 1) * ct * p1 - (k - 1) * p2) / k;
          p2 = p1;
          p1 = pl;
          a += (double)(2 * k + 1) * pl * m[k];
          if (k <= N - 1) b += (double)(2 * k + 1) * pl * (m[k] - f) / (1.0 - f);
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
        if (wbar > tiny && fbar > tiny && stau > tiny && fbeam > tiny) {
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
