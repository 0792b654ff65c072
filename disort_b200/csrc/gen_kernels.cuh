// gen_kernels.cuh — the general solver's own kernels (DisortSolver::solve):
// per-instance setup and the user-angle intensities of one azimuth mode.
//
// The per-layer eigensystems and particular solutions (flux_layer_kernel<N,
// true>) and the boundary-value problem (flux_bvp*_kernel<N, true>) are shared
// with the flux solver; these kernels add what only the general solver has:
// ragged layer counts, user optical depths, the azimuth-mode schedule and
// intensities at user polar angles and azimuths.
#pragma once

#include "dsp_device.cuh"
#include "flux_setup.cuh"

namespace dsp {

// Setup of one instance per warp (disortSet, DisortSolver.cpp:641-866, and the
// decisions of DisortSolver::solve, :21-234).  Validation follows
// DisortConfig::validate (DisortConfig.cpp:72-249).
static __global__ void __launch_bounds__(128) gen_setup_kernel(FluxParams p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = blockIdx.x * 4 + warp;
  if (slot >= p.n) return;
  const GenView& g = p.g;
  const int i = g.ids[slot];
  const int N = p.N, L = g.Ls[i];
  const int NT = g.user_tau ? g.user_tau : L + 1;
  const GenLayout gly = GenLayout::make(L > 0 ? L : 0, N, NT > 0 ? NT : 0);
  const InstLayout& il = gly.il;
  double* rec = p.inst_rec + g.inst_off[slot];
  const uint32_t fl = p.flags;
  const bool thermal = (fl & DSP_FLAG_THERMAL) != 0;
  const bool dlbc = (fl & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const bool ifb = (fl & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  const bool only_fluxes = (fl & DSP_GFLAG_ONLY_FLUXES) != 0;
  const bool user_mu = (fl & DSP_GFLAG_USER_MU) != 0;
  const double fbeam = p.fbeam(i), umu0 = p.umu0(i), alb = p.alb(i), emis = p.emis(i);
  const double wlo = p.wlo(i), whi = p.whi(i), ttop = p.ttop(i), tbot = p.tbot(i);
  const int nmom = g.nmoms[i], pc = p.pc;
  const long long base = g.in_off[i];
  // index_from_bottom: inputs come bottom-up (reverseInputArrays, IndexConversion.hpp:16-40)
  auto dtau_at = [&](int lc) { return g.dtau[base + (ifb ? L - 1 - lc : lc)]; };
  auto ssa_at = [&](int lc) { return g.ssa[base + (ifb ? L - 1 - lc : lc)]; };
  auto pm_row = [&](int lc) { return g.pmom + (base + (ifb ? L - 1 - lc : lc)) * (long long)pc; };
  auto temp_at = [&](int lev) { return g.temp[base + i + (ifb ? L - lev : lev)]; };
  if (lane == 0) {
    for (int k = 0; k < 16; ++k) rec[k] = 0.0;
    rec[H_NT] = NT;
  }

  // ---- validate (DisortConfig.cpp:72-249) -------------------------------
  bool bad = L <= 0 || nmom < 0 || pc < (nmom > N ? nmom : N) + 1;
  if (!__any_sync(0xffffffffu, bad)) {
    for (int lc = lane; lc < L; lc += 32) {
      if (dtau_at(lc) < 0.0) bad = true;
      if (ssa_at(lc) < 0.0 || ssa_at(lc) > 1.0) bad = true;
    }
    if (thermal)
      for (int lev = lane; lev <= L; lev += 32)
        if (temp_at(lev) < 0.0) bad = true;
    if (user_mu) {
      const double* um = g.umu.row(i);
      for (int iu = lane; iu < g.numu_in; iu += 32) {
        if (fabs(um[iu]) > 1.0) bad = true;
        if (iu > 0 && um[iu] <= um[iu - 1]) bad = true;
      }
    }
    if (!only_fluxes) {
      const double* ph = g.phi.row(i);
      for (int j = lane; j < g.nphi; j += 32)
        if (ph[j] < 0.0 || ph[j] > 360.0) bad = true;
    }
    if (lane == 0) {
      if (thermal && (wlo < 0.0 || whi < wlo)) bad = true;
      if (dlbc && !thermal) bad = true;
      if (fbeam < 0.0) bad = true;
      if ((umu0 <= 0.0 || umu0 > 1.0) && fbeam > 0.0) bad = true;
      // the albedo is checked for a Lambertian surface only; a BRDF excludes the
      // diffusion lower boundary (DisortConfig.cpp:144-146, 160-163)
      if (g.brdf_type == DSP_BRDF_LAMBERTIAN && (alb < 0.0 || alb > 1.0)) bad = true;
      if (g.brdf_type != DSP_BRDF_LAMBERTIAN && dlbc) bad = true;
      if ((fl & DSP_FLAG_DELTA_M_PLUS) && nmom < N + 1) bad = true;
      // bottom_radius > 0 with the pseudo-spherical beam (DisortConfig.cpp:189-196)
      if ((fl & DSP_FLAG_SPHERICAL_BEAM) && !(p.rbot(i) > 0.0)) bad = true;
      if (thermal) {
        if (wlo < 0.0 || whi <= wlo) bad = true;
        if (ttop < 0.0 || tbot < 0.0) bad = true;
        if (emis < 0.0 || emis > 1.0) bad = true;
      }
    }
  }
  if (__any_sync(0xffffffffu, bad)) {
    if (lane == 0) set_status(p.status, i, DSP_ERR_INVALID_INPUT);
    return;
  }

  // ---- delta-M decisions (DisortSolver.cpp:72-112) ------------------------
  bool dm_local = false, dmp_fail = false;
  for (int lc = lane; lc < L; lc += 32) {
    const double pmN = pm_row(lc)[N];
    if (pmN != 0.0) dm_local = true;
    if (fl & DSP_FLAG_DELTA_M_PLUS) {
      const double pmN1 = pm_row(lc)[N + 1];
      if (pmN < 1e-4 || pmN1 < 0.7 * pmN) dmp_fail = true;
    }
  }
  bool deltam = __any_sync(0xffffffffu, dm_local);
  const bool dmplus = (fl & DSP_FLAG_DELTA_M_PLUS) && !__any_sync(0xffffffffu, dmp_fail);
  if (dmplus) deltam = false;

  // ---- per-layer scaling (disortSet, DisortSolver.cpp:663-747) -------------
  for (int lc = lane; lc < L; lc += 32) {
    const double w0 = ssa_at(lc), dt = dtau_at(lc);
    const double* pml = pm_row(lc);
    double f = 0.0, sig = 0.0, ws = w0, dts = dt, mode = 0.0;
    if (!deltam && !dmplus) {
      mode = 0.0;
    } else if (!dmplus || pml[N - 1] == pml[N] || pml[N] == pml[N + 1]) {
      f = pml[N];
      ws = w0 * (1.0 - f) / (1.0 - f * w0);
      dts = (1.0 - f * w0) * dt;
      mode = 1.0;
    } else {
      const double pmv = pml[N], pm1 = pml[N + 1];
      const double M = static_cast<double>(N);
      sig = ((M + 1.0) * (M + 1.0) - M * M) / (log(pmv * pmv) - log(pm1 * pm1));
      const double c = exp(M * M / (2.0 * sig));
      f = c * pmv;
      ws = w0 * (1.0 - f) / (1.0 - f * w0);
      dts = (1.0 - f * w0) * dt;
      mode = 2.0;
    }
    rec[il.dtau_s + lc] = dts;
    rec[il.ssa_s + lc] = ws;
    rec[il.fsc + lc] = f;
    rec[il.sig + lc] = sig;
    rec[il.mode + lc] = mode;
  }
  if (thermal)
    for (int lev = lane; lev <= L; lev += 32) rec[il.pkag + lev] = planck2(wlo, whi, temp_at(lev), p.pk);
  __syncwarp();

  if (lane == 0) {
    const double abscut = 10.0;
    double tauc = 0.0, taus = 0.0, abstau = 0.0;
    int ncut = L;
    rec[il.tauc] = 0.0;
    rec[il.tau_s] = 0.0;
    for (int lc = 0; lc < L; ++lc) {
      if (abstau < abscut) ncut = lc + 1;
      abstau += (1.0 - ssa_at(lc)) * dtau_at(lc);
      tauc = tauc + dtau_at(lc);
      rec[il.tauc + lc + 1] = tauc;
      if (!deltam && !dmplus) taus = tauc;
      else taus = taus + rec[il.dtau_s + lc];
      rec[il.tau_s + lc + 1] = taus;
    }
    // beam transmission for lc < ncut of the absorption loop (DisortSolver.cpp:749-790);
    // later entries stay zero, as on a freshly constructed reference solver
    for (int lev = 0; lev <= L; ++lev) rec[il.btr + lev] = 0.0;
    if (fbeam > 0.0) {
      rec[il.btr] = 1.0;
      for (int lc = 0; lc < ncut; ++lc) rec[il.btr + lc + 1] = exp(-rec[il.tau_s + lc + 1] / umu0);
    }
    const bool lyrcut = (abstau >= abscut && !thermal && L > 1);
    if (!lyrcut) ncut = L;
    // boundary Planck terms (DisortSolver.cpp:186-202)
    double ptop = 0.0, pbot = 0.0, pbotd = 0.0;
    if (thermal) {
      ptop = planck2(wlo, whi, ttop, p.pk) * emis;
      pbot = planck2(wlo, whi, tbot, p.pk);
      if (dlbc) {
        const double bl = planck2(wlo, whi, temp_at(L - 1), p.pk);
        const double dl = rec[il.dtau_s + L - 1];
        if (dl > 0.0) pbotd = (pbot - bl) / dl;
      }
    }
    // highest azimuth mode (DisortSolver.cpp:218-234).  The reference reads
    // mu_user[1] and mu_user[2] (one past the index it means); entries past the
    // list count as 0 here.  Without intensities only mode 0 contributes.
    const int numu = (user_mu && !only_fluxes) ? g.numu_in : N;
    const double* um = (user_mu && !only_fluxes) ? g.umu.row(i) : nullptr;
    auto umu_at = [&](int k) { return (um && k < numu) ? um[k] : 0.0; };
    const bool indep = (fbeam == 0.0) || (fabs(1.0 - umu0) < 1.e-5) || only_fluxes ||
                       (numu == 1 && fabs(1.0 - umu_at(1)) < 1.e-5) ||
                       (numu == 1 && fabs(1.0 + umu_at(1)) < 1.e-5) ||
                       (numu == 2 && fabs(1.0 + umu_at(1)) < 1.e-5 && fabs(1.0 - umu_at(2)) < 1.e-5);
    const int naz = (indep || g.numu == 0) ? 0 : N - 1;
    rec[H_NCUT] = ncut;
    rec[H_LYRCUT] = lyrcut ? 1.0 : 0.0;
    rec[H_PTOP] = ptop;
    rec[H_PBOT] = pbot;
    rec[H_PBOTD] = pbotd;
    rec[H_DELTAM] = deltam ? 1.0 : 0.0;
    rec[H_DMPLUS] = dmplus ? 1.0 : 0.0;
    rec[H_FBEAM] = fbeam;
    rec[H_UMU0] = umu0;
    rec[H_ALB] = alb;
    rec[H_FISOT] = p.fisot(i);
    rec[H_FISOB] = p.fisob(i);
    rec[H_NAZ] = naz;
  }
  __syncwarp();
  // ---- output depths and their layers (DisortSolver.cpp:801-817) -----------
  const double total = rec[il.tauc + L];
  const double* ut_in = g.user_tau ? g.utau.row(i) : nullptr;
  for (int lu = lane; lu < NT; lu += 32) {
    double tau;
    if (ut_in) tau = ifb ? total - ut_in[NT - 1 - lu] : ut_in[lu];
    else tau = rec[il.tauc + lu];
    int lc;
    for (lc = 0; lc < L - 1; ++lc)
      if (tau >= rec[il.tauc + lc] && tau <= rec[il.tauc + lc + 1]) break;
    double tus = tau;
    if (deltam || dmplus) tus = rec[il.tau_s + lc] + (1.0 - ssa_at(lc) * rec[il.fsc + lc]) * (tau - rec[il.tauc + lc]);
    rec[gly.utau + lu] = tau;
    rec[gly.utaus + lu] = tus;
    rec[gly.lyr + lu] = lc;
  }
}

// Intensities at the user angles for mode m (computeUserIntensities,
// DisortSolver.cpp:2938-3268): one warp per instance, a lane per (level, angle)
// pair, looping over the layers between the level and the boundary.
template <int N>
__global__ void __launch_bounds__(128) gen_intensity_kernel(FluxParams p) {
  constexpr int NN = N / 2;
  constexpr double PI = 3.14159265358979323846;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = blockIdx.x * 4 + warp;
  if (slot >= p.n) return;
  const GenView& g = p.g;
  const int i = g.ids[slot];
  const int L = g.Ls[i];
  const int NT = g.user_tau ? g.user_tau : L + 1;
  const int m = g.m, numu = g.numu, nphi = g.nphi;
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  auto orow = [&](int lu) { return (long long)i * g.ntau_out + (ifb ? NT - 1 - lu : lu); };
  const int st0 = p.status ? p.status[i] : 0;
  if (st0 == DSP_ERR_INVALID_INPUT || st0 == DSP_ERR_EIGEN) {
    if (m == 0) {
      const double qnan = __longlong_as_double(0x7ff8000000000000ll);
      for (int k = lane; k < NT * numu; k += 32) {
        const int lu = k / numu, iu = k % numu;
        g.out_iavg[orow(lu) * g.numu_out + iu] = qnan;
        for (int j = 0; j < nphi; ++j) g.out_int[(orow(lu) * g.numu_out + iu) * nphi + j] = qnan;
      }
    }
    return;
  }
  const double* rec = p.inst_rec + g.inst_off[slot];
  if (m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  const GenLayout gly = GenLayout::make(L, N, NT);
  const InstLayout& il = gly.il;
  const double* mu = p.tables + tab_mu(N);
  const double* wt = p.tables + tab_wt(N);
  const int ncut = (int)rec[H_NCUT];
  const bool lyrcut = rec[H_LYRCUT] != 0.0;
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0 && m == 0;
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double fbeam = rec[H_FBEAM], umu0 = rec[H_UMU0], alb = rec[H_ALB];
  const bool beam = fbeam > 0.0;
  const double* taus = rec + il.tau_s;
  const double* dts = rec + il.dtau_s;
  const double* btr = rec + il.btr;
  const double* utaus = rec + gly.utaus;
  const double* lyr = rec + gly.lyr;
  const double* lrec0 = p.layer_rec + g.lay_off[slot] * g.lstride;
  const double* cc0 = g.cc + g.lay_off[slot] * N;
  auto LR = [&](int l) { return lrec0 + (long long)l * g.lstride; };
  const double* um = g.umu.row(i);

  // bottom-boundary reflection of the mode-0 downward field (DisortSolver.cpp:3180-3218):
  // S = sum_iq mu w dfuint(iq), in the reference's order iq = NN-1 .. 0
  double bsum = 0.0;
  // bidirectional surface: this mode's table; its user rows receive the
  // reflected sum of each user angle in their last slot
  double* sft = g.brdf ? g.brdf + (long long)slot * brdf_stride(N, g.numu) : nullptr;
  const bool lambert_bnd = (m == 0) && !lyrcut && !dlbc && !sft;
  if (sft && !lyrcut) {
    // sum_iq (1 + delta_m0) R_m(mu_u, mu_iq) mu_iq w_iq dfuint(iq) per user angle
    // (DisortSolver.cpp:3180-3218), dfuint as below, summed across the warp
    const double* lr = LR(L - 1);
    const double* G = lr + lrec_G(N);
    const double* x = cc0 + (long long)(L - 1) * N;
    double dfu = 0.0;
    const int iq = lane;
    if (iq < NN) {
      for (int jq = 0; jq < NN; ++jq) dfu += G[iq * N + jq] * x[jq];
      for (int jq = NN; jq < N; ++jq) dfu += G[iq * N + jq] * x[jq] * exp(-lr[lrec_eig(N) + jq] * dts[L - 1]);
      if (beam) dfu += lr[lrec_zb(N) + iq] * btr[L];
      if (thermal) dfu += lr[lrec_z0(N) + iq] + lr[lrec_z1(N) + iq] * taus[L];
    }
    const double cpl = m == 0 ? 2.0 : 1.0;
    for (int iu = 0; iu < numu; ++iu) {
      double* ur = sft + (NN + iu) * brdf_row(N);
      double v = iq < NN ? cpl * ur[NN - iq] * mu[NN - iq - 1] * wt[NN - iq - 1] * dfu : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if (lane == 0) ur[NN + 2] = v;
    }
    __syncwarp();
  }
  if (lambert_bnd) {
    const double* lr = LR(L - 1);
    const double* G = lr + lrec_G(N);
    const double* x = cc0 + (long long)(L - 1) * N;
    double dfu = 0.0;
    const int iq = lane;
    if (iq < NN) {
      for (int jq = 0; jq < NN; ++jq) dfu += G[iq * N + jq] * x[jq];
      for (int jq = NN; jq < N; ++jq) dfu += G[iq * N + jq] * x[jq] * exp(-lr[lrec_eig(N) + jq] * dts[L - 1]);
      if (beam) dfu += lr[lrec_zb(N) + iq] * btr[L];
      if (p.flags & DSP_FLAG_THERMAL) dfu += lr[lrec_z0(N) + iq] + lr[lrec_z1(N) + iq] * taus[L];
    }
    for (int k = NN - 1; k >= 0; --k) {
      const double v = __shfl_sync(0xffffffffu, dfu, k);
      bsum += 2.0 * mu[NN - k - 1] * wt[NN - k - 1] * v;
    }
  }

  double maxr = 0.0;
  for (int k = lane; k < NT * numu; k += 32) {
    const int lu = k / numu, iu = k % numu;
    const double umv = um[iu];
    const int y = (int)lyr[lu];
    double I = 0.0;
    if (!(lyrcut && y >= ncut)) {
      const double ut = utaus[lu];
      const double exp0 = beam ? exp(-ut / umu0) : 0.0;
      const bool neg = umv < 0.0;
      const int ls = neg ? 0 : y + 1, le = neg ? y - 1 : ncut - 1;
      const double sgn = neg ? -1.0 : 1.0;
      double palint = 0.0, plkint = 0.0;
      // layers entirely between the level and the boundary
      for (int lc = ls; lc <= le; ++lc) {
        const double* lr = LR(lc);
        const double* gu = lr + glrec_gu(N) + iu * N;
        const double* x = cc0 + (long long)lc * N;
        const double* kk = lr + lrec_eig(N);
        const double dt = dts[lc];
        const double e1 = exp((ut - taus[lc]) / umv);
        const double e2 = exp((ut - taus[lc + 1]) / umv);
        if (thermal) {
          const double f0n = sgn * (e1 - e2);
          const double f1n = sgn * ((taus[lc] + umv) * e1 - (taus[lc + 1] + umv) * e2);
          const double* zu = lr + glrec_gu(N) + numu * N + numu;
          plkint += zu[iu] * f0n + zu[numu + iu] * f1n;
        }
        if (beam) {
          const double den = 1.0 + umv / umu0;
          double expn;
          if (fabs(den) < 0.0001) expn = (dt / umu0) * exp0;
          else expn = (e1 * btr[lc] - e2 * btr[lc + 1]) * sgn / den;
          palint += lr[glrec_gu(N) + numu * N + iu] * expn;
        }
        double wk[NN];
#pragma unroll
        for (int iq = 0; iq < NN; ++iq) {
          wk[iq] = exp(kk[iq] * dt);
          const double den = 1.0 + umv * kk[iq];
          double expn;
          if (fabs(den) < 0.0001) expn = (dt / umv) * e2;
          else expn = sgn * (e1 * wk[iq] - e2) / den;
          palint += (gu[iq] * x[iq]) * expn;
        }
#pragma unroll
        for (int iq = NN; iq < N; ++iq) {
          const double den = 1.0 + umv * kk[iq];
          double expn;
          if (fabs(den) < 0.0001) expn = -(dt / umv) * e1;
          else expn = sgn * (e1 - e2 * wk[N - 1 - iq]) / den;
          palint += (gu[iq] * x[iq]) * expn;
        }
      }
      // the part of the level's own layer on the boundary side
      const double dt1 = ut - taus[y], dt2 = ut - taus[y + 1];
      if ((fabs(dt1) >= 1e-6 || !neg) && (fabs(dt2) >= 1e-6 || neg)) {
        const double* lr = LR(y);
        const double* gu = lr + glrec_gu(N) + iu * N;
        const double* x = cc0 + (long long)y * N;
        const double* kk = lr + lrec_eig(N);
        const double e1c = neg ? exp(dt1 / umv) : 0.0;
        const double e2c = neg ? 0.0 : exp(dt2 / umv);
        if (beam) {
          const double den = 1.0 + umv / umu0;
          double expn;
          if (fabs(den) < 0.0001) expn = (dt1 / umu0) * exp0;
          else if (neg) expn = (exp0 - btr[y] * e1c) / den;
          else expn = (exp0 - btr[y + 1] * e2c) / den;
          palint += lr[glrec_gu(N) + numu * N + iu] * expn;
        }
        const double dty = dts[y];
#pragma unroll 4
        for (int iq = 0; iq < NN; ++iq) {
          const double den = 1.0 + umv * kk[iq];
          double expn;
          if (fabs(den) < 0.0001) expn = -dt2 / umv * e2c;
          else if (neg) expn = (exp(-kk[iq] * dt2) - exp(kk[iq] * dty) * e1c) / den;
          else expn = (exp(-kk[iq] * dt2) - e2c) / den;
          palint += (gu[iq] * x[iq]) * expn;
        }
#pragma unroll 4
        for (int iq = NN; iq < N; ++iq) {
          const double den = 1.0 + umv * kk[iq];
          double expn;
          if (fabs(den) < 0.0001) expn = -(dt1 / umv) * e1c;
          else if (neg) expn = (exp(-kk[iq] * dt1) - e1c) / den;
          else expn = (exp(-kk[iq] * dt1) - exp(-kk[iq] * dty) * e2c) / den;
          palint += (gu[iq] * x[iq]) * expn;
        }
        if (thermal) {
          const double expn = neg ? e1c : e2c;
          const double fact = neg ? taus[y] + umv : taus[y + 1] + umv;
          const double f0n = 1.0 - expn;
          const double f1n = ut + umv - fact * expn;
          const double* zu = lr + glrec_gu(N) + numu * N + numu;
          plkint += zu[iu] * f0n + zu[numu + iu] * f1n;
        }
      }
      // boundary terms
      double bndint = 0.0;
      bool bnd_skip = false;
      if (neg && m == 0) {
        bndint = (rec[H_FISOT] + rec[H_PTOP]) * exp(ut / umv);
      } else if (!neg) {
        if (dlbc) {
          if (lyrcut || m > 0) bnd_skip = true;
          else bndint = (rec[H_PBOT] + umv * rec[H_PBOTD]) * exp((ut - taus[L]) / umv);
        } else if (lyrcut || (m > 0 && !sft)) {
          bnd_skip = true;
        } else if (sft) {
          // bidirectional surface at user angles (DisortSolver.cpp:3213-3220); the
          // isotropic bottom flux enters at every mode, as the reference adds it
          const double* ur = sft + (NN + iu) * brdf_row(N);
          const double bnddir = umu0 * fbeam / PI * ur[0] * btr[L];
          const double emit = m == 0 ? ur[NN + 1] * rec[H_PBOT] : 0.0;
          bndint = (ur[NN + 2] + bnddir + emit + rec[H_FISOB]) * exp((ut - taus[L]) / umv);
        } else {
          // Lambertian surface at user angles: set for mu > 0 only (DisortSolver.cpp:2655-2662)
          const double rho = umv > 0.0 ? alb : 0.0, em = umv > 0.0 ? 1.0 - alb : 0.0;
          const double bnddir = umu0 * fbeam / PI * rho * btr[L];
          bndint = (rho * bsum + bnddir + em * rec[H_PBOT] + rec[H_FISOB]) * exp((ut - taus[L]) / umv);
        }
      }
      I = bnd_skip ? palint + plkint : palint + plkint + bndint;
    }
    // accumulate the Fourier series (DisortSolver.cpp:3228-3266)
    const long long o2 = orow(lu) * g.numu_out + iu;
    if (m == 0) {
      g.out_iavg[o2] = I;
      for (int j = 0; j < nphi; ++j) g.out_int[o2 * nphi + j] = I;
    } else {
      const double* ph = g.phi.row(i);
      const double phi0 = g.phi0(i);
      for (int j = 0; j < nphi; ++j) {
        const double phirad = (ph[j] - phi0) * PI / 180.0;
        const double az = I * cos(static_cast<double>(m) * phirad);
        double& acc = g.out_int[o2 * nphi + j];
        acc += az;
        const double uu = fabs(acc);
        double ratio;
        if (uu == 0.0) ratio = 1.0 + fabs(az);
        else if (fabs(az) == 0.0) ratio = 0.0;
        else ratio = fabs(az) / uu;
        maxr = fmax(maxr, ratio);
      }
    }
  }
  // azimuthal convergence (DisortSolver.cpp:337-347)
  if (m > 0 && g.accur > 0.0) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) maxr = fmax(maxr, __shfl_xor_sync(0xffffffffu, maxr, off));
    if (lane == 0) {
      double* wrec = p.inst_rec + g.inst_off[slot];
      double kconv = wrec[H_KCONV];
      if (maxr <= g.accur) kconv += 1.0;
      wrec[H_KCONV] = kconv;
      if (kconv >= 2.0) wrec[H_DONE] = 1.0;
    }
  }
}

}  // namespace dsp
