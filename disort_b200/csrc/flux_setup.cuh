// flux_setup.cuh — per-instance setup: validation, delta-M / delta-M+ scaling,
// optical-depth scans, absorption cut, beam transmission and level Planck values.
//
// One warp per instance; lanes run over layers/levels, lane 0 does the scans in
// the reference's sequential order so cumulative depths round identically.
#pragma once

#include "dsp_device.cuh"

namespace dsp {

// planckFunction / planckFunction2 (Planck.cpp:35-169).  NaN where the reference throws.
__device__ __forceinline__ double planck_kernel(double v) { return v * v * v / (exp(v) - 1.0); }

static __device__ double planck2(double lo, double hi, double T, const PlanckConsts& pk) {
  constexpr double C2 = 1.438786, A1 = 1.0 / 3.0, A2 = -1.0 / 8.0, A3 = 1.0 / 60.0,
                   A4 = -1.0 / 5040.0, A5 = 1.0 / 272160.0, A6 = -1.0 / 13305600.0, VCUT = 1.5;
  if (T < 0.0 || hi < lo || lo < 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  if (T < 1.e-4) return 0.0;
  if (hi == lo) {
    const double arg = exp(-C2 * hi / T);
    return pk.c1 * hi * hi * hi * arg / (1.0 - arg);
  }
  const double v0 = C2 * lo / T, v1 = C2 * hi / T;
  if (v0 > 2.220446049250313e-16 && v1 < pk.vmax && (hi - lo) / hi < 1.e-2) {
    const double hh = v1 - v0;
    double oldval = 0.0;
    const double val0 = planck_kernel(v0) + planck_kernel(v1);
    for (int n = 1; n <= 10; ++n) {
      const double del = hh / (2.0 * n);
      double val = val0;
      for (int k = 1; k <= 2 * n - 1; ++k) val += 2.0 * (1 + k % 2) * planck_kernel(v0 + k * del);
      val *= del * A1;
      if (fabs((val - oldval) / val) <= 1.e-6) return pk.sigdpi * pow(T, 4.0) * pk.conc * val;
      oldval = val;
    }
    return pk.sigdpi * pow(T, 4.0) * pk.conc * oldval;
  }
  const double v[2] = {v0, v1};
  double pp[2] = {0.0, 0.0}, d[2] = {0.0, 0.0};
  int smallv = 0;
  const double vcp[7] = {10.25, 5.7, 3.9, 2.9, 2.3, 1.9, 0.0};
  for (int i = 0; i < 2; ++i) {
    if (v[i] < VCUT) {
      smallv++;
      const double vsq = v[i] * v[i];
      pp[i] = pk.conc * vsq * v[i] * (A1 + v[i] * (A2 + v[i] * (A3 + vsq * (A4 + vsq * (A5 + vsq * A6)))));
    } else {
      int mmax = 1;
      while (v[i] < vcp[mmax - 1]) mmax++;
      const double ex = exp(-v[i]);
      double exm = 1.0;
      d[i] = 0.0;
      for (int m = 1; m <= mmax; ++m) {
        const double mv = m * v[i];
        exm *= ex;
        d[i] += exm * (6.0 + mv * (6.0 + mv * (3.0 + mv))) / (m * m * m * m);
      }
      d[i] *= pk.conc;
    }
  }
  double ans;
  if (smallv == 2) ans = pp[1] - pp[0];
  else if (smallv == 1) ans = 1.0 - pp[0] - d[1];
  else ans = d[0] - d[1];
  ans *= pk.sigdpi * pow(T, 4.0);
  if (ans == 0.0) return 0.0;
  return ans;
}

// Henyey-Greenstein moments of a DSP_FLAG_HG_G batch: moment k of (instance i,
// layer lc) is g^k formed by k successive products from 1, the order of
// fillHenyeyGreenstein (PhaseFunction.cpp:6-19), so it equals a host-side fill
// bit for bit.  One thread per output element: consecutive threads write
// consecutive doubles of out[i][lc][k].
static __global__ void __launch_bounds__(256) hg_moments_kernel(DArr g, long long n_rows, int L, int pc,
                                                                double* out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n_rows * pc) return;
  const long long row = t / pc;
  const int k = (int)(t - row * pc);
  const long long i = row / L;
  const double gv = g(i, row - i * L);
  double gk = 1.0;
  for (int j = 0; j < k; ++j) gk *= gv;
  out[t] = gk;
}

// Four instances per 128-thread CTA, one warp each.
static __global__ void __launch_bounds__(128) flux_setup_kernel(FluxParams p) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * 4 + warp;
  if (i >= p.n) return;
  const int N = p.N, L = p.L;
  const InstLayout& il = p.il;
  double* rec = p.inst_rec + (long long)i * il.stride;
  const bool thermal = (p.flags & DSP_FLAG_THERMAL) != 0;
  const bool dlbc = (p.flags & DSP_FLAG_DIFFUSION_LOWER_BC) != 0;
  const double fbeam = p.fbeam(i), umu0 = p.umu0(i), alb = p.alb(i), emis = p.emis(i);
  const double wlo = p.wlo(i), whi = p.whi(i), ttop = p.ttop(i), tbot = p.tbot(i);
  // index_from_bottom: inputs are given bottom-up (IndexConversion.hpp:42-52);
  // the solver works top-down, so layer lc reads entry L-1-lc, level lev entry L-lev
  const bool ifb = (p.flags & DSP_FLAG_INDEX_FROM_BOTTOM) != 0;
  const double* dtau_in = p.dtau.row(i);
  const double* ssa_in = p.ssa.row(i);
  const double* pm_in = p.pmom.row(i);
  const double* temp_in = thermal ? p.temp.row(i) : nullptr;
  const int pc = p.pc;
  auto dtau_at = [&](int lc) { return dtau_in[ifb ? L - 1 - lc : lc]; };
  auto ssa_at = [&](int lc) { return ssa_in[ifb ? L - 1 - lc : lc]; };
  auto pm_row = [&](int lc) { return pm_in + (long long)(ifb ? L - 1 - lc : lc) * pc; };
  auto temp_at = [&](int lev) { return temp_in[ifb ? L - lev : lev]; };

  // ---- validate() (DisortFluxConfig.cpp:43-143) -------------------------
  bool bad = false;
  for (int lc = lane; lc < L; lc += 32) {
    if (dtau_at(lc) < 0.0) bad = true;
    if (ssa_at(lc) < 0.0 || ssa_at(lc) > 1.0) bad = true;
  }
  if (thermal)
    for (int lev = lane; lev <= L; lev += 32)
      if (temp_at(lev) < 0.0) bad = true;
  if (lane == 0) {
    if (dlbc && !thermal) bad = true;
    if (fbeam < 0.0) bad = true;
    if (fbeam > 0.0 && (umu0 <= 0.0 || umu0 > 1.0)) bad = true;
    if (alb < 0.0 || alb > 1.0) bad = true;
    if (thermal) {
      if (wlo < 0.0 || wlo > whi) bad = true;
      if (ttop < 0.0 || tbot < 0.0) bad = true;
      if (emis < 0.0 || emis > 1.0) bad = true;
    }
    if ((p.flags & DSP_FLAG_DELTA_M_PLUS) && p.nmom < N + 1) bad = true;
    // bottom_radius > 0 with the pseudo-spherical beam (DisortFluxConfig.cpp:127-133)
    if ((p.flags & DSP_FLAG_SPHERICAL_BEAM) && !(p.rbot(i) > 0.0)) bad = true;
  }
  if (__any_sync(0xffffffffu, bad)) {
    if (lane == 0) set_status(p.status, i, DSP_ERR_INVALID_INPUT);
    return;
  }

  // ---- delta-M decisions (FluxSolver.cpp:56-81) -------------------------
  bool dm_local = false, dmp_fail = false;
  for (int lc = lane; lc < L; lc += 32) {
    const double pmN = pm_row(lc)[N];
    if (pmN != 0.0) dm_local = true;
    if (p.flags & DSP_FLAG_DELTA_M_PLUS) {
      const double pmN1 = pm_row(lc)[N + 1];
      if (pmN < 1e-4 || pmN1 < 0.7 * pmN) dmp_fail = true;
    }
  }
  bool deltam = __any_sync(0xffffffffu, dm_local);
  bool dmplus = (p.flags & DSP_FLAG_DELTA_M_PLUS) && !__any_sync(0xffffffffu, dmp_fail);
  if (dmplus) deltam = false;

  // ---- per-layer scaling (disortSet, FluxSolver.cpp:333-387) -------------
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
  // Planck at the levels (computeIsotropicSource, FluxSolver.cpp:748-752)
  if (thermal)
    for (int lev = lane; lev <= L; lev += 32) rec[il.pkag + lev] = planck2(wlo, whi, temp_at(lev), p.pk);
  __syncwarp();

  if (lane == 0) {
    // cumulative depths, absorption cut (FluxSolver.cpp:312-331, 429-435)
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
    // beam transmission for lc < ncut of the absorption loop (FluxSolver.cpp:391-412);
    // later entries stay zero, as on a freshly constructed reference solver
    for (int lev = 0; lev <= L; ++lev) rec[il.btr + lev] = 0.0;
    if (fbeam > 0.0) {
      rec[il.btr] = 1.0;
      for (int lc = 0; lc < ncut; ++lc) rec[il.btr + lc + 1] = exp(-rec[il.tau_s + lc + 1] / umu0);
    }
    const bool lyrcut = (abstau >= abscut && !thermal && L > 1);
    if (!lyrcut) ncut = L;
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
    // Legendre at -mu0 (FluxSolver.cpp:601-602), m = 0 recurrence
    if (fbeam > 0.0) {
      const double x = -umu0;
      double y0 = 1.0, y1 = x;
      rec[il.yb + 0] = 1.0;
      rec[il.yb + 1] = x;
      for (int l = 2; l <= N - 1; ++l) {
        const double y2 = ((2.0 * l - 1.0) * x * y1 - (l - 1.0) * y0) / l;
        rec[il.yb + l] = y2;
        y0 = y1;
        y1 = y2;
      }
    }
  }
}

}  // namespace dsp
