// gen_brdf.cuh — bidirectional surfaces of the general solver: the four
// reflectance models of DisortSolver (DisortSolver.cpp:2710-2936) on the
// device, and the kernel that forms a mode's surface table
// (computeSurfaceBidir, DisortSolver.cpp:2582-2708).
//
// The surface's Fourier coefficient of mode m between two polar cosines is
//   R_m(mu, mu') = (2 - delta_m0) sum_k w_k R(mu, mu', pi x_k) cos(m pi x_k)
// over the 100 positive nodes x_k of a 200-node Gauss rule on (-1, 1)
// (weights summing to 1 over the positive half), and the directional
// emissivity of mode 0 is
//   e(mu) = 1 - sum_{j<200} w_j sum_{k<100} w_k x_k R(mu, x_k, pi x_j).
// One CTA per instance forms every entry of the mode's table; a thread per
// (row, column) entry sums its 100 azimuth nodes, and the 20,000-term
// emissivity sums are split over the CTA and reduced in shared memory.
#pragma once

#include "dsp_device.cuh"

namespace dsp {

namespace brdf_detail {
constexpr double PI = 3.14159265358979323846;
}
using brdf_detail::PI;

// ---- reflectance models --------------------------------------------------
// Parameters in the order of the C ABI (dsp.h, dsp_general_batch::brdf_params).

// Hapke opposition-effect model (Hapke 1993, eq. 8.89; DisortSolver.cpp:2710-2732)
__device__ inline double brdf_hapke_d(const double* bp, double mu, double mup, double dphi) {
  const double b0 = bp[0], hh = bp[1], w = bp[2];
  const double cg = mu * mup + sqrt((1.0 - mu * mu) * (1.0 - mup * mup)) * cos(dphi);
  const double half_angle = 0.5 * acos(cg);
  const double opposition = b0 * hh / (hh + tan(half_angle));
  const double gamma = sqrt(1.0 - w);
  const double h_in = (1.0 + 2.0 * mup) / (1.0 + 2.0 * gamma * mup);
  const double h_out = (1.0 + 2.0 * mu) / (1.0 + 2.0 * gamma * mu);
  return 0.25 * w * ((1.0 + opposition) * (1.0 + 0.5 * cg) + h_in * h_out - 1.0) / (mu + mup);
}

// Rahman-Pinty-Verstraete model (DisortSolver.cpp:2734-2780), without the
// clamping of grazing cosines (the reference passes badmu = 0); its azimuth is
// measured from the backward direction
__device__ inline double brdf_rpv_d(const double* bp, double mu1, double mu2, double dphi) {
  const double rho0 = bp[0], k = bp[1], th = bp[2], sigma = bp[3], t1 = bp[4], t2 = bp[5], scale = bp[6];
  const double phi = PI - dphi;
  if (phi == 1.0e-4 && mu1 == mu2) {  // the exact hot-spot direction
    const double hot = rho0 * (pow(2.0 * mu1 * mu1 * mu1, k - 1.0) * (1.0 - th) / ((1.0 + th) * (1.0 + th)) *
                                   (2.0 - rho0) + sigma / mu1) *
                       (t1 * exp(PI * t2) + 1.0);
    return hot * scale;
  }
  const double minnaert = pow(mu1 * mu2 * (mu1 + mu2), k - 1.0);
  const double cphi = cos(phi);
  const double s1 = sqrt(1.0 - mu1 * mu1), s2 = sqrt(1.0 - mu2 * mu2);
  const double cg = mu1 * mu2 + s1 * s2 * cphi;
  const double hg = (1.0 - th * th) / pow(1.0 + 2.0 * th * cg + th * th, 1.5);
  const double ta = s1 / mu1, tb = s2 / mu2;
  const double G = sqrt(ta * ta + tb * tb - 2.0 * ta * tb * cphi);
  const double hot = 1.0 + (1.0 - rho0) / (1.0 + G);
  const double snow = 1.0 + t1 * exp(t2 * (PI - acos(cg)));
  const double v = rho0 * (minnaert * hg * hot + sigma / mu1) * snow * scale;
  return v < 0.0 ? 0.0 : v;
}

// Ross-thick + Li-sparse-reciprocal kernels (DisortSolver.cpp:2782-2836):
// crown height-to-base ratio 2, branch-to-radius ratio 1, hot-spot width 1.5 deg
__device__ inline double brdf_rossli_d(const double* bp, double mu, double mup, double dphi) {
  const double iso = bp[0], vol = bp[1], geo = bp[2];
  const double si = sqrt(1.0 - mup * mup), sr = sqrt(1.0 - mu * mu);
  const double ti = mup > 0.0 ? si / mup : 0.0, tr = mu > 0.0 ? sr / mu : 0.0;
  double sphi, cphi;
  sincos(dphi, &sphi, &cphi);
  const double ca = fmin(fmax(mup * mu + si * sr * cphi, -1.0), 1.0);
  const double alpha = acos(ca);
  const double hot = 1.0 + 1.0 / (1.0 + alpha / (1.5 * PI / 180.0));
  const double k_vol =
      4.0 / (3.0 * PI) * (1.0 / (mup + mu)) * ((PI / 2.0 - alpha) * ca + sin(alpha)) * hot - 1.0 / 3.0;
  // branch/radius ratio 1: the projected angles are the angles themselves
  const double ci1 = 1.0 / sqrt(1.0 + ti * ti), cr1 = 1.0 / sqrt(1.0 + tr * tr);
  const double si1 = ti * ci1, sr1 = tr * cr1;
  const double ca1 = ci1 * cr1 + si1 * sr1 * cphi;
  const double d2 = fmax(ti * ti + tr * tr - 2.0 * ti * tr * cphi, 0.0);
  const double tt = ti * tr * sphi;
  const double ct = 2.0 * (ci1 * cr1) / (ci1 + cr1) * sqrt(d2 + tt * tt);
  const double t = (ct >= -1.0 && ct <= 1.0) ? acos(ct) : 0.0;
  const double k_geo =
      (ci1 + cr1) / (PI * ci1 * cr1) * (t - sin(t) * cos(t) - PI) + (1.0 + ca1) / (2.0 * ci1 * cr1);
  return fmax(iso + vol * k_vol + geo * k_geo, 0.0);
}

// Tsang's shadowing function of the Cox-Munk surface (DisortSolver.cpp:2838-2851)
__device__ inline double brdf_shadow_d(double c, double s2) {
  const double s = sqrt(1.0 - c * c);
  if (s < 1e-15) return 0.0;
  const double cot = c / s;
  return 0.5 * (sqrt(s2 / PI) / cot * exp(-cot * cot / s2) - erfc(cot / sqrt(s2)));
}

// Cox-Munk sea surface: Gaussian slopes of variance 0.003 + 0.00512 u10 with
// Fresnel reflection (DisortSolver.cpp:2853-2900)
__device__ inline double brdf_cox_munk_d(const double* bp, double mu, double mup, double dphi) {
  const double u10 = bp[0], n_t = bp[3];
  const bool shadow = bp[4] != 0.0;
  const double si = sqrt(1.0 - mup * mup), sr = sqrt(1.0 - mu * mu);
  const double ct = -mup * mu + si * sr * cos(dphi);
  const double omc = 1.0 - ct;
  if (omc < 1e-15) return 0.0;
  const double mun2 = (mup + mu) * (mup + mu) / (2.0 * omc);  // squared cosine of the facet normal
  if (mun2 < 1e-15) return 0.0;
  const double s2 = 0.003 + 0.00512 * u10;
  const double slopes = 1.0 / (PI * s2) * exp(-(1.0 - mun2) / (s2 * mun2));
  const double cli = sqrt(0.5 * (1.0 + ct));
  const double sli = sqrt(fmax(0.0, 1.0 - cli * cli));
  const double slt = sli / n_t;
  if (slt >= 1.0) return 0.0;
  const double clt = sqrt(1.0 - slt * slt);
  const double rs = (cli - n_t * clt) / (cli + n_t * clt);
  const double rp = (n_t * cli - clt) / (clt + n_t * cli);
  double v = slopes * (0.5 * (rs * rs + rp * rp)) / (4.0 * mup * mu * mun2 * mun2);
  if (shadow) v *= 1.0 / (brdf_shadow_d(mup, s2) + brdf_shadow_d(mu, s2) + 1.0);
  return fmax(v, 0.0);
}

// bidirReflectivity (DisortSolver.cpp:2902-2936): outgoing mu, incoming mup
__device__ inline double brdf_eval(int type, const double* bp, double mu, double mup, double dphi) {
  switch (type) {
    case DSP_BRDF_RPV: return brdf_rpv_d(bp, mu, mup, dphi);
    case DSP_BRDF_COX_MUNK: return brdf_cox_munk_d(bp, mu, mup, dphi);
    case DSP_BRDF_AMBRALS: return brdf_rossli_d(bp, mu, mup, dphi);
    case DSP_BRDF_HAPKE: return brdf_hapke_d(bp, mu, mup, dphi);
  }
  return 0.0;
}

// ---- the mode's surface table --------------------------------------------
// One CTA of 128 threads per chunk slot.  Rows: quadrature angles 0..NN-1, then
// the user polar angles (zero rows for mu <= 0, as the reference fills only
// upward user angles); columns: beam, NN diffuse streams, emissivity (mode 0).
template <int N>
__global__ void __launch_bounds__(128) gen_brdf_kernel(FluxParams p) {
  constexpr int NN = N / 2, RW = brdf_row(N), NQ = 100;
  __shared__ double s_mu[NQ], s_wt[NQ], s_cw[NQ];  // positive azimuth nodes, weights, w cos(m pi x)
  __shared__ double s_red[128];
  const int slot = blockIdx.x;
  if (slot >= p.n) return;
  const GenView& g = p.g;
  const int i = g.ids[slot];
  const int st0 = p.status ? p.status[i] : 0;
  if (st0 == DSP_ERR_INVALID_INPUT || st0 == DSP_ERR_EIGEN) return;
  const double* rec = p.inst_rec + g.inst_off[slot];
  const int m = g.m;
  if (m > (int)rec[H_NAZ] || rec[H_DONE] != 0.0) return;
  const int t = threadIdx.x;
  for (int k = t; k < NQ; k += blockDim.x) {
    const double x = g.brdf_q[k], w = g.brdf_q[200 + k];
    s_mu[k] = x;
    s_wt[k] = w;
    s_cw[k] = (m == 0) ? w : w * cos(static_cast<double>(m) * PI * x);
  }
  __syncthreads();
  const double* bp = g.brdf_par.row(i);
  const int type = g.brdf_type;
  const double* mu = p.tables + tab_mu(N);
  const double* um = g.umu.row(i);
  const int rows = NN + g.numu;
  const bool beam = rec[H_FBEAM] > 0.0;
  const double umu0 = rec[H_UMU0];
  const double fac = (m == 0) ? 1.0 : 2.0;
  double* tab = g.brdf + (long long)slot * brdf_stride(N, g.numu);
  auto row_mu = [&](int r) { return r < NN ? mu[r] : um[r - NN]; };
  // reflectance entries
  for (int e = t; e < rows * (NN + 1); e += blockDim.x) {
    const int r = e / (NN + 1), c = e % (NN + 1);
    const double out = row_mu(r);
    double v = 0.0;
    if (out > 0.0 && (c > 0 || beam)) {
      const double in = c == 0 ? umu0 : mu[c - 1];
      double s = 0.0;
      for (int k = 0; k < NQ; ++k) s += s_cw[k] * brdf_eval(type, bp, out, in, PI * s_mu[k]);
      v = fac * s;
    }
    tab[r * RW + c] = v;
    // the beam column of the user rows, per mode, for the intensity correction
    if (c == 0 && r >= NN) {
      double* modes = tab + brdf_beam_modes(N, g.numu) + (r - NN) * N;
      if (m == 0)
        for (int mm = 1; mm < N; ++mm) modes[mm] = 0.0;
      modes[m] = v;
    }
  }
  // directional emissivity (mode 0); the azimuth nodes x_j run over both halves
  for (int r = 0; r < rows; ++r) {
    const double out = row_mu(r);
    if (m != 0 || !(out > 0.0)) {
      if (t == 0) tab[r * RW + NN + 1] = 0.0;
      continue;
    }
    double s = 0.0;
    for (int e = t; e < 2 * NQ * NQ; e += blockDim.x) {
      const int j = e / NQ, k = e % NQ;
      const double xj = j < NQ ? s_mu[j] : -s_mu[j - NQ], wj = s_wt[j < NQ ? j : j - NQ];
      s += wj * s_wt[k] * s_mu[k] * brdf_eval(type, bp, out, s_mu[k], PI * xj);
    }
    s_red[t] = s;
    __syncthreads();
    for (int h = 64; h > 0; h >>= 1) {
      if (t < h) s_red[t] += s_red[t + h];
      __syncthreads();
    }
    if (t == 0) tab[r * RW + NN + 1] = 1.0 - s_red[0];
    __syncthreads();
  }
}

}  // namespace dsp
