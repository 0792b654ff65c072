// oracle_common.hpp — CPU restatement of DisORT++ numerics used by the oracle.
//
// TEST INFRASTRUCTURE ONLY.  This directory is the correctness oracle for the
// B200 engine: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg may load it.  The product (disort_b200, libdsp.so) never links or calls it.
//
// The reference (DisORT++) is C++17 on top of Eigen 3.4, which is not present
// here, so the reference cannot be compiled; this is a restatement of its
// algorithms in plain C++, with the dense linear algebra written from textbook
// algorithms (Golub & Van Loan).  Each routine cites the reference lines it
// follows.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------
// Planck band integral (Planck.cpp:35-169, constants Planck.hpp:10-22)
// ---------------------------------------------------------------------------
namespace planck_const {
constexpr double C2 = 1.438786;
constexpr double SIGMA = 5.67032E-8;
constexpr double VCUT = 1.5;
constexpr double A1 = 1.0 / 3.0;
constexpr double A2 = -1.0 / 8.0;
constexpr double A3 = 1.0 / 60.0;
constexpr double A4 = -1.0 / 5040.0;
constexpr double A5 = 1.0 / 272160.0;
constexpr double A6 = -1.0 / 13305600.0;
}  // namespace planck_const

struct PlanckData {
  double vmax, sigdpi, conc, c1;
  PlanckData() {
    vmax = std::log(std::numeric_limits<double>::max());
    sigdpi = planck_const::SIGMA / M_PI;
    conc = 15.0 / std::pow(M_PI, 4.0);
    c1 = 1.1911e-8;
  }
};
inline const PlanckData& planck_data() {
  static const PlanckData d;
  return d;
}

inline double planck_kernel(double v) { return v * v * v / (std::exp(v) - 1.0); }

// planckFunction (Planck.cpp:35-144).  Returns NaN where the reference throws.
inline double planck_function(double wnumlo, double wnumhi, double temp) {
  using namespace planck_const;
  const PlanckData& pd = planck_data();
  if (temp < 0.0 || wnumhi <= wnumlo || wnumlo < 0.0) return std::nan("");
  if (temp < 1.e-4) return 0.0;
  double v[2] = {C2 * wnumlo / temp, C2 * wnumhi / temp};
  // Simpson's rule for close wavenumbers (Planck.cpp:53-85)
  if (v[0] > std::numeric_limits<double>::epsilon() && v[1] < pd.vmax &&
      (wnumhi - wnumlo) / wnumhi < 1.e-2) {
    const double hh = v[1] - v[0];
    double oldval = 0.0;
    const double val0 = planck_kernel(v[0]) + planck_kernel(v[1]);
    for (int n = 1; n <= 10; ++n) {
      const double del = hh / (2.0 * n);
      double val = val0;
      for (int k = 1; k <= 2 * n - 1; ++k) val += 2.0 * (1 + k % 2) * planck_kernel(v[0] + k * del);
      val *= del * A1;
      if (std::abs((val - oldval) / val) <= 1.e-6)
        return pd.sigdpi * std::pow(temp, 4.0) * pd.conc * val;
      oldval = val;
    }
    return pd.sigdpi * std::pow(temp, 4.0) * pd.conc * oldval;
  }
  // Power / exponential series (Planck.cpp:87-143)
  double p[2] = {0.0, 0.0}, d[2] = {0.0, 0.0};
  int smallv = 0;
  constexpr double vcp[7] = {10.25, 5.7, 3.9, 2.9, 2.3, 1.9, 0.0};
  for (int i = 0; i < 2; ++i) {
    if (v[i] < VCUT) {
      smallv++;
      const double vsq = v[i] * v[i];
      p[i] = pd.conc * vsq * v[i] * (A1 + v[i] * (A2 + v[i] * (A3 + vsq * (A4 + vsq * (A5 + vsq * A6)))));
    } else {
      int mmax = 1;
      while (v[i] < vcp[mmax - 1]) mmax++;
      const double ex = std::exp(-v[i]);
      double exm = 1.0;
      d[i] = 0.0;
      for (int m = 1; m <= mmax; ++m) {
        const double mv = m * v[i];
        exm *= ex;
        d[i] += exm * (6.0 + mv * (6.0 + mv * (3.0 + mv))) / (m * m * m * m);
      }
      d[i] *= pd.conc;
    }
  }
  double ans;
  if (smallv == 2) ans = p[1] - p[0];
  else if (smallv == 1) ans = 1.0 - p[0] - d[1];
  else ans = d[0] - d[1];
  ans *= pd.sigdpi * std::pow(temp, 4.0);
  if (ans == 0.0) return 0.0;
  return ans;
}

// planckFunction2 (Planck.cpp:146-169): single-wavenumber form when lo == hi.
inline double planck_function2(double wnumlo, double wnumhi, double temp) {
  if (temp < 0.0 || wnumhi < wnumlo || wnumlo < 0.0) return std::nan("");
  if (temp < 1.e-4) return 0.0;
  if (wnumhi == wnumlo) {
    const double wvn = wnumhi;
    const double arg = std::exp(-planck_const::C2 * wvn / temp);
    return planck_data().c1 * wvn * wvn * wvn * arg / (1.0 - arg);
  }
  return planck_function(wnumlo, wnumhi, temp);
}

// planckFunctionDeriv2 (Planck.cpp:171-214): dB/dT of the band (or single
// wavenumber) Planck function, from the closed form of the derivative of the
// band integral (4 B / T minus the boundary terms of the integration limits).
inline double planck_function_deriv2(double wnumlo, double wnumhi, double temp) {
  using namespace planck_const;
  if (temp < 0.0 || wnumhi < wnumlo || wnumlo < 0.0) return std::nan("");
  if (temp < 1.e-4) return 0.0;
  auto fkernel = [](double v) -> double {  // v^3 / (e^v - 1), v^2 near 0
    if (v < 1.e-6) return v * v;
    const double em = std::exp(-v);
    return v * v * v * em / (1.0 - em);
  };
  if (wnumhi == wnumlo) {
    const double wvn = wnumhi;
    const double x = C2 * wvn / temp;
    const double em = std::exp(-x);
    const double b = planck_data().c1 * wvn * wvn * wvn * em / (1.0 - em);
    return b * (x / temp) / (1.0 - em);
  }
  const double sigdpi = SIGMA / M_PI;
  const double conc = 15.0 / std::pow(M_PI, 4.0);
  const double v0 = C2 * wnumlo / temp;
  const double v1 = C2 * wnumhi / temp;
  const double B = planck_function2(wnumlo, wnumhi, temp);
  const double boundary = sigdpi * conc * temp * temp * temp * (v1 * fkernel(v1) - v0 * fkernel(v0));
  return 4.0 * B / temp - boundary;
}

// ---------------------------------------------------------------------------
// Gauss-Legendre quadrature on (0,1), mirrored (FluxSolver.cpp:257-290)
// mu[0..n-1] > 0, mu[n..2n-1] = -mu[0..n-1]; w likewise.
// ---------------------------------------------------------------------------
inline bool gauss_quadrature(int n, double* mu, double* w) {
  const double eps = 3.0e-14;
  const int max_iter = 10;
  for (int i = 1; i <= n; ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (n + 0.5));
    double z1, pp;
    int iter = 0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= n; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
      if (++iter > max_iter) return false;
    } while (std::abs(z - z1) > eps);
    mu[i - 1] = 0.5 * (1.0 + z);
    w[i - 1] = 1.0 / ((1.0 - z * z) * pp * pp);
  }
  for (int i = 0; i < n; ++i) {
    mu[n + i] = -mu[i];
    w[n + i] = w[i];
  }
  return true;
}

// ---------------------------------------------------------------------------
// Normalised associated Legendre polynomials (Legendre.cpp:67-120)
// ylm[l * ld + i] = P_l^m(mu[i]).  For m > 0 the seed reads row m-1, which must
// hold the values left by the call for mode m-1 (Legendre.cpp:90-103).
// ---------------------------------------------------------------------------
inline void legendre_flat(int nmu, int m, int ld, int twonm1, const double* mu, double* ylm) {
  if (m == 0) {
    for (int i = 0; i < nmu; ++i) {
      ylm[0 * ld + i] = 1.0;
      if (twonm1 >= 1) ylm[1 * ld + i] = mu[i];
    }
    for (int l = 2; l <= twonm1; ++l)
      for (int i = 0; i < nmu; ++i)
        ylm[l * ld + i] = ((2.0 * l - 1.0) * mu[i] * ylm[(l - 1) * ld + i] - (l - 1.0) * ylm[(l - 2) * ld + i]) / l;
  } else {
    for (int i = 0; i < nmu; ++i) {
      ylm[m * ld + i] = -std::sqrt((1.0 - 1.0 / (2.0 * m)) * (1.0 - mu[i] * mu[i])) * ylm[(m - 1) * ld + i];
      if (m + 1 <= twonm1) ylm[(m + 1) * ld + i] = std::sqrt(2.0 * m + 1.0) * mu[i] * ylm[m * ld + i];
    }
    for (int l = m + 2; l <= twonm1; ++l) {
      const double tmp1 = std::sqrt(static_cast<double>((l - m) * (l + m)));
      const double tmp2 = std::sqrt(static_cast<double>((l - m - 1) * (l + m - 1)));
      for (int i = 0; i < nmu; ++i)
        ylm[l * ld + i] = ((2.0 * l - 1.0) * mu[i] * ylm[(l - 1) * ld + i] - tmp2 * ylm[(l - 2) * ld + i]) / tmp1;
    }
  }
}

// ---------------------------------------------------------------------------
// Dense linear algebra, row-major n x n with leading dimension ld.
// ---------------------------------------------------------------------------

// LU with partial (row) pivoting, in place: the stand-in for Eigen::PartialPivLU
// used at FluxSolver.cpp:634 and :758.  Returns false on an exactly zero pivot.
inline bool lu_factor(double* a, int n, int ld, int* piv) {
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = std::abs(a[k * ld + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = std::abs(a[i * ld + k]);
      if (v > amax) { amax = v; p = i; }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[k * ld + j], a[p * ld + j]);
    const double akk = a[k * ld + k];
    if (akk == 0.0) { ok = false; continue; }
    for (int i = k + 1; i < n; ++i) {
      const double lik = a[i * ld + k] / akk;
      a[i * ld + k] = lik;
      for (int j = k + 1; j < n; ++j) a[i * ld + j] -= lik * a[k * ld + j];
    }
  }
  return ok;
}

inline void lu_solve(const double* a, int n, int ld, const int* piv, double* b) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k) std::swap(b[k], b[piv[k]]);
  for (int i = 1; i < n; ++i) {
    double s = b[i];
    for (int j = 0; j < i; ++j) s -= a[i * ld + j] * b[j];
    b[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < n; ++j) s -= a[i * ld + j] * b[j];
    b[i] = s / a[i * ld + i];
  }
}

// Cholesky A = L L^T from the lower triangle (Eigen::LLT semantics used at
// FluxSolver.cpp:523-524): fails on a non-positive pivot.  L is written to l
// (full n x n, zeros above the diagonal).
inline bool cholesky_lower(const double* a, int n, int ld, double* l) {
  for (int i = 0; i < n * ld; ++i) l[i] = 0.0;
  for (int j = 0; j < n; ++j) {
    double d = a[j * ld + j];
    for (int k = 0; k < j; ++k) d -= l[j * ld + k] * l[j * ld + k];
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    l[j * ld + j] = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = a[i * ld + j];
      for (int k = 0; k < j; ++k) s -= l[i * ld + k] * l[j * ld + k];
      l[i * ld + j] = s / ljj;
    }
  }
  return true;
}

// Symmetric eigensolver (stand-in for Eigen::SelfAdjointEigenSolver,
// FluxSolver.cpp:542): Householder tridiagonalisation followed by implicit
// symmetric QR steps with Wilkinson shifts (Golub & Van Loan, Alg. 8.3.1 and
// 8.3.3).  Reads the lower triangle of a.  Eigenvalues ascending in evals,
// eigenvectors as columns of z (row-major, ld).  Work arrays are local.
inline void sym_eigen(const double* a_in, int n, int ld, double* evals, double* z) {
  constexpr int NMAX = 64;
  double a[NMAX * NMAX];
  double d[NMAX], e[NMAX];
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const int ii = std::max(i, j), jj = std::min(i, j);
      a[i * n + j] = a_in[ii * ld + jj];
    }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) z[i * ld + j] = (i == j) ? 1.0 : 0.0;
  // Householder tridiagonalisation: A <- H A H, Z <- Z H
  double v[NMAX], p[NMAX], w[NMAX];
  for (int k = 0; k + 2 < n; ++k) {
    double xnorm2 = 0.0;
    for (int i = k + 1; i < n; ++i) xnorm2 += a[i * n + k] * a[i * n + k];
    const double x0 = a[(k + 1) * n + k];
    double tail2 = xnorm2 - x0 * x0;
    if (tail2 == 0.0) continue;
    const double alpha = (x0 >= 0.0) ? -std::sqrt(xnorm2) : std::sqrt(xnorm2);
    for (int i = k + 1; i < n; ++i) v[i] = a[i * n + k];
    v[k + 1] -= alpha;
    double vnorm2 = 0.0;
    for (int i = k + 1; i < n; ++i) vnorm2 += v[i] * v[i];
    const double beta = 2.0 / vnorm2;
    // p = beta * A_sub v
    for (int i = k + 1; i < n; ++i) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += a[i * n + j] * v[j];
      p[i] = beta * s;
    }
    double vp = 0.0;
    for (int i = k + 1; i < n; ++i) vp += v[i] * p[i];
    const double kk = 0.5 * beta * vp;
    for (int i = k + 1; i < n; ++i) w[i] = p[i] - kk * v[i];
    for (int i = k + 1; i < n; ++i)
      for (int j = k + 1; j < n; ++j) a[i * n + j] -= v[i] * w[j] + w[i] * v[j];
    a[(k + 1) * n + k] = alpha;
    a[k * n + k + 1] = alpha;
    for (int i = k + 2; i < n; ++i) { a[i * n + k] = 0.0; a[k * n + i] = 0.0; }
    // Z <- Z (I - beta v v^T)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = k + 1; j < n; ++j) s += z[i * ld + j] * v[j];
      s *= beta;
      for (int j = k + 1; j < n; ++j) z[i * ld + j] -= s * v[j];
    }
  }
  for (int i = 0; i < n; ++i) d[i] = a[i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = a[(i + 1) * n + i];
  e[n - 1] = 0.0;
  // implicit symmetric QR with Wilkinson shift on (d, e)
  const double eps = std::numeric_limits<double>::epsilon();
  int q = n - 1;
  int iter = 0;
  while (q > 0 && iter < 60 * n) {
    // deflate
    for (int i = 0; i < q; ++i)
      if (std::abs(e[i]) <= eps * (std::abs(d[i]) + std::abs(d[i + 1]))) e[i] = 0.0;
    while (q > 0 && e[q - 1] == 0.0) --q;
    if (q == 0) break;
    int p0 = q - 1;
    while (p0 > 0 && e[p0 - 1] != 0.0) --p0;
    ++iter;
    // Wilkinson shift from the trailing 2x2 of block [p0..q]
    const double dd = 0.5 * (d[q - 1] - d[q]);
    const double ee = e[q - 1];
    const double sgn = (dd >= 0.0) ? 1.0 : -1.0;
    const double mu = d[q] - ee * ee / (dd + sgn * std::hypot(dd, ee));
    double x = d[p0] - mu;
    double y = e[p0];
    for (int k = p0; k < q; ++k) {
      // Givens rotation zeroing y against x
      double c, s;
      if (y == 0.0) { c = 1.0; s = 0.0; }
      else if (std::abs(y) > std::abs(x)) { const double t = -x / y; s = 1.0 / std::sqrt(1.0 + t * t); c = s * t; }
      else { const double t = -y / x; c = 1.0 / std::sqrt(1.0 + t * t); s = c * t; }
      if (k > p0) e[k - 1] = c * x - s * y;
      const double dk = d[k], dk1 = d[k + 1], ek = e[k];
      // T(k:k+1,k:k+1) <- G^T T G, G = [c s; -s c]
      d[k] = c * c * dk - 2.0 * c * s * ek + s * s * dk1;
      d[k + 1] = s * s * dk + 2.0 * c * s * ek + c * c * dk1;
      e[k] = c * s * (dk - dk1) + (c * c - s * s) * ek;
      if (k + 1 < q) {
        x = e[k];
        y = -s * e[k + 1];
        e[k + 1] *= c;
      }
      for (int i = 0; i < n; ++i) {
        const double zk = z[i * ld + k], zk1 = z[i * ld + k + 1];
        z[i * ld + k] = c * zk - s * zk1;
        z[i * ld + k + 1] = s * zk + c * zk1;
      }
    }
  }
  // sort ascending (Eigen's order); columns of z follow
  for (int i = 0; i < n; ++i) evals[i] = d[i];
  for (int i = 0; i < n - 1; ++i) {
    int kmin = i;
    for (int j = i + 1; j < n; ++j)
      if (evals[j] < evals[kmin]) kmin = j;
    if (kmin != i) {
      std::swap(evals[i], evals[kmin]);
      for (int r = 0; r < n; ++r) std::swap(z[r * ld + i], z[r * ld + kmin]);
    }
  }
}

// ---------------------------------------------------------------------------
// Bidirectional surface reflectance (DisortSolver.cpp:2710-2936).  `bp` holds
// the parameters of the model in the C ABI's order (include/dsp.h,
// dsp_general_batch::brdf_params):
//   RPV      rho0, k, theta, sigma, t1, t2, scale
//   CoxMunk  u10, pcl, xsal, refractive_index, do_shadow (0 / 1)
//   Ambrals  iso, vol, geo
//   Hapke    b0, hh, w
// ---------------------------------------------------------------------------
enum { BRDF_LAMBERT = 0, BRDF_RPV = 1, BRDF_COX_MUNK = 2, BRDF_AMBRALS = 3, BRDF_HAPKE = 4 };

// bidirReflectivityHapke (DisortSolver.cpp:2710-2732)
inline double brdf_hapke(const double* bp, double mu, double mup, double dphi) {
  const double b0 = bp[0], hh = bp[1], w = bp[2];
  const double ctheta = mu * mup + std::sqrt((1.0 - mu * mu) * (1.0 - mup * mup)) * std::cos(dphi);
  const double thetah = std::acos(ctheta);
  const double p = 1.0 + 0.5 * ctheta;
  const double b = b0 * hh / (hh + std::tan(0.5 * thetah));
  const double gam = std::sqrt(1.0 - w);
  const double h0 = (1.0 + 2.0 * mup) / (1.0 + 2.0 * gam * mup);
  const double h = (1.0 + 2.0 * mu) / (1.0 + 2.0 * gam * mu);
  return 0.25 * w * ((1.0 + b) * p + h0 * h - 1.0) / (mu + mup);
}

// bidirReflectivityRpv (DisortSolver.cpp:2734-2780), called with badmu = 0
// (DisortSolver.cpp:2915-2918): no clamping of the cosines
inline double brdf_rpv(const double* bp, double mu1, double mu2, double phi) {
  const double rho0 = bp[0], k = bp[1], th = bp[2], sigma = bp[3], t1 = bp[4], t2 = bp[5], scale = bp[6];
  phi = M_PI - phi;  // RPV measures the azimuth from the backward direction
  const double hspot = rho0 * (std::pow(2.0 * mu1 * mu1 * mu1, k - 1.0) * (1.0 - th) / ((1.0 + th) * (1.0 + th)) *
                                   (2.0 - rho0) + sigma / mu1) *
                       (t1 * std::exp(M_PI * t2) + 1.0);
  if (phi == 1.0e-4 && mu1 == mu2) return hspot * scale;
  const double m = std::pow(mu1 * mu2 * (mu1 + mu2), k - 1.0);
  const double cosphi = std::cos(phi);
  const double sin1 = std::sqrt(1.0 - mu1 * mu1), sin2 = std::sqrt(1.0 - mu2 * mu2);
  const double cosg = mu1 * mu2 + sin1 * sin2 * cosphi;
  const double g = std::acos(cosg);
  const double f = (1.0 - th * th) / std::pow(1.0 + 2.0 * th * cosg + th * th, 1.5);
  const double tan1 = sin1 / mu1, tan2 = sin2 / mu2;
  const double capg = std::sqrt(tan1 * tan1 + tan2 * tan2 - 2.0 * tan1 * tan2 * cosphi);
  const double hval = 1.0 + (1.0 - rho0) / (1.0 + capg);
  const double t = 1.0 + t1 * std::exp(t2 * (M_PI - g));
  const double ans = rho0 * (m * f * hval + sigma / mu1) * t * scale;
  return ans < 0.0 ? 0.0 : ans;
}

// bidirReflectivityRossLi (DisortSolver.cpp:2782-2836): Ross-thick volume and
// Li-sparse-reciprocal geometric kernels, crown height/base 2, branch/radius 1,
// hot-spot width 1.5 degrees
inline double brdf_rossli(const double* bp, double mu, double mup, double dphi) {
  const double iso = bp[0], vol = bp[1], geo = bp[2];
  const double hb = 2.0, br = 1.0, alpha0 = 1.5 * M_PI / 180.0;
  const double sin_i = std::sqrt(1.0 - mup * mup), sin_r = std::sqrt(1.0 - mu * mu);
  const double tan_i = mup > 0.0 ? sin_i / mup : 0.0, tan_r = mu > 0.0 ? sin_r / mu : 0.0;
  double cos_a = mup * mu + sin_i * sin_r * std::cos(dphi);
  cos_a = std::min(std::max(cos_a, -1.0), 1.0);
  const double alpha = std::acos(cos_a), sin_a = std::sin(alpha);
  const double cc = 1.0 + 1.0 / (1.0 + alpha / alpha0);
  const double f_vol = 4.0 / (3.0 * M_PI) * (1.0 / (mup + mu)) * ((M_PI / 2.0 - alpha) * cos_a + sin_a) * cc - 1.0 / 3.0;
  const double ti = br * tan_i, tr = br * tan_r;
  const double ci = 1.0 / std::sqrt(1.0 + ti * ti), cr = 1.0 / std::sqrt(1.0 + tr * tr);
  const double si = ti * ci, sr = tr * cr;
  const double cos_a1 = ci * cr + si * sr * std::cos(dphi);
  double g2 = ti * ti + tr * tr - 2.0 * ti * tr * std::cos(dphi);
  if (g2 < 0.0) g2 = 0.0;
  const double cos_t = hb * (ci * cr) / (ci + cr) * std::sqrt(g2 + std::pow(ti * tr * std::sin(dphi), 2));
  double t = 0.0;
  if (cos_t >= -1.0 && cos_t <= 1.0) t = std::acos(cos_t);
  const double f_geo = (ci + cr) / (M_PI * ci * cr) * (t - std::sin(t) * std::cos(t) - M_PI) + (1.0 + cos_a1) / (2.0 * ci * cr);
  return std::max(iso + vol * f_vol + geo * f_geo, 0.0);
}

// shadowEta (DisortSolver.cpp:2838-2851): Tsang's shadowing function
inline double brdf_shadow_eta(double cos_theta, double sigma_sq) {
  const double sin_theta = std::sqrt(1.0 - cos_theta * cos_theta);
  if (sin_theta < 1e-15) return 0.0;
  const double cot = cos_theta / sin_theta;
  const double t1 = std::sqrt(sigma_sq / M_PI) / cot * std::exp(-cot * cot / sigma_sq);
  const double t2 = std::erfc(cot / std::sqrt(sigma_sq));
  return 0.5 * (t1 - t2);
}

// bidirReflectivityCoxMunk (DisortSolver.cpp:2853-2900)
inline double brdf_cox_munk(const double* bp, double mu, double mup, double dphi) {
  const double u10 = bp[0], nt = bp[3];
  const bool shadow = bp[4] != 0.0;
  const double sin_i = std::sqrt(1.0 - mup * mup), sin_r = std::sqrt(1.0 - mu * mu);
  const double cos_theta = -mup * mu + sin_i * sin_r * std::cos(dphi);
  const double omc = 1.0 - cos_theta;
  if (omc < 1e-15) return 0.0;
  const double mun2 = (mup + mu) * (mup + mu) / (2.0 * omc);
  if (mun2 < 1e-15) return 0.0;
  const double s2 = 0.003 + 0.00512 * u10;
  const double p_slope = 1.0 / (M_PI * s2) * std::exp(-(1.0 - mun2) / (s2 * mun2));
  const double ni = 1.0;
  const double cos_li = std::sqrt(0.5 * (1.0 + cos_theta));
  const double sin_li = std::sqrt(std::max(0.0, 1.0 - cos_li * cos_li));
  const double sin_lt = ni * sin_li / nt;
  if (sin_lt >= 1.0) return 0.0;
  const double cos_lt = std::sqrt(1.0 - sin_lt * sin_lt);
  const double rs = (ni * cos_li - nt * cos_lt) / (ni * cos_li + nt * cos_lt);
  const double rp = (nt * cos_li - ni * cos_lt) / (ni * cos_lt + nt * cos_li);
  const double rf = 0.5 * (rs * rs + rp * rp);
  double v = (p_slope * rf) / (4.0 * mup * mu * mun2 * mun2);
  if (shadow) v *= 1.0 / (brdf_shadow_eta(mup, s2) + brdf_shadow_eta(mu, s2) + 1.0);
  return std::max(v, 0.0);
}

// bidirReflectivity (DisortSolver.cpp:2902-2936)
inline double brdf_value(int type, const double* bp, double mu, double mup, double dphi) {
  switch (type) {
    case BRDF_HAPKE: return brdf_hapke(bp, mu, mup, dphi);
    case BRDF_RPV: return brdf_rpv(bp, mu, mup, dphi);
    case BRDF_COX_MUNK: return brdf_cox_munk(bp, mu, mup, dphi);
    case BRDF_AMBRALS: return brdf_rossli(bp, mu, mup, dphi);
  }
  return std::numeric_limits<double>::quiet_NaN();
}

// computeSurfaceBidir (DisortSolver.cpp:2582-2708) for one azimuth mode m:
//   rq[iq][0]      direct-beam reflectance at quadrature angle iq
//   rq[iq][1 + jq] diffuse reflectance, incoming stream jq, outgoing iq
//   eq[iq]         directional emissivity (mode 0)
//   ru[iu][...], eu[iu] the same at the user polar angles (mu > 0 only)
// with the 100-point half-range Gauss quadrature of the azimuth (NMUG = 200,
// DisortSolver.cpp:484-496).  Lambertian: the albedo at mode 0, zero above.
struct SurfaceTables {
  int NN = 0, numu = 0;
  std::vector<double> rq, eq, ru, eu;
  std::vector<double> gmu, gwt;  // the azimuth quadrature, 200 nodes
  void init(int nn, int nu) {
    NN = nn;
    numu = nu;
    rq.assign((size_t)NN * (NN + 1), 0.0);
    eq.assign(NN, 0.0);
    ru.assign((size_t)std::max(numu, 1) * (NN + 1), 0.0);
    eu.assign(std::max(numu, 1), 0.0);
    gmu.assign(200, 0.0);
    gwt.assign(200, 0.0);
    gauss_quadrature(100, gmu.data(), gwt.data());
  }
  double& RQ(int iq, int j) { return rq[(size_t)iq * (NN + 1) + j]; }
  double& RU(int iu, int j) { return ru[(size_t)iu * (NN + 1) + j]; }
  void fill(int type, const double* bp, double alb, int m, const double* mu, const double* umu, bool user,
            double fbeam, double umu0) {
    const double d0 = m == 0 ? 1.0 : 0.0;
    std::fill(rq.begin(), rq.end(), 0.0);
    std::fill(eq.begin(), eq.end(), 0.0);
    auto fourier = [&](double a, double b) {
      double s = 0.0;
      for (int k = 0; k < 100; ++k)
        s += gwt[k] * brdf_value(type, bp, a, b, M_PI * gmu[k]) * std::cos(static_cast<double>(m) * M_PI * gmu[k]);
      return (2.0 - d0) * s;
    };
    auto emissivity = [&](double a) {
      double dref = 0.0;
      for (int jg = 0; jg < 200; ++jg) {
        double s = 0.0;
        for (int k = 0; k < 100; ++k) s += gwt[k] * gmu[k] * brdf_value(type, bp, a, gmu[k], M_PI * gmu[jg]);
        dref += gwt[jg] * s;
      }
      return 1.0 - dref;
    };
    if (type == BRDF_LAMBERT) {
      if (m == 0)
        for (int iq = 0; iq < NN; ++iq) {
          eq[iq] = 1.0 - alb;
          for (int j = 0; j <= NN; ++j) RQ(iq, j) = alb;
        }
    } else {
      for (int iq = 0; iq < NN; ++iq) {
        for (int jq = 0; jq < NN; ++jq) RQ(iq, jq + 1) = fourier(mu[iq], mu[jq]);
        if (fbeam > 0.0) RQ(iq, 0) = fourier(mu[iq], umu0);
      }
      if (m == 0)
        for (int iq = 0; iq < NN; ++iq) eq[iq] = emissivity(mu[iq]);
    }
    if (!user) return;
    std::fill(ru.begin(), ru.end(), 0.0);
    std::fill(eu.begin(), eu.end(), 0.0);
    for (int iu = 0; iu < numu; ++iu) {
      const double u = umu[iu];
      if (u <= 0.0) continue;
      if (type == BRDF_LAMBERT) {
        if (m == 0) {
          for (int j = 0; j <= NN; ++j) RU(iu, j) = alb;
          eu[iu] = 1.0 - alb;
        }
      } else {
        for (int jq = 0; jq < NN; ++jq) RU(iu, jq + 1) = fourier(u, mu[jq]);
        if (fbeam > 0.0) RU(iu, 0) = fourier(u, umu0);
        if (m == 0) eu[iu] = emissivity(u);
      }
    }
  }
};

}  // namespace oracle
