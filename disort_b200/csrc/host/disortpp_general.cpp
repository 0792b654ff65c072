// disortpp_general.cpp — the general DisORT++ API (DisortConfig, DisortResult,
// DisortSolver, solveSpectralBands) on top of dsp_general_bands_solve.
//
// DisortConfig's constructor, allocate() and validate() follow
// DisortConfig.cpp:10-248 rule for rule and message for message; the solver
// entry points follow DisortSolver::solve's handling of the config
// (DisortSolver.cpp:20-67, 640-660, 840-850) and the spectral loops of
// python_bindings.cpp:89-127, with every band of a loop in one GPU batch.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/disortpp/disortpp.hpp"
#include "../../../include/dsp.h"

namespace disortpp {

namespace detail {
std::mutex& engine_mutex();
dsp_context engine_context_locked();
}  // namespace detail

// ---------------------------------------------------------------------------
// DisortConfig
// ---------------------------------------------------------------------------
DisortConfig::DisortConfig(int nlyr, int nstr, int nmom)
    : num_layers(nlyr), num_phase_func_moments(nmom), num_streams(nstr) {
  if (num_layers <= 0) throw std::invalid_argument("num_layers must be positive");
  if (num_streams < 4 || num_streams % 2 != 0) throw std::invalid_argument("num_streams must be even and >= 4");
  if (num_phase_func_moments < 0) throw std::invalid_argument("num_phase_func_moments must be non-negative");
}

void DisortConfig::allocate() {
  delta_tau.resize(num_layers);
  single_scat_albedo.resize(num_layers);
  phase_function_moments.resize(num_layers, std::vector<double>(nmomNstr() + 1, 0.0));
  if (flags.use_thermal_emission) temperature.resize(num_layers + 1);
  if (num_user_tau > 0) tau_user.resize(num_user_tau);
  if (num_user_mu > 0) mu_user.resize(num_user_mu);
  if (!flags.comp_only_fluxes && num_phi > 0) phi_user.resize(num_phi);
  if (flags.use_spherical_beam) {
    if (bottom_radius <= 0.0)
      throw std::invalid_argument("bottom_radius must be positive when use_spherical_beam=true");
    level_altitudes.resize(num_layers + 1);
  }
  if (flags.intensity_corr_buras && !flags.intensity_corr_nakajima && num_phase_func_angles > 0) {
    mu_phase_function.resize(num_phase_func_angles);
    phase_function.resize(num_layers, std::vector<double>(num_phase_func_angles, 0.0));
  }
}

void DisortConfig::validate() const {
  if (num_layers <= 0) throw std::invalid_argument("num_layers must be positive");
  if (num_streams < 4) throw std::invalid_argument("num_streams must be >= 4");
  if (num_streams % 2 != 0) throw std::invalid_argument("num_streams must be even");
  if (num_phase_func_moments < 0) throw std::invalid_argument("num_phase_func_moments must be non-negative");
  if (delta_tau.size() < static_cast<size_t>(num_layers)) throw std::invalid_argument("delta_tau array is too small");
  if (single_scat_albedo.size() < static_cast<size_t>(num_layers))
    throw std::invalid_argument("single_scat_albedo array is too small");
  if (static_cast<int>(phase_function_moments.size()) < num_layers)
    throw std::invalid_argument("phase_function_moments must have at least num_layers layers");
  for (int lc = 0; lc < num_layers; ++lc)
    if (static_cast<int>(phase_function_moments[lc].size()) < nmomNstr() + 1)
      throw std::invalid_argument("phase_function_moments[" + std::to_string(lc) +
                                  "] must have at least nmomNstr()+1 elements");
  for (int lc = 0; lc < num_layers; ++lc) {
    if (delta_tau[lc] < 0.0) throw std::invalid_argument("delta_tau[" + std::to_string(lc) + "] is negative");
    if (single_scat_albedo[lc] < 0.0 || single_scat_albedo[lc] > 1.0)
      throw std::invalid_argument("single_scat_albedo[" + std::to_string(lc) + "] must be in [0, 1]");
  }
  if (flags.use_thermal_emission) {
    if (temperature.size() < static_cast<size_t>(num_layers + 1))
      throw std::invalid_argument("temperature array is too small (need num_layers+1 when use_thermal_emission=true)");
    for (int lev = 0; lev <= num_layers; ++lev)
      if (temperature[lev] < 0.0) throw std::invalid_argument("temperature[" + std::to_string(lev) + "] is negative");
    if (wavenumber_low < 0.0 || wavenumber_high < wavenumber_low)
      throw std::invalid_argument("Invalid wavenumber range for Planck function");
  }
  if (flags.use_diffusion_lower_bc) {
    if (!flags.use_thermal_emission)
      throw std::invalid_argument("use_diffusion_lower_bc requires use_thermal_emission = true");
    if (!flags.use_lambertian_surface)
      throw std::invalid_argument(
          "use_diffusion_lower_bc requires use_lambertian_surface = true (BRDF is incompatible)");
  }
  if (bc.direct_beam_flux < 0.0) throw std::invalid_argument("direct_beam_flux must be non-negative");
  if ((bc.direct_beam_mu <= 0.0 || bc.direct_beam_mu > 1.0) && bc.direct_beam_flux > 0.0)
    throw std::invalid_argument("direct_beam_mu must be in (0, 1] when direct_beam_flux > 0");
  if (flags.use_lambertian_surface && (bc.surface_albedo < 0.0 || bc.surface_albedo > 1.0))
    throw std::invalid_argument("surface_albedo must be in [0, 1] when use_lambertian_surface=true");
  if (flags.use_user_mu) {
    if (num_user_mu <= 0) throw std::invalid_argument("num_user_mu must be positive when use_user_mu=true");
    if (mu_user.size() < static_cast<size_t>(num_user_mu)) throw std::invalid_argument("mu_user array is too small");
    for (int iu = 0; iu < num_user_mu; ++iu) {
      if (std::abs(mu_user[iu]) > 1.0)
        throw std::invalid_argument("mu_user[" + std::to_string(iu) + "] out of range [-1, 1]");
      if (iu > 0 && mu_user[iu] <= mu_user[iu - 1]) throw std::invalid_argument("mu_user must be in increasing order");
    }
  }
  if (flags.use_spherical_beam) {
    if (bottom_radius <= 0.0)
      throw std::invalid_argument("bottom_radius must be positive when use_spherical_beam=true");
    if (level_altitudes.size() < static_cast<size_t>(num_layers + 1))
      throw std::invalid_argument(
          "level_altitudes array is too small (need num_layers+1 when use_spherical_beam=true)");
  }
  if (!flags.comp_only_fluxes && flags.ibcnd != BoundaryConditionType::Special) {
    if (num_phi <= 0) throw std::invalid_argument("num_phi must be positive when comp_only_fluxes=false");
    if (phi_user.size() < static_cast<size_t>(num_phi)) throw std::invalid_argument("phi_user array is too small");
    for (int j = 0; j < num_phi; ++j)
      if (phi_user[j] < 0.0 || phi_user[j] > 360.0)
        throw std::invalid_argument("phi_user[" + std::to_string(j) + "] must be in [0, 360]");
  }
  if (flags.use_delta_m_plus && num_phase_func_moments < num_streams + 1)
    throw std::invalid_argument(
        "use_delta_m_plus=true requires num_phase_func_moments >= num_streams + 1 (need moments M and M+1)");
  if (accuracy_fourier_series < 0.0)
    throw std::invalid_argument("accuracy_fourier_series must be non-negative (0 = disabled)");
  if (flags.use_thermal_emission) {
    if (wavenumber_low < 0.0 || wavenumber_high <= wavenumber_low)
      throw std::invalid_argument("use_thermal_emission=true requires 0 <= wavenumber_low < wavenumber_high");
    if (bc.temperature_top < 0.0 || bc.temperature_bottom < 0.0)
      throw std::invalid_argument(
          "use_thermal_emission=true requires non-negative temperature_top and temperature_bottom");
    if (bc.emissivity_top < 0.0 || bc.emissivity_top > 1.0)
      throw std::invalid_argument("use_thermal_emission=true requires 0 <= emissivity_top <= 1");
    if (static_cast<int>(temperature.size()) < num_layers + 1)
      throw std::invalid_argument("use_thermal_emission=true requires temperature array of size num_layers+1");
  }
}

void DisortConfig::setHenyeyGreenstein(double g, int lc) {
  phase_function::fillHenyeyGreenstein(phase_function_moments, nmomNstr(), num_layers, g, lc);
}
void DisortConfig::setIsotropic(int lc) {
  phase_function::fillIsotropic(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortConfig::setRayleigh(int lc) {
  phase_function::fillRayleigh(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortConfig::setHazeGarciaSiewert(int lc) {
  phase_function::fillHazeGarciaSiewert(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortConfig::setCloudGarciaSiewert(int lc) {
  phase_function::fillCloudGarciaSiewert(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortConfig::setPhaseFunction(PhaseFunction type, double g, int lc) {
  phase_function::fillPhaseFunction(phase_function_moments, nmomNstr(), num_layers, type, g, lc);
}

// ---------------------------------------------------------------------------
// DisortResult (DisortResult.cpp:6-46)
// ---------------------------------------------------------------------------
void DisortResult::allocate(int ntau, int numu, int nphi, int nstr, bool special_bc, bool compute_intensity,
                            bool output_fourier_expansion) {
  ntau_ = ntau;
  numu_ = numu;
  nphi_ = nphi;
  for (auto* v : {&flux_direct_beam, &flux_down, &flux_up, &flux_tau_divergence, &mean_intensity,
                  &mean_intensity_down, &mean_intensity_up, &mean_intensity_direct_beam})
    v->assign(ntau, 0.0);
  mu_angles.assign(numu, 0.0);
  if (special_bc) {
    albedo_medium.resize(numu);
    transmissivity_medium.resize(numu);
  }
  if (compute_intensity) {
    intensity.assign(ntau, std::vector<std::vector<double>>(numu, std::vector<double>(nphi, 0.0)));
    intensity_azimuth_avg.assign(ntau, std::vector<double>(numu, 0.0));
    if (output_fourier_expansion)
      intensity_fourier_expansion.assign(ntau,
                                         std::vector<std::vector<double>>(numu, std::vector<double>(nstr + 1, 0.0)));
  }
}

namespace {

bool engine_streams(int n) {
  for (int s : {4, 6, 8, 10, 12, 14, 16, 32, 64})
    if (s == n) return true;
  return false;
}

// What DisortSolver implements and this engine does not: rejected after
// validate() so that a config the reference rejects gets the reference's message.
void check_engine(const DisortConfig& c) {
  const DisortFlags& f = c.flags;
  if (!engine_streams(c.num_streams))
    throw std::invalid_argument("num_streams=" + std::to_string(c.num_streams) +
                                " is not supported by the B200 engine (supported: 4, 6, 8, 10, 12, 14, 16, 32, 64)");
  // ibcnd = Special forces a Lambertian surface (computeAlbTrans,
  // DisortSolver.cpp:4038-4043): no BRDF is evaluated
  if (!f.use_lambertian_surface && f.ibcnd != BoundaryConditionType::Special) {
    // the model's spec must be present; the reference finds out inside its
    // solve (bidirReflectivity, DisortSolver.cpp:2902-2936) with these errors
    switch (f.brdf_type) {
      case BrdfType::RPV:
        if (!c.brdf.rpv) throw std::runtime_error("bidirReflectivity: RPV BRDF selected but rpv spec is null");
        break;
      case BrdfType::CoxMunk:
        if (!c.brdf.cox_munk)
          throw std::runtime_error("bidirReflectivity: Cox-Munk BRDF selected but cox_munk spec is null");
        break;
      case BrdfType::Ambrals:
        if (!c.brdf.ambrals)
          throw std::runtime_error("bidirReflectivity: Ross-Li/Ambrals BRDF selected but ambrals spec is null");
        break;
      case BrdfType::Hapke:
        break;  // defaults apply without a spec
      default:
        throw std::runtime_error("bidirReflectivity: unknown BRDF type");
    }
  }
  // the Buras-Emde correction (DisortSolver.cpp:362-367) interpolates the tabulated
  // phase function between angles: it needs two and every layer's values
  if (f.intensity_corr_buras && !f.intensity_corr_nakajima && c.num_phase_func_angles > 0) {
    const size_t na = static_cast<size_t>(c.num_phase_func_angles);
    bool ok = na >= 2 && c.mu_phase_function.size() >= na &&
              c.phase_function.size() >= static_cast<size_t>(c.num_layers);
    for (int lc = 0; ok && lc < c.num_layers; ++lc) ok = c.phase_function[lc].size() >= na;
    if (!ok)
      throw std::invalid_argument(
          "intensity_corr_buras with a tabulated phase function needs num_phase_func_angles >= 2, "
          "mu_phase_function and phase_function of every layer");
  }
  // output_fourier_expansion: the reference allocates its results without the
  // expansion (DisortSolver.cpp:122-126), so the array stays empty; so here
  // validate() does not look at the user optical depths; the reference reads
  // tau_user[0 .. num_user_tau-1] whatever its size
  if (f.use_user_tau && (c.num_user_tau <= 0 || c.tau_user.size() < static_cast<size_t>(c.num_user_tau)))
    throw std::invalid_argument("use_user_tau=true requires num_user_tau > 0 and num_user_tau values in tau_user");
}

// reverseInputArrays (IndexConversion.hpp:16-38), applied to a copy that is
// only validated, so messages that name an index name the reference's index.
void validate_as_reference(const DisortConfig& c) {
  if (!c.flags.index_from_bottom) {
    c.validate();
    return;
  }
  DisortConfig r = c;
  std::reverse(r.delta_tau.begin(), r.delta_tau.end());
  std::reverse(r.single_scat_albedo.begin(), r.single_scat_albedo.end());
  std::reverse(r.phase_function_moments.begin(), r.phase_function_moments.end());
  std::reverse(r.temperature.begin(), r.temperature.end());
  std::reverse(r.level_altitudes.begin(), r.level_altitudes.end());
  r.validate();
}

// Gauss-Legendre nodes on (0,1) in the reference's order (FluxSolver.cpp:257-290):
// Newton iteration on P_NN from cos(pi (i - 1/4) / (NN + 1/2)).
std::vector<double> quadrature_angles(int NN) {
  std::vector<double> mu(NN);
  for (int i = 1; i <= NN; ++i) {
    double z = std::cos(M_PI * (i - 0.25) / (NN + 0.5)), z1, pp;
    int iter = 0;
    do {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= NN; ++j) {
        const double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = NN * (z * p1 - p2) / (z * z - 1.0);
      z1 = z;
      z = z1 - p1 / pp;
    } while (std::fabs(z - z1) > 3.0e-14 && ++iter <= 10);
    mu[i - 1] = 0.5 * (1.0 + z);
  }
  return mu;
}

// The config changes DisortSolver::solve makes (DisortSolver.cpp:26-67,
// 650-660, 843-850): allocation of an empty config, output levels at the layer
// boundaries, computational output angles, moment 0 set to 1.
void fill_automatic(DisortConfig& c) {
  const int L = c.num_layers, N = c.num_streams, NN = N / 2;
  if (!c.flags.use_user_tau) {
    c.num_user_tau = L + 1;
    c.tau_user.resize(L + 1);
    const bool ifb = c.flags.index_from_bottom;
    double t = 0.0;
    c.tau_user[0] = 0.0;
    for (int lc = 0; lc < L; ++lc) {
      t += c.delta_tau[ifb ? L - 1 - lc : lc];
      c.tau_user[lc + 1] = t;
    }
  }
  if (!c.flags.use_user_mu || c.flags.comp_only_fluxes) {
    c.num_user_mu = N;
    c.mu_user.resize(N);
    const std::vector<double> mu = quadrature_angles(NN);
    for (int iu = 0; iu < NN; ++iu) c.mu_user[iu] = -mu[NN - 1 - iu];
    for (int iu = NN; iu < N; ++iu) c.mu_user[iu] = mu[iu - NN];
  }
  for (int lc = 0; lc < L; ++lc) c.phase_function_moments[lc][0] = 1.0;
}

struct GenPacked {
  std::vector<int32_t> nstr, nlyr, nmom;
  std::vector<int64_t> off;
  std::vector<double> dtau, ssa, pmom, temp, zalt, utau, umu, phi;
  std::vector<double> lo, hi, alb, emis, fbeam, fisot, fisob;
  double mu0 = 0.5, phi0 = 0.0, ttop = 0.0, tbot = 0.0, rbot = 0.0;
  double bpar[DSP_BRDF_PARAMS] = {};  // the surface model's parameters, shared by every band
  std::vector<double> mup, phasef;   // tabulated phase function (Buras-Emde correction)
};

// One batch for the whole loop.  `c` already carries the automatic fields.
// Layer arrays are CSR per band (overrides or copies of the base); user angle
// and depth lists and the scalars without overrides are shared (stride 0).
dsp_general_batch pack_general(const DisortConfig& c, const std::vector<std::pair<double, double>>& bands,
                               const SpectralOverrides& ov, GenPacked& pk) {
  const int n = static_cast<int>(bands.size());
  const int L = c.num_layers, pc = c.nmomNstr() + 1;
  const DisortFlags& f = c.flags;
  dsp_general_batch b{};
  b.n_inst = n;
  b.flags = (f.use_thermal_emission ? DSP_FLAG_THERMAL : 0u) | (f.use_delta_m_plus ? DSP_FLAG_DELTA_M_PLUS : 0u) |
            (f.use_diffusion_lower_bc ? DSP_FLAG_DIFFUSION_LOWER_BC : 0u) |
            (f.index_from_bottom ? DSP_FLAG_INDEX_FROM_BOTTOM : 0u) | (f.use_user_tau ? DSP_GFLAG_USER_TAU : 0u) |
            (f.use_user_mu && !f.comp_only_fluxes ? DSP_GFLAG_USER_MU : 0u) |
            (f.comp_only_fluxes ? DSP_GFLAG_ONLY_FLUXES : 0u) |
            (f.use_spherical_beam ? DSP_FLAG_SPHERICAL_BEAM : 0u) |
            (f.intensity_corr_buras ? DSP_GFLAG_INTENSITY_CORR : 0u);
  pk.nstr.assign(n, c.num_streams);
  pk.nlyr.assign(n, L);
  pk.nmom.assign(n, c.num_phase_func_moments);
  pk.off.resize(n + 1);
  for (int i = 0; i <= n; ++i) pk.off[i] = static_cast<int64_t>(i) * L;
  b.num_streams = pk.nstr.data();
  b.num_layers = pk.nlyr.data();
  b.layer_offset = pk.off.data();
  b.num_phase_func_moments = pk.nmom.data();
  b.pmom_count = pc;
  const size_t nl = static_cast<size_t>(n) * L;
  pk.dtau.resize(nl);
  pk.ssa.resize(nl);
  pk.pmom.resize(nl * pc);
  for (int i = 0; i < n; ++i) {
    const std::vector<double>& dt = ov.delta_tau.empty() ? c.delta_tau : ov.delta_tau[i];
    const std::vector<double>& ss = ov.single_scat_albedo.empty() ? c.single_scat_albedo : ov.single_scat_albedo[i];
    const auto& pm = ov.phase_function_moments.empty() ? c.phase_function_moments : ov.phase_function_moments[i];
    const size_t o = static_cast<size_t>(i) * L;
    std::copy(dt.begin(), dt.begin() + L, pk.dtau.begin() + o);
    std::copy(ss.begin(), ss.begin() + L, pk.ssa.begin() + o);
    for (int lc = 0; lc < L; ++lc) {
      double* row = pk.pmom.data() + (o + lc) * pc;
      std::copy(pm[lc].begin(), pm[lc].begin() + pc, row);
      row[0] = 1.0;  // disortSet sets moment 0 (DisortSolver.cpp:666-668)
    }
  }
  b.delta_tau = pk.dtau.data();
  b.single_scat_albedo = pk.ssa.data();
  b.phase_function_moments = pk.pmom.data();
  if (f.use_thermal_emission) {
    pk.temp.resize(static_cast<size_t>(n) * (L + 1));
    for (int i = 0; i < n; ++i)
      std::copy(c.temperature.begin(), c.temperature.begin() + L + 1, pk.temp.begin() + static_cast<size_t>(i) * (L + 1));
    b.temperature = pk.temp.data();
  }
  if (f.use_spherical_beam) {  // the same column geometry for every band
    pk.zalt.resize(static_cast<size_t>(n) * (L + 1));
    for (int i = 0; i < n; ++i)
      std::copy(c.level_altitudes.begin(), c.level_altitudes.begin() + L + 1,
                pk.zalt.begin() + static_cast<size_t>(i) * (L + 1));
    pk.rbot = c.bottom_radius;
    b.level_altitudes = pk.zalt.data();
    b.bottom_radius = {&pk.rbot, 0};
  }
  if (f.use_user_tau) {
    pk.utau.assign(c.tau_user.begin(), c.tau_user.begin() + c.num_user_tau);
    b.num_user_tau = c.num_user_tau;
    b.tau_user = {pk.utau.data(), 0};
  }
  // with comp_only_fluxes the reference replaces mu_user by the computational
  // angles (DisortSolver.cpp:62-66) and computes no intensities
  if (f.use_user_mu && !f.comp_only_fluxes) {
    pk.umu.assign(c.mu_user.begin(), c.mu_user.begin() + c.num_user_mu);
    b.num_user_mu = c.num_user_mu;
    b.mu_user = {pk.umu.data(), 0};
  }
  if (!f.comp_only_fluxes) {
    pk.phi.assign(c.phi_user.begin(), c.phi_user.begin() + c.num_phi);
    b.num_phi = c.num_phi;
    b.phi_user = {pk.phi.data(), 0};
  }
  b.accuracy_fourier_series = c.accuracy_fourier_series;
  pk.lo.resize(n);
  pk.hi.resize(n);
  for (int i = 0; i < n; ++i) {
    pk.lo[i] = bands[i].first;
    pk.hi[i] = bands[i].second;
  }
  b.wavenumber_low = {pk.lo.data(), 1};
  b.wavenumber_high = {pk.hi.data(), 1};
  auto scalar = [&](const std::vector<double>& per, double base, std::vector<double>& dst) -> dsp_darray {
    if (per.empty()) {
      dst.assign(1, base);
      return {dst.data(), 0};
    }
    dst = per;
    return {dst.data(), 1};
  };
  b.surface_albedo = scalar(ov.surface_albedo, c.bc.surface_albedo, pk.alb);
  b.emissivity_top = scalar(ov.emissivity_top, c.bc.emissivity_top, pk.emis);
  b.direct_beam_flux = scalar(ov.direct_beam_flux, c.bc.direct_beam_flux, pk.fbeam);
  b.isotropic_flux_top = scalar(ov.isotropic_flux_top, c.bc.isotropic_flux_top, pk.fisot);
  b.isotropic_flux_bottom = scalar(ov.isotropic_flux_bottom, c.bc.isotropic_flux_bottom, pk.fisob);
  pk.mu0 = c.bc.direct_beam_mu;
  pk.phi0 = c.bc.direct_beam_phi;
  pk.ttop = c.bc.temperature_top;
  pk.tbot = c.bc.temperature_bottom;
  b.direct_beam_mu = {&pk.mu0, 0};
  b.direct_beam_phi = {&pk.phi0, 0};
  b.temperature_top = {&pk.ttop, 0};
  b.temperature_bottom = {&pk.tbot, 0};
  if (f.intensity_corr_buras && !f.intensity_corr_nakajima && c.num_phase_func_angles > 0) {
    // the Buras-Emde method: the table, layer rows per band in the batch's layer order
    const int na = c.num_phase_func_angles;
    b.flags |= DSP_GFLAG_INTENSITY_CORR_BE;
    b.num_phase_func_angles = na;
    pk.mup.assign(c.mu_phase_function.begin(), c.mu_phase_function.begin() + na);
    b.mu_phase_function = {pk.mup.data(), 0};
    pk.phasef.resize(static_cast<size_t>(n) * L * na);
    for (int i = 0; i < n; ++i)
      for (int lc = 0; lc < L; ++lc)
        std::copy(c.phase_function[lc].begin(), c.phase_function[lc].begin() + na,
                  pk.phasef.begin() + (static_cast<size_t>(i) * L + lc) * na);
    b.phase_function = pk.phasef.data();
  }
  if (!f.use_lambertian_surface) {  // the spec in the C ABI's parameter order
    b.brdf_type = static_cast<int32_t>(f.brdf_type);
    double* q = pk.bpar;
    switch (f.brdf_type) {
      case BrdfType::RPV: {
        const RpvBrdfSpec& r = *c.brdf.rpv;
        const double v[7] = {r.rho0, r.k, r.theta, r.sigma, r.t1, r.t2, r.scale};
        std::copy(v, v + 7, q);
        break;
      }
      case BrdfType::CoxMunk: {
        const CoxMunkBrdfSpec& r = *c.brdf.cox_munk;
        const double v[5] = {r.u10, r.pcl, r.xsal, r.refractive_index, r.do_shadow ? 1.0 : 0.0};
        std::copy(v, v + 5, q);
        break;
      }
      case BrdfType::Ambrals: {
        const AmbralsBrdfSpec& r = *c.brdf.ambrals;
        q[0] = r.iso, q[1] = r.vol, q[2] = r.geo;
        break;
      }
      default: {
        const HapkeBrdfSpec r = c.brdf.hapke ? *c.brdf.hapke : HapkeBrdfSpec{};
        q[0] = r.b0, q[1] = r.hh, q[2] = r.w;
        break;
      }
    }
    b.brdf_params = {q, 0};
  }
  return b;
}

// Band i's effective config is the base with override i applied
// (applyOverrides, python_bindings.cpp:62-71); validate it with validate()'s
// rules and messages.  The base config was validated with the band-free rules.
void validate_band(const DisortConfig& c, const SpectralOverrides& ov, size_t i, double lo, double hi) {
  const int L = c.num_layers;
  const bool ifb = c.flags.index_from_bottom;
  if (!ov.delta_tau.empty() || !ov.single_scat_albedo.empty() || !ov.phase_function_moments.empty()) {
    const std::vector<double>& dt = ov.delta_tau.empty() ? c.delta_tau : ov.delta_tau[i];
    const std::vector<double>& ss = ov.single_scat_albedo.empty() ? c.single_scat_albedo : ov.single_scat_albedo[i];
    const auto& pm = ov.phase_function_moments.empty() ? c.phase_function_moments : ov.phase_function_moments[i];
    if (dt.size() < static_cast<size_t>(L)) throw std::invalid_argument("delta_tau array is too small");
    if (ss.size() < static_cast<size_t>(L)) throw std::invalid_argument("single_scat_albedo array is too small");
    if (static_cast<int>(pm.size()) < L)
      throw std::invalid_argument("phase_function_moments must have at least num_layers layers");
    for (int lc = 0; lc < L; ++lc)
      if (static_cast<int>(pm[ifb ? L - 1 - lc : lc].size()) < c.nmomNstr() + 1)
        throw std::invalid_argument("phase_function_moments[" + std::to_string(lc) +
                                    "] must have at least nmomNstr()+1 elements");
    for (int lc = 0; lc < L; ++lc) {
      const int k = ifb ? L - 1 - lc : lc;
      if (dt[k] < 0.0) throw std::invalid_argument("delta_tau[" + std::to_string(lc) + "] is negative");
      if (ss[k] < 0.0 || ss[k] > 1.0)
        throw std::invalid_argument("single_scat_albedo[" + std::to_string(lc) + "] must be in [0, 1]");
    }
  }
  if (c.flags.use_thermal_emission && (lo < 0.0 || hi < lo))
    throw std::invalid_argument("Invalid wavenumber range for Planck function");
  const double fbeam = ov.direct_beam_flux.empty() ? c.bc.direct_beam_flux : ov.direct_beam_flux[i];
  const double alb = ov.surface_albedo.empty() ? c.bc.surface_albedo : ov.surface_albedo[i];
  const double emis = ov.emissivity_top.empty() ? c.bc.emissivity_top : ov.emissivity_top[i];
  if (fbeam < 0.0) throw std::invalid_argument("direct_beam_flux must be non-negative");
  if ((c.bc.direct_beam_mu <= 0.0 || c.bc.direct_beam_mu > 1.0) && fbeam > 0.0)
    throw std::invalid_argument("direct_beam_mu must be in (0, 1] when direct_beam_flux > 0");
  if (c.flags.use_lambertian_surface && (alb < 0.0 || alb > 1.0))
    throw std::invalid_argument("surface_albedo must be in [0, 1] when use_lambertian_surface=true");
  if (c.flags.use_thermal_emission) {
    if (lo < 0.0 || hi <= lo)
      throw std::invalid_argument("use_thermal_emission=true requires 0 <= wavenumber_low < wavenumber_high");
    if (emis < 0.0 || emis > 1.0)
      throw std::invalid_argument("use_thermal_emission=true requires 0 <= emissivity_top <= 1");
  }
}

// The base config with every per-band field neutralised, through validate().
void validate_base(const DisortConfig& c, const SpectralOverrides& ov) {
  DisortConfig v = c;
  if (!ov.delta_tau.empty() || !ov.single_scat_albedo.empty() || !ov.phase_function_moments.empty()) {
    v.delta_tau.assign(c.num_layers, 0.0);
    v.single_scat_albedo.assign(c.num_layers, 0.0);
    v.phase_function_moments.assign(c.num_layers, std::vector<double>(c.nmomNstr() + 1, 0.0));
  }
  v.bc.direct_beam_flux = 0.0;
  v.bc.surface_albedo = 0.0;
  v.bc.emissivity_top = 1.0;
  v.wavenumber_low = 0.0;
  v.wavenumber_high = 1.0;
  validate_as_reference(v);
}

// Solve every band of `c` (automatic fields filled) and return the results.
std::vector<DisortResult> run_general(const DisortConfig& c, const std::vector<std::pair<double, double>>& bands,
                                      const SpectralOverrides& ov) {
  const size_t n = bands.size();
  std::vector<DisortResult> res(n);
  if (n == 0) return res;
  const DisortFlags& f = c.flags;
  const int ntau = c.num_user_tau, numu = c.num_user_mu, nphi = c.num_phi;
  const bool compute_intensity = !f.comp_only_fluxes;
  const bool do_int = f.use_user_mu && !f.comp_only_fluxes;
  GenPacked pk;
  dsp_general_batch b = pack_general(c, bands, ov, pk);
  std::vector<double> flux(8 * n * static_cast<size_t>(ntau));
  std::vector<double> inten, iavg;
  if (do_int) {
    inten.resize(n * static_cast<size_t>(ntau) * numu * nphi);
    iavg.resize(n * static_cast<size_t>(ntau) * numu);
  }
  std::vector<int32_t> status(n, 0);
  // temperature Jacobians (DisortSolver.cpp:2130-2358): [n][ntau][L+2] per output
  const bool jac = f.compute_temperature_jacobian;
  const int ndof = c.num_layers + 2;
  std::vector<double> jbuf;
  dsp_general_jac_out jo{};
  if (jac) {
    const size_t per = n * static_cast<size_t>(ntau) * ndof;
    jbuf.resize(6 * per);
    double** jp[6] = {&jo.flux_up, &jo.flux_down, &jo.mean_intensity, &jo.mean_intensity_down,
                      &jo.mean_intensity_up, &jo.flux_divergence};
    for (int k = 0; k < 6; ++k) *jp[k] = jbuf.data() + k * per;
    jo.ndof_out = ndof;
  }
  dsp_general_out o{};
  for (int k = 0; k < 8; ++k) o.flux[k] = flux.data() + static_cast<size_t>(k) * n * ntau;
  o.intensity = do_int ? inten.data() : nullptr;
  o.intensity_azimuth_avg = do_int ? iavg.data() : nullptr;
  o.status = status.data();
  o.ntau_out = ntau;
  o.numu_out = do_int ? numu : 0;
  {
    std::lock_guard<std::mutex> lk(detail::engine_mutex());
    dsp_context ctx = detail::engine_context_locked();
    const dsp_status st = jac ? dsp_general_bands_solve_jac(ctx, &b, &o, &jo) : dsp_general_bands_solve(ctx, &b, &o);
    if (st != DSP_OK)
      throw std::runtime_error(std::string("disortpp: GPU solve failed: ") + dsp_status_string(st) + ": " +
                               dsp_context_last_error(ctx));
  }
  for (size_t i = 0; i < n; ++i)
    if (status[i] == DSP_ERR_INVALID_INPUT || status[i] == DSP_ERR_UNSUPPORTED)
      throw std::invalid_argument("band " + std::to_string(i) + ": " + dsp_status_string((dsp_status)status[i]));
  for (size_t i = 0; i < n; ++i) {
    DisortResult& r = res[i];
    r.allocate(ntau, numu, nphi, c.num_streams, false, compute_intensity, false);
    std::vector<double>* dst[8] = {&r.flux_direct_beam, &r.flux_down, &r.flux_up, &r.flux_tau_divergence,
                                   &r.mean_intensity, &r.mean_intensity_down, &r.mean_intensity_up,
                                   &r.mean_intensity_direct_beam};
    for (int k = 0; k < 8; ++k) {
      const double* src = o.flux[k] + i * ntau;
      std::copy(src, src + ntau, dst[k]->begin());
    }
    std::copy(c.mu_user.begin(), c.mu_user.begin() + numu, r.mu_angles.begin());
    if (do_int) {
      for (int lu = 0; lu < ntau; ++lu)
        for (int iu = 0; iu < numu; ++iu) {
          const size_t row = (i * ntau + lu) * static_cast<size_t>(numu) + iu;
          std::copy(inten.begin() + row * nphi, inten.begin() + (row + 1) * nphi, r.intensity[lu][iu].begin());
          r.intensity_azimuth_avg[lu][iu] = iavg[row];
        }
    }
    // Jacobians when asked for with thermal emission on; otherwise empty, as the
    // reference clears them (DisortSolver.cpp:2143-2151)
    std::vector<std::vector<double>>* jd[6] = {&r.flux_up_temperature_jac, &r.flux_down_temperature_jac,
                                               &r.mean_intensity_temperature_jac,
                                               &r.mean_intensity_down_temperature_jac,
                                               &r.mean_intensity_up_temperature_jac,
                                               &r.flux_divergence_temperature_jac};
    for (int k = 0; k < 6; ++k) {
      jd[k]->clear();
      if (!jac || !f.use_thermal_emission) continue;
      const double* src = jbuf.data() + static_cast<size_t>(k) * n * ntau * ndof + i * static_cast<size_t>(ntau) * ndof;
      jd[k]->resize(ntau);
      for (int lu = 0; lu < ntau; ++lu) (*jd[k])[lu].assign(src + lu * ndof, src + (lu + 1) * ndof);
    }
  }
  return res;
}

// ibcnd = Special over every band (DisortSolver.cpp:52-58, 169-176, 4025-4163):
// dsp_general_bands_albtrans; the results carry the mirrored cosines, zero
// fluxes and intensities, and the albedo and transmissivity of the medium in the
// first half of arrays sized like the mirrored list, as the reference's.
std::vector<DisortResult> run_special(const DisortConfig& c0, const std::vector<std::pair<double, double>>& bands,
                                      const SpectralOverrides& ov) {
  const size_t n = bands.size();
  std::vector<DisortResult> res(n);
  if (n == 0) return res;
  DisortConfig c = c0;
  const int N = c.num_streams, NN = N / 2;
  const bool user_mu = c.flags.use_user_mu;
  const int half = user_mu ? c.num_user_mu : NN;
  std::vector<double> mirrored(2 * half);
  if (user_mu) {
    for (int iu = 0; iu < half; ++iu) {
      mirrored[half + iu] = c.mu_user[iu];
      mirrored[iu] = -c.mu_user[half - 1 - iu];
    }
  } else {  // the quadrature cosines as the reference orders them (descending)
    const std::vector<double> mu = quadrature_angles(NN);
    for (int iu = 0; iu < NN; ++iu) mirrored[iu] = -mu[NN - 1 - iu];
    for (int iu = NN; iu < N; ++iu) mirrored[iu] = mu[iu - NN];
  }
  // the batch of the general solver's layers and moments, nothing else
  c.flags.use_thermal_emission = false;
  c.flags.use_spherical_beam = false;
  c.flags.use_user_tau = false;
  c.flags.comp_only_fluxes = true;
  c.flags.use_lambertian_surface = true;
  c.flags.intensity_corr_buras = false;
  c.flags.use_user_mu = false;
  fill_automatic(c);
  GenPacked pk;
  dsp_general_batch b = pack_general(c, bands, ov, pk);
  b.flags &= (DSP_FLAG_DELTA_M_PLUS | DSP_FLAG_INDEX_FROM_BOTTOM);
  if (user_mu) {
    pk.umu.assign(c0.mu_user.begin(), c0.mu_user.begin() + half);
    b.flags |= DSP_GFLAG_USER_MU;
    b.num_user_mu = half;
    b.mu_user = {pk.umu.data(), 0};
  }
  std::vector<double> am(n * half), tm(n * half), sa(n), st(n);
  std::vector<int32_t> status(n, 0);
  dsp_albtrans_out o{am.data(), tm.data(), sa.data(), st.data(), status.data(), half};
  {
    std::lock_guard<std::mutex> lk(detail::engine_mutex());
    dsp_context ctx = detail::engine_context_locked();
    const dsp_status e = dsp_general_bands_albtrans(ctx, &b, &o);
    if (e != DSP_OK)
      throw std::runtime_error(std::string("disortpp: GPU solve failed: ") + dsp_status_string(e) + ": " +
                               dsp_context_last_error(ctx));
  }
  for (size_t i = 0; i < n; ++i)
    if (status[i] == DSP_ERR_INVALID_INPUT || status[i] == DSP_ERR_UNSUPPORTED)
      throw std::invalid_argument("band " + std::to_string(i) + ": " + dsp_status_string((dsp_status)status[i]));
  const int ntau = c0.flags.use_user_tau ? c0.num_user_tau : c0.num_layers + 1;
  for (size_t i = 0; i < n; ++i) {
    DisortResult& r = res[i];
    r.allocate(ntau, 2 * half, c0.num_phi, N, true, !c0.flags.comp_only_fluxes, false);
    r.mu_angles = mirrored;
    std::copy(am.begin() + i * half, am.begin() + (i + 1) * half, r.albedo_medium.begin());
    std::copy(tm.begin() + i * half, tm.begin() + (i + 1) * half, r.transmissivity_medium.begin());
    r.spherical_albedo = sa[i];
    r.spherical_transmissivity = st[i];
  }
  return res;
}

void check_override_sizes(const SpectralOverrides& ov, size_t n) {
  auto check = [&](size_t got, const char* name) {
    if (got != 0 && got != n)
      throw std::invalid_argument(std::string(name) + " override has " + std::to_string(got) + " entries for " +
                                  std::to_string(n) + " bands");
  };
  check(ov.delta_tau.size(), "delta_tau");
  check(ov.single_scat_albedo.size(), "single_scat_albedo");
  check(ov.phase_function_moments.size(), "phase_function_moments");
  check(ov.surface_albedo.size(), "surface_albedo");
  check(ov.emissivity_top.size(), "emissivity_top");
  check(ov.direct_beam_flux.size(), "direct_beam_flux");
  check(ov.isotropic_flux_top.size(), "isotropic_flux_top");
  check(ov.isotropic_flux_bottom.size(), "isotropic_flux_bottom");
}

}  // namespace

DisortResult DisortSolver::solve(DisortConfig& config) {
  if (config.delta_tau.empty()) config.allocate();
  validate_as_reference(config);
  check_engine(config);
  if (config.flags.ibcnd == BoundaryConditionType::Special) {
    std::vector<std::pair<double, double>> one{{config.wavenumber_low, config.wavenumber_high}};
    DisortResult r = run_special(config, one, SpectralOverrides{})[0];
    // the config as the reference leaves it: automatic depths and moment 0, the
    // cosines halved back (DisortSolver.cpp:4615-4620 of computeAlbTrans)
    const int half = config.flags.use_user_mu ? config.num_user_mu : config.num_streams / 2;
    const std::vector<double> mirrored = r.mu_angles;
    fill_automatic(config);
    config.mu_user = mirrored;
    config.mu_user.resize(std::max(mirrored.size(), static_cast<size_t>(2 * half + 1)), 0.0);
    for (int iu = 1; iu <= half; ++iu) config.mu_user[iu] = config.mu_user[iu + half];
    config.num_user_mu = half;
    return r;
  }
  fill_automatic(config);
  std::vector<std::pair<double, double>> one{{config.wavenumber_low, config.wavenumber_high}};
  return run_general(config, one, SpectralOverrides{})[0];
}

std::vector<DisortResult> solveSpectralBands(const DisortConfig& config,
                                             const std::vector<std::pair<double, double>>& bands,
                                             const SpectralOverrides& ov) {
  DisortConfig c = config;  // the loop's configs are copies (python_bindings.cpp:108)
  if (c.delta_tau.empty()) c.allocate();
  check_override_sizes(ov, bands.size());
  validate_base(c, ov);
  for (size_t i = 0; i < bands.size(); ++i) validate_band(c, ov, i, bands[i].first, bands[i].second);
  if (bands.empty()) return {};
  check_engine(c);
  if (c.flags.ibcnd == BoundaryConditionType::Special) return run_special(c, bands, ov);
  fill_automatic(c);
  return run_general(c, bands, ov);
}

std::vector<DisortResult> solveSpectral(const DisortConfig& config, const std::vector<double>& wavenumbers,
                                        const SpectralOverrides& ov) {
  std::vector<std::pair<double, double>> bands;
  bands.reserve(wavenumbers.size());
  for (double w : wavenumbers) bands.emplace_back(w, w);
  return solveSpectralBands(config, bands, ov);
}

}  // namespace disortpp
