// disortpp.hpp — the DisORT++ C++ API, served by the B200 engine.
//
// Same class names, fields, defaults, methods and exceptions as the reference
// (src/DisortFluxConfig.hpp:15-93, src/FluxResult.hpp:14-51,
// src/FluxSolver.hpp:28-49, src/python_bindings.cpp:51-211), so a C++ caller
// recompiles against this header and links libdisortpp.so instead of the
// reference library.  Every solve runs on the GPU through the C ABI of dsp.h;
// there is no CPU solve path.
#pragma once

#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace disortpp {

enum class PhaseFunction {
  Isotropic = 1,
  Rayleigh = 2,
  HenyeyGreenstein = 3,
  HazeGarciaSiewert = 4,
  CloudGarciaSiewert = 5
};

// Phase-function moment fillers (PhaseFunction.cpp:6-117).
namespace phase_function {
void fillHenyeyGreenstein(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers, double g, int lc);
void fillIsotropic(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers, int lc);
void fillRayleigh(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers, int lc);
void fillHazeGarciaSiewert(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers, int lc);
void fillCloudGarciaSiewert(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers, int lc);
void fillPhaseFunction(std::vector<std::vector<double>>& moments, int nmom_nstr, int num_layers,
                       PhaseFunction type, double g, int lc);
}  // namespace phase_function

// DisortFluxConfig (DisortFluxConfig.hpp:15-93).
class DisortFluxConfig {
 public:
  int num_layers = 0;
  int num_streams = 0;
  int num_phase_func_moments = 0;
  int nmomNstr() const { return num_phase_func_moments > num_streams ? num_phase_func_moments : num_streams; }

  bool use_thermal_emission = false;
  bool use_spherical_beam = false;
  bool use_delta_m_plus = false;
  bool use_diffusion_lower_bc = false;
  bool index_from_bottom = false;
  bool compute_temperature_jacobian = false;

  double direct_beam_flux = 0.0;
  double direct_beam_mu = 0.5;
  double isotropic_flux_top = 0.0;
  double isotropic_flux_bottom = 0.0;
  double temperature_top = 0.0;
  double temperature_bottom = 0.0;
  double emissivity_top = 1.0;
  double surface_albedo = 0.0;

  double wavenumber_low = 0.0;
  double wavenumber_high = 0.0;
  double bottom_radius = 0.0;

  std::vector<double> delta_tau;
  std::vector<double> single_scat_albedo;
  std::vector<std::vector<double>> phase_function_moments;
  std::vector<double> temperature;
  std::vector<double> level_altitudes;

  DisortFluxConfig() = default;
  DisortFluxConfig(int nlyr, int nstr, int nmom = 0);
  void allocate();
  void validate() const;  // throws std::invalid_argument with the reference's messages

  double& phaseFunctionMoments(int k, int lc) { return phase_function_moments[lc][k]; }
  const double& phaseFunctionMoments(int k, int lc) const { return phase_function_moments[lc][k]; }
  void setHenyeyGreenstein(double g, int lc = -1);
  void setIsotropic(int lc = -1);
  void setRayleigh(int lc = -1);
  void setHazeGarciaSiewert(int lc = -1);
  void setCloudGarciaSiewert(int lc = -1);
  void setPhaseFunction(PhaseFunction type, double g = 0.0, int lc = -1);
};

// FluxResult (FluxResult.hpp:14-51).
struct FluxResult {
  std::vector<double> flux_direct_beam;
  std::vector<double> flux_down;
  std::vector<double> flux_up;
  std::vector<double> flux_tau_divergence;
  std::vector<double> mean_intensity;
  std::vector<double> mean_intensity_down;
  std::vector<double> mean_intensity_up;
  std::vector<double> mean_intensity_direct_beam;
  std::vector<std::vector<double>> flux_up_temperature_jac;
  std::vector<std::vector<double>> flux_down_temperature_jac;
  std::vector<std::vector<double>> mean_intensity_temperature_jac;
  std::vector<std::vector<double>> mean_intensity_down_temperature_jac;
  std::vector<std::vector<double>> mean_intensity_up_temperature_jac;
  std::vector<std::vector<double>> flux_divergence_temperature_jac;

  int num_levels() const { return static_cast<int>(flux_up.size()); }
  void allocate(int num_layers);
  double totalFluxDown(int lev) const { return flux_direct_beam[lev] + flux_down[lev]; }
  double netFlux(int lev) const { return flux_direct_beam[lev] + flux_down[lev] - flux_up[lev]; }
};

// Per-band override lists of the spectral loops (python_bindings.cpp:51-60).
struct SpectralOverrides {
  std::vector<std::vector<double>> delta_tau;
  std::vector<std::vector<double>> single_scat_albedo;
  std::vector<std::vector<std::vector<double>>> phase_function_moments;
  std::vector<double> surface_albedo;
  std::vector<double> emissivity_top;
  std::vector<double> direct_beam_flux;
  std::vector<double> isotropic_flux_top;
  std::vector<double> isotropic_flux_bottom;
};

// One flux solve of `config` with `nstr` streams on the engine's GPU.
FluxResult solveFluxOne(const DisortFluxConfig& config, int nstr);

// DisortFluxSolver<NStr> (FluxSolver.hpp:28-49): solve() validates and runs one
// instance on the GPU.
template <int NStr>
class DisortFluxSolver {
  static_assert(NStr >= 4, "NStr must be >= 4 (use a dedicated two-stream solver for NStr=2)");
  static_assert(NStr % 2 == 0, "NStr must be even");

 public:
  static constexpr int NN = NStr / 2;
  DisortFluxSolver() = default;
  FluxResult solve(const DisortFluxConfig& config) { return solveFluxOne(config, NStr); }
};

// Spectral loops (python_bindings.cpp:148-211): all bands in one GPU batch.
std::vector<FluxResult> solveFluxSpectralBands(const DisortFluxConfig& config,
                                               const std::vector<std::pair<double, double>>& wavenumber_bands,
                                               const SpectralOverrides& ov = {});
std::vector<FluxResult> solveFluxSpectral(const DisortFluxConfig& config, const std::vector<double>& wavenumbers,
                                          const SpectralOverrides& ov = {});

// Array form of solveFluxSpectralBands: every output [n_bands][num_layers+1]
// row-major in `out8` order flux_direct_beam, flux_down, flux_up,
// flux_tau_divergence, mean_intensity, mean_intensity_down, mean_intensity_up,
// mean_intensity_direct_beam (no reference counterpart: skips the per-band
// FluxResult objects for large sweeps).
void solveFluxSpectralBandsInto(const DisortFluxConfig& config,
                                const std::vector<std::pair<double, double>>& wavenumber_bands,
                                const SpectralOverrides& ov, double* out8[8]);

// ---------------------------------------------------------------------------
// General solver (DisortConfig.hpp:11-243, DisortResult.hpp:16-125,
// DisortSolver.hpp:87): plane-parallel or pseudo-spherical beam geometry,
// Lambertian or bidirectional (BRDF) surface, Fourier azimuth modes, fluxes,
// intensities at user optical depths and angles, temperature Jacobians.
// Special boundary conditions (ibcnd = Special) fill albedo_medium and
// transmissivity_medium; output_fourier_expansion leaves
// intensity_fourier_expansion empty, as the reference does.  Stream counts
// outside 4-16/32/64 pass validate() like in the reference and are rejected
// with std::invalid_argument when solved.
// ---------------------------------------------------------------------------
enum class BoundaryConditionType { General = 0, Special = 1 };
enum class BrdfType { None = 0, RPV = 1, CoxMunk = 2, Ambrals = 3, Hapke = 4 };

struct DisortFlags {
  bool use_user_tau = false;
  bool use_user_mu = false;
  BoundaryConditionType ibcnd = BoundaryConditionType::General;
  bool use_lambertian_surface = true;
  bool use_thermal_emission = false;
  bool use_spherical_beam = false;
  bool comp_only_fluxes = false;
  BrdfType brdf_type = BrdfType::None;
  bool intensity_corr_buras = false;
  bool intensity_corr_nakajima = false;
  bool use_delta_m_plus = false;
  bool use_diffusion_lower_bc = false;
  bool output_fourier_expansion = false;
  bool index_from_bottom = false;
  bool compute_temperature_jacobian = false;
};

struct BoundaryConditions {
  double direct_beam_flux = 0.0;
  double direct_beam_mu = 0.5;
  double direct_beam_phi = 0.0;
  double isotropic_flux_top = 0.0;
  double isotropic_flux_bottom = 0.0;
  double temperature_top = 0.0;
  double temperature_bottom = 0.0;
  double emissivity_top = 1.0;
  double surface_albedo = 0.0;
};

// BRDF parameter sets (DisortConfig.hpp:48-111), used by DisortSolver when
// flags.use_lambertian_surface is false (the model chosen by flags.brdf_type).
struct RpvBrdfSpec {
  double rho0 = 0.0, k = 0.0, theta = 0.0, sigma = 0.0, t1 = 0.0, t2 = 0.0, scale = 1.0;
};
struct AmbralsBrdfSpec {
  double iso = 0.0, vol = 0.0, geo = 0.0;
};
struct CoxMunkBrdfSpec {
  double u10 = 0.0, pcl = 0.0, xsal = 0.0, refractive_index = 1.34;
  bool do_shadow = true;
};
struct HapkeBrdfSpec {
  double b0 = 1.0, hh = 0.06, w = 0.6;
};
struct BrdfSpecification {
  std::optional<RpvBrdfSpec> rpv;
  std::optional<AmbralsBrdfSpec> ambrals;
  std::optional<CoxMunkBrdfSpec> cox_munk;
  std::optional<HapkeBrdfSpec> hapke;
  void setRpv(const RpvBrdfSpec& spec) { rpv = spec; }
  void setAmbrals(const AmbralsBrdfSpec& spec) { ambrals = spec; }
  void setCoxMunk(const CoxMunkBrdfSpec& spec) { cox_munk = spec; }
  void setHapke(const HapkeBrdfSpec& spec) { hapke = spec; }
};

class DisortConfig {
 public:
  DisortFlags flags;
  BoundaryConditions bc;
  BrdfSpecification brdf;
  int num_layers = 0;
  int num_phase_func_moments = 0;
  int num_streams = 0;
  int num_user_tau = 0;
  int num_user_mu = 0;
  int num_phi = 0;
  int num_phase_func_angles = 0;
  int nmomNstr() const { return num_phase_func_moments > num_streams ? num_phase_func_moments : num_streams; }
  double wavenumber_low = 0.0;
  double wavenumber_high = 0.0;
  double accuracy_fourier_series = 0.0;
  double bottom_radius = 0.0;
  std::vector<double> delta_tau;
  std::vector<double> single_scat_albedo;
  std::vector<std::vector<double>> phase_function_moments;
  std::vector<double> temperature;
  std::vector<double> level_altitudes;
  std::vector<double> tau_user;
  std::vector<double> mu_user;
  std::vector<double> phi_user;
  std::vector<double> mu_phase_function;
  std::vector<std::vector<double>> phase_function;

  DisortConfig() = default;
  DisortConfig(int nlyr, int nstr, int nmom = 0);
  void allocate();
  void validate() const;  // std::invalid_argument with the reference's messages
  double& phaseFunctionMoments(int k, int lc) { return phase_function_moments[lc][k]; }
  const double& phaseFunctionMoments(int k, int lc) const { return phase_function_moments[lc][k]; }
  void setHenyeyGreenstein(double g, int lc = -1);
  void setIsotropic(int lc = -1);
  void setRayleigh(int lc = -1);
  void setHazeGarciaSiewert(int lc = -1);
  void setCloudGarciaSiewert(int lc = -1);
  void setPhaseFunction(PhaseFunction type, double g = 0.0, int lc = -1);
};

// DisortResult (DisortResult.hpp:16-125).  The special-boundary-condition
// outputs, the Fourier expansion and the temperature Jacobians stay empty.
class DisortResult {
 public:
  std::vector<double> flux_direct_beam, flux_down, flux_up, flux_tau_divergence, mean_intensity,
      mean_intensity_down, mean_intensity_up, mean_intensity_direct_beam;
  std::vector<double> albedo_medium, transmissivity_medium;
  double spherical_albedo = 0.0;
  double spherical_transmissivity = 0.0;
  std::vector<double> mu_angles;
  std::vector<std::vector<std::vector<double>>> intensity;  // [lu][iu][j]
  std::vector<std::vector<double>> intensity_azimuth_avg;   // [lu][iu]
  std::vector<std::vector<std::vector<double>>> intensity_fourier_expansion;
  std::vector<std::vector<double>> flux_up_temperature_jac, flux_down_temperature_jac, mean_intensity_temperature_jac,
      mean_intensity_down_temperature_jac, mean_intensity_up_temperature_jac, flux_divergence_temperature_jac;

  int num_user_tau() const { return ntau_; }
  int num_user_mu() const { return numu_; }
  int num_phi() const { return nphi_; }
  void allocate(int num_user_tau, int num_user_mu, int num_phi, int num_streams, bool special_bc,
                bool compute_intensity, bool output_fourier_expansion);
  double& intensities(int iu, int lu, int j) { return intensity[lu][iu][j]; }
  const double& intensities(int iu, int lu, int j) const { return intensity[lu][iu][j]; }
  double& intensitiesAzimuthAvg(int iu, int lu) { return intensity_azimuth_avg[lu][iu]; }
  const double& intensitiesAzimuthAvg(int iu, int lu) const { return intensity_azimuth_avg[lu][iu]; }
  double totalFluxDown(int lu) const { return flux_direct_beam[lu] + flux_down[lu]; }
  double netFlux(int lu) const { return flux_direct_beam[lu] + flux_down[lu] - flux_up[lu]; }

 private:
  int ntau_ = 0, numu_ = 0, nphi_ = 0;
};

// DisortSolver::solve (DisortSolver.cpp:20-399): one instance on the GPU.  Like
// the reference it allocates a config whose delta_tau is empty and fills in the
// automatic dimensions of `config`: tau_user at the layer boundaries without
// user optical depths, mu_user at the computational angles without user angles
// (or with comp_only_fluxes), and phase-function moment 0 set to 1.
class DisortSolver {
 public:
  DisortResult solve(DisortConfig& config);
};

// Spectral loops of the general solver (python_bindings.cpp:89-127): every band
// in one dsp_general_bands_solve call.
std::vector<DisortResult> solveSpectralBands(const DisortConfig& config,
                                             const std::vector<std::pair<double, double>>& wavenumber_bands,
                                             const SpectralOverrides& ov = {});
std::vector<DisortResult> solveSpectral(const DisortConfig& config, const std::vector<double>& wavenumbers,
                                        const SpectralOverrides& ov = {});

}  // namespace disortpp
