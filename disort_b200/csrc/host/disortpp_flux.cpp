// disortpp_flux.cpp — DisORT++ flux API (include/disortpp/disortpp.hpp) on top
// of the C ABI.  Validation mirrors DisortFluxConfig::validate
// (DisortFluxConfig.cpp:43-143) message for message; every solve is one batched
// dsp_flux_bands_solve call.
#include <dlfcn.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "../../../include/disortpp/disortpp.hpp"
#include "../../../include/dsp.h"

namespace disortpp {

#include "phase_tables.inc"

// ---------------------------------------------------------------------------
// phase functions (PhaseFunction.cpp:6-117)
// ---------------------------------------------------------------------------
namespace phase_function {
namespace {
void range(int num_layers, int lc, int& lo, int& hi) {
  lo = (lc < 0) ? 0 : lc;
  hi = (lc < 0) ? num_layers - 1 : lc;
}
}  // namespace

void fillHenyeyGreenstein(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, double g, int lc) {
  int lo, hi;
  range(num_layers, lc, lo, hi);
  for (int layer = lo; layer <= hi; ++layer) {
    double gk = 1.0;
    for (int k = 0; k <= nmom_nstr; ++k) {
      m[layer][k] = gk;
      gk *= g;
    }
  }
}

void fillIsotropic(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, int lc) {
  int lo, hi;
  range(num_layers, lc, lo, hi);
  for (int layer = lo; layer <= hi; ++layer)
    for (int k = 0; k <= nmom_nstr; ++k) m[layer][k] = (k == 0) ? 1.0 : 0.0;
}

void fillRayleigh(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, int lc) {
  int lo, hi;
  range(num_layers, lc, lo, hi);
  for (int layer = lo; layer <= hi; ++layer)
    for (int k = 0; k <= nmom_nstr; ++k) m[layer][k] = (k == 0) ? 1.0 : (k == 2) ? 0.1 : 0.0;
}

void fillHazeGarciaSiewert(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, int lc) {
  int lo, hi;
  range(num_layers, lc, lo, hi);
  for (int layer = lo; layer <= hi; ++layer) {
    m[layer][0] = 1.0;
    for (int k = 1; k <= nmom_nstr; ++k) m[layer][k] = (k <= kHazeCount) ? kHazeL[k - 1] / (2 * k + 1) : 0.0;
  }
}

void fillCloudGarciaSiewert(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, int lc) {
  int lo, hi;
  range(num_layers, lc, lo, hi);
  for (int layer = lo; layer <= hi; ++layer) {
    m[layer][0] = 1.0;
    for (int k = 1; k <= nmom_nstr; ++k) m[layer][k] = (k <= 298) ? kCloudC1[k - 1] / (2 * k + 1) : 0.0;
  }
}

void fillPhaseFunction(std::vector<std::vector<double>>& m, int nmom_nstr, int num_layers, PhaseFunction type,
                       double g, int lc) {
  switch (type) {
    case PhaseFunction::Isotropic: fillIsotropic(m, nmom_nstr, num_layers, lc); break;
    case PhaseFunction::Rayleigh: fillRayleigh(m, nmom_nstr, num_layers, lc); break;
    case PhaseFunction::HenyeyGreenstein: fillHenyeyGreenstein(m, nmom_nstr, num_layers, g, lc); break;
    case PhaseFunction::HazeGarciaSiewert: fillHazeGarciaSiewert(m, nmom_nstr, num_layers, lc); break;
    case PhaseFunction::CloudGarciaSiewert: fillCloudGarciaSiewert(m, nmom_nstr, num_layers, lc); break;
  }
}
}  // namespace phase_function

// ---------------------------------------------------------------------------
// DisortFluxConfig
// ---------------------------------------------------------------------------
DisortFluxConfig::DisortFluxConfig(int nlyr, int nstr, int nmom)
    : num_layers(nlyr), num_streams(nstr), num_phase_func_moments(nmom) {
  if (num_layers <= 0) throw std::invalid_argument("num_layers must be > 0");
  if (num_streams < 4 || num_streams % 2 != 0) throw std::invalid_argument("num_streams must be even and >= 4");
  if (num_phase_func_moments < 0) throw std::invalid_argument("num_phase_func_moments must be >= 0");
}

void DisortFluxConfig::allocate() {
  delta_tau.resize(num_layers, 0.0);
  single_scat_albedo.resize(num_layers, 0.0);
  const int nmom_size = nmomNstr() + 1;
  phase_function_moments.resize(num_layers);
  for (int lc = 0; lc < num_layers; ++lc) phase_function_moments[lc].resize(nmom_size, 0.0);
  if (use_thermal_emission) temperature.resize(num_layers + 1, 0.0);
  if (use_spherical_beam) level_altitudes.resize(num_layers + 1, 0.0);
}

void DisortFluxConfig::validate() const {
  if (num_layers <= 0) throw std::invalid_argument("num_layers must be > 0");
  if (num_streams < 4 || num_streams % 2 != 0) throw std::invalid_argument("num_streams must be even and >= 4");
  if (num_phase_func_moments < 0) throw std::invalid_argument("num_phase_func_moments must be >= 0");
  if (static_cast<int>(delta_tau.size()) < num_layers)
    throw std::invalid_argument("delta_tau size (" + std::to_string(delta_tau.size()) + ") < num_layers (" +
                                std::to_string(num_layers) + ")");
  if (static_cast<int>(single_scat_albedo.size()) < num_layers)
    throw std::invalid_argument("single_scat_albedo size < num_layers");
  if (static_cast<int>(phase_function_moments.size()) < num_layers)
    throw std::invalid_argument("phase_function_moments size < num_layers");
  const int nmom_needed = nmomNstr() + 1;
  for (int lc = 0; lc < num_layers; ++lc)
    if (static_cast<int>(phase_function_moments[lc].size()) < nmom_needed)
      throw std::invalid_argument("phase_function_moments[" + std::to_string(lc) + "] size < nmomNstr()+1");
  for (int lc = 0; lc < num_layers; ++lc) {
    if (delta_tau[lc] < 0.0) throw std::invalid_argument("delta_tau[" + std::to_string(lc) + "] must be >= 0");
    if (single_scat_albedo[lc] < 0.0 || single_scat_albedo[lc] > 1.0)
      throw std::invalid_argument("single_scat_albedo[" + std::to_string(lc) + "] must be in [0, 1]");
  }
  if (use_diffusion_lower_bc && !use_thermal_emission)
    throw std::invalid_argument("use_diffusion_lower_bc requires use_thermal_emission = true");
  if (direct_beam_flux < 0.0) throw std::invalid_argument("direct_beam_flux must be >= 0");
  if (direct_beam_flux > 0.0 && (direct_beam_mu <= 0.0 || direct_beam_mu > 1.0))
    throw std::invalid_argument("direct_beam_mu must be in (0, 1] when direct_beam_flux > 0");
  if (surface_albedo < 0.0 || surface_albedo > 1.0) throw std::invalid_argument("surface_albedo must be in [0, 1]");
  if (use_thermal_emission) {
    if (static_cast<int>(temperature.size()) < num_layers + 1)
      throw std::invalid_argument("temperature size < num_layers + 1");
    for (int lev = 0; lev <= num_layers; ++lev)
      if (temperature[lev] < 0.0) throw std::invalid_argument("temperature[" + std::to_string(lev) + "] must be >= 0");
    if (wavenumber_low < 0.0 || wavenumber_low > wavenumber_high)
      throw std::invalid_argument("wavenumber: need 0 <= wavenumber_low <= wavenumber_high");
    if (temperature_top < 0.0 || temperature_bottom < 0.0)
      throw std::invalid_argument("temperature_top and temperature_bottom must be >= 0");
    if (emissivity_top < 0.0 || emissivity_top > 1.0) throw std::invalid_argument("emissivity_top must be in [0, 1]");
  }
  if (use_spherical_beam) {
    if (bottom_radius <= 0.0) throw std::invalid_argument("bottom_radius must be > 0 when use_spherical_beam is true");
    if (static_cast<int>(level_altitudes.size()) < num_layers + 1)
      throw std::invalid_argument("level_altitudes size < num_layers + 1");
  }
  if (use_delta_m_plus && num_phase_func_moments < num_streams + 1)
    throw std::invalid_argument("use_delta_m_plus requires num_phase_func_moments >= num_streams + 1");
}

void DisortFluxConfig::setHenyeyGreenstein(double g, int lc) {
  phase_function::fillHenyeyGreenstein(phase_function_moments, nmomNstr(), num_layers, g, lc);
}
void DisortFluxConfig::setIsotropic(int lc) {
  phase_function::fillIsotropic(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortFluxConfig::setRayleigh(int lc) {
  phase_function::fillRayleigh(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortFluxConfig::setHazeGarciaSiewert(int lc) {
  phase_function::fillHazeGarciaSiewert(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortFluxConfig::setCloudGarciaSiewert(int lc) {
  phase_function::fillCloudGarciaSiewert(phase_function_moments, nmomNstr(), num_layers, lc);
}
void DisortFluxConfig::setPhaseFunction(PhaseFunction type, double g, int lc) {
  phase_function::fillPhaseFunction(phase_function_moments, nmomNstr(), num_layers, type, g, lc);
}

void FluxResult::allocate(int num_layers) {
  const size_t n = static_cast<size_t>(num_layers) + 1;
  for (auto* v : {&flux_direct_beam, &flux_down, &flux_up, &flux_tau_divergence, &mean_intensity,
                  &mean_intensity_down, &mean_intensity_up, &mean_intensity_direct_beam})
    v->assign(n, 0.0);
}

// ---------------------------------------------------------------------------
// engine access
// ---------------------------------------------------------------------------
namespace detail {

std::mutex& engine_mutex() {
  static std::mutex mu;
  return mu;
}

// The library's one engine context (device DSP_DEVICE, default 0); call with
// engine_mutex() held.
dsp_context engine_context_locked() {
  static dsp_context ctx = nullptr;
  if (!ctx) {
    const char* d = std::getenv("DSP_DEVICE");
    const int dev = d ? std::atoi(d) : 0;
    if (dsp_context_create(dev, nullptr, &ctx) != DSP_OK)
      throw std::runtime_error("disortpp: no CUDA device available for the B200 engine");
    // launch schedules: DSP_SCHEDULE_FILE, else the autotuned table installed
    // beside this library (lib/../tuning/b200.txt), when present
    std::string path;
    if (const char* e = std::getenv("DSP_SCHEDULE_FILE")) {
      path = e;
    } else {
      Dl_info info;
      if (dladdr(reinterpret_cast<void*>(&engine_context_locked), &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        const size_t cut = so.find_last_of('/');
        path = (cut == std::string::npos ? std::string(".") : so.substr(0, cut)) + "/../tuning/b200.txt";
      }
    }
    if (!path.empty()) {
      if (FILE* f = std::fopen(path.c_str(), "r")) {
        std::fclose(f);
        if (dsp_context_load_schedule_file(ctx, path.c_str()) != DSP_OK)
          throw std::runtime_error(std::string("disortpp: schedule file: ") + dsp_context_last_error(ctx));
      }
    }
  }
  return ctx;
}

}  // namespace detail

namespace {

std::mutex& g_mu = detail::engine_mutex();
dsp_context context_locked() { return detail::engine_context_locked(); }

bool supported(int n) {
  for (int s : {4, 6, 8, 10, 12, 14, 16, 32, 64})
    if (s == n) return true;
  return false;
}

// One band's effective configuration is the base config with override i applied
// (applyOverrides, python_bindings.cpp:73-82); check it with validate()'s rules
// and messages.  Rules that involve no override were checked once on the base.
void validate_band(const DisortFluxConfig& base, const SpectralOverrides& ov, size_t i, double lo, double hi) {
  const int L = base.num_layers;
  if (!ov.delta_tau.empty() || !ov.single_scat_albedo.empty() || !ov.phase_function_moments.empty()) {
    const std::vector<double>& dt = ov.delta_tau.empty() ? base.delta_tau : ov.delta_tau[i];
    const std::vector<double>& ss = ov.single_scat_albedo.empty() ? base.single_scat_albedo : ov.single_scat_albedo[i];
    const auto& pm = ov.phase_function_moments.empty() ? base.phase_function_moments : ov.phase_function_moments[i];
    if (static_cast<int>(dt.size()) < L)
      throw std::invalid_argument("delta_tau size (" + std::to_string(dt.size()) + ") < num_layers (" +
                                  std::to_string(L) + ")");
    if (static_cast<int>(ss.size()) < L) throw std::invalid_argument("single_scat_albedo size < num_layers");
    if (static_cast<int>(pm.size()) < L) throw std::invalid_argument("phase_function_moments size < num_layers");
    const int need = base.nmomNstr() + 1;
    for (int lc = 0; lc < L; ++lc)
      if (static_cast<int>(pm[lc].size()) < need)
        throw std::invalid_argument("phase_function_moments[" + std::to_string(lc) + "] size < nmomNstr()+1");
    for (int lc = 0; lc < L; ++lc) {
      if (dt[lc] < 0.0) throw std::invalid_argument("delta_tau[" + std::to_string(lc) + "] must be >= 0");
      if (ss[lc] < 0.0 || ss[lc] > 1.0)
        throw std::invalid_argument("single_scat_albedo[" + std::to_string(lc) + "] must be in [0, 1]");
    }
  }
  const double fbeam = ov.direct_beam_flux.empty() ? base.direct_beam_flux : ov.direct_beam_flux[i];
  const double alb = ov.surface_albedo.empty() ? base.surface_albedo : ov.surface_albedo[i];
  const double emis = ov.emissivity_top.empty() ? base.emissivity_top : ov.emissivity_top[i];
  if (fbeam < 0.0) throw std::invalid_argument("direct_beam_flux must be >= 0");
  if (fbeam > 0.0 && (base.direct_beam_mu <= 0.0 || base.direct_beam_mu > 1.0))
    throw std::invalid_argument("direct_beam_mu must be in (0, 1] when direct_beam_flux > 0");
  if (alb < 0.0 || alb > 1.0) throw std::invalid_argument("surface_albedo must be in [0, 1]");
  if (base.use_thermal_emission) {
    if (lo < 0.0 || lo > hi) throw std::invalid_argument("wavenumber: need 0 <= wavenumber_low <= wavenumber_high");
    if (emis < 0.0 || emis > 1.0) throw std::invalid_argument("emissivity_top must be in [0, 1]");
  }
}

// the rules that no override touches, with the base arrays where they are used
void validate_base(const DisortFluxConfig& c, const SpectralOverrides& ov) {
  DisortFluxConfig v = c;
  // the checks of overridden fields happen per band; neutralise them here
  if (!ov.delta_tau.empty() || !ov.single_scat_albedo.empty() || !ov.phase_function_moments.empty()) {
    v.delta_tau.assign(c.num_layers, 0.0);
    v.single_scat_albedo.assign(c.num_layers, 0.0);
    v.phase_function_moments.assign(c.num_layers, std::vector<double>(c.nmomNstr() + 1, 0.0));
  }
  v.direct_beam_flux = 0.0;
  v.surface_albedo = 0.0;
  v.emissivity_top = 1.0;
  v.wavenumber_low = 0.0;
  v.wavenumber_high = 0.0;
  v.validate();
}

struct Packed {
  std::vector<double> lo, hi, dtau, ssa, pmom, temp, alb, emis, fbeam, fisot, fisob, zalt;
  double mu0 = 0.5, ttop = 0.0, tbot = 0.0, rbot = 0.0;
};

// Build a dsp_flux_batch for the whole loop: overrides become per-instance
// arrays, everything else is shared (stride 0).
dsp_flux_batch pack(const DisortFluxConfig& c, const std::vector<std::pair<double, double>>& bands,
                    const SpectralOverrides& ov, Packed& pk) {
  const int n = static_cast<int>(bands.size());
  const int L = c.num_layers;
  const int pc = c.nmomNstr() + 1;
  dsp_flux_batch b{};
  b.n_inst = n;
  b.num_streams = c.num_streams;
  b.num_layers = L;
  b.num_phase_func_moments = c.num_phase_func_moments;
  b.pmom_count = pc;
  b.flags = (c.use_thermal_emission ? DSP_FLAG_THERMAL : 0u) | (c.use_delta_m_plus ? DSP_FLAG_DELTA_M_PLUS : 0u) |
            (c.use_diffusion_lower_bc ? DSP_FLAG_DIFFUSION_LOWER_BC : 0u) |
            (c.index_from_bottom ? DSP_FLAG_INDEX_FROM_BOTTOM : 0u) |
            (c.use_spherical_beam ? DSP_FLAG_SPHERICAL_BEAM : 0u);
  pk.lo.resize(n);
  pk.hi.resize(n);
  for (int i = 0; i < n; ++i) {
    pk.lo[i] = bands[i].first;
    pk.hi[i] = bands[i].second;
  }
  b.wavenumber_low = {pk.lo.data(), 1};
  b.wavenumber_high = {pk.hi.data(), 1};
  auto layers = [&](const std::vector<std::vector<double>>& per, const std::vector<double>& base,
                    std::vector<double>& dst) -> dsp_darray {
    if (per.empty()) {
      dst.assign(base.begin(), base.begin() + L);
      return {dst.data(), 0};
    }
    dst.resize(static_cast<size_t>(n) * L);
    for (int i = 0; i < n; ++i)
      for (int lc = 0; lc < L; ++lc) dst[static_cast<size_t>(i) * L + lc] = per[i][lc];
    return {dst.data(), L};
  };
  b.delta_tau = layers(ov.delta_tau, c.delta_tau, pk.dtau);
  b.single_scat_albedo = layers(ov.single_scat_albedo, c.single_scat_albedo, pk.ssa);
  if (ov.phase_function_moments.empty()) {
    pk.pmom.resize(static_cast<size_t>(L) * pc);
    for (int lc = 0; lc < L; ++lc)
      for (int k = 0; k < pc; ++k) pk.pmom[static_cast<size_t>(lc) * pc + k] = c.phase_function_moments[lc][k];
    b.phase_function_moments = {pk.pmom.data(), 0};
  } else {
    pk.pmom.resize(static_cast<size_t>(n) * L * pc);
    for (int i = 0; i < n; ++i)
      for (int lc = 0; lc < L; ++lc)
        for (int k = 0; k < pc; ++k)
          pk.pmom[(static_cast<size_t>(i) * L + lc) * pc + k] = ov.phase_function_moments[i][lc][k];
    b.phase_function_moments = {pk.pmom.data(), static_cast<int64_t>(L) * pc};
  }
  if (c.use_thermal_emission) {
    pk.temp.assign(c.temperature.begin(), c.temperature.begin() + L + 1);
    b.temperature = {pk.temp.data(), 0};
  }
  if (c.use_spherical_beam) {  // one column geometry for every band
    pk.zalt.assign(c.level_altitudes.begin(), c.level_altitudes.begin() + L + 1);
    pk.rbot = c.bottom_radius;
    b.level_altitudes = {pk.zalt.data(), 0};
    b.bottom_radius = {&pk.rbot, 0};
  }
  auto scalar = [&](const std::vector<double>& per, double base, std::vector<double>& dst) -> dsp_darray {
    if (per.empty()) {
      dst.assign(1, base);
      return {dst.data(), 0};
    }
    dst = per;
    return {dst.data(), 1};
  };
  b.surface_albedo = scalar(ov.surface_albedo, c.surface_albedo, pk.alb);
  b.emissivity_top = scalar(ov.emissivity_top, c.emissivity_top, pk.emis);
  b.direct_beam_flux = scalar(ov.direct_beam_flux, c.direct_beam_flux, pk.fbeam);
  b.isotropic_flux_top = scalar(ov.isotropic_flux_top, c.isotropic_flux_top, pk.fisot);
  b.isotropic_flux_bottom = scalar(ov.isotropic_flux_bottom, c.isotropic_flux_bottom, pk.fisob);
  pk.mu0 = c.direct_beam_mu;
  pk.ttop = c.temperature_top;
  pk.tbot = c.temperature_bottom;
  b.direct_beam_mu = {&pk.mu0, 0};
  b.temperature_top = {&pk.ttop, 0};
  b.temperature_bottom = {&pk.tbot, 0};
  return b;
}

// jac6 (null unless compute_temperature_jacobian): the six Jacobian arrays,
// each [n][L+1][L+2]
void run(const DisortFluxConfig& c, const std::vector<std::pair<double, double>>& bands, const SpectralOverrides& ov,
         double* out8[8], double* jac6[6] = nullptr) {
  if (!supported(c.num_streams))
    throw std::invalid_argument("Unsupported num_streams=" + std::to_string(c.num_streams) +
                                ". Supported values: 4, 6, 8, 10, 12, 14, 16, 32, 64");
  const size_t n = bands.size();
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
  validate_base(c, ov);
  for (size_t i = 0; i < n; ++i) validate_band(c, ov, i, bands[i].first, bands[i].second);
  if (n == 0) return;
  Packed pk;
  dsp_flux_batch b = pack(c, bands, ov, pk);
  std::vector<int32_t> status(n, 0);
  dsp_flux_out o{out8[0], out8[1], out8[2], out8[3], out8[4], out8[5], out8[6], out8[7], status.data()};
  std::lock_guard<std::mutex> lk(g_mu);
  dsp_context ctx = context_locked();
  dsp_status st;
  if (jac6) {
    const dsp_flux_jac_out j{jac6[0], jac6[1], jac6[2], jac6[3], jac6[4], jac6[5]};
    st = dsp_flux_bands_solve_jac(ctx, &b, &o, &j);
  } else {
    st = dsp_flux_bands_solve(ctx, &b, &o);
  }
  if (st != DSP_OK)
    throw std::runtime_error(std::string("disortpp: GPU solve failed: ") + dsp_status_string(st) + ": " +
                             dsp_context_last_error(ctx));
  for (size_t i = 0; i < n; ++i)
    if (status[i] == DSP_ERR_INVALID_INPUT || status[i] == DSP_ERR_UNSUPPORTED)
      throw std::invalid_argument("band " + std::to_string(i) + ": " + dsp_status_string((dsp_status)status[i]));
}

// jbuf: the six Jacobian arrays back to back ([6][n][L+1][L+2]), or empty
std::vector<FluxResult> to_results(size_t n, int L, const std::vector<double>& buf,
                                   const std::vector<double>& jbuf = {}) {
  std::vector<FluxResult> res(n);
  const size_t nlev = static_cast<size_t>(L) + 1, ndof = static_cast<size_t>(L) + 2;
  for (size_t i = 0; i < n; ++i) {
    FluxResult& r = res[i];
    std::vector<double>* dst[8] = {&r.flux_direct_beam, &r.flux_down, &r.flux_up, &r.flux_tau_divergence,
                                   &r.mean_intensity, &r.mean_intensity_down, &r.mean_intensity_up,
                                   &r.mean_intensity_direct_beam};
    for (int f = 0; f < 8; ++f) {
      const double* src = buf.data() + (static_cast<size_t>(f) * n + i) * nlev;
      dst[f]->assign(src, src + nlev);
    }
    if (!jbuf.empty()) {
      std::vector<std::vector<double>>* jd[6] = {&r.flux_up_temperature_jac, &r.flux_down_temperature_jac,
                                                 &r.mean_intensity_temperature_jac,
                                                 &r.mean_intensity_down_temperature_jac,
                                                 &r.mean_intensity_up_temperature_jac,
                                                 &r.flux_divergence_temperature_jac};
      for (int f = 0; f < 6; ++f) {
        jd[f]->resize(nlev);
        for (size_t lu = 0; lu < nlev; ++lu) {
          const double* src = jbuf.data() + ((static_cast<size_t>(f) * n + i) * nlev + lu) * ndof;
          (*jd[f])[lu].assign(src, src + ndof);
        }
      }
    }
  }
  return res;
}

}  // namespace

void solveFluxSpectralBandsInto(const DisortFluxConfig& config,
                                const std::vector<std::pair<double, double>>& bands, const SpectralOverrides& ov,
                                double* out8[8]) {
  if (config.compute_temperature_jacobian)
    throw std::invalid_argument("temperature Jacobians are returned by solve_flux_spectral_bands");
  run(config, bands, ov, out8);
}

std::vector<FluxResult> solveFluxSpectralBands(const DisortFluxConfig& config,
                                               const std::vector<std::pair<double, double>>& bands,
                                               const SpectralOverrides& ov) {
  const size_t n = bands.size();
  const size_t nlev = static_cast<size_t>(config.num_layers) + 1;
  std::vector<double> buf(8 * n * nlev);
  double* out8[8];
  for (int f = 0; f < 8; ++f) out8[f] = buf.data() + static_cast<size_t>(f) * n * nlev;
  // Jacobians are returned when asked for with thermal emission on; otherwise
  // they stay empty, as the reference clears them (FluxSolver.cpp:1299-1307)
  const bool jac = config.compute_temperature_jacobian;
  std::vector<double> jbuf;
  double* jac6[6];
  if (jac) {
    const size_t per = n * nlev * (nlev + 1);
    jbuf.resize(6 * per);
    for (int f = 0; f < 6; ++f) jac6[f] = jbuf.data() + f * per;
  }
  run(config, bands, ov, out8, jac ? jac6 : nullptr);
  if (jac && !config.use_thermal_emission) jbuf.clear();
  return to_results(n, config.num_layers, buf, jbuf);
}

std::vector<FluxResult> solveFluxSpectral(const DisortFluxConfig& config, const std::vector<double>& wavenumbers,
                                          const SpectralOverrides& ov) {
  std::vector<std::pair<double, double>> bands;
  bands.reserve(wavenumbers.size());
  for (double w : wavenumbers) bands.emplace_back(w, w);
  return solveFluxSpectralBands(config, bands, ov);
}

FluxResult solveFluxOne(const DisortFluxConfig& config, int nstr) {
  config.validate();
  if (config.num_streams != nstr)
    throw std::invalid_argument("DisortFluxSolver<" + std::to_string(nstr) + ">::solve: config.num_streams=" +
                                std::to_string(config.num_streams) + " does not match template NStr");
  std::vector<std::pair<double, double>> one{{config.wavenumber_low, config.wavenumber_high}};
  return solveFluxSpectralBands(config, one, SpectralOverrides{})[0];
}

}  // namespace disortpp
