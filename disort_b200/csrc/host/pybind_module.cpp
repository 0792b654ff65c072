// pybind_module.cpp — the `disortpp` Python API served by the B200 engine.
//
// Mirrors the reference module (src/python_bindings.cpp:213-763): the same
// class, property, function and keyword names, the same immutable-tuple
// getters for vector fields (:21-44), the GIL released around
// solves.  Added: solve_flux_spectral_bands_arrays, which takes numpy arrays and
// returns numpy arrays [n_bands, num_layers+1] without per-band objects.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "../../../include/disortpp/disortpp.hpp"

namespace py = pybind11;
using namespace disortpp;

namespace {

// Vector members read back as immutable tuples (a snapshot: element assignment on
// the result cannot silently edit a temporary copy) and are replaced whole on
// assignment, which is how the reference module exposes them.
py::tuple as_tuple(const std::vector<double>& v) { return py::tuple(py::cast(v)); }
py::tuple as_tuple(const std::vector<std::vector<double>>& v) {
  py::tuple t(v.size());
  for (size_t i = 0; i < v.size(); ++i) t[i] = as_tuple(v[i]);
  return t;
}
template <class C, class V>
auto tuple_getter(V C::*member) {
  return [member](const C& c) { return as_tuple(c.*member); };
}
template <class C, class V>
auto whole_setter(V C::*member) {
  return [member](C& c, const V& v) { c.*member = v; };
}

}  // namespace

namespace {

template <int N>
void bind_flux_solver(py::module_& m, const char* name, const char* doc) {
  py::class_<DisortFluxSolver<N>>(m, name, doc)
      .def(py::init<>())
      .def(
          "solve",
          [](DisortFluxSolver<N>& self, const DisortFluxConfig& config) {
            py::gil_scoped_release release;
            return self.solve(config);
          },
          py::arg("config"));
}

SpectralOverrides make_overrides(std::vector<std::vector<double>> delta_tau,
                                 std::vector<std::vector<double>> single_scat_albedo,
                                 std::vector<std::vector<std::vector<double>>> phase_function_moments,
                                 std::vector<double> surface_albedo, std::vector<double> emissivity_top,
                                 std::vector<double> direct_beam_flux, std::vector<double> isotropic_flux_top,
                                 std::vector<double> isotropic_flux_bottom) {
  return SpectralOverrides{std::move(delta_tau),        std::move(single_scat_albedo),
                           std::move(phase_function_moments), std::move(surface_albedo),
                           std::move(emissivity_top),   std::move(direct_beam_flux),
                           std::move(isotropic_flux_top), std::move(isotropic_flux_bottom)};
}

// numpy array (or None) -> nested vectors, shape-checked
std::vector<std::vector<double>> rows2(const py::object& o, size_t n) {
  std::vector<std::vector<double>> out;
  if (o.is_none()) return out;
  auto a = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(o);
  if (!a || a.ndim() != 2 || (size_t)a.shape(0) != n) throw std::invalid_argument("expected an array [n_bands, num_layers]");
  out.resize(n);
  const double* p = a.data();
  for (size_t i = 0; i < n; ++i) out[i].assign(p + i * a.shape(1), p + (i + 1) * a.shape(1));
  return out;
}

std::vector<std::vector<std::vector<double>>> rows3(const py::object& o, size_t n) {
  std::vector<std::vector<std::vector<double>>> out;
  if (o.is_none()) return out;
  auto a = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(o);
  if (!a || a.ndim() != 3 || (size_t)a.shape(0) != n)
    throw std::invalid_argument("expected an array [n_bands, num_layers, nmom+1]");
  out.resize(n);
  const double* p = a.data();
  const size_t L = a.shape(1), K = a.shape(2);
  for (size_t i = 0; i < n; ++i) {
    out[i].resize(L);
    for (size_t l = 0; l < L; ++l) out[i][l].assign(p + (i * L + l) * K, p + (i * L + l + 1) * K);
  }
  return out;
}

std::vector<double> vec1(const py::object& o) {
  if (o.is_none()) return {};
  auto a = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(o);
  if (!a) throw std::invalid_argument("expected a 1-D array");
  return std::vector<double>(a.data(), a.data() + a.size());
}

}  // namespace

PYBIND11_MODULE(_disortpp, m) {
  m.doc() = "DisORT++ API on the B200-native DISORT engine (FP64, sm_100a)";
  m.attr("__version__") = "1.0";

  py::enum_<PhaseFunction>(m, "PhaseFunction")
      .value("Isotropic", PhaseFunction::Isotropic)
      .value("Rayleigh", PhaseFunction::Rayleigh)
      .value("HenyeyGreenstein", PhaseFunction::HenyeyGreenstein)
      .value("HazeGarciaSiewert", PhaseFunction::HazeGarciaSiewert)
      .value("CloudGarciaSiewert", PhaseFunction::CloudGarciaSiewert);

  py::enum_<BoundaryConditionType>(m, "BoundaryConditionType")
      .value("General", BoundaryConditionType::General)
      .value("Special", BoundaryConditionType::Special);

  py::enum_<BrdfType>(m, "BrdfType")
      .value("NONE", BrdfType::None)
      .value("RPV", BrdfType::RPV)
      .value("CoxMunk", BrdfType::CoxMunk)
      .value("Ambrals", BrdfType::Ambrals)
      .value("Hapke", BrdfType::Hapke);

  py::class_<DisortFlags>(m, "DisortFlags")
      .def(py::init<>())
      .def_readwrite("use_user_tau", &DisortFlags::use_user_tau)
      .def_readwrite("use_user_mu", &DisortFlags::use_user_mu)
      .def_readwrite("ibcnd", &DisortFlags::ibcnd)
      .def_readwrite("use_lambertian_surface", &DisortFlags::use_lambertian_surface)
      .def_readwrite("use_thermal_emission", &DisortFlags::use_thermal_emission)
      .def_readwrite("use_spherical_beam", &DisortFlags::use_spherical_beam)
      .def_readwrite("comp_only_fluxes", &DisortFlags::comp_only_fluxes)
      .def_readwrite("brdf_type", &DisortFlags::brdf_type)
      .def_readwrite("intensity_corr_buras", &DisortFlags::intensity_corr_buras)
      .def_readwrite("intensity_corr_nakajima", &DisortFlags::intensity_corr_nakajima)
      .def_readwrite("use_delta_m_plus", &DisortFlags::use_delta_m_plus)
      .def_readwrite("use_diffusion_lower_bc", &DisortFlags::use_diffusion_lower_bc)
      .def_readwrite("output_fourier_expansion", &DisortFlags::output_fourier_expansion)
      .def_readwrite("index_from_bottom", &DisortFlags::index_from_bottom)
      .def_readwrite("compute_temperature_jacobian", &DisortFlags::compute_temperature_jacobian);

  py::class_<BoundaryConditions>(m, "BoundaryConditions")
      .def(py::init<>())
      .def_readwrite("direct_beam_flux", &BoundaryConditions::direct_beam_flux)
      .def_readwrite("direct_beam_mu", &BoundaryConditions::direct_beam_mu)
      .def_readwrite("direct_beam_phi", &BoundaryConditions::direct_beam_phi)
      .def_readwrite("isotropic_flux_top", &BoundaryConditions::isotropic_flux_top)
      .def_readwrite("isotropic_flux_bottom", &BoundaryConditions::isotropic_flux_bottom)
      .def_readwrite("temperature_top", &BoundaryConditions::temperature_top)
      .def_readwrite("temperature_bottom", &BoundaryConditions::temperature_bottom)
      .def_readwrite("emissivity_top", &BoundaryConditions::emissivity_top)
      .def_readwrite("surface_albedo", &BoundaryConditions::surface_albedo);

  py::class_<RpvBrdfSpec>(m, "RpvBrdfSpec")
      .def(py::init<>())
      .def_readwrite("rho0", &RpvBrdfSpec::rho0)
      .def_readwrite("k", &RpvBrdfSpec::k)
      .def_readwrite("theta", &RpvBrdfSpec::theta)
      .def_readwrite("sigma", &RpvBrdfSpec::sigma)
      .def_readwrite("t1", &RpvBrdfSpec::t1)
      .def_readwrite("t2", &RpvBrdfSpec::t2)
      .def_readwrite("scale", &RpvBrdfSpec::scale);
  py::class_<AmbralsBrdfSpec>(m, "AmbralsBrdfSpec")
      .def(py::init<>())
      .def_readwrite("iso", &AmbralsBrdfSpec::iso)
      .def_readwrite("vol", &AmbralsBrdfSpec::vol)
      .def_readwrite("geo", &AmbralsBrdfSpec::geo);
  py::class_<CoxMunkBrdfSpec>(m, "CoxMunkBrdfSpec")
      .def(py::init<>())
      .def_readwrite("u10", &CoxMunkBrdfSpec::u10)
      .def_readwrite("pcl", &CoxMunkBrdfSpec::pcl)
      .def_readwrite("xsal", &CoxMunkBrdfSpec::xsal)
      .def_readwrite("refractive_index", &CoxMunkBrdfSpec::refractive_index)
      .def_readwrite("do_shadow", &CoxMunkBrdfSpec::do_shadow);
  py::class_<HapkeBrdfSpec>(m, "HapkeBrdfSpec")
      .def(py::init<>())
      .def_readwrite("b0", &HapkeBrdfSpec::b0)
      .def_readwrite("hh", &HapkeBrdfSpec::hh)
      .def_readwrite("w", &HapkeBrdfSpec::w);
  py::class_<BrdfSpecification>(m, "BrdfSpecification")
      .def(py::init<>())
      .def_readwrite("rpv", &BrdfSpecification::rpv)
      .def_readwrite("ambrals", &BrdfSpecification::ambrals)
      .def_readwrite("cox_munk", &BrdfSpecification::cox_munk)
      .def_readwrite("hapke", &BrdfSpecification::hapke)
      .def("set_rpv", &BrdfSpecification::setRpv, py::arg("spec"))
      .def("set_ambrals", &BrdfSpecification::setAmbrals, py::arg("spec"))
      .def("set_cox_munk", &BrdfSpecification::setCoxMunk, py::arg("spec"))
      .def("set_hapke", &BrdfSpecification::setHapke, py::arg("spec"));

  py::class_<DisortConfig>(m, "DisortConfig")
      .def(py::init<>())
      .def(py::init<int, int, int>(), py::arg("num_layers"), py::arg("num_streams"),
           py::arg("num_phase_func_moments") = 0)
      .def_readwrite("flags", &DisortConfig::flags)
      .def_readwrite("bc", &DisortConfig::bc)
      .def_readwrite("brdf", &DisortConfig::brdf)
      .def_readwrite("num_layers", &DisortConfig::num_layers)
      .def_readwrite("num_phase_func_moments", &DisortConfig::num_phase_func_moments)
      .def_readwrite("num_streams", &DisortConfig::num_streams)
      .def_readwrite("num_user_tau", &DisortConfig::num_user_tau)
      .def_readwrite("num_user_mu", &DisortConfig::num_user_mu)
      .def_readwrite("num_phi", &DisortConfig::num_phi)
      .def_readwrite("num_phase_func_angles", &DisortConfig::num_phase_func_angles)
      .def_readwrite("wavenumber_low", &DisortConfig::wavenumber_low)
      .def_readwrite("wavenumber_high", &DisortConfig::wavenumber_high)
      .def_readwrite("accuracy_fourier_series", &DisortConfig::accuracy_fourier_series)
      .def_readwrite("bottom_radius", &DisortConfig::bottom_radius)
      .def_property("delta_tau", tuple_getter(&DisortConfig::delta_tau), whole_setter(&DisortConfig::delta_tau))
      .def_property("single_scat_albedo", tuple_getter(&DisortConfig::single_scat_albedo), whole_setter(&DisortConfig::single_scat_albedo))
      .def_property("phase_function_moments", tuple_getter(&DisortConfig::phase_function_moments), whole_setter(&DisortConfig::phase_function_moments))
      .def_property("temperature", tuple_getter(&DisortConfig::temperature), whole_setter(&DisortConfig::temperature))
      .def_property("level_altitudes", tuple_getter(&DisortConfig::level_altitudes), whole_setter(&DisortConfig::level_altitudes))
      .def_property("tau_user", tuple_getter(&DisortConfig::tau_user), whole_setter(&DisortConfig::tau_user))
      .def_property("mu_user", tuple_getter(&DisortConfig::mu_user), whole_setter(&DisortConfig::mu_user))
      .def_property("phi_user", tuple_getter(&DisortConfig::phi_user), whole_setter(&DisortConfig::phi_user))
      .def_property("mu_phase_function", tuple_getter(&DisortConfig::mu_phase_function), whole_setter(&DisortConfig::mu_phase_function))
      .def_property("phase_function", tuple_getter(&DisortConfig::phase_function), whole_setter(&DisortConfig::phase_function))
      .def("nmom_nstr", &DisortConfig::nmomNstr)
      .def("allocate", &DisortConfig::allocate)
      .def("validate", &DisortConfig::validate)
      .def("set_henyey_greenstein", &DisortConfig::setHenyeyGreenstein, py::arg("g"), py::arg("lc") = -1)
      .def("set_isotropic", &DisortConfig::setIsotropic, py::arg("lc") = -1)
      .def("set_rayleigh", &DisortConfig::setRayleigh, py::arg("lc") = -1)
      .def("set_haze_garcia_siewert", &DisortConfig::setHazeGarciaSiewert, py::arg("lc") = -1)
      .def("set_cloud_garcia_siewert", &DisortConfig::setCloudGarciaSiewert, py::arg("lc") = -1)
      .def("set_phase_function", &DisortConfig::setPhaseFunction, py::arg("type"), py::arg("g") = 0.0,
           py::arg("lc") = -1);

  py::class_<DisortResult>(m, "DisortResult")
      .def(py::init<>())
      .def_readwrite("flux_direct_beam", &DisortResult::flux_direct_beam)
      .def_readwrite("flux_down", &DisortResult::flux_down)
      .def_readwrite("flux_up", &DisortResult::flux_up)
      .def_readwrite("flux_tau_divergence", &DisortResult::flux_tau_divergence)
      .def_readwrite("mean_intensity", &DisortResult::mean_intensity)
      .def_readwrite("mean_intensity_down", &DisortResult::mean_intensity_down)
      .def_readwrite("mean_intensity_up", &DisortResult::mean_intensity_up)
      .def_readwrite("mean_intensity_direct_beam", &DisortResult::mean_intensity_direct_beam)
      .def_readwrite("albedo_medium", &DisortResult::albedo_medium)
      .def_readwrite("transmissivity_medium", &DisortResult::transmissivity_medium)
      .def_readwrite("spherical_albedo", &DisortResult::spherical_albedo)
      .def_readwrite("spherical_transmissivity", &DisortResult::spherical_transmissivity)
      .def_readwrite("flux_up_temperature_jac", &DisortResult::flux_up_temperature_jac)
      .def_readwrite("flux_down_temperature_jac", &DisortResult::flux_down_temperature_jac)
      .def_readwrite("mean_intensity_temperature_jac", &DisortResult::mean_intensity_temperature_jac)
      .def_readwrite("mean_intensity_down_temperature_jac", &DisortResult::mean_intensity_down_temperature_jac)
      .def_readwrite("mean_intensity_up_temperature_jac", &DisortResult::mean_intensity_up_temperature_jac)
      .def_readwrite("flux_divergence_temperature_jac", &DisortResult::flux_divergence_temperature_jac)
      .def_readwrite("mu_angles", &DisortResult::mu_angles)
      .def_readwrite("intensity", &DisortResult::intensity)
      .def_readwrite("intensity_azimuth_avg", &DisortResult::intensity_azimuth_avg)
      .def_readwrite("intensity_fourier_expansion", &DisortResult::intensity_fourier_expansion)
      .def("num_user_tau", &DisortResult::num_user_tau)
      .def("num_user_mu", &DisortResult::num_user_mu)
      .def("num_phi", &DisortResult::num_phi)
      .def("total_flux_down", &DisortResult::totalFluxDown, py::arg("lu"))
      .def("net_flux", &DisortResult::netFlux, py::arg("lu"))
      .def("intensities", py::overload_cast<int, int, int>(&DisortResult::intensities, py::const_), py::arg("iu"),
           py::arg("lu"), py::arg("j"))
      .def("intensities_azimuth_avg", py::overload_cast<int, int>(&DisortResult::intensitiesAzimuthAvg, py::const_),
           py::arg("iu"), py::arg("lu"));

  py::class_<DisortSolver>(m, "DisortSolver", "General discrete ordinates radiative transfer solver")
      .def(py::init<>())
      .def(
          "solve",
          [](DisortSolver& self, DisortConfig& config) {
            py::gil_scoped_release release;
            return self.solve(config);
          },
          py::arg("config"),
          "Solve the radiative transfer problem. Note: config may be modified by the solver to set automatic "
          "dimensions.");

  py::class_<DisortFluxConfig>(m, "DisortFluxConfig")
      .def(py::init<>())
      .def(py::init<int, int, int>(), py::arg("num_layers"), py::arg("num_streams"),
           py::arg("num_phase_func_moments") = 0)
      .def_readwrite("num_layers", &DisortFluxConfig::num_layers)
      .def_readwrite("num_streams", &DisortFluxConfig::num_streams)
      .def_readwrite("num_phase_func_moments", &DisortFluxConfig::num_phase_func_moments)
      .def_readwrite("use_thermal_emission", &DisortFluxConfig::use_thermal_emission)
      .def_readwrite("use_spherical_beam", &DisortFluxConfig::use_spherical_beam)
      .def_readwrite("use_delta_m_plus", &DisortFluxConfig::use_delta_m_plus)
      .def_readwrite("use_diffusion_lower_bc", &DisortFluxConfig::use_diffusion_lower_bc)
      .def_readwrite("index_from_bottom", &DisortFluxConfig::index_from_bottom)
      .def_readwrite("compute_temperature_jacobian", &DisortFluxConfig::compute_temperature_jacobian)
      .def_readwrite("direct_beam_flux", &DisortFluxConfig::direct_beam_flux)
      .def_readwrite("direct_beam_mu", &DisortFluxConfig::direct_beam_mu)
      .def_readwrite("isotropic_flux_top", &DisortFluxConfig::isotropic_flux_top)
      .def_readwrite("isotropic_flux_bottom", &DisortFluxConfig::isotropic_flux_bottom)
      .def_readwrite("temperature_top", &DisortFluxConfig::temperature_top)
      .def_readwrite("temperature_bottom", &DisortFluxConfig::temperature_bottom)
      .def_readwrite("emissivity_top", &DisortFluxConfig::emissivity_top)
      .def_readwrite("surface_albedo", &DisortFluxConfig::surface_albedo)
      .def_readwrite("wavenumber_low", &DisortFluxConfig::wavenumber_low)
      .def_readwrite("wavenumber_high", &DisortFluxConfig::wavenumber_high)
      .def_readwrite("bottom_radius", &DisortFluxConfig::bottom_radius)
      .def_property("delta_tau", tuple_getter(&DisortFluxConfig::delta_tau), whole_setter(&DisortFluxConfig::delta_tau))
      .def_property("single_scat_albedo", tuple_getter(&DisortFluxConfig::single_scat_albedo), whole_setter(&DisortFluxConfig::single_scat_albedo))
      .def_property("phase_function_moments", tuple_getter(&DisortFluxConfig::phase_function_moments), whole_setter(&DisortFluxConfig::phase_function_moments))
      .def_property("temperature", tuple_getter(&DisortFluxConfig::temperature), whole_setter(&DisortFluxConfig::temperature))
      .def_property("level_altitudes", tuple_getter(&DisortFluxConfig::level_altitudes), whole_setter(&DisortFluxConfig::level_altitudes))
      .def("nmom_nstr", &DisortFluxConfig::nmomNstr)
      .def("allocate", &DisortFluxConfig::allocate)
      .def("validate", &DisortFluxConfig::validate)
      .def("set_henyey_greenstein", &DisortFluxConfig::setHenyeyGreenstein, py::arg("g"), py::arg("lc") = -1)
      .def("set_isotropic", &DisortFluxConfig::setIsotropic, py::arg("lc") = -1)
      .def("set_rayleigh", &DisortFluxConfig::setRayleigh, py::arg("lc") = -1)
      .def("set_haze_garcia_siewert", &DisortFluxConfig::setHazeGarciaSiewert, py::arg("lc") = -1)
      .def("set_cloud_garcia_siewert", &DisortFluxConfig::setCloudGarciaSiewert, py::arg("lc") = -1)
      .def("set_phase_function", &DisortFluxConfig::setPhaseFunction, py::arg("type"), py::arg("g") = 0.0,
           py::arg("lc") = -1);

  py::class_<FluxResult>(m, "FluxResult")
      .def(py::init<>())
      .def_readwrite("flux_direct_beam", &FluxResult::flux_direct_beam)
      .def_readwrite("flux_down", &FluxResult::flux_down)
      .def_readwrite("flux_up", &FluxResult::flux_up)
      .def_readwrite("flux_tau_divergence", &FluxResult::flux_tau_divergence)
      .def_readwrite("mean_intensity", &FluxResult::mean_intensity)
      .def_readwrite("mean_intensity_down", &FluxResult::mean_intensity_down)
      .def_readwrite("mean_intensity_up", &FluxResult::mean_intensity_up)
      .def_readwrite("mean_intensity_direct_beam", &FluxResult::mean_intensity_direct_beam)
      .def_readwrite("flux_up_temperature_jac", &FluxResult::flux_up_temperature_jac)
      .def_readwrite("flux_down_temperature_jac", &FluxResult::flux_down_temperature_jac)
      .def_readwrite("mean_intensity_temperature_jac", &FluxResult::mean_intensity_temperature_jac)
      .def_readwrite("mean_intensity_down_temperature_jac", &FluxResult::mean_intensity_down_temperature_jac)
      .def_readwrite("mean_intensity_up_temperature_jac", &FluxResult::mean_intensity_up_temperature_jac)
      .def_readwrite("flux_divergence_temperature_jac", &FluxResult::flux_divergence_temperature_jac)
      .def("num_levels", &FluxResult::num_levels)
      .def("total_flux_down", &FluxResult::totalFluxDown, py::arg("lev"))
      .def("net_flux", &FluxResult::netFlux, py::arg("lev"));

  bind_flux_solver<4>(m, "DisortFluxSolver4", "Flux-only solver with 4 streams");
  bind_flux_solver<6>(m, "DisortFluxSolver6", "Flux-only solver with 6 streams");
  bind_flux_solver<8>(m, "DisortFluxSolver8", "Flux-only solver with 8 streams");
  bind_flux_solver<10>(m, "DisortFluxSolver10", "Flux-only solver with 10 streams");
  bind_flux_solver<12>(m, "DisortFluxSolver12", "Flux-only solver with 12 streams");
  bind_flux_solver<14>(m, "DisortFluxSolver14", "Flux-only solver with 14 streams");
  bind_flux_solver<16>(m, "DisortFluxSolver16", "Flux-only solver with 16 streams");
  bind_flux_solver<32>(m, "DisortFluxSolver32", "Flux-only solver with 32 streams");
  bind_flux_solver<64>(m, "DisortFluxSolver64", "Flux-only solver with 64 streams");

  m.def(
      "create_flux_solver",
      [](int nstr) -> py::object {
        switch (nstr) {
          case 4: return py::cast(DisortFluxSolver<4>());
          case 6: return py::cast(DisortFluxSolver<6>());
          case 8: return py::cast(DisortFluxSolver<8>());
          case 10: return py::cast(DisortFluxSolver<10>());
          case 12: return py::cast(DisortFluxSolver<12>());
          case 14: return py::cast(DisortFluxSolver<14>());
          case 16: return py::cast(DisortFluxSolver<16>());
          case 32: return py::cast(DisortFluxSolver<32>());
          case 64: return py::cast(DisortFluxSolver<64>());
          default:
            throw std::invalid_argument("Unsupported nstr=" + std::to_string(nstr) +
                                        ". Supported values: 4, 6, 8, 10, 12, 14, 16, 32, 64");
        }
      },
      py::arg("nstr"), "Create a flux-only solver for the given number of streams (4, 6, 8, 10, 12, 14, 16, 32, or 64)");

  m.def(
      "solve_spectral",
      [](DisortConfig config, const std::vector<double>& wavenumbers, std::vector<std::vector<double>> delta_tau,
         std::vector<std::vector<double>> single_scat_albedo,
         std::vector<std::vector<std::vector<double>>> phase_function_moments, std::vector<double> surface_albedo,
         std::vector<double> emissivity_top, std::vector<double> direct_beam_flux,
         std::vector<double> isotropic_flux_top, std::vector<double> isotropic_flux_bottom) {
        SpectralOverrides ov = make_overrides(std::move(delta_tau), std::move(single_scat_albedo),
                                              std::move(phase_function_moments), std::move(surface_albedo),
                                              std::move(emissivity_top), std::move(direct_beam_flux),
                                              std::move(isotropic_flux_top), std::move(isotropic_flux_bottom));
        py::gil_scoped_release release;
        return solveSpectral(config, wavenumbers, ov);
      },
      py::arg("config"), py::arg("wavenumbers"), py::arg("delta_tau") = std::vector<std::vector<double>>{},
      py::arg("single_scat_albedo") = std::vector<std::vector<double>>{},
      py::arg("phase_function_moments") = std::vector<std::vector<std::vector<double>>>{},
      py::arg("surface_albedo") = std::vector<double>{}, py::arg("emissivity_top") = std::vector<double>{},
      py::arg("direct_beam_flux") = std::vector<double>{}, py::arg("isotropic_flux_top") = std::vector<double>{},
      py::arg("isotropic_flux_bottom") = std::vector<double>{},
      "Solve for a list of single wavenumbers (wavenumber_low = wavenumber_high = wn), all in one GPU batch. "
      "Optional per-wavelength arrays override the corresponding config values. Returns a list of DisortResult.");

  m.def(
      "solve_spectral_bands",
      [](DisortConfig config, const std::vector<std::pair<double, double>>& wavenumber_bands,
         std::vector<std::vector<double>> delta_tau, std::vector<std::vector<double>> single_scat_albedo,
         std::vector<std::vector<std::vector<double>>> phase_function_moments, std::vector<double> surface_albedo,
         std::vector<double> emissivity_top, std::vector<double> direct_beam_flux,
         std::vector<double> isotropic_flux_top, std::vector<double> isotropic_flux_bottom) {
        SpectralOverrides ov = make_overrides(std::move(delta_tau), std::move(single_scat_albedo),
                                              std::move(phase_function_moments), std::move(surface_albedo),
                                              std::move(emissivity_top), std::move(direct_beam_flux),
                                              std::move(isotropic_flux_top), std::move(isotropic_flux_bottom));
        py::gil_scoped_release release;
        return solveSpectralBands(config, wavenumber_bands, ov);
      },
      py::arg("config"), py::arg("wavenumber_bands"), py::arg("delta_tau") = std::vector<std::vector<double>>{},
      py::arg("single_scat_albedo") = std::vector<std::vector<double>>{},
      py::arg("phase_function_moments") = std::vector<std::vector<std::vector<double>>>{},
      py::arg("surface_albedo") = std::vector<double>{}, py::arg("emissivity_top") = std::vector<double>{},
      py::arg("direct_beam_flux") = std::vector<double>{}, py::arg("isotropic_flux_top") = std::vector<double>{},
      py::arg("isotropic_flux_bottom") = std::vector<double>{},
      "Solve for a list of wavenumber bands (pairs of (low, high)), all in one GPU batch. Optional "
      "per-wavelength arrays override the corresponding config values. Returns a list of DisortResult.");

  m.def(
      "solve_flux_spectral",
      [](DisortFluxConfig& config, const std::vector<double>& wavenumbers, std::vector<std::vector<double>> delta_tau,
         std::vector<std::vector<double>> single_scat_albedo,
         std::vector<std::vector<std::vector<double>>> phase_function_moments, std::vector<double> surface_albedo,
         std::vector<double> emissivity_top, std::vector<double> direct_beam_flux,
         std::vector<double> isotropic_flux_top, std::vector<double> isotropic_flux_bottom) {
        SpectralOverrides ov = make_overrides(std::move(delta_tau), std::move(single_scat_albedo),
                                              std::move(phase_function_moments), std::move(surface_albedo),
                                              std::move(emissivity_top), std::move(direct_beam_flux),
                                              std::move(isotropic_flux_top), std::move(isotropic_flux_bottom));
        py::gil_scoped_release release;
        return solveFluxSpectral(config, wavenumbers, ov);
      },
      py::arg("config"), py::arg("wavenumbers"), py::arg("delta_tau") = std::vector<std::vector<double>>{},
      py::arg("single_scat_albedo") = std::vector<std::vector<double>>{},
      py::arg("phase_function_moments") = std::vector<std::vector<std::vector<double>>>{},
      py::arg("surface_albedo") = std::vector<double>{}, py::arg("emissivity_top") = std::vector<double>{},
      py::arg("direct_beam_flux") = std::vector<double>{}, py::arg("isotropic_flux_top") = std::vector<double>{},
      py::arg("isotropic_flux_bottom") = std::vector<double>{},
      "Solve for fluxes at a list of single wavenumbers (all bands in one GPU batch). Returns a list of FluxResult.");

  m.def(
      "solve_flux_spectral_bands",
      [](DisortFluxConfig& config, const std::vector<std::pair<double, double>>& wavenumber_bands,
         std::vector<std::vector<double>> delta_tau, std::vector<std::vector<double>> single_scat_albedo,
         std::vector<std::vector<std::vector<double>>> phase_function_moments, std::vector<double> surface_albedo,
         std::vector<double> emissivity_top, std::vector<double> direct_beam_flux,
         std::vector<double> isotropic_flux_top, std::vector<double> isotropic_flux_bottom) {
        SpectralOverrides ov = make_overrides(std::move(delta_tau), std::move(single_scat_albedo),
                                              std::move(phase_function_moments), std::move(surface_albedo),
                                              std::move(emissivity_top), std::move(direct_beam_flux),
                                              std::move(isotropic_flux_top), std::move(isotropic_flux_bottom));
        py::gil_scoped_release release;
        return solveFluxSpectralBands(config, wavenumber_bands, ov);
      },
      py::arg("config"), py::arg("wavenumber_bands"), py::arg("delta_tau") = std::vector<std::vector<double>>{},
      py::arg("single_scat_albedo") = std::vector<std::vector<double>>{},
      py::arg("phase_function_moments") = std::vector<std::vector<std::vector<double>>>{},
      py::arg("surface_albedo") = std::vector<double>{}, py::arg("emissivity_top") = std::vector<double>{},
      py::arg("direct_beam_flux") = std::vector<double>{}, py::arg("isotropic_flux_top") = std::vector<double>{},
      py::arg("isotropic_flux_bottom") = std::vector<double>{},
      "Solve for fluxes at a list of wavenumber bands (pairs of (low, high)), all bands in one GPU batch. "
      "Returns a list of FluxResult.");

  m.def(
      "solve_flux_spectral_bands_arrays",
      [](DisortFluxConfig& config, py::object wavenumber_bands, py::object delta_tau, py::object single_scat_albedo,
         py::object phase_function_moments, py::object surface_albedo, py::object emissivity_top,
         py::object direct_beam_flux, py::object isotropic_flux_top, py::object isotropic_flux_bottom) {
        auto wb = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(wavenumber_bands);
        if (!wb || wb.ndim() != 2 || wb.shape(1) != 2)
          throw std::invalid_argument("wavenumber_bands must be an array [n_bands, 2]");
        const size_t n = wb.shape(0);
        std::vector<std::pair<double, double>> bands(n);
        for (size_t i = 0; i < n; ++i) bands[i] = {wb.at(i, 0), wb.at(i, 1)};
        SpectralOverrides ov{rows2(delta_tau, n),    rows2(single_scat_albedo, n), rows3(phase_function_moments, n),
                             vec1(surface_albedo),   vec1(emissivity_top),         vec1(direct_beam_flux),
                             vec1(isotropic_flux_top), vec1(isotropic_flux_bottom)};
        const size_t nlev = static_cast<size_t>(config.num_layers) + 1;
        const char* names[8] = {"flux_direct_beam", "flux_down",         "flux_up",           "flux_tau_divergence",
                                "mean_intensity",   "mean_intensity_down", "mean_intensity_up", "mean_intensity_direct_beam"};
        std::vector<py::array_t<double>> arrs;
        double* out8[8];
        for (int f = 0; f < 8; ++f) {
          arrs.emplace_back(std::vector<py::ssize_t>{(py::ssize_t)n, (py::ssize_t)nlev});
          out8[f] = arrs.back().mutable_data();
        }
        {
          py::gil_scoped_release release;
          solveFluxSpectralBandsInto(config, bands, ov, out8);
        }
        py::dict d;
        for (int f = 0; f < 8; ++f) d[names[f]] = arrs[f];
        return d;
      },
      py::arg("config"), py::arg("wavenumber_bands"), py::arg("delta_tau") = py::none(),
      py::arg("single_scat_albedo") = py::none(), py::arg("phase_function_moments") = py::none(),
      py::arg("surface_albedo") = py::none(), py::arg("emissivity_top") = py::none(),
      py::arg("direct_beam_flux") = py::none(), py::arg("isotropic_flux_top") = py::none(),
      py::arg("isotropic_flux_bottom") = py::none(),
      "solve_flux_spectral_bands with numpy arrays in and a dict of numpy arrays [n_bands, num_layers+1] out.");
}
