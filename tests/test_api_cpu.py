"""The DisORT++ Python API surface (no GPU needed): names, defaults, validation
messages and phase-function fillers, as the reference module defines them
(src/python_bindings.cpp:213-763, src/DisortFluxConfig.cpp:43-143)."""
import math

import pytest

import disort_b200 as disortpp


def test_names_and_defaults():
    for n in (4, 6, 8, 10, 12, 14, 16, 32, 64):
        assert hasattr(disortpp, f"DisortFluxSolver{n}")
    c = disortpp.DisortFluxConfig(3, 8)
    assert (c.num_layers, c.num_streams, c.num_phase_func_moments) == (3, 8, 0)
    assert c.direct_beam_mu == 0.5 and c.emissivity_top == 1.0 and c.surface_albedo == 0.0
    assert c.nmom_nstr() == 8
    c.allocate()
    assert isinstance(c.delta_tau, tuple) and len(c.delta_tau) == 3
    assert len(c.phase_function_moments) == 3 and len(c.phase_function_moments[0]) == 9
    with pytest.raises(TypeError):
        c.delta_tau[0] = 1.0  # immutable tuple getter, like the reference
    c.delta_tau = [0.1, 0.2, 0.3]
    assert c.delta_tau == (0.1, 0.2, 0.3)


def test_constructor_and_validate_messages():
    with pytest.raises(ValueError, match="num_layers must be > 0"):
        disortpp.DisortFluxConfig(0, 8)
    with pytest.raises(ValueError, match="num_streams must be even and >= 4"):
        disortpp.DisortFluxConfig(2, 5)
    c = disortpp.DisortFluxConfig(2, 4)
    c.allocate()
    c.delta_tau = [0.1, -1.0]
    with pytest.raises(ValueError, match=r"delta_tau\[1\] must be >= 0"):
        c.validate()
    c.delta_tau = [0.1, 0.2]
    c.single_scat_albedo = [0.5, 1.5]
    with pytest.raises(ValueError, match=r"single_scat_albedo\[1\] must be in \[0, 1\]"):
        c.validate()
    c.single_scat_albedo = [0.5, 0.5]
    c.direct_beam_flux = 1.0
    c.direct_beam_mu = 0.0
    with pytest.raises(ValueError, match="direct_beam_mu must be in"):
        c.validate()
    c.direct_beam_mu = 0.5
    c.use_delta_m_plus = True
    with pytest.raises(ValueError, match="use_delta_m_plus requires"):
        c.validate()
    with pytest.raises(ValueError, match="Unsupported nstr=18"):
        disortpp.create_flux_solver(18)


def test_phase_function_fillers():
    c = disortpp.DisortFluxConfig(2, 4, 6)
    c.allocate()
    c.set_henyey_greenstein(0.5)
    assert c.phase_function_moments[1] == tuple(0.5 ** k for k in range(7))
    c.set_rayleigh(0)
    assert c.phase_function_moments[0] == (1.0, 0.0, 0.1, 0.0, 0.0, 0.0, 0.0)
    c.set_isotropic()
    assert c.phase_function_moments[1] == (1.0,) + (0.0,) * 6
    c.set_haze_garcia_siewert(1)
    assert math.isclose(c.phase_function_moments[1][1], 2.41260 / 3)
    c.set_phase_function(disortpp.PhaseFunction.CloudGarciaSiewert, 0.0, 0)
    assert math.isclose(c.phase_function_moments[0][2], 3.883 / 5)


# ---------------------------------------------------------------------------
# general path (DisortConfig.cpp:10-248, python_bindings.cpp:221-380)
# ---------------------------------------------------------------------------
def test_general_names_and_defaults():
    for name in ("DisortConfig", "DisortFlags", "BoundaryConditions", "DisortResult", "DisortSolver",
                 "solve_spectral", "solve_spectral_bands", "BoundaryConditionType", "BrdfType",
                 "RpvBrdfSpec", "AmbralsBrdfSpec", "CoxMunkBrdfSpec", "HapkeBrdfSpec", "BrdfSpecification"):
        assert hasattr(disortpp, name), name
    f = disortpp.DisortFlags()
    assert f.use_lambertian_surface and not f.use_user_tau and not f.comp_only_fluxes
    assert f.ibcnd == disortpp.BoundaryConditionType.General and f.brdf_type == disortpp.BrdfType.NONE
    bc = disortpp.BoundaryConditions()
    assert (bc.direct_beam_mu, bc.emissivity_top, bc.direct_beam_phi) == (0.5, 1.0, 0.0)
    c = disortpp.DisortConfig(3, 8, 4)
    assert c.nmom_nstr() == 8 and c.accuracy_fourier_series == 0.0
    c.num_user_tau, c.num_user_mu, c.num_phi = 2, 3, 4
    c.allocate()
    assert len(c.delta_tau) == 3 and len(c.phase_function_moments[2]) == 9
    assert (len(c.tau_user), len(c.mu_user), len(c.phi_user)) == (2, 3, 4)
    assert disortpp.HapkeBrdfSpec().hh == 0.06 and disortpp.CoxMunkBrdfSpec().refractive_index == 1.34
    r = disortpp.DisortResult()
    assert (r.num_user_tau(), r.num_user_mu(), r.num_phi()) == (0, 0, 0)


def _general_cfg(nlyr=3, nstr=8):
    c = disortpp.DisortConfig(nlyr, nstr)
    c.flags.comp_only_fluxes = True
    c.allocate()
    c.delta_tau = [0.5] * nlyr
    c.single_scat_albedo = [0.5] * nlyr
    c.set_isotropic()
    return c


def test_general_constructor_and_validate_messages():
    with pytest.raises(ValueError, match="num_layers must be positive"):
        disortpp.DisortConfig(0, 8)
    with pytest.raises(ValueError, match="num_streams must be even and >= 4"):
        disortpp.DisortConfig(2, 6 + 1)
    with pytest.raises(ValueError, match="num_phase_func_moments must be non-negative"):
        disortpp.DisortConfig(2, 8, -1)
    c = _general_cfg()
    c.validate()
    c.delta_tau = [0.5, -1.0, 0.5]
    with pytest.raises(ValueError, match=r"delta_tau\[1\] is negative"):
        c.validate()
    c.delta_tau = [0.5] * 3
    c.flags.comp_only_fluxes = False
    with pytest.raises(ValueError, match="num_phi must be positive when comp_only_fluxes=false"):
        c.validate()
    c.num_phi = 2
    c.phi_user = [0.0, 400.0]
    with pytest.raises(ValueError, match=r"phi_user\[1\] must be in \[0, 360\]"):
        c.validate()
    c.phi_user = [0.0, 90.0]
    c.flags.use_user_mu = True
    c.num_user_mu = 2
    c.mu_user = [0.5, 0.1]
    with pytest.raises(ValueError, match="mu_user must be in increasing order"):
        c.validate()
    c.mu_user = [0.1, 0.5]
    c.accuracy_fourier_series = -1.0
    with pytest.raises(ValueError, match="accuracy_fourier_series must be non-negative"):
        c.validate()
    c.accuracy_fourier_series = 0.0
    c.flags.use_thermal_emission = True
    c.temperature = [250.0] * 4
    c.wavenumber_low = c.wavenumber_high = 500.0
    with pytest.raises(ValueError, match="requires 0 <= wavenumber_low < wavenumber_high"):
        c.validate()


def test_general_index_from_bottom_reports_reference_index():
    """The reference validates after reversing the layer arrays (DisortSolver.cpp:31-37)."""
    c = _general_cfg()
    c.flags.index_from_bottom = True
    c.delta_tau = [-1.0, 0.5, 0.5]
    with pytest.raises(ValueError, match=r"delta_tau\[2\] is negative"):
        disortpp.DisortSolver().solve(c)


def test_general_engine_rejections_before_any_gpu_work():
    solver = disortpp.DisortSolver()
    cases = [
        (lambda c: (setattr(c.flags, "intensity_corr_buras", True), setattr(c, "num_phase_func_angles", 8)),
         "needs num_phase_func_angles >= 2, mu_phase_function and phase_function"),
    ]
    for mutate, msg in cases:
        c = _general_cfg()
        mutate(c)
        with pytest.raises(ValueError, match=msg):
            solver.solve(c)
    # a bidirectional surface without a model, or without its spec, fails like the
    # reference's bidirReflectivity (DisortSolver.cpp:2902-2936)
    c = _general_cfg()
    c.flags.use_lambertian_surface = False
    with pytest.raises(RuntimeError, match="unknown BRDF type"):
        solver.solve(c)
    for kind, msg in ((disortpp.BrdfType.RPV, "rpv spec is null"), (disortpp.BrdfType.CoxMunk, "cox_munk spec"),
                      (disortpp.BrdfType.Ambrals, "ambrals spec")):
        c.flags.brdf_type = kind
        with pytest.raises(RuntimeError, match=msg):
            solver.solve(c)
    c = disortpp.DisortConfig(2, 18)
    c.flags.comp_only_fluxes = True
    c.allocate()
    with pytest.raises(ValueError, match="num_streams=18 is not supported by the B200 engine"):
        solver.solve(c)
    c = _general_cfg()
    c.flags.use_user_tau = True
    with pytest.raises(ValueError, match="use_user_tau=true requires num_user_tau > 0"):
        solver.solve(c)


def test_general_spectral_loop_validation():
    c = _general_cfg()
    c.flags.use_thermal_emission = True
    c.temperature = [250.0] * 4
    # solve_spectral sets wavenumber_low = wavenumber_high, which thermal emission rejects
    with pytest.raises(ValueError, match="requires 0 <= wavenumber_low < wavenumber_high"):
        disortpp.solve_spectral(c, [500.0, 510.0])
    bands = [(500.0, 510.0), (510.0, 520.0)]
    with pytest.raises(ValueError, match=r"single_scat_albedo\[0\] must be in \[0, 1\]"):
        disortpp.solve_spectral_bands(c, bands, single_scat_albedo=[[0.5] * 3, [1.5, 0.5, 0.5]])
    with pytest.raises(ValueError, match="surface_albedo override has 1 entries for 2 bands"):
        disortpp.solve_spectral_bands(c, bands, surface_albedo=[0.1])
