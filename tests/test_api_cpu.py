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
