"""The DisORT++ Python API on the GPU, checked against the CPU oracle the way the
reference's own tests build configurations (tests/test_flux_solver.cpp)."""
import numpy as np
import pytest

import disort_b200 as disortpp
import oracle_lib
from disort_b200 import capi, workloads
from parity import assert_parity

pytestmark = pytest.mark.gpu


def _flux_cfg(nlyr=5, nstr=16):
    c = disortpp.DisortFluxConfig(nlyr, nstr)
    c.direct_beam_flux = 1.0
    c.direct_beam_mu = 0.6
    c.surface_albedo = 0.2
    c.use_thermal_emission = True
    c.wavenumber_low, c.wavenumber_high = 500.0, 520.0
    c.temperature_top, c.temperature_bottom = 200.0, 290.0
    c.allocate()
    c.delta_tau = [0.1, 0.5, 1.0, 2.0, 0.3][:nlyr]
    c.single_scat_albedo = [0.9, 0.5, 0.2, 0.95, 0.7][:nlyr]
    c.temperature = [200.0 + 20 * k for k in range(nlyr + 1)]
    c.set_henyey_greenstein(0.75)
    return c


def _as_workload(c, lo, hi):
    pm = np.array(c.phase_function_moments)
    return dict(n_inst=1, num_streams=c.num_streams, num_layers=c.num_layers,
                num_phase_func_moments=c.num_phase_func_moments, pmom_count=pm.shape[1],
                flags=capi.FLAG_THERMAL if c.use_thermal_emission else 0,
                arrays=dict(wavenumber_low=lo, wavenumber_high=hi, delta_tau=np.array(c.delta_tau),
                            single_scat_albedo=np.array(c.single_scat_albedo), phase_function_moments=pm,
                            temperature=np.array(c.temperature), surface_albedo=c.surface_albedo,
                            emissivity_top=c.emissivity_top, direct_beam_flux=c.direct_beam_flux,
                            direct_beam_mu=c.direct_beam_mu, isotropic_flux_top=c.isotropic_flux_top,
                            isotropic_flux_bottom=c.isotropic_flux_bottom, temperature_top=c.temperature_top,
                            temperature_bottom=c.temperature_bottom))


def test_flux_solver_object_matches_oracle():
    c = _flux_cfg()
    r = disortpp.DisortFluxSolver16().solve(c)
    assert r.num_levels() == 6
    ref, st = oracle_lib.flux_solve(_as_workload(c, 500.0, 520.0))
    got = {f: np.array(getattr(r, f))[None, :] for f in capi.FLUX_OUT_FIELDS}
    assert_parity(got, ref, "DisortFluxSolver16")
    with pytest.raises(ValueError, match="does not match template NStr"):
        disortpp.DisortFluxSolver8().solve(c)


def test_spectral_bands_with_overrides_match_oracle():
    c = _flux_cfg()
    rng = np.random.default_rng(3)
    n = 40
    bands = [(300.0 + 5 * i, 305.0 + 5 * i) for i in range(n)]
    dtau = rng.uniform(0.01, 3.0, (n, 5))
    alb = rng.uniform(0, 0.5, n)
    res = disortpp.solve_flux_spectral_bands(c, bands, delta_tau=dtau.tolist(), surface_albedo=alb.tolist())
    arr = disortpp.solve_flux_spectral_bands_arrays(c, np.array(bands), delta_tau=dtau, surface_albedo=alb)
    for i in range(n):
        w = _as_workload(c, *bands[i])
        w["arrays"]["delta_tau"] = dtau[i]
        w["arrays"]["surface_albedo"] = alb[i]
        ref, st = oracle_lib.flux_solve(w)
        got = {f: np.array(getattr(res[i], f))[None, :] for f in capi.FLUX_OUT_FIELDS}
        assert_parity(got, ref, f"band {i}")
        for f in capi.FLUX_OUT_FIELDS:
            np.testing.assert_array_equal(arr[f][i], got[f][0])
    # an invalid override is reported with the reference's message
    bad = dtau.copy()
    bad[7, 2] = -1.0
    with pytest.raises(ValueError, match=r"delta_tau\[2\] must be >= 0"):
        disortpp.solve_flux_spectral_bands(c, bands, delta_tau=bad.tolist())


def test_single_wavenumber_spectral_loop():
    c = _flux_cfg(3, 8)
    res = disortpp.solve_flux_spectral(c, [600.0, 900.0])
    w = _as_workload(c, 900.0, 900.0)
    ref, st = oracle_lib.flux_solve(w)
    assert_parity({f: np.array(getattr(res[1], f))[None, :] for f in capi.FLUX_OUT_FIELDS}, ref, "lo == hi")
