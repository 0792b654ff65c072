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


# ---------------------------------------------------------------------------
# general path: DisortSolver / solve_spectral_bands against the general oracle
# ---------------------------------------------------------------------------
from parity import assert_parity_general  # noqa: E402


def _general_cfg(nlyr=4, nstr=16, user_tau=True, user_mu=True, only_fluxes=False):
    c = disortpp.DisortConfig(nlyr, nstr, nstr + 4)
    f = c.flags
    f.use_user_tau, f.use_user_mu, f.comp_only_fluxes = user_tau, user_mu, only_fluxes
    f.use_thermal_emission = True
    c.wavenumber_low, c.wavenumber_high = 500.0, 520.0
    c.bc.direct_beam_flux, c.bc.direct_beam_mu, c.bc.direct_beam_phi = 1.0, 0.6, 30.0
    c.bc.surface_albedo, c.bc.isotropic_flux_top = 0.2, 0.05
    c.bc.temperature_top, c.bc.temperature_bottom = 200.0, 290.0
    c.num_user_tau, c.num_user_mu, c.num_phi = 3, 4, 3
    c.allocate()
    c.delta_tau = [0.1, 0.5, 1.0, 2.0][:nlyr]
    c.single_scat_albedo = [0.9, 0.5, 0.2, 0.95][:nlyr]
    c.temperature = [200.0 + 20 * k for k in range(nlyr + 1)]
    c.set_henyey_greenstein(0.75)
    if user_tau:
        c.tau_user = [0.0, 0.35, 3.6]
    if user_mu:
        c.mu_user = [-0.8, -0.2, 0.3, 1.0]
    c.phi_user = [0.0, 45.0, 170.0]
    return c


def _oracle_inst(c, lo, hi, **over):
    inst = dict(num_streams=c.num_streams, num_layers=c.num_layers,
                num_phase_func_moments=c.num_phase_func_moments,
                delta_tau=list(c.delta_tau), single_scat_albedo=list(c.single_scat_albedo),
                phase_function_moments=[list(r) for r in c.phase_function_moments],
                temperature=list(c.temperature), wavenumber_low=lo, wavenumber_high=hi,
                surface_albedo=c.bc.surface_albedo, emissivity_top=c.bc.emissivity_top,
                direct_beam_flux=c.bc.direct_beam_flux, direct_beam_mu=c.bc.direct_beam_mu,
                direct_beam_phi=c.bc.direct_beam_phi, isotropic_flux_top=c.bc.isotropic_flux_top,
                isotropic_flux_bottom=c.bc.isotropic_flux_bottom, temperature_top=c.bc.temperature_top,
                temperature_bottom=c.bc.temperature_bottom)
    f = c.flags
    if f.use_user_tau:
        inst["tau_user"] = list(c.tau_user)[:c.num_user_tau]
    if f.use_user_mu and not f.comp_only_fluxes:
        inst["mu_user"] = list(c.mu_user)[:c.num_user_mu]
    if not f.comp_only_fluxes:
        inst["phi_user"] = list(c.phi_user)[:c.num_phi]
    inst.update(over)
    return inst


def _general_flags(c):
    f = c.flags
    return ((capi.FLAG_THERMAL if f.use_thermal_emission else 0)
            | (capi.FLAG_INDEX_FROM_BOTTOM if f.index_from_bottom else 0)
            | (capi.GFLAG_USER_TAU if f.use_user_tau else 0)
            | (capi.GFLAG_USER_MU if f.use_user_mu and not f.comp_only_fluxes else 0)
            | (capi.GFLAG_ONLY_FLUXES if f.comp_only_fluxes else 0))


def _as_outputs(results, with_intensity):
    got = {f: np.array([getattr(r, f) for r in results]) for f in capi.FLUX_OUT_FIELDS}
    if with_intensity:
        got["intensity"] = np.array([r.intensity for r in results])
        got["intensity_azimuth_avg"] = np.array([r.intensity_azimuth_avg for r in results])
    return got


def _oracle(c, insts, with_intensity):
    ref = oracle_lib.general_solve(capi.pack_general(insts, _general_flags(c), c.accuracy_fourier_series))
    assert (ref["status"] == 0).all()
    if not with_intensity:
        ref = {f: ref[f] for f in capi.FLUX_OUT_FIELDS}
    return ref


@pytest.mark.parametrize("ifb", [False, True])
def test_disort_solver_matches_oracle(ifb):
    c = _general_cfg()
    c.flags.index_from_bottom = ifb
    r = disortpp.DisortSolver().solve(c)
    assert (r.num_user_tau(), r.num_user_mu(), r.num_phi()) == (3, 4, 3)
    assert r.mu_angles == [-0.8, -0.2, 0.3, 1.0]
    ref = _oracle(c, [_oracle_inst(c, 500.0, 520.0)], True)
    assert_parity_general(_as_outputs([r], True), ref, f"DisortSolver ifb={ifb}")
    assert r.intensities(3, 2, 1) == r.intensity[2][3][1]
    assert r.intensities_azimuth_avg(1, 0) == r.intensity_azimuth_avg[0][1]


def test_disort_solver_automatic_dimensions():
    """Without user depths and angles the config is completed like the reference's
    (outputs at the layer boundaries, computational angles, intensity arrays
    allocated at those angles and left zero)."""
    c = _general_cfg(user_tau=False, user_mu=False)
    r = disortpp.DisortSolver().solve(c)
    L, N = c.num_layers, c.num_streams
    assert c.num_user_tau == L + 1 and r.num_user_tau() == L + 1
    np.testing.assert_allclose(c.tau_user, np.concatenate([[0.0], np.cumsum(c.delta_tau)]), rtol=0, atol=0)
    assert c.num_user_mu == N and r.mu_angles == list(c.mu_user)
    mu = np.array(c.mu_user)
    assert np.all(np.diff(mu[:N // 2]) != 0) and np.allclose(mu[:N // 2], -mu[N // 2:][::-1])
    assert all(row[0] == 1.0 for row in c.phase_function_moments)
    assert np.array(r.intensity).shape == (L + 1, N, 3) and not np.array(r.intensity).any()
    ref = _oracle(c, [_oracle_inst(c, 500.0, 520.0)], False)
    assert_parity_general(_as_outputs([r], False), ref, "automatic dimensions")


def test_disort_solver_only_fluxes():
    c = _general_cfg(only_fluxes=True)
    r = disortpp.DisortSolver().solve(c)
    assert r.intensity == [] and r.num_user_mu() == c.num_streams
    ref = _oracle(c, [_oracle_inst(c, 500.0, 520.0)], False)
    assert_parity_general(_as_outputs([r], False), ref, "comp_only_fluxes")


def test_general_spectral_bands_with_overrides_match_oracle():
    c = _general_cfg()
    c.accuracy_fourier_series = 1e-4
    rng = np.random.default_rng(5)
    n = 24
    bands = [(300.0 + 5 * i, 305.0 + 5 * i) for i in range(n)]
    dtau = rng.uniform(0.01, 3.0, (n, 4))
    alb = rng.uniform(0, 0.5, n)
    fbeam = rng.uniform(0.5, 2.0, n)
    res = disortpp.solve_spectral_bands(c, bands, delta_tau=dtau.tolist(), surface_albedo=alb.tolist(),
                                        direct_beam_flux=fbeam.tolist())
    insts = [_oracle_inst(c, *bands[i], delta_tau=list(dtau[i]), surface_albedo=float(alb[i]),
                          direct_beam_flux=float(fbeam[i])) for i in range(n)]
    ref = _oracle(c, insts, True)
    assert_parity_general(_as_outputs(res, True), ref, "solve_spectral_bands")
    # the caller's config is not modified by the spectral loop
    assert c.num_user_tau == 3 and list(c.delta_tau) == [0.1, 0.5, 1.0, 2.0]


def test_flux_solver_temperature_jacobians():
    """compute_temperature_jacobian through the DisORT++ API: FluxResult's six
    *_temperature_jac fields ([L+1][L+2]) equal the oracle's within the
    Jacobian tolerance of test_jacobian_gpu.py; empty without thermal emission,
    as the reference clears them."""
    c = _flux_cfg()
    c.compute_temperature_jacobian = True
    r = disortpp.DisortFluxSolver16().solve(c)
    out, st, jac = oracle_lib.flux_solve_jac(_as_workload(c, 500.0, 520.0))
    assert st[0] == 0
    names = dict(flux_up="flux_up_temperature_jac", flux_down="flux_down_temperature_jac",
                 mean_intensity="mean_intensity_temperature_jac",
                 mean_intensity_down="mean_intensity_down_temperature_jac",
                 mean_intensity_up="mean_intensity_up_temperature_jac",
                 flux_divergence="flux_divergence_temperature_jac")
    for f, attr in names.items():
        got = np.array(getattr(r, attr))
        assert got.shape == (6, 7)
        ref = jac[f][0]
        scale = np.abs(ref).max()
        assert np.all(np.abs(got - ref) <= 3e-8 * np.maximum(np.abs(ref), 1e-3 * scale)), f
    # spectral loop: one Jacobian per band
    res = disortpp.solve_flux_spectral_bands(c, [(500.0, 520.0), (600.0, 610.0)])
    assert len(res[1].flux_up_temperature_jac) == 6 and len(res[1].flux_up_temperature_jac[0]) == 7
    np.testing.assert_array_equal(np.array(res[0].flux_up_temperature_jac), np.array(r.flux_up_temperature_jac))
    c.use_thermal_emission = False
    r = disortpp.DisortFluxSolver16().solve(c)
    assert len(r.flux_up_temperature_jac) == 0


def test_general_solver_temperature_jacobians():
    """DisortSolver with compute_temperature_jacobian (the reference's
    buildThermalConfig, test_jacobian.cpp:19-70): DisortResult's Jacobians
    ([ntau][L+2]) equal the oracle's, and agree with the flux solver's
    (FluxSolverMatchesDisortSolver, 1e-6 relative)."""
    from test_jacobian_oracle import general_thermal
    Tlev = [210.0, 240.0, 265.0, 282.0]
    c = disortpp.DisortConfig(3, 16)
    c.flags.use_thermal_emission = True
    c.flags.use_user_tau = False
    c.flags.use_user_mu = False
    c.flags.comp_only_fluxes = False
    c.flags.compute_temperature_jacobian = True
    c.bc.direct_beam_flux = 0.0
    c.bc.surface_albedo = 0.1
    c.bc.temperature_bottom = 290.0
    c.bc.temperature_top = 0.0
    c.bc.emissivity_top = 1.0
    c.wavenumber_low, c.wavenumber_high = 500.0, 800.0
    c.accuracy_fourier_series = 1e-4
    c.num_phi = 1
    c.allocate()
    c.phi_user = [0.0]
    c.delta_tau = [0.4] * 3
    c.single_scat_albedo = [0.3] * 3
    c.phase_function_moments = [[1.0, 0.09] + [0.0] * 15 for _ in range(3)]
    c.temperature = Tlev
    r = disortpp.DisortSolver().solve(c)
    _, jac = oracle_lib.general_solve_jac(general_thermal(Tlev, 290.0, 16, 0.3))
    got = np.array(r.flux_up_temperature_jac)
    assert got.shape == (4, 5)
    ref = jac["flux_up"][0][:4, :5]
    scale = np.abs(ref).max()
    assert np.all(np.abs(got - ref) <= 3e-8 * np.maximum(np.abs(ref), 1e-3 * scale))


# ---------------------------------------------------------------------------
# pseudo-spherical beam through both solver objects
# ---------------------------------------------------------------------------
def test_flux_solver_spherical_beam():
    """SphericalBeam16 (test_flux_solver.cpp:309-358) through DisortFluxSolver16
    and the spectral-band loop."""
    c = disortpp.DisortFluxConfig(5, 16)
    c.use_spherical_beam = True
    c.direct_beam_flux, c.direct_beam_mu, c.surface_albedo = 1.0, 0.3, 0.1
    c.bottom_radius = 6371.0
    c.allocate()
    c.delta_tau = [0.1] * 5
    c.single_scat_albedo = [0.9] * 5
    c.set_isotropic()
    c.level_altitudes = [100.0, 80.0, 60.0, 40.0, 20.0, 0.0]
    r = disortpp.DisortFluxSolver16().solve(c)
    w = _as_workload(c, 0.0, 0.0)
    w["flags"] |= capi.FLAG_SPHERICAL_BEAM
    w["arrays"].update(level_altitudes=np.array(c.level_altitudes), bottom_radius=6371.0, temperature=None)
    ref, st = oracle_lib.flux_solve(w)
    assert st[0] == 0
    assert_parity({f: np.array(getattr(r, f))[None, :] for f in capi.FLUX_OUT_FIELDS}, ref, "spherical flux")
    res = disortpp.solve_flux_spectral_bands(c, [(500.0, 510.0), (600.0, 610.0)])
    assert_parity({f: np.array(getattr(res[1], f))[None, :] for f in capi.FLUX_OUT_FIELDS}, ref, "spherical bands")
    c.bottom_radius = 0.0
    with pytest.raises(ValueError, match="bottom_radius"):
        disortpp.DisortFluxSolver16().solve(c)


@pytest.mark.parametrize("ifb", [False, True])
def test_disort_solver_spherical_beam(ifb):
    c = _general_cfg()
    c.flags.use_spherical_beam = True
    c.flags.index_from_bottom = ifb
    c.bottom_radius = 6371.0
    z = [8.0, 6.0, 4.0, 2.0, 0.0]
    c.level_altitudes = z[::-1] if ifb else z
    r = disortpp.DisortSolver().solve(c)
    inst = _oracle_inst(c, 500.0, 520.0, level_altitudes=list(c.level_altitudes), bottom_radius=6371.0)
    ref = oracle_lib.general_solve(capi.pack_general([inst], _general_flags(c) | capi.FLAG_SPHERICAL_BEAM))
    assert (ref["status"] == 0).all()
    assert_parity_general(_as_outputs([r], True), ref, f"DisortSolver spherical ifb={ifb}")
