"""Temperature Jacobians of the flux oracle, checked as the reference checks its own.

The reference validates computeThermalJacobian (FluxSolver.cpp:1294-1497)
against central finite differences of the forward solve, over every temperature
degree of freedom (the L+1 level temperatures and the surface) and every output
level (tests/test_jacobian.cpp:73-181, 206-251, 361-378), with the tolerances
of those tests; the index_from_bottom layout check follows
test_jacobian.cpp:316-352.
The same FD check runs here on the oracle's analytic Jacobian, which is then
the checker of the GPU's.
"""
import numpy as np
import pytest

import oracle_lib
from disort_b200 import capi


def thermal_column(Tlev, Tsurf, nstr, ssa, beam=0.0, flags=0, n=1):
    """The reference's test problem (test_jacobian.cpp:19-70, 120-144): layers of
    optical depth 0.4, moment 1 = 0.3 ssa, band 500-800 cm^-1, albedo 0.1."""
    L = len(Tlev) - 1
    pc = nstr + 1
    pm = np.zeros((L, pc))
    pm[:, 0] = 1.0
    pm[:, 1] = 0.3 * ssa
    return dict(n_inst=n, num_streams=nstr, num_layers=L, num_phase_func_moments=0, pmom_count=pc,
                flags=capi.FLAG_THERMAL | flags,
                arrays=dict(wavenumber_low=500.0, wavenumber_high=800.0, delta_tau=np.full(L, 0.4),
                            single_scat_albedo=np.full(L, ssa), phase_function_moments=pm,
                            temperature=np.array(Tlev, dtype=np.float64), surface_albedo=0.1,
                            emissivity_top=1.0, direct_beam_flux=beam, direct_beam_mu=0.5,
                            temperature_top=0.0, temperature_bottom=Tsurf))


def fd_check(Tlev, Tsurf, nstr, ssa, beam, rtol, atol=1e-9, flags=0):
    L = len(Tlev) - 1
    out, st, jac = oracle_lib.flux_solve_jac(thermal_column(Tlev, Tsurf, nstr, ssa, beam, flags))
    assert st[0] == 0
    for dof in range(L + 2):
        T0 = Tlev[dof] if dof <= L else Tsurf
        h = 1e-3 * max(abs(T0), 1.0)
        Tp, Tm = list(Tlev), list(Tlev)
        Tsp = Tsm = Tsurf
        if dof <= L:
            Tp[dof] += h
            Tm[dof] -= h
        else:
            Tsp += h
            Tsm -= h
        op, _ = oracle_lib.flux_solve(thermal_column(Tp, Tsp, nstr, ssa, beam, flags))
        om, _ = oracle_lib.flux_solve(thermal_column(Tm, Tsm, nstr, ssa, beam, flags))
        for jf, of in capi.JAC_OF.items():
            fd = (op[of][0] - om[of][0]) / (2.0 * h)
            ana = jac[jf][0, :, dof]
            tol = rtol * np.maximum(np.abs(fd), np.abs(ana)) + atol
            assert np.all(np.abs(ana - fd) <= tol), (jf, dof, ana, fd)


def test_planck_derivative_vs_fd():
    """test_jacobian.cpp:186-199: dB/dT against a central difference of B
    (plus a single-wavenumber band)."""
    lib = oracle_lib.load()
    for lo, hi in ((500.0, 800.0), (100.0, 110.0), (1.0, 3000.0), (2000.0, 2001.0), (900.0, 900.0)):
        for T in (50.0, 150.0, 300.0, 1200.0):
            h = 1e-4 * T
            fd = (lib.oracle_planck(lo, hi, T + h) - lib.oracle_planck(lo, hi, T - h)) / (2 * h)
            ana = jac_planck_deriv(lib, lo, hi, T)
            assert abs(ana - fd) <= 1e-5 * max(abs(fd), abs(ana)) + 1e-12, (lo, hi, T, ana, fd)


def jac_planck_deriv(lib, lo, hi, T):
    import ctypes
    lib.oracle_planck_deriv.restype = ctypes.c_double
    lib.oracle_planck_deriv.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
    return lib.oracle_planck_deriv(lo, hi, T)


@pytest.mark.parametrize("name,Tlev,Tsurf,nstr,ssa,beam,rtol", [
    ("flux_single_layer", [200.0, 260.0], 280.0, 8, 0.0, 0.0, 1e-3),             # :361-364
    ("flux_multilayer_scattering", [205.0 + 9.0 * i for i in range(9)], 290.0, 16, 0.7, 0.0, 2e-3),  # :366-371
    ("flux_thermal_plus_beam", [210.0, 245.0, 275.0], 288.0, 16, 0.5, 1.0, 1.5e-3),  # :373-377
    ("single_layer", [200.0, 260.0], 280.0, 8, 0.0, 0.0, 1e-3),                  # :206-210
    ("multilayer_profile", [200.0 + 8.0 * i for i in range(11)], 285.0, 16, 0.0, 0.0, 1e-3),  # :216-222
    ("scattering_half", [210.0, 235.0, 255.0, 270.0, 280.0], 290.0, 16, 0.5, 0.0, 1.5e-3),  # :228-232
    ("scattering_high", [210.0, 235.0, 255.0, 270.0, 280.0], 290.0, 16, 0.9, 0.0, 2e-3),  # :234-238
    ("thermal_plus_beam", [200.0, 240.0, 270.0], 288.0, 16, 0.6, 1.0, 1.5e-3),  # :244-248
    ("four_streams", [220.0, 240.0, 260.0, 275.0], 285.0, 4, 0.4, 0.0, 2e-3),
])
def test_flux_jacobian_vs_finite_differences(name, Tlev, Tsurf, nstr, ssa, beam, rtol):
    fd_check(Tlev, Tsurf, nstr, ssa, beam, rtol)


def test_flux_jacobian_diffusion_lower_bc_vs_finite_differences():
    fd_check([200.0, 240.0, 270.0, 280.0], 288.0, 16, 0.6, 0.0, 2e-3, flags=capi.FLAG_DIFFUSION_LOWER_BC)


def test_index_from_bottom_reverses_rows_and_level_columns():
    """test_jacobian.cpp:316-352: rows reversed, level columns reversed, the
    surface column kept last, 1e-9 relative."""
    Tlev = [210.0, 240.0, 265.0, 285.0]
    L = len(Tlev) - 1
    _, _, j0 = oracle_lib.flux_solve_jac(thermal_column(Tlev, 295.0, 16, 0.3))
    _, _, j1 = oracle_lib.flux_solve_jac(thermal_column(Tlev[::-1], 295.0, 16, 0.3,
                                                        flags=capi.FLAG_INDEX_FROM_BOTTOM))
    for f in capi.JAC_FIELDS:
        a = j1[f][0]
        b = j0[f][0][::-1]
        b = np.concatenate([b[:, L::-1], b[:, L + 1:]], axis=1)
        assert np.all(np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), np.abs(b)) + 1e-12), f


def test_no_thermal_gives_zero_jacobian():
    w = thermal_column([220.0, 250.0, 275.0], 285.0, 8, 0.0)
    w["flags"] = 0
    w["arrays"]["direct_beam_flux"] = 1.0
    out, st, jac = oracle_lib.flux_solve_jac(w)
    assert st[0] == 0
    for f in capi.JAC_FIELDS:
        assert np.all(jac[f] == 0.0)


def test_double_and_extended_oracle_jacobians_agree():
    """The double build of the oracle against its extended-precision build (the
    GPU Jacobians' checker): within 3e-8 of max(|entry|, 1e-3 of the output's
    largest entry in the instance) on thermal-sweep columns -- double rounding
    alone moves single entries by up to ~1.4e-8 there."""
    from disort_b200 import workloads
    w = workloads.subset(workloads.thermal_sweep(), np.arange(0, 20000, 800))
    for extra in (0, capi.FLAG_DIFFUSION_LOWER_BC):
        _, _, a = oracle_lib.flux_solve_jac(w, extra_flags=extra)
        _, _, b = oracle_lib.flux_solve_jac(w, extra_flags=extra, ext=True)
        for f in capi.JAC_FIELDS:
            scale = np.abs(b[f]).reshape(b[f].shape[0], -1).max(axis=1)[:, None, None]
            assert np.all(np.abs(a[f] - b[f]) <= 3e-8 * np.maximum(np.abs(b[f]), 1e-3 * scale)), f


# ---------------------------------------------------------------------------
# DisortSolver (general path): test_jacobian.cpp:19-115, 206-249, 284-409
# ---------------------------------------------------------------------------
def general_thermal(Tlev, Tsurf, nstr, ssa, beam=0.0, flags=0):
    """buildThermalConfig (test_jacobian.cpp:19-70): outputs at the layer
    boundaries, intensities at the quadrature angles, one azimuth, accuracy 1e-4."""
    L = len(Tlev) - 1
    pm = np.zeros((L, nstr + 1))
    pm[:, 0] = 1.0
    pm[:, 1] = 0.3 * ssa
    inst = dict(num_streams=nstr, num_layers=L, num_phase_func_moments=0, delta_tau=np.full(L, 0.4),
                single_scat_albedo=np.full(L, ssa), phase_function_moments=pm,
                temperature=np.array(Tlev, dtype=np.float64), wavenumber_low=500.0, wavenumber_high=800.0,
                surface_albedo=0.1, emissivity_top=1.0, direct_beam_flux=beam, direct_beam_mu=0.5,
                direct_beam_phi=0.0, temperature_top=0.0, temperature_bottom=Tsurf, phi_user=[0.0])
    return capi.pack_general([inst], capi.FLAG_THERMAL | flags, accuracy_fourier_series=1e-4)


def general_fd_check(Tlev, Tsurf, nstr, ssa, beam, rtol, atol=1e-9):
    L = len(Tlev) - 1
    out, jac = oracle_lib.general_solve_jac(general_thermal(Tlev, Tsurf, nstr, ssa, beam))
    assert out["status"][0] == 0
    for dof in range(L + 2):
        T0 = Tlev[dof] if dof <= L else Tsurf
        h = 1e-3 * max(abs(T0), 1.0)
        Tp, Tm = list(Tlev), list(Tlev)
        Tsp = Tsm = Tsurf
        if dof <= L:
            Tp[dof] += h
            Tm[dof] -= h
        else:
            Tsp += h
            Tsm -= h
        op = oracle_lib.general_solve(general_thermal(Tp, Tsp, nstr, ssa, beam))
        om = oracle_lib.general_solve(general_thermal(Tm, Tsm, nstr, ssa, beam))
        for jf, of in capi.JAC_OF.items():
            fd = (op[of][0] - om[of][0]) / (2.0 * h)
            ana = jac[jf][0, :, dof]
            assert np.all(np.abs(ana - fd) <= rtol * np.maximum(np.abs(fd), np.abs(ana)) + atol), (jf, dof)


@pytest.mark.parametrize("name,Tlev,Tsurf,nstr,ssa,beam,rtol", [
    ("single_layer", [200.0, 260.0], 280.0, 8, 0.0, 0.0, 1e-3),                   # :206-210
    ("multilayer_profile", [200.0 + 8.0 * i for i in range(11)], 285.0, 16, 0.0, 0.0, 1e-3),  # :216-222
    ("scattering_half", [210.0, 235.0, 255.0, 270.0, 280.0], 290.0, 16, 0.5, 0.0, 1.5e-3),  # :228-232
    ("scattering_high", [210.0, 235.0, 255.0, 270.0, 280.0], 290.0, 16, 0.9, 0.0, 2e-3),  # :234-238
    ("thermal_plus_beam", [200.0, 240.0, 270.0], 288.0, 16, 0.6, 1.0, 1.5e-3),  # :244-248
])
def test_general_jacobian_vs_finite_differences(name, Tlev, Tsurf, nstr, ssa, beam, rtol):
    general_fd_check(Tlev, Tsurf, nstr, ssa, beam, rtol)


def test_general_and_flux_jacobians_agree():
    """FluxSolverMatchesDisortSolver (test_jacobian.cpp:381-409): 1e-6 relative, 1e-9 absolute."""
    Tlev = [210.0, 240.0, 265.0, 282.0]
    _, jg = oracle_lib.general_solve_jac(general_thermal(Tlev, 290.0, 16, 0.0))
    _, _, jf = oracle_lib.flux_solve_jac(thermal_column(Tlev, 290.0, 16, 0.0))
    for f in ("flux_up", "flux_down", "flux_divergence"):
        a, b = jg[f][0], jf[f][0]
        assert np.all(np.abs(a - b) <= 1e-6 * np.maximum(np.abs(a), np.abs(b)) + 1e-9), f


def test_general_jacobian_index_from_bottom_and_user_taus():
    """IndexFromBottomReversal (test_jacobian.cpp:316-352) on the general solver,
    and Jacobians at user optical depths inside layers (the rows follow the
    user depths, scaled like the fluxes)."""
    Tlev = [210.0, 240.0, 265.0, 285.0]
    L = 3
    _, j0 = oracle_lib.general_solve_jac(general_thermal(Tlev, 295.0, 16, 0.3))
    _, j1 = oracle_lib.general_solve_jac(general_thermal(Tlev[::-1], 295.0, 16, 0.3,
                                                         flags=capi.FLAG_INDEX_FROM_BOTTOM))
    for f in capi.JAC_FIELDS:
        a = j1[f][0]
        b = j0[f][0][::-1]
        b = np.concatenate([b[:, L::-1], b[:, L + 1:]], axis=1)
        assert np.all(np.abs(a - b) <= 1e-9 * np.maximum(np.abs(a), np.abs(b)) + 1e-12), f
    # user taus at the layer boundaries reproduce the level rows
    taus = np.concatenate([[0.0], np.cumsum([0.4] * L)])
    d2 = capi.pack_general([dict(num_streams=16, num_layers=L, num_phase_func_moments=0,
                                 delta_tau=np.full(L, 0.4), single_scat_albedo=np.full(L, 0.3),
                                 phase_function_moments=np.c_[np.ones(L), np.full(L, 0.09), np.zeros((L, 15))],
                                 temperature=np.array(Tlev), wavenumber_low=500.0, wavenumber_high=800.0,
                                 surface_albedo=0.1, temperature_bottom=295.0, phi_user=[0.0],
                                 tau_user=taus)], capi.FLAG_THERMAL | capi.GFLAG_USER_TAU,
                           accuracy_fourier_series=1e-4)
    _, ju = oracle_lib.general_solve_jac(d2)
    for f in capi.JAC_FIELDS:
        np.testing.assert_allclose(ju[f][0], j0[f][0], rtol=1e-12, atol=1e-18)
