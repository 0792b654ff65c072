"""The CPU oracle against the reference's own known-answer tests.

Every expected value and tolerance comes from DisORT++ tests/test_solver.cpp
(extracted into tests/golden/reference_goldens.json by
tests/golden/make_reference_goldens.py).  Fluxes are compared at the output
levels that coincide with layer boundaries (the flux solver's output grid).
The Delta-M+ regression cases carry 13 significant digits, so the oracle is
additionally held to 1e-9 relative there.
"""
import numpy as np
import pytest

import golden_cases
import oracle_lib
from disort_b200 import capi

CASES = golden_cases.load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_flux_goldens(case):
    w = golden_cases.flux_workload(case)
    out, status = oracle_lib.flux_solve(w)
    assert status[0] == 0
    checked = 0
    for e in case["expect_flux"]:
        lev = golden_cases.level_of(case, e["index"])
        if lev is None:
            continue
        got = out[e["field"]][0, lev]
        assert abs(got - e["value"]) <= e["tol"], (e, got)
        if case["name"].startswith("DeltaMPlus.") and e["value"] != 0.0:
            assert abs(got - e["value"]) <= 1e-9 * abs(e["value"]), (e, got)
        checked += 1
    assert checked > 0


def test_quadrature_and_planck_sanity():
    import ctypes
    lib = oracle_lib.load()
    for n in (4, 16, 64):
        mu = np.zeros(n); w = np.zeros(n); y = np.zeros((n + 1) * n)
        assert lib.oracle_quadrature(n, mu.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     y.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
        assert abs(w[: n // 2].sum() - 1.0) < 1e-13
        assert np.all(mu[: n // 2] > 0) and np.allclose(mu[n // 2:], -mu[: n // 2])
    # Stefan-Boltzmann limit of the band integral over (0, 50000) cm^-1 at 300 K
    sigma = 5.67032e-8
    b = lib.oracle_planck(0.0, 50000.0, 300.0)
    assert abs(b - sigma * 300.0 ** 4 / np.pi) / b < 1e-5
    # single-wavenumber branch and zero-temperature branch
    assert lib.oracle_planck(1000.0, 1000.0, 300.0) > 0
    assert lib.oracle_planck(100.0, 200.0, 0.0) == 0.0


def test_extended_precision_build_reproduces_goldens_and_double_build():
    """The extended-precision build of the oracle (the checker of the deep 32/64
    stream GPU cases) passes the same known-answer tests, and on deep 64-stream
    columns the double build stays within 1e-8 of it (its own rounding reaches
    ~7e-9 of small upward fluxes there)."""
    from disort_b200 import workloads
    from parity import worst
    for case in CASES:
        w = golden_cases.flux_workload(case)
        out, st = oracle_lib.flux_solve(w, ext=True)
        assert st[0] == 0
        for e in case["expect_flux"]:
            lev = golden_cases.level_of(case, e["index"])
            if lev is not None:
                assert abs(out[e["field"]][0, lev] - e["value"]) <= e["tol"]
    rng = np.random.default_rng(254)
    n, N, L = 6, 64, 120
    pc = N + 2
    w = dict(n_inst=n, num_streams=N, num_layers=L, num_phase_func_moments=N + 1, pmom_count=pc,
             flags=capi.FLAG_DELTA_M_PLUS,
             arrays=dict(delta_tau=np.clip(rng.lognormal(-3, 2, (n, L)), 1e-6, 50),
                         single_scat_albedo=rng.uniform(0, 0.99, (n, L)),
                         phase_function_moments=workloads.hg_moments(rng.uniform(0.5, 0.95, (n, L)), pc),
                         surface_albedo=rng.uniform(0, 0.6, n), direct_beam_flux=1.0,
                         direct_beam_mu=rng.uniform(0.1, 1.0, n)))
    a, _ = oracle_lib.flux_solve(w)
    b, _ = oracle_lib.flux_solve(w, ext=True)
    assert worst(a, b)[0] <= 10.0


SPH = golden_cases.load_spherical_cases()


@pytest.mark.parametrize("case", SPH, ids=[c["name"] for c in SPH])
def test_oracle_spherical_goldens(case):
    """The reference's pseudo-spherical known-answer test (C-DISORT values, the
    general solver's fluxes, which the flux solver reproduces): Chapman factors,
    beam transmission and the spherical particular solution."""
    w = golden_cases.flux_workload(case)
    out, status = oracle_lib.flux_solve(w)
    assert status[0] == 0
    for e in case["expect_flux"]:
        got = out[e["field"]][0, golden_cases.level_of(case, e["index"])]
        assert abs(got - e["value"]) <= e["tol"], (e, got)
    # the plane-parallel solve of the same column differs (the Chapman correction)
    w["flags"] &= ~capi.FLAG_SPHERICAL_BEAM
    pp, _ = oracle_lib.flux_solve(w)
    assert pp["flux_direct_beam"][0, 2] < 2.49e-2 < out["flux_direct_beam"][0, 2]


def test_oracle_spherical_tends_to_plane_parallel():
    """A very large radius makes the shells flat: the spherical fluxes approach
    the plane-parallel ones."""
    from disort_b200 import workloads
    from parity import worst
    w = workloads.subset(workloads.beam_sweep(64), np.arange(64))
    L = w["num_layers"]
    w["arrays"]["level_altitudes"] = np.linspace(40.0, 0.0, L + 1)
    pp, _ = oracle_lib.flux_solve(w)
    prev = np.inf
    for radius in (6.371e3, 6.371e5, 6.371e7):  # km: the Earth, then flatter shells
        w["arrays"]["bottom_radius"] = radius
        sp, st = oracle_lib.flux_solve(w, extra_flags=capi.FLAG_SPHERICAL_BEAM)
        assert not st.any()
        gap = worst(sp, pp)[0]
        assert gap < prev / 50.0  # the Chapman correction shrinks like 1 / radius
        prev = gap
    assert prev < 1e4  # within ~1e-5 relative at 6.4e7 km


def test_spherical_double_and_extended_builds_agree():
    """The rounding floor of the pseudo-spherical source at 32 and 64 streams:
    the double build of the oracle within 3e-8 of its extended-precision build
    (the checker of those GPU cases)."""
    from test_flux_gpu import spherical_columns
    for nstr in (32, 64):
        w = spherical_columns(nstr, 12, 12, seed=400 + nstr)
        for extra in (0, capi.FLAG_INDEX_FROM_BOTTOM):
            if extra:
                w["arrays"]["level_altitudes"] = w["arrays"]["level_altitudes"][::-1].copy()
            a, _ = oracle_lib.flux_solve(w, extra_flags=extra)
            b, _ = oracle_lib.flux_solve(w, extra_flags=extra, ext=True)
            for f in capi.FLUX_OUT_FIELDS:
                np.testing.assert_allclose(a[f], b[f], rtol=3e-8, atol=1e-12)
