"""GPU parity of the Nakajima-Tanaka intensity correction (and the BRDF beam
correction) on the general path against the oracle.

The reference's IntensityCorrection* known-answer cases (tests/test_solver.cpp)
and random delta-M columns at every stream count, with user angles in the
aureole of the beam (the IMS term), exactly opposite to it (the dither branch of
the single-scattering sum), deep columns with the absorption cut, bottom-up
indexing, device pointers and the C++/Python solver object.  Tolerances as the
general path: 1e-9 relative + 1e-12 absolute, intensities against the
instance's largest intensity.
"""
import numpy as np
import pytest

import golden_cases
import gpu_lib
import oracle_lib
from disort_b200 import capi, workloads
from parity import assert_parity_general
from test_general_gpu import with_streams

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_corrected_cases(engine_only=True)


def both(insts, flags):
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_solve(d)
    got, rc = gpu_lib.general_solve(d)
    assert rc == 0, gpu_lib.context().last_error()
    return got, ref, d


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_intcor_reference_goldens(case):
    inst, flags = golden_cases.general_instance(case)
    got, ref, _ = both([inst], flags)
    assert got["status"][0] == ref["status"][0] == 0
    if max(case["single_scat_albedo"]) >= 1.0:
        assert_parity_general(got, ref, case["name"], rtol=1e-8, atol=2e-9)
    else:
        assert_parity_general(got, ref, case["name"])
    for e in case["expect_intensity"]:
        assert abs(got["intensity"][0, e["lu"], e["iu"], e["j"]] - e["value"]) <= e["tol"]


def corr_mix(n, seed, nstr, layers=(3, 12), extra_moments=8):
    """Delta-M (not delta-M+) beam columns with user angles around the
    anti-solar direction -mu0 (aureole) and exactly at it."""
    insts, _ = workloads.general_mix(n, seed=seed, nstr=(4,), layers=layers)
    insts = with_streams(insts, nstr)
    rng = np.random.default_rng(seed)
    for c in insts:
        N = c["num_streams"]
        g = c["phase_function_moments"][:, 1]
        mu0 = float(rng.uniform(0.15, 0.9))
        c.update(num_phase_func_moments=N + extra_moments,
                 phase_function_moments=workloads.hg_moments(g, N + extra_moments + 1),
                 direct_beam_mu=mu0, direct_beam_phi=float(rng.uniform(0.0, 40.0)),
                 mu_user=[-1.0, -mu0 - 0.04, -mu0, -mu0 + 0.05, 0.3, 0.8])
    flags = capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU | capi.GFLAG_INTENSITY_CORR
    return insts, flags


@pytest.mark.parametrize("nstr", [(4, 8), (16,), (6, 10, 12, 14), (32,), (64,)])
def test_intcor_mix(nstr):
    n = 3 if nstr == (64,) else 10
    insts, flags = corr_mix(n, seed=60 + len(nstr) + nstr[0], nstr=nstr, layers=(3, 6) if nstr == (64,) else (3, 12))
    got, ref, _ = both(insts, flags)
    assert (got["status"] == 0).all()
    assert_parity_general(got, ref, f"intensity correction N {nstr}")
    # the correction moves the intensities and leaves fluxes and averages alone
    plain, _, _ = both(insts, flags & ~capi.GFLAG_INTENSITY_CORR)
    np.testing.assert_array_equal(plain["flux_up"], got["flux_up"])
    np.testing.assert_array_equal(plain["intensity_azimuth_avg"], got["intensity_azimuth_avg"])
    assert np.abs(plain["intensity"] - got["intensity"]).max() > 0.0


def test_intcor_lyrcut_bottom_up_and_device_pointers():
    insts, flags = corr_mix(6, seed=5, nstr=(8, 16), layers=(25, 35))
    for c in insts:  # deep absorbing columns: the absorption cut drops the lower layers
        c["delta_tau"] = np.full(c["num_layers"], 1.5)
        c["single_scat_albedo"] = np.full(c["num_layers"], 0.3)
    got, ref, _ = both(insts, flags)
    assert_parity_general(got, ref, "lyrcut")
    insts, flags = corr_mix(6, seed=6, nstr=(8, 16))
    got, ref, _ = both(insts, flags | capi.FLAG_INDEX_FROM_BOTTOM)
    assert_parity_general(got, ref, "index_from_bottom")
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_solve(d)
    got, rc = gpu_lib.general_solve_device(d)
    assert rc == 0
    assert_parity_general(got, ref, "device pointers")


def test_intcor_with_brdf_surface():
    """Both corrections at once: Nakajima-Tanaka over an RPV surface plus the
    reflected-beam correction; under delta-M+ only the BRDF one is skipped."""
    insts, flags = corr_mix(8, seed=9, nstr=(8, 16))
    for c in insts:
        c.update(brdf_type=capi.BRDF_RPV, brdf_params=[0.15, 0.8, -0.1, 0.0, 0.0, 0.0, 1.0])
    got, ref, _ = both(insts, flags)
    assert_parity_general(got, ref, "NT + BRDF")
    got, ref, _ = both(insts, flags | capi.FLAG_DELTA_M_PLUS)
    assert_parity_general(got, ref, "delta-M+ with BRDF")


def test_intcor_through_solver_object():
    """DisortSolver with intensity_corr_buras and intensity_corr_nakajima equals the
    C ABI call; the Buras-Emde selection is refused."""
    import disort_b200 as db
    cfg = db.DisortConfig(2, 8, 12)
    f = cfg.flags
    f.use_user_tau, f.use_user_mu = True, True
    f.intensity_corr_buras, f.intensity_corr_nakajima = True, True
    cfg.num_user_tau, cfg.num_user_mu, cfg.num_phi = 2, 3, 2
    cfg.allocate()
    cfg.delta_tau = [0.4, 1.1]
    cfg.single_scat_albedo = [0.9, 0.7]
    cfg.set_henyey_greenstein(0.8)
    cfg.tau_user = [0.0, 1.5]
    cfg.mu_user = [-0.5, -0.2, 0.6]
    cfg.phi_user = [0.0, 30.0]
    cfg.bc.direct_beam_flux, cfg.bc.direct_beam_mu = 1.0, 0.5
    r = db.DisortSolver().solve(cfg)
    inst = dict(num_streams=8, num_layers=2, num_phase_func_moments=12, delta_tau=[0.4, 1.1],
                single_scat_albedo=[0.9, 0.7], phase_function_moments=workloads.hg_moments(np.array([0.8, 0.8]), 13),
                direct_beam_flux=1.0, direct_beam_mu=0.5, tau_user=[0.0, 1.5], mu_user=[-0.5, -0.2, 0.6],
                phi_user=[0.0, 30.0])
    got, ref, _ = both([inst], capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU | capi.GFLAG_INTENSITY_CORR)
    np.testing.assert_allclose(np.asarray(r.intensity), got["intensity"][0], rtol=1e-12, atol=1e-15)
    f.intensity_corr_nakajima = False
    cfg.num_phase_func_angles = 8
    with pytest.raises(ValueError, match="needs num_phase_func_angles >= 2"):
        db.DisortSolver().solve(cfg)


def tabulate(insts, na=121):
    """Each layer's HG phase function tabulated on na uniform cosines (the
    Buras-Emde method's input)."""
    mu = np.linspace(-1.0, 1.0, na)
    for c in insts:
        g = np.asarray(c["phase_function_moments"])[:, 1]
        d = 1.0 + g[:, None] ** 2 - 2.0 * g[:, None] * mu[None, :]
        c["mu_phase_function"] = mu
        c["phase_function"] = (1.0 - g[:, None] ** 2) / (d * np.sqrt(d))
    return insts


@pytest.mark.parametrize("nstr", [(4, 8), (16,), (32,), (64,)])
def test_buras_emde_mix(nstr):
    n = 3 if nstr == (64,) else 8
    insts, flags = corr_mix(n, seed=80 + nstr[0], nstr=nstr, layers=(3, 6) if nstr == (64,) else (3, 12))
    insts = tabulate(insts)
    flags |= capi.GFLAG_INTENSITY_CORR_BE
    got, ref, _ = both(insts, flags)
    assert (got["status"] == 0).all() and (ref["status"] == 0).all()
    assert_parity_general(got, ref, f"Buras-Emde N {nstr}")
    nt, _, _ = both(insts, flags & ~capi.GFLAG_INTENSITY_CORR_BE)
    assert np.abs(nt["intensity"] - got["intensity"]).max() > 0.0  # a different method


def test_buras_emde_levels_bottom_up_and_device_pointers():
    """Output at the layer boundaries (a different number of depths per
    instance), bottom-up indexing and device pointers."""
    insts, flags = corr_mix(6, seed=88, nstr=(8, 16))
    insts = tabulate(insts, na=64)
    flags |= capi.GFLAG_INTENSITY_CORR_BE
    lv = [dict(c) for c in insts]
    for c in lv:
        c.pop("tau_user")
    got, ref, _ = both(lv, flags & ~capi.GFLAG_USER_TAU)
    assert_parity_general(got, ref, "Buras-Emde at the levels")
    got, ref, _ = both(insts, flags | capi.FLAG_INDEX_FROM_BOTTOM)
    assert_parity_general(got, ref, "Buras-Emde bottom-up")
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_solve(d)
    got, rc = gpu_lib.general_solve_device(d)
    assert rc == 0
    assert_parity_general(got, ref, "Buras-Emde device pointers")


def test_buras_emde_through_solver_object():
    import disort_b200 as db
    cfg = db.DisortConfig(2, 8, 12)
    f = cfg.flags
    f.use_user_tau, f.use_user_mu = True, True
    f.intensity_corr_buras, f.intensity_corr_nakajima = True, False
    cfg.num_user_tau, cfg.num_user_mu, cfg.num_phi = 2, 3, 2
    cfg.num_phase_func_angles = 41
    cfg.allocate()
    cfg.delta_tau = [0.4, 1.1]
    cfg.single_scat_albedo = [0.9, 0.7]
    cfg.set_henyey_greenstein(0.8)
    mu = np.linspace(-1.0, 1.0, 41)
    d = 1.0 + 0.64 - 1.6 * mu
    tab = (1.0 - 0.64) / (d * np.sqrt(d))
    cfg.mu_phase_function = list(mu)
    cfg.phase_function = [list(tab), list(tab)]
    cfg.tau_user = [0.0, 1.5]
    cfg.mu_user = [-0.5, -0.2, 0.6]
    cfg.phi_user = [0.0, 30.0]
    cfg.bc.direct_beam_flux, cfg.bc.direct_beam_mu = 1.0, 0.5
    r = db.DisortSolver().solve(cfg)
    inst = dict(num_streams=8, num_layers=2, num_phase_func_moments=12, delta_tau=[0.4, 1.1],
                single_scat_albedo=[0.9, 0.7], phase_function_moments=workloads.hg_moments(np.array([0.8, 0.8]), 13),
                direct_beam_flux=1.0, direct_beam_mu=0.5, tau_user=[0.0, 1.5], mu_user=[-0.5, -0.2, 0.6],
                phi_user=[0.0, 30.0], mu_phase_function=mu, phase_function=np.stack([tab, tab]))
    fl = capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU | capi.GFLAG_INTENSITY_CORR | capi.GFLAG_INTENSITY_CORR_BE
    got, ref, _ = both([inst], fl)
    np.testing.assert_allclose(np.asarray(r.intensity), got["intensity"][0], rtol=1e-12, atol=1e-15)


def test_deep_columns_brdf_and_correction_against_extended_oracle():
    """32 and 64 streams, 60-100 layers, an RPV surface and the Nakajima-Tanaka
    correction over every azimuth mode: against the extended-precision oracle,
    each element allowed 1e-9 (intensities: of the instance's largest) times
    max(1, twice the instance's FP64 spread: how far the double oracle on the
    given inputs and on one-ulp-perturbed copies strays from the extended one,
    in those units), the bench's parity of record."""
    import bench
    insts, flags = corr_mix(2, seed=77, nstr=(32, 64), layers=(60, 100))
    for c in insts:
        c.update(brdf_type=capi.BRDF_RPV, brdf_params=[0.12, 0.85, -0.15, 0.0, 0.0, 0.0, 1.0])
    d = capi.pack_general(insts, flags)
    got, rc = gpu_lib.general_solve(d)
    assert rc == 0 and (got["status"] == 0).all()
    ext = oracle_lib.general_solve(d, ext=True)
    floor = [oracle_lib.general_solve(d)]
    for k in range(bench.ULP_COPIES):
        rng = np.random.default_rng(1000 + k)
        floor.append(oracle_lib.general_solve(capi.pack_general([bench.ulp_perturbed(c, rng) for c in insts], flags)))
    assert all((np.asarray(f["status"]) == 0).all() for f in floor)
    r = bench.general_parity(got, np.arange(len(insts)), ext, floor_ref=floor)
    assert r["passes"], r
