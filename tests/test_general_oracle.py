"""The general-solver oracle (oracle/general_oracle.hpp) pinned on the CPU.

1. Every flux and intensity expectation of the reference's known-answer tests
   (tests/golden/reference_goldens.json, from tests/test_solver.cpp).
2. The reference's own cross-solver check (test_flux_solver.cpp:104-539): the
   general solver's mode-0 fluxes equal the flux solver's to 1e-12 relative.
3. index_from_bottom, and the validation rules of DisortConfig::validate.
"""
from __future__ import annotations

import numpy as np
import pytest

import golden_cases as gc
import oracle_lib
from disort_b200 import capi

CASES = gc.load_cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_general_oracle_goldens(case):
    inst, flags = gc.general_instance(case)
    o = oracle_lib.general_solve(capi.pack_general([inst], flags))
    assert o["status"][0] == 0
    for e in case["expect_flux"]:
        v = o[e["field"]][0, e["index"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)
    for e in case["expect_intensity"]:
        v = o["intensity"][0, e["lu"], e["iu"], e["j"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)


def random_instance(rng, N, L, thermal, beam, dmplus=False, ssa_max=0.99):
    g = rng.uniform(0.0, 0.9, L)
    nmom = N + 1 if dmplus else 0
    nm = max(nmom, N)
    pm = g[:, None] ** np.arange(nm + 1)[None, :]
    inst = dict(num_streams=N, num_layers=L, num_phase_func_moments=nmom,
                delta_tau=np.clip(rng.lognormal(-1.0, 1.5, L), 1e-6, 50.0),
                single_scat_albedo=rng.uniform(0.0, ssa_max, L), phase_function_moments=pm,
                surface_albedo=float(rng.uniform(0, 0.6)))
    if thermal:
        inst.update(temperature=180.0 + 140.0 * np.arange(L + 1) / L + rng.uniform(-10, 10, L + 1),
                    wavenumber_low=500.0, wavenumber_high=520.0, temperature_bottom=300.0,
                    temperature_top=50.0, emissivity_top=0.9)
    if beam:
        inst.update(direct_beam_flux=1.7, direct_beam_mu=float(rng.uniform(0.1, 1.0)),
                    isotropic_flux_top=0.3)
    return inst


def flux_oracle_of(inst, flags):
    pm = np.asarray(inst["phase_function_moments"])
    arrays = dict(delta_tau=np.asarray(inst["delta_tau"]), single_scat_albedo=np.asarray(inst["single_scat_albedo"]),
                  phase_function_moments=pm, temperature=inst.get("temperature"))
    for f in ("wavenumber_low", "wavenumber_high", "surface_albedo", "emissivity_top", "direct_beam_flux",
              "direct_beam_mu", "isotropic_flux_top", "isotropic_flux_bottom", "temperature_top",
              "temperature_bottom"):
        arrays[f] = float(inst.get(f, capi.GENERAL_SCALAR_DEFAULTS[f]))
    w = dict(n_inst=1, num_streams=inst["num_streams"], num_layers=inst["num_layers"],
             num_phase_func_moments=inst["num_phase_func_moments"], pmom_count=pm.shape[1],
             flags=flags & 0xFF, arrays=arrays)
    return oracle_lib.flux_solve(w)


@pytest.mark.parametrize("N", [4, 8, 16, 32])
@pytest.mark.parametrize("kind", ["thermal", "beam", "both", "dmplus", "dlbc", "ifb"])
def test_general_matches_flux_oracle(N, kind):
    rng = np.random.default_rng(100 + N)
    thermal = kind in ("thermal", "both", "dlbc", "ifb")
    beam = kind in ("beam", "both", "dmplus", "ifb")
    flags = (capi.FLAG_THERMAL if thermal else 0) | capi.GFLAG_ONLY_FLUXES
    if kind == "dmplus":
        flags |= capi.FLAG_DELTA_M_PLUS
    if kind == "dlbc":
        flags |= capi.FLAG_DIFFUSION_LOWER_BC
    if kind == "ifb":
        flags |= capi.FLAG_INDEX_FROM_BOTTOM
    L = 7
    for _ in range(3):
        inst = random_instance(rng, N, L, thermal, beam, dmplus=kind == "dmplus")
        og = oracle_lib.general_solve(capi.pack_general([inst], flags))
        of, st = flux_oracle_of(inst, flags)
        assert og["status"][0] == 0 and st[0] == 0
        for f in capi.FLUX_OUT_FIELDS:
            a, b = og[f][0, :L + 1], of[f][0]
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()), err_msg=f)


def test_general_lyrcut_matches_flux_oracle():
    """Deep absorbing beam-only column: the absorption cut drops the lower layers."""
    rng = np.random.default_rng(7)
    inst = random_instance(rng, 8, 6, thermal=False, beam=True, ssa_max=0.2)
    inst["delta_tau"] = np.array([2.0, 5.0, 8.0, 10.0, 3.0, 1.0])
    og = oracle_lib.general_solve(capi.pack_general([inst], capi.GFLAG_ONLY_FLUXES))
    of, st = flux_oracle_of(inst, 0)
    for f in capi.FLUX_OUT_FIELDS:
        np.testing.assert_allclose(og[f][0], of[f][0], rtol=1e-12, atol=1e-14, err_msg=f)
    assert og["flux_up"][0, -1] == 0.0  # below the cut


def test_general_index_from_bottom_reverses():
    rng = np.random.default_rng(11)
    inst = random_instance(rng, 8, 5, thermal=True, beam=True)
    inst.update(tau_user=[0.0, 0.05, 1.0], mu_user=[-0.7, -0.2, 0.3, 1.0], phi_user=[0.0, 45.0, 170.0])
    flags = capi.FLAG_THERMAL | capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU
    top = oracle_lib.general_solve(capi.pack_general([inst], flags))
    tot = float(np.sum(inst["delta_tau"]))
    rev = dict(inst)
    rev.update(delta_tau=inst["delta_tau"][::-1].copy(), single_scat_albedo=inst["single_scat_albedo"][::-1].copy(),
               phase_function_moments=inst["phase_function_moments"][::-1].copy(),
               temperature=inst["temperature"][::-1].copy(), tau_user=[tot - t for t in inst["tau_user"][::-1]])
    bot = oracle_lib.general_solve(capi.pack_general([rev], flags | capi.FLAG_INDEX_FROM_BOTTOM))
    for f in capi.FLUX_OUT_FIELDS + ("intensity", "intensity_azimuth_avg"):
        np.testing.assert_allclose(bot[f][0][::-1], top[f][0], rtol=1e-12, atol=1e-15, err_msg=f)


def test_general_azimuth_modes_matter():
    """With an oblique beam and azimuth-dependent output the m > 0 modes contribute."""
    rng = np.random.default_rng(5)
    inst = random_instance(rng, 16, 3, thermal=False, beam=True)
    inst.update(direct_beam_mu=0.6, tau_user=[0.0, 0.5], mu_user=[-0.5, 0.5], phi_user=[0.0, 90.0, 180.0])
    o = oracle_lib.general_solve(capi.pack_general([inst], capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU))
    I = o["intensity"][0]
    assert np.all(np.isfinite(I))
    assert np.abs(I[:, :, 0] - I[:, :, 2]).max() > 1e-3 * np.abs(I).max()
    np.testing.assert_array_equal(o["intensity_azimuth_avg"][0].shape, (2, 2))


@pytest.mark.parametrize("mutate", [
    lambda i, f: (i.update(num_layers=0, delta_tau=[], single_scat_albedo=[], phase_function_moments=np.zeros((0, 17))) or i, f),
    lambda i, f: (i.update(single_scat_albedo=np.r_[1.5, i["single_scat_albedo"][1:]]) or i, f),
    lambda i, f: (i.update(delta_tau=np.r_[-1.0, i["delta_tau"][1:]]) or i, f),
    lambda i, f: (i.update(mu_user=[0.5, 0.2]) or i, f),
    lambda i, f: (i.update(mu_user=[-0.5, 1.5]) or i, f),
    lambda i, f: (i.update(phi_user=[-10.0]) or i, f),
    lambda i, f: (i.update(direct_beam_mu=0.0) or i, f),
    lambda i, f: (i, f | capi.FLAG_DIFFUSION_LOWER_BC),
    lambda i, f: (i, f | capi.FLAG_DELTA_M_PLUS),
])
def test_general_validation(mutate):
    rng = np.random.default_rng(3)
    inst = random_instance(rng, 16, 3, thermal=False, beam=True)
    inst.update(tau_user=[0.0], mu_user=[-0.5, 0.5], phi_user=[0.0])
    inst, flags = mutate(inst, capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU)
    if inst["num_layers"] == 0:
        d = capi.pack_general([inst], flags, pmom_count=17)
    else:
        d = capi.pack_general([inst], flags)
    o = oracle_lib.general_solve(d)
    assert o["status"][0] == capi.DSP_ERR_INVALID_INPUT


# ---------------------------------------------------------------------------
# pseudo-spherical beam of the general solver
# ---------------------------------------------------------------------------
def test_general_spherical_golden():
    """SphericalGeometry (tests/test_solver.cpp:4459-4533): the C-DISORT
    fluxes of the general solver with the Chapman correction, 1e-3."""
    case = gc.load_spherical_cases()[0]
    inst, flags = gc.general_instance(case)
    inst.update(level_altitudes=case["level_altitudes"], bottom_radius=case["bottom_radius"])
    o = oracle_lib.general_solve(capi.pack_general([inst], flags | capi.FLAG_SPHERICAL_BEAM))
    assert o["status"][0] == 0
    for e in case["expect_flux"]:
        v = o[e["field"]][0, e["index"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)


@pytest.mark.parametrize("nstr", [4, 16])
def test_general_spherical_equals_flux_spherical(nstr):
    """SphericalBeam4/16 (test_flux_solver.cpp:309-358): the flux solver and
    the general solver agree to 1e-12 on a spherical-shell column."""
    from disort_b200 import workloads
    L = 5
    zalt = [100.0, 80.0, 60.0, 40.0, 20.0, 0.0]
    pm = workloads.hg_moments(np.zeros(L), nstr + 1)
    inst = dict(num_streams=nstr, num_layers=L, num_phase_func_moments=0, delta_tau=np.full(L, 0.1),
                single_scat_albedo=np.full(L, 0.9), phase_function_moments=pm, surface_albedo=0.1,
                direct_beam_flux=1.0, direct_beam_mu=0.3, level_altitudes=zalt, bottom_radius=6371.0)
    o = oracle_lib.general_solve(capi.pack_general([inst], capi.FLAG_SPHERICAL_BEAM | capi.GFLAG_ONLY_FLUXES))
    w = dict(n_inst=1, num_streams=nstr, num_layers=L, num_phase_func_moments=0, pmom_count=nstr + 1,
             flags=capi.FLAG_SPHERICAL_BEAM,
             arrays=dict(delta_tau=np.full(L, 0.1), single_scat_albedo=np.full(L, 0.9), phase_function_moments=pm,
                         surface_albedo=0.1, direct_beam_flux=1.0, direct_beam_mu=0.3,
                         level_altitudes=np.array(zalt), bottom_radius=6371.0))
    f, st = oracle_lib.flux_solve(w)
    assert o["status"][0] == 0 and st[0] == 0
    for k in capi.FLUX_OUT_FIELDS:
        np.testing.assert_allclose(o[k][0, :L + 1], f[k][0], rtol=1e-12, atol=1e-14, err_msg=k)


BRDF_CASES = gc.load_brdf_cases()


@pytest.mark.parametrize("case", BRDF_CASES, ids=[c["name"] for c in BRDF_CASES])
def test_general_oracle_brdf_goldens(case):
    """Bidirectional surfaces (Hapke, RPV) against the reference's C-DISORT goldens;
    disotest 6d-6h with the BRDF correction of the reflected beam."""
    inst, flags = gc.general_instance(case)
    o = oracle_lib.general_solve(capi.pack_general([inst], flags))
    assert o["status"][0] == 0
    assert case["expect_flux"] or case["expect_intensity"]
    for e in case["expect_flux"]:
        v = o[e["field"]][0, e["index"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)
    for e in case["expect_intensity"]:
        v = o["intensity"][0, e["lu"], e["iu"], e["j"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)


CORR_CASES = gc.load_corrected_cases()


@pytest.mark.parametrize("case", CORR_CASES, ids=[c["name"] for c in CORR_CASES])
def test_general_oracle_intensity_correction_goldens(case):
    """The Nakajima-Tanaka correction against the reference's C-DISORT goldens
    (IntensityCorrection*, disotest 12a); without it the intensities miss them."""
    inst, flags = gc.general_instance(case)
    o = oracle_lib.general_solve(capi.pack_general([inst], flags))
    assert o["status"][0] == 0
    for e in case["expect_flux"]:
        v = o[e["field"]][0, e["index"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)
    for e in case["expect_intensity"]:
        v = o["intensity"][0, e["lu"], e["iu"], e["j"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)
    plain = oracle_lib.general_solve(capi.pack_general([inst], flags & ~capi.GFLAG_INTENSITY_CORR))
    np.testing.assert_array_equal(plain["flux_up"], o["flux_up"])
    np.testing.assert_array_equal(plain["intensity_azimuth_avg"], o["intensity_azimuth_avg"])


@pytest.mark.parametrize("model", [capi.BRDF_RPV, capi.BRDF_COX_MUNK, capi.BRDF_AMBRALS, capi.BRDF_HAPKE])
def test_general_oracle_brdf_conserves_energy_sense(model):
    """Every surface model: a non-absorbing, non-emitting column over a BRDF
    reflects no more than it receives (net flux at the surface >= 0) and the
    surface's reflection raises the upward flux over a black surface."""
    params = {capi.BRDF_RPV: [0.1, 0.9, -0.2, 0.0, 0.0, 0.0, 1.0],
              capi.BRDF_COX_MUNK: [5.0, 0.0, 0.0, 1.34, 1.0],
              capi.BRDF_AMBRALS: [0.1, 0.05, 0.02],
              capi.BRDF_HAPKE: [1.0, 0.06, 0.6]}[model]
    rng = np.random.default_rng(11 + model)
    inst = random_instance(rng, 8, 5, thermal=False, beam=True)
    inst.update(mu_user=[-0.7, -0.2, 0.3, 0.8], phi_user=[0.0, 90.0, 180.0])
    flags = capi.GFLAG_USER_MU
    black = oracle_lib.general_solve(capi.pack_general([dict(inst, surface_albedo=0.0)], flags))
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, brdf_type=model, brdf_params=params)], flags))
    assert o["status"][0] == 0 and black["status"][0] == 0
    L = inst["num_layers"]
    down = o["flux_down"][0, L] + o["flux_direct_beam"][0, L]
    assert o["flux_up"][0, L] <= down
    assert o["flux_up"][0, 0] > black["flux_up"][0, 0]
    assert np.isfinite(o["intensity"][0]).all()


def test_general_oracle_brdf_rejections():
    """A BRDF with the diffusion lower boundary is invalid (DisortConfig.cpp:144-146);
    an unknown model too; a BRDF ignores surface_albedo (no [0, 1] check)."""
    rng = np.random.default_rng(5)
    inst = random_instance(rng, 8, 3, thermal=True, beam=False)
    hap = dict(brdf_type=capi.BRDF_HAPKE, brdf_params=[1.0, 0.06, 0.6])
    fl = capi.FLAG_THERMAL | capi.GFLAG_ONLY_FLUXES
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, **hap)], fl))
    assert o["status"][0] == 0
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, **hap)], fl | capi.FLAG_DIFFUSION_LOWER_BC))
    assert o["status"][0] == capi.DSP_ERR_INVALID_INPUT
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, brdf_type=9, brdf_params=[1.0])], fl))
    assert o["status"][0] == capi.DSP_ERR_INVALID_INPUT
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, surface_albedo=7.0, **hap)], fl))
    assert o["status"][0] == 0
    o = oracle_lib.general_solve(capi.pack_general([dict(inst, surface_albedo=7.0)], fl))
    assert o["status"][0] == capi.DSP_ERR_INVALID_INPUT


SPECIAL_CASES = gc.load_special_cases()


@pytest.mark.parametrize("case", SPECIAL_CASES, ids=[c["name"] for c in SPECIAL_CASES])
def test_general_oracle_special_bc_goldens(case):
    """ibcnd = Special: albedo and transmissivity of the medium (computeAlbTrans)
    against the reference's C-DISORT values, spherical-albedo correction included."""
    inst, flags = gc.general_instance(case)
    o = oracle_lib.general_albtrans(capi.pack_general([inst], flags))
    assert o["status"][0] == 0
    assert case["expect_albtrans"]
    for e in case["expect_albtrans"]:
        v = o[e["field"]][0, e["index"]]
        assert abs(v - e["value"]) <= e["tol"], (e, v)
    assert 0.0 < o["spherical_albedo"][0] < 1.0 and 0.0 < o["spherical_transmissivity"][0] < 1.0


def test_general_oracle_special_bc_reciprocity():
    """Without a surface the albedo of the medium at mu equals the beam albedo of a
    general solve lit at mu (flux_up at the top / (mu F0)), and the transmissivity the
    total downward flux at the bottom (the reference's 13b/13d verification)."""
    rng = np.random.default_rng(13)
    for L in (1, 3):
        inst = random_instance(rng, 16, L, thermal=False, beam=False)
        inst.update(surface_albedo=0.0, mu_user=[0.3, 0.5, 0.9])
        a = oracle_lib.general_albtrans(capi.pack_general([inst], capi.GFLAG_USER_MU))
        assert a["status"][0] == 0
        assert a["spherical_albedo"][0] == 0.0
        for k, mu0 in enumerate((0.3, 0.5, 0.9)):
            beam = dict(inst, direct_beam_flux=1.0 / mu0, direct_beam_mu=mu0, isotropic_flux_top=0.0)
            beam.pop("mu_user")
            g = oracle_lib.general_solve(capi.pack_general([beam], capi.GFLAG_ONLY_FLUXES))
            np.testing.assert_allclose(a["albedo_medium"][0, k], g["flux_up"][0, 0], rtol=1e-3)
            np.testing.assert_allclose(a["transmissivity_medium"][0, k],
                                       g["flux_down"][0, L] + g["flux_direct_beam"][0, L], rtol=1e-3)
