"""GPU parity of bidirectional (BRDF) surfaces on the general path against the oracle.

The reference's Hapke and RPV known-answer cases (tests/test_solver.cpp) and
random columns over every surface model (RPV, Cox-Munk, Ross-Li/Ambrals,
Hapke) at every stream count, with the beam's azimuth modes, thermal emission,
temperature Jacobians, device pointers and the C++/Python solver objects.
Tolerances are those of the general path (1e-9 relative + 1e-12 absolute;
intensities against the instance's largest intensity).
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
BRDF_CASES = golden_cases.load_brdf_cases()
MODELS = {
    capi.BRDF_RPV: [0.1, 0.9, -0.2, 0.0, 0.0, 0.0, 1.0],
    capi.BRDF_COX_MUNK: [5.0, 0.0, 0.0, 1.34, 1.0],
    capi.BRDF_AMBRALS: [0.1, 0.05, 0.02],
    capi.BRDF_HAPKE: [1.0, 0.06, 0.6],
}


def both(insts, flags, accuracy=0.0):
    d = capi.pack_general(insts, flags, accuracy_fourier_series=accuracy)
    ref = oracle_lib.general_solve(d)
    got, rc = gpu_lib.general_solve(d)
    assert rc == 0, gpu_lib.context().last_error()
    return got, ref, d


@pytest.mark.parametrize("case", BRDF_CASES, ids=[c["name"] for c in BRDF_CASES])
def test_brdf_reference_goldens(case):
    inst, flags = golden_cases.general_instance(case)
    got, ref, _ = both([inst], flags)
    assert got["status"][0] == ref["status"][0] == 0
    # conservative scattering (HapkeBRDF1): the reference's own cross-solver
    # tolerance there is 1e-8 relative, 2e-9 absolute (test_flux_solver.cpp:135-136)
    if max(case["single_scat_albedo"]) >= 1.0:
        assert_parity_general(got, ref, case["name"], rtol=1e-8, atol=2e-9)
    else:
        assert_parity_general(got, ref, case["name"])
    for e in case["expect_flux"]:
        assert abs(got[e["field"]][0, e["index"]] - e["value"]) <= e["tol"]
    for e in case["expect_intensity"]:
        assert abs(got["intensity"][0, e["lu"], e["iu"], e["j"]] - e["value"]) <= e["tol"]


def brdf_mix(model, n, seed, nstr, layers=(3, 14), thermal=False, params=None):
    insts, flags = workloads.general_mix(n, seed=seed, nstr=(4,), layers=layers)
    insts = with_streams(insts, nstr)
    rng = np.random.default_rng(seed)
    for c in insts:
        c["brdf_type"] = model
        p = list(params or MODELS[model])
        if model == capi.BRDF_RPV:
            p[0] = float(rng.uniform(0.05, 0.3))  # rho0 per instance
        elif model == capi.BRDF_COX_MUNK:
            p[0] = float(rng.uniform(1.0, 12.0))  # wind speed per instance
        c["brdf_params"] = p
        if thermal:
            L = c["num_layers"]
            c.update(temperature=200.0 + 100.0 * np.arange(L + 1) / L, wavenumber_low=600.0,
                     wavenumber_high=640.0, temperature_bottom=305.0, temperature_top=20.0)
    if thermal:
        flags |= capi.FLAG_THERMAL
    return insts, flags


@pytest.mark.parametrize("model", list(MODELS), ids=["rpv", "cox_munk", "ambrals", "hapke"])
@pytest.mark.parametrize("nstr", [(4, 8), (16,), (6, 10, 12, 14), (32,), (64,)])
def test_brdf_mix_every_model(model, nstr):
    n = 3 if nstr == (64,) else 10
    layers = (3, 6) if nstr == (64,) else (3, 14)
    insts, flags = brdf_mix(model, n, seed=40 + model + len(nstr), nstr=nstr, layers=layers)
    got, ref, _ = both(insts, flags)
    assert (got["status"] == 0).all() and (ref["status"] == 0).all()
    assert_parity_general(got, ref, f"brdf {model} N {nstr}")


@pytest.mark.parametrize("model", [capi.BRDF_RPV, capi.BRDF_HAPKE])
def test_brdf_thermal_and_lyrcut(model):
    """Thermal emission (surface emissivity from the BRDF) and deep beam-only
    columns where the absorption cut drops the surface from the problem."""
    insts, flags = brdf_mix(model, 8, seed=90 + model, nstr=(8, 16), thermal=True)
    got, ref, _ = both(insts, flags)
    assert (got["status"] == 0).all()
    assert_parity_general(got, ref, "thermal")
    insts, flags = brdf_mix(model, 6, seed=95 + model, nstr=(8,), layers=(30, 40))
    for c in insts:
        c["delta_tau"] = np.full(c["num_layers"], 2.0)
        c["single_scat_albedo"] = np.full(c["num_layers"], 0.2)
    got, ref, _ = both(insts, flags)
    assert_parity_general(got, ref, "lyrcut")


def test_brdf_device_pointers_and_fluxes_only():
    insts, flags = brdf_mix(capi.BRDF_AMBRALS, 6, seed=7, nstr=(8, 16))
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_solve(d)
    got, rc = gpu_lib.general_solve_device(d)
    assert rc == 0
    assert_parity_general(got, ref, "device pointers")
    for c in insts:
        c.pop("mu_user")
    fl = (flags & ~capi.GFLAG_USER_MU) | capi.GFLAG_ONLY_FLUXES
    got, ref, _ = both(insts, fl)
    assert_parity_general(got, ref, "fluxes only")


def test_brdf_invalid_combinations():
    """A BRDF with the diffusion lower boundary is an invalid instance; an
    unknown model or missing parameters reject the call."""
    insts, flags = brdf_mix(capi.BRDF_HAPKE, 3, seed=3, nstr=(8,), thermal=True)
    d = capi.pack_general(insts, flags | capi.FLAG_DIFFUSION_LOWER_BC)
    got, rc = gpu_lib.general_solve(d)
    assert rc == 0
    assert (got["status"] == capi.DSP_ERR_INVALID_INPUT).all()
    d = capi.pack_general(insts, flags)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    batch.brdf_type = 7
    assert gpu_lib.context().general_bands_solve(batch, o) == capi.DSP_ERR_INVALID_INPUT
    batch.brdf_type = capi.BRDF_HAPKE
    batch.brdf_params = capi.DArray(None, 0)
    assert gpu_lib.context().general_bands_solve(batch, o) == capi.DSP_ERR_INVALID_INPUT


def test_brdf_temperature_jacobians():
    """Temperature Jacobians over a BRDF surface: its emissivity and reflection
    enter the replayed boundary rows."""
    insts, flags = brdf_mix(capi.BRDF_RPV, 5, seed=21, nstr=(8, 16), thermal=True)
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_solve_jac(d)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    jac, jo, keep3 = capi.alloc_general_jac_numpy(d)
    assert gpu_lib.context().general_bands_solve_jac(batch, o, jo) == 0
    assert_parity_general(outs, ref[0], "fluxes")
    for f in capi.JAC_FIELDS:
        a, b = jac[f], ref[1][f]
        scale = np.maximum(np.abs(b), 1e-3 * np.abs(b).max(axis=(1, 2), keepdims=True))
        assert np.all(np.abs(a - b) <= 3e-8 * scale + 1e-15), f


def test_brdf_through_solver_objects():
    """disort_b200.DisortSolver with a Hapke and an RPV surface equals the C ABI call;
    an RPV surface without its spec raises like the reference."""
    import disort_b200 as db
    cfg = db.DisortConfig(2, 8, 9)
    cfg.flags.use_user_tau = False
    cfg.flags.use_user_mu = True
    cfg.flags.use_lambertian_surface = False
    cfg.flags.brdf_type = db.BrdfType.Hapke
    cfg.num_user_mu = 2
    cfg.num_phi = 2
    cfg.allocate()
    cfg.delta_tau = [0.3, 0.7]
    cfg.single_scat_albedo = [0.8, 0.6]
    cfg.set_henyey_greenstein(0.6)
    cfg.mu_user = [-0.4, 0.6]
    cfg.phi_user = [0.0, 120.0]
    cfg.bc.direct_beam_flux = 1.0
    cfg.bc.direct_beam_mu = 0.7
    r = db.DisortSolver().solve(cfg)
    inst = dict(num_streams=8, num_layers=2, num_phase_func_moments=9, delta_tau=[0.3, 0.7],
                single_scat_albedo=[0.8, 0.6], phase_function_moments=workloads.hg_moments(np.array([0.6, 0.6]), 10),
                direct_beam_flux=1.0, direct_beam_mu=0.7, mu_user=[-0.4, 0.6], phi_user=[0.0, 120.0],
                brdf_type=capi.BRDF_HAPKE, brdf_params=MODELS[capi.BRDF_HAPKE])
    got, ref, _ = both([inst], capi.GFLAG_USER_MU)
    np.testing.assert_allclose(np.asarray(r.flux_up), got["flux_up"][0, :3], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(np.asarray(r.intensity), got["intensity"][0, :3, :2, :], rtol=1e-12, atol=1e-15)
    cfg.flags.brdf_type = db.BrdfType.RPV
    with pytest.raises(RuntimeError, match="rpv spec is null"):
        db.DisortSolver().solve(cfg)
    spec = db.RpvBrdfSpec()
    spec.rho0, spec.k, spec.theta, spec.scale = 0.1, 0.9, -0.2, 1.0
    cfg.brdf.set_rpv(spec)
    r = db.DisortSolver().solve(cfg)
    inst.update(brdf_type=capi.BRDF_RPV, brdf_params=[0.1, 0.9, -0.2, 0.0, 0.0, 0.0, 1.0])
    got, ref, _ = both([inst], capi.GFLAG_USER_MU)
    np.testing.assert_allclose(np.asarray(r.flux_up), got["flux_up"][0, :3], rtol=1e-12, atol=1e-15)
