"""GPU parity of the general path (dsp_general_bands_solve) against the CPU oracle.

Every test calls libdsp.so through its C ABI with the same dsp_general_batch
the oracle receives.  Fluxes must agree element-wise within 1e-9 relative plus
1e-12 absolute; intensities within 1e-9 of max(|value|, the instance's largest
|intensity|) plus 1e-12 (an intensity is a Fourier sum over azimuth modes whose
terms cancel, so a single element can sit far below the field it comes from).
"""
import numpy as np
import pytest

import golden_cases
import gpu_lib
import oracle_lib
from disort_b200 import capi, workloads
from parity import assert_parity_general, worst_general

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_cases()


def both(insts, flags, accuracy=0.0, ext=False):
    d = capi.pack_general(insts, flags, accuracy_fourier_series=accuracy)
    ref = oracle_lib.general_solve(d, ext=ext)
    got, rc = gpu_lib.general_solve(d)
    assert rc == 0, gpu_lib.context().last_error()
    return got, ref, d


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_general_reference_goldens(case):
    inst, flags = golden_cases.general_instance(case)
    got, ref, _ = both([inst], flags)
    assert got["status"][0] == ref["status"][0] == 0
    # conservative scattering takes the other factorisation; the reference's own
    # cross-solver tolerance there is 1e-8 relative, 2e-9 absolute (test_flux_solver.cpp:135-136)
    if max(case["single_scat_albedo"]) >= 1.0:
        assert_parity_general(got, ref, case["name"], rtol=1e-8, atol=2e-9)
    else:
        assert_parity_general(got, ref, case["name"])
    for e in case["expect_flux"]:
        assert abs(got[e["field"]][0, e["index"]] - e["value"]) <= e["tol"]
    for e in case["expect_intensity"]:
        assert abs(got["intensity"][0, e["lu"], e["iu"], e["j"]] - e["value"]) <= e["tol"]


def with_streams(insts, Ns):
    """Re-target mixed-batch instances to the stream counts Ns (cycled): N+1 HG moments."""
    for k, p in enumerate(insts):
        N = Ns[k % len(Ns)]
        g = p["phase_function_moments"][:, 1]
        p.update(num_streams=N, num_phase_func_moments=N + 1,
                 phase_function_moments=workloads.hg_moments(g, N + 2))
    return insts


@pytest.mark.parametrize("nstr", [(4, 8), (16,), (6, 10, 12, 14), (32,)])
def test_general_mix_small(nstr):
    insts, flags = workloads.general_mix(24, seed=30 + len(nstr), nstr=(4,), layers=(2, 12))
    insts = with_streams(insts, nstr)
    got, ref, _ = both(insts, flags)
    assert np.all(got["status"] == 0) and np.all(ref["status"] == 0)
    assert_parity_general(got, ref, f"general mix N={nstr}")


def test_general_mix_n64():
    insts, flags = workloads.general_mix(2, seed=41, nstr=(64,), layers=(3, 5))
    got, ref, _ = both(insts, flags)
    assert np.all(got["status"] == 0)
    assert_parity_general(got, ref, "general mix N=64")


def test_general_ragged_mixed_streams_one_batch():
    """One batch holding every supported stream count and ragged layer counts."""
    Ns = capi.SUPPORTED_NSTR[:-1]
    insts, flags = workloads.general_mix(2 * len(Ns), seed=50, nstr=(4,), layers=(1, 9))
    insts = with_streams(insts, Ns)
    got, ref, _ = both(insts, flags)
    assert np.all(got["status"] == 0)
    assert_parity_general(got, ref, "ragged mixed-N batch")


@pytest.mark.parametrize("kind", ["thermal", "thermal_beam", "dlbc", "ifb", "levels", "only_fluxes"])
def test_general_sources_and_options(kind):
    rng = np.random.default_rng(7)
    insts = []
    for k in range(6):
        N = (4, 8, 16)[k % 3]
        L = int(rng.integers(2, 9))
        g = rng.uniform(0.1, 0.9, L)
        inst = dict(num_streams=N, num_layers=L, num_phase_func_moments=0,
                    delta_tau=np.clip(rng.lognormal(-1.0, 1.5, L), 1e-6, 20.0),
                    single_scat_albedo=rng.uniform(0.0, 0.95, L), phase_function_moments=workloads.hg_moments(g, N + 1),
                    surface_albedo=float(rng.uniform(0, 0.5)), tau_user=[0.0, 0.3, 1.0],
                    mu_user=[-0.9, -0.3, 0.2, 0.7], phi_user=[0.0, 30.0, 200.0])
        if kind.startswith("thermal") or kind in ("dlbc", "ifb"):
            inst.update(temperature=200.0 + 100.0 * np.arange(L + 1) / L, wavenumber_low=600.0,
                        wavenumber_high=640.0, temperature_bottom=310.0, temperature_top=40.0, emissivity_top=0.8)
        if kind in ("thermal_beam", "ifb", "levels", "only_fluxes"):
            inst.update(direct_beam_flux=2.0, direct_beam_mu=float(rng.uniform(0.2, 0.95)), direct_beam_phi=25.0,
                        isotropic_flux_top=0.2, isotropic_flux_bottom=0.1)
        insts.append(inst)
    flags = capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU
    if kind in ("thermal", "thermal_beam", "dlbc", "ifb"):
        flags |= capi.FLAG_THERMAL
    if kind == "dlbc":
        flags |= capi.FLAG_DIFFUSION_LOWER_BC
    if kind == "ifb":
        flags |= capi.FLAG_INDEX_FROM_BOTTOM
    if kind == "levels":
        flags &= ~capi.GFLAG_USER_TAU
    if kind == "only_fluxes":
        flags |= capi.GFLAG_ONLY_FLUXES
    got, ref, _ = both(insts, flags)
    assert np.all(got["status"] == 0) and np.all(ref["status"] == 0)
    assert_parity_general(got, ref, kind)


def test_general_absorption_cut():
    """Deep absorbing beam-only columns: levels below the cut are zero."""
    rng = np.random.default_rng(9)
    insts = []
    for k in range(4):
        L = 6
        insts.append(dict(num_streams=8, num_layers=L, num_phase_func_moments=0,
                          delta_tau=np.array([2.0, 5.0, 8.0, 10.0, 3.0, 1.0]) * (1 + 0.1 * k),
                          single_scat_albedo=np.full(L, 0.2), phase_function_moments=workloads.hg_moments(np.full(L, 0.6), 9),
                          direct_beam_flux=1.0, direct_beam_mu=0.4 + 0.1 * k, surface_albedo=0.3,
                          tau_user=[0.0, 3.0, 40.0], mu_user=[-0.5, 0.5], phi_user=[0.0, 90.0]))
    got, ref, _ = both(insts, capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU)
    assert_parity_general(got, ref, "lyrcut")
    assert np.all(got["flux_up"][:, 2] == 0.0) and np.all(got["intensity"][:, 2] == 0.0)


def test_general_convergence_early_exit():
    insts, flags = workloads.general_mix(8, seed=61, nstr=(16,), layers=(2, 6))
    got, ref, _ = both(insts, flags, accuracy=1e-3)
    assert_parity_general(got, ref, "accuracy 1e-3")


def test_general_invalid_and_unsupported_instances():
    insts, flags = workloads.general_mix(5, seed=71, nstr=(8,), layers=(2, 4))
    insts[1]["single_scat_albedo"] = np.r_[1.5, insts[1]["single_scat_albedo"][1:]]
    insts[3]["num_streams"] = 18  # even, >= 4, but no kernel instantiation
    insts[3]["num_phase_func_moments"] = 19
    insts[3]["phase_function_moments"] = workloads.hg_moments(np.full(insts[3]["num_layers"], 0.7), 20)
    got, ref, _ = both(insts, flags)
    assert got["status"][1] == capi.DSP_ERR_INVALID_INPUT
    assert got["status"][3] == capi.DSP_ERR_UNSUPPORTED
    for k in (1, 3):
        assert np.all(np.isnan(got["flux_up"][k])) and np.all(np.isnan(got["intensity"][k]))
    keep = [0, 2, 4]
    assert np.all(got["status"][keep] == 0)
    sub = lambda o: {f: o[f][keep] for f in o if f != "status"}
    assert_parity_general(sub(got), sub(ref), "valid instances beside invalid ones")


def test_general_device_pointers_match_host():
    insts, flags = workloads.general_mix(10, seed=81, nstr=(4, 16), layers=(2, 8))
    d = capi.pack_general(insts, flags)
    host, rc = gpu_lib.general_solve(d)
    assert rc == 0
    dev, rc2 = gpu_lib.general_solve_device(d)
    assert rc2 == 0, gpu_lib.context().last_error()
    for f in host:
        np.testing.assert_array_equal(dev[f], host[f], err_msg=f)


def config3_sample():
    """A stratified sample of the ragged general mix at its own sizes: the mix's
    real distribution (N in {4, 8, 16, 32, 64}, 10-120 layers, delta-M+, beam
    only so the absorption cut fires, user optical depths top/middle/bottom, five
    polar angles, four azimuths, every azimuth mode), four instances of each of
    N = 4, 8, 16, and for N = 32 and 64 four deep columns (90 layers or more) and
    one shallow one."""
    insts, flags = workloads.general_mix(1200, seed=3)
    pick = []
    for N in (4, 8, 16):
        pick += [i for i, p in enumerate(insts) if p["num_streams"] == N][:4]
    for N in (32, 64):
        pick += [i for i, p in enumerate(insts) if p["num_streams"] == N and p["num_layers"] >= 90][:4]
        pick += [i for i, p in enumerate(insts) if p["num_streams"] == N and p["num_layers"] < 40][:1]
    return [insts[i] for i in pick], flags


def test_general_mix_at_full_sizes():
    from disort_b200 import flops
    insts, flags = config3_sample()
    assert sum(p["num_layers"] >= 90 for p in insts if p["num_streams"] == 64) >= 4
    cut = [flops.absorption_cut(p["delta_tau"], p["single_scat_albedo"], False) < p["num_layers"] for p in insts]
    assert sum(cut) >= 5  # the absorption cut shortens several columns
    # checker: the extended-precision oracle build (at 64 streams double rounding in
    # the restatement reaches 1e-9 of some fluxes; the double build is held to 1e-8)
    got, ref, d = both(insts, flags, ext=True)
    assert np.all(got["status"] == 0) and np.all(ref["status"] == 0)
    assert_parity_general(got, ref, "general mix at full sizes")
    assert worst_general(oracle_lib.general_solve(d), ref)[0] <= 10.0
    # the same instances through device pointers give the same numbers
    dgot, rc = gpu_lib.general_solve_device(capi.pack_general(insts, flags))
    assert rc == 0
    for f in got:
        np.testing.assert_array_equal(got[f], dgot[f])


# ---------------------------------------------------------------------------
# pseudo-spherical beam (DisortSolver.cpp:740-790, 1396-1530)
# ---------------------------------------------------------------------------
def spherical_mix(n, seed, nstr, layers=(3, 16), bottom_up=False, thermal=False):
    """Beam instances of the mixed batch through spherical shells (altitudes
    2 km per layer over a 6371 km radius), intensities at user angles in every
    azimuth mode; bottom_up gives the layer arrays and altitudes bottom-up."""
    insts, flags = workloads.general_mix(n, seed=seed, nstr=(4,), layers=layers)
    insts = with_streams(insts, nstr)
    rng = np.random.default_rng(seed + 1)
    for p in insts:
        L = p["num_layers"]
        z = np.linspace(2.0 * L, 0.0, L + 1)
        p.update(level_altitudes=z[::-1] if bottom_up else z, bottom_radius=6371.0,
                 direct_beam_phi=float(rng.uniform(0, 90)))
        if thermal:
            lo = float(rng.uniform(300, 1500))
            p.update(temperature=200 + 100 * rng.random(L + 1), wavenumber_low=lo, wavenumber_high=lo * 1.01,
                     temperature_bottom=300.0)
    flags |= capi.FLAG_SPHERICAL_BEAM
    if bottom_up:
        flags |= capi.FLAG_INDEX_FROM_BOTTOM
    if thermal:
        flags |= capi.FLAG_THERMAL
    return insts, flags


def test_general_spherical_golden():
    """SphericalGeometry (tests/test_solver.cpp:4459-4533) through the general path."""
    case = golden_cases.load_spherical_cases()[0]
    inst, flags = golden_cases.general_instance(case)
    inst.update(level_altitudes=case["level_altitudes"], bottom_radius=case["bottom_radius"])
    got, ref, _ = both([inst], flags | capi.FLAG_SPHERICAL_BEAM)
    assert got["status"][0] == ref["status"][0] == 0
    assert_parity_general(got, ref, case["name"])
    for e in case["expect_flux"]:
        assert abs(got[e["field"]][0, e["index"]] - e["value"]) <= e["tol"]


@pytest.mark.parametrize("nstr", [(4, 8), (16,), (6, 10, 12, 14), (32,), (64,)])
def test_general_spherical_beam(nstr):
    """Spherical-shell instances at every stream count, with all azimuth modes
    (each mode has its own spherical particular solution), then bottom-up
    indexing and a thermal source with them.  At 32 and 64 streams the N x N
    LU of I + xba M - C (xba = 1 / Chapman factor, often within a few percent of
    a 1 / mu_i) carries rounding of ~2e-8 relative: there the checker is the
    extended-precision oracle build, at 5e-8."""
    big = max(nstr) >= 32
    rtol = 5e-8 if big else 1e-9
    # theoretically-zero fluxes (the downward diffuse flux at the top) come out
    # as cancellation noise: 1.3e-12 in the extended build itself at 64 streams
    atol = 1e-11 if big else 1e-12
    n = 2 if 64 in nstr else 12
    for kw in (dict(), dict(bottom_up=True), dict(thermal=True)):
        insts, flags = spherical_mix(n, seed=600 + sum(nstr), nstr=nstr, layers=(3, 5) if 64 in nstr else (3, 16),
                                     **kw)
        got, ref, _ = both(insts, flags, ext=big)
        assert np.all(got["status"] == 0) and np.all(ref["status"] == 0), (got["status"], ref["status"])
        assert_parity_general(got, ref, f"spherical N={nstr} {kw}", rtol=rtol, atol=atol)


def test_general_spherical_invalid_radius_and_missing_altitudes():
    insts, flags = spherical_mix(4, seed=7, nstr=(8,))
    insts[1]["bottom_radius"] = -1.0
    insts[3]["bottom_radius"] = 0.0
    got, ref, _ = both(insts, flags)
    assert list(got["status"]) == [0, capi.DSP_ERR_INVALID_INPUT, 0, capi.DSP_ERR_INVALID_INPUT]
    assert np.all(got["status"] == ref["status"])
    ok = [0, 2]
    assert_parity_general({k: v[ok] for k, v in got.items() if k != "status"},
                          {k: v[ok] for k, v in ref.items() if k != "status"}, "valid rows")
    d = capi.pack_general(insts, flags)
    batch, keep = capi.make_general_batch(d)
    batch.level_altitudes = None
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    assert gpu_lib.context().general_bands_solve(batch, o) == capi.DSP_ERR_INVALID_INPUT


def test_general_spherical_device_pointers_match_host():
    insts, flags = spherical_mix(6, seed=11, nstr=(4, 16))
    d = capi.pack_general(insts, flags)
    host, rc = gpu_lib.general_solve(d)
    dev, rc2 = gpu_lib.general_solve_device(d)
    assert rc == 0 and rc2 == 0, gpu_lib.context().last_error()
    for f in capi.FLUX_OUT_FIELDS + ("intensity", "intensity_azimuth_avg", "status"):
        np.testing.assert_array_equal(host[f], dev[f], err_msg=f)
