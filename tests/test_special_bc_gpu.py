"""GPU parity of ibcnd = Special (albedo and transmissivity of the medium,
dsp_general_bands_albtrans) against the oracle's restatement of computeAlbTrans.

The reference's 13a/13c known-answer cases, random columns at every stream
count with and without user angles, one and several layers, delta-M+, bottom-up
input and the spherical-albedo correction, and the C++/Python DisortSolver.
Tolerance: 1e-9 relative + 1e-12 absolute.
"""
import numpy as np
import pytest

import golden_cases
import gpu_lib
import oracle_lib
from disort_b200 import capi, workloads
from test_general_gpu import with_streams

pytestmark = pytest.mark.gpu
CASES = golden_cases.load_special_cases()
FIELDS = ("albedo_medium", "transmissivity_medium", "spherical_albedo", "spherical_transmissivity")


def gpu_albtrans(d):
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_albtrans_numpy(d)
    rc = gpu_lib.context().general_bands_albtrans(batch, o)
    assert rc == 0, gpu_lib.context().last_error()
    return outs


def check(insts, flags, label):
    d = capi.pack_general(insts, flags)
    ref = oracle_lib.general_albtrans(d)
    got = gpu_albtrans(d)
    assert (got["status"] == 0).all() and (ref["status"] == 0).all(), (got["status"], ref["status"])
    for f in FIELDS:
        a, b = got[f], ref[f]
        assert np.all(np.abs(a - b) <= 1e-9 * np.abs(b) + 1e-12), (label, f, np.max(np.abs(a - b)))
    return got


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_special_bc_reference_goldens(case):
    inst, flags = golden_cases.general_instance(case)
    got = check([inst], flags, case["name"])
    for e in case["expect_albtrans"]:
        assert abs(got[e["field"]][0, e["index"]] - e["value"]) <= e["tol"]


@pytest.mark.parametrize("nstr", [(4,), (8,), (16,), (32,), (64,)])
def test_special_bc_mix(nstr):
    n = 3 if nstr == (64,) else 8
    insts, _ = workloads.general_mix(n, seed=130 + nstr[0], nstr=(4,), layers=(1, 6) if nstr == (64,) else (1, 14))
    insts = with_streams(insts, nstr)
    rng = np.random.default_rng(nstr[0])
    for k, c in enumerate(insts):
        c["surface_albedo"] = 0.0 if k % 3 == 0 else float(rng.uniform(0.05, 0.8))
        c["mu_user"] = [0.15, 0.5, 0.85]
    check(insts, capi.GFLAG_USER_MU, f"user angles N {nstr}")
    check(insts, capi.GFLAG_USER_MU | capi.FLAG_DELTA_M_PLUS, f"delta-M+ N {nstr}")
    check(insts, capi.GFLAG_USER_MU | capi.FLAG_INDEX_FROM_BOTTOM, f"bottom-up N {nstr}")
    for c in insts:
        c.pop("mu_user")
    check(insts, 0, f"quadrature angles N {nstr}")


def test_special_bc_through_solver_object():
    """DisortSolver with ibcnd = Special on the 13a configuration: the C ABI's
    numbers, arrays sized like the mirrored cosines, the config's cosines halved."""
    import disort_b200 as db
    cfg = db.DisortConfig(1, 16)
    cfg.flags.ibcnd = db.BoundaryConditionType.Special
    cfg.flags.use_user_tau = False
    cfg.flags.use_user_mu = True
    cfg.flags.use_lambertian_surface = False  # ignored: the special case forces a Lambertian surface
    cfg.bc.surface_albedo = 0.5
    cfg.num_user_mu = 1
    cfg.allocate()
    cfg.delta_tau = [1.0]
    cfg.single_scat_albedo = [0.99]
    cfg.mu_user = [0.5]
    cfg.set_henyey_greenstein(0.8)
    r = db.DisortSolver().solve(cfg)
    assert list(r.mu_angles) == [-0.5, 0.5]
    assert len(r.albedo_medium) == 2
    assert abs(r.albedo_medium[0] - 5.4525838793e-01) <= 1e-3 * 5.4525838793e-01
    assert abs(r.transmissivity_medium[0] - 8.4499871160e-01) <= 1e-3 * 8.4499871160e-01
    assert cfg.num_user_mu == 1
    inst = dict(num_streams=16, num_layers=1, num_phase_func_moments=0, delta_tau=[1.0], single_scat_albedo=[0.99],
                phase_function_moments=workloads.hg_moments(np.array([0.8]), 17), surface_albedo=0.5,
                mu_user=[0.5])
    got = gpu_albtrans(capi.pack_general([inst], capi.GFLAG_USER_MU))
    np.testing.assert_allclose(r.albedo_medium[0], got["albedo_medium"][0, 0], rtol=1e-13)
    np.testing.assert_allclose(r.spherical_albedo, got["spherical_albedo"][0], rtol=1e-13)
