"""The bench's parity measure of the general leg (bench.general_parity) on CPU.

Fluxes are compared element-wise at 1e-9 relative + 1e-12 absolute;
intensities against the instance's largest intensity; with FP64 evaluations
given as `floor_ref` (the double oracle build on the given inputs and on
one-ulp-perturbed copies of them), an element's allowance widens to twice the
instance's FP64 spread (the farthest of those evaluations from the extended
build over that field, in units of the plain allowance)."""
import numpy as np

import bench
from disort_b200 import capi


def outputs(n=3, nt=4, nu=2, nphi=2, seed=0):
    rng = np.random.default_rng(seed)
    o = {f: rng.uniform(0.1, 1.0, (n, nt)) for f in capi.FLUX_OUT_FIELDS}
    o["intensity"] = rng.uniform(0.1, 1.0, (n, nt, nu, nphi))
    o["intensity_azimuth_avg"] = rng.uniform(0.1, 1.0, (n, nt, nu))
    return o


def perturbed(o, rel, field="flux_up", at=(1, 2)):
    p = {k: v.copy() for k, v in o.items()}
    p[field][at] *= 1.0 + rel
    return p


def test_plain_parity_threshold():
    ref = outputs()
    idx = np.arange(3)
    assert bench.general_parity(perturbed(ref, 5e-10), idx, ref)["passes"]
    r = bench.general_parity(perturbed(ref, 5e-9), idx, ref)
    assert not r["passes"] and r["at"].startswith("flux_up(1, 2)")


def test_intensity_scaled_by_instance_maximum():
    """A small intensity in an instance whose largest intensity is big passes
    at the same absolute error that a relative test would fail."""
    ref = outputs()
    ref["intensity"][0] *= 1e-6
    ref["intensity"][0, 0, 0, 0] = 1.0  # the instance's largest
    got = {k: v.copy() for k, v in ref.items()}
    got["intensity"][0, 1, 1, 1] += 5e-10  # 5e-10 of the instance maximum
    assert bench.general_parity(got, np.arange(3), ref)["passes"]


def test_fp64_spread_allowance():
    ext = outputs()
    dbl = perturbed(ext, 3e-9, at=(1, 0))  # the double build: 3e-9 off in instance 1
    idx = np.arange(3)
    # the GPU 5e-9 off elsewhere in instance 1: within twice the instance's spread
    gpu = perturbed(ext, 5e-9, at=(1, 3))
    assert not bench.general_parity(gpu, idx, ext)["passes"]
    assert bench.general_parity(gpu, idx, ext, floor_ref=dbl)["passes"]
    # 7e-9 is more than twice the spread; and the spread of instance 1 does not
    # cover instance 2
    assert not bench.general_parity(perturbed(ext, 7e-9, at=(1, 3)), idx, ext, floor_ref=dbl)["passes"]
    assert not bench.general_parity(perturbed(ext, 5e-9, at=(2, 3)), idx, ext, floor_ref=dbl)["passes"]


def test_spread_over_several_evaluations():
    """The spread is the farthest of several FP64 evaluations, in units of the
    plain allowance; one that did not solve the instance adds nothing, and
    noise far below the absolute tolerance next to nothing."""
    ext = outputs()
    idx = np.arange(3)
    near = perturbed(ext, 1e-10, at=(1, 0))
    far = perturbed(ext, 3e-9, at=(1, 0))
    gpu = perturbed(ext, 5e-9, at=(1, 3))
    assert not bench.general_parity(gpu, idx, ext, floor_ref=[near])["passes"]
    r = bench.general_parity(gpu, idx, ext, floor_ref=[near, far])
    b = ext["flux_up"][1, 0]
    assert r["passes"] and abs(r["fp64_spread_max"] - 3e-9 * b / (1e-9 * b + 1e-12)) < 1e-6
    far["status"] = np.array([0, 5, 0])
    assert not bench.general_parity(gpu, idx, ext, floor_ref=[near, far])["passes"]
    tiny = {k: v.copy() for k, v in ext.items()}
    tiny["flux_down"][1] = 1e-18
    wild = perturbed(tiny, 10.0, field="flux_down", at=(1, 0))
    r = bench.general_parity(tiny, idx, tiny, floor_ref=wild)
    assert r["passes"] and r["fp64_spread_max"] < 1e-4


def test_ulp_perturbed_copy():
    """Every layer input moves by exactly one ulp; the zeroth moment, zero
    entries and the albedo bound stay; the user depths follow the new total."""
    from disort_b200 import workloads
    insts, _ = workloads.general_mix(4, seed=1)
    c = dict(insts[0])
    c["single_scat_albedo"] = np.asarray(c["single_scat_albedo"], dtype=np.float64).copy()
    c["single_scat_albedo"][:2] = (1.0, 0.0)
    p = bench.ulp_perturbed(c, np.random.default_rng(0))
    for k in ("delta_tau", "single_scat_albedo", "phase_function_moments"):
        a, b = np.asarray(c[k], dtype=np.float64), np.asarray(p[k])
        moved = a != b
        assert np.all(np.abs(b[moved] - a[moved]) <= np.spacing(np.abs(a[moved])) * 1.0000001)
    a = np.asarray(c["phase_function_moments"])
    assert np.array_equal(np.asarray(p["phase_function_moments"])[..., 0], a[..., 0])
    assert p["single_scat_albedo"][0] <= 1.0 and p["single_scat_albedo"][1] == 0.0
    tot = workloads.column_total(p["delta_tau"])
    assert p["tau_user"][-1] == tot and p["tau_user"][1] == tot / 2.0
