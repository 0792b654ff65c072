"""GPU temperature Jacobians (dsp_flux_bands_solve_jac) against the oracle.

The oracle's analytic Jacobian is itself checked against finite differences of
the forward solve (test_jacobian_oracle.py, after the reference's
tests/test_jacobian.cpp).  Jacobian entries are derivatives formed with
cancellation (the flux divergence's, in particular, subtracts the Planck
derivative from the mean-intensity one): two builds of the same oracle source,
double and extended-precision intermediates, differ by up to 1.4e-8 of an
entry on thermal-sweep columns, and theoretically-zero entries (the downward
flux at the top) are rounding noise of the larger entries of their output.  So
every GPU entry must satisfy |gpu - oracle| <= 3e-8 * max(|oracle|, 1e-3 * s),
s the largest |entry| of that output's Jacobian in the instance -- the bound the
two oracle builds are held to (test_jacobian_oracle.py), and thirty times
tighter than the reference's own cross-solver Jacobian check (1e-6 relative,
test_jacobian.cpp:381-409).  The fluxes of the same call are held to the usual
1e-9 / 1e-12 parity.
"""
import numpy as np
import pytest

import gpu_lib
import oracle_lib
from disort_b200 import capi, workloads
from parity import assert_parity
from test_jacobian_oracle import thermal_column

pytestmark = pytest.mark.gpu

RTOL = 3e-8
FLOOR = 1e-3


def jac_ratio(got: dict, ref: dict) -> tuple[float, str]:
    worst, where = 0.0, ""
    for f in capi.JAC_FIELDS:
        a, b = got[f], ref[f]
        flat = np.abs(np.where(np.isnan(b), 0.0, b)).reshape(b.shape[0], -1)
        scale = flat.max(axis=1)[:, None, None]
        denom = RTOL * np.maximum(np.abs(b), FLOOR * scale) + 1e-300
        r = np.where(np.isnan(a) & np.isnan(b), 0.0, np.abs(a - b) / denom)
        r = np.where(np.isnan(r), np.inf, r)
        k = float(r.max())
        if k > worst:
            idx = np.unravel_index(int(np.argmax(r)), r.shape)
            worst, where = k, f"{f}{tuple(int(x) for x in idx)} gpu={a[idx]!r} ref={b[idx]!r}"
    return worst, where


def check(w, extra_flags=0, label=""):
    out, st, jac, rc = gpu_lib.flux_solve_jac(w, extra_flags)
    assert rc == 0, gpu_lib.context().last_error()
    rout, rst, rjac = oracle_lib.flux_solve_jac(w, extra_flags=extra_flags)
    assert np.all(st == rst)
    ok = st == 0
    assert_parity({k: v[ok] for k, v in out.items()}, {k: v[ok] for k, v in rout.items()}, label)
    r, where = jac_ratio(jac, rjac)
    assert r <= 1.0, f"{label}: Jacobian parity ratio {r:.3g} at {where}"
    return out, st, jac


@pytest.mark.parametrize("name,Tlev,Tsurf,nstr,ssa,beam", [
    ("flux_single_layer", [200.0, 260.0], 280.0, 8, 0.0, 0.0),
    ("flux_multilayer_scattering", [205.0 + 9.0 * i for i in range(9)], 290.0, 16, 0.7, 0.0),
    ("thermal_plus_beam", [200.0, 240.0, 270.0], 288.0, 16, 0.6, 1.0),
    ("four_streams", [220.0, 240.0, 260.0, 275.0], 285.0, 4, 0.4, 0.0),
    ("scattering_high_12", [210.0, 235.0, 255.0, 270.0, 280.0], 290.0, 12, 0.9, 0.0),
])
def test_reference_jacobian_problems(name, Tlev, Tsurf, nstr, ssa, beam):
    check(thermal_column(Tlev, Tsurf, nstr, ssa, beam), label=name)


@pytest.mark.parametrize("extra", [0, capi.FLAG_INDEX_FROM_BOTTOM, capi.FLAG_DIFFUSION_LOWER_BC,
                                   capi.FLAG_DELTA_M_PLUS])
def test_thermal_sweep_jacobians(extra):
    """Thermal-sweep columns (60 layers, 16 streams), also bottom-up, with the
    diffusion lower boundary, and delta-M+ (moments g^k: the global fallback
    keeps delta-M)."""
    w = workloads.subset(workloads.thermal_sweep(), np.arange(0, 20000, 800))
    check(w, extra, label=f"thermal sweep flags={extra}")


@pytest.mark.parametrize("nstr", [6, 10, 14, 32, 64])
def test_jacobians_other_stream_counts(nstr):
    w = workloads.thermal_sweep(n_bands=5, num_layers=30 if nstr < 64 else 20, num_streams=nstr, seed=80 + nstr)
    check(w, label=f"N={nstr}")


def test_deep_column_more_degrees_of_freedom_than_a_pass():
    """90 layers: 92 degrees of freedom, two passes of the 64-thread Jacobian CTA."""
    w = workloads.thermal_sweep(n_bands=3, num_layers=90, num_streams=8, seed=91)
    check(w, label="L=90")


def test_jacobian_device_pointers_equal_host_pointers_and_edge_cases():
    w = workloads.subset(workloads.thermal_sweep(), np.arange(0, 20000, 1000))
    w["arrays"]["single_scat_albedo"] = w["arrays"]["single_scat_albedo"].copy()
    w["arrays"]["single_scat_albedo"][3, 7] = 1.5  # invalid instance: NaN Jacobian
    out, st, jac = check(w, label="with an invalid instance")
    assert st[3] == capi.DSP_ERR_INVALID_INPUT and np.all(np.isnan(jac["flux_up"][3]))
    dout, dst, djac, rc = gpu_lib.flux_solve_jac_device(w)
    assert rc == 0
    for f in capi.JAC_FIELDS:
        np.testing.assert_array_equal(jac[f], djac[f])
    # without thermal emission the Jacobians are zero
    w2 = workloads.beam_sweep(16)
    out, st, jac, rc = gpu_lib.flux_solve_jac(w2)
    assert rc == 0 and not st.any()
    for f in capi.JAC_FIELDS:
        assert np.all(jac[f] == 0.0)
    # the plain entry point rejects the Jacobian flag
    _, _, rc = gpu_lib.flux_solve(w, extra_flags=capi.FLAG_TEMPERATURE_JAC)
    assert rc == capi.DSP_ERR_UNSUPPORTED


def test_jacobians_with_spherical_beam():
    """Thermal Jacobians are unchanged in form under the pseudo-spherical beam
    (its source does not depend on temperature)."""
    from test_flux_gpu import spherical_columns
    check(spherical_columns(16, 20, 6, seed=77, thermal=True), label="spherical + thermal")


# ---------------------------------------------------------------------------
# general path (dsp_general_bands_solve_jac, DisortSolver)
# ---------------------------------------------------------------------------
def general_check(insts, flags, label, accuracy=0.0):
    d = capi.pack_general(insts, flags, accuracy_fourier_series=accuracy)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    jac, jo, keep3 = capi.alloc_general_jac_numpy(d)
    rc = gpu_lib.context().general_bands_solve_jac(batch, o, jo)
    assert rc == 0, gpu_lib.context().last_error()
    rout, rjac = oracle_lib.general_solve_jac(d)
    assert np.all(outs["status"] == rout["status"])
    from parity import assert_parity_general
    ok = outs["status"] == 0
    assert_parity_general({k: v[ok] for k, v in outs.items() if k != "status"},
                          {k: v[ok] for k, v in rout.items() if k != "status"}, label)
    # compare each instance's own columns (L_i + 2) and rows
    for i in np.nonzero(ok)[0]:
        L = insts[i]["num_layers"]
        nt = d["num_user_tau"] if flags & capi.GFLAG_USER_TAU else L + 1
        got = {f: jac[f][i:i + 1, :nt, :L + 2] for f in capi.JAC_FIELDS}
        ref = {f: rjac[f][i:i + 1, :nt, :L + 2] for f in capi.JAC_FIELDS}
        r, where = jac_ratio(got, ref)
        assert r <= 1.0, f"{label} instance {i}: Jacobian parity ratio {r:.3g} at {where}"
    return outs, jac


def general_thermal_mix(n, seed, nstr=(4, 8, 16, 32), user_tau=True):
    rng = np.random.default_rng(seed)
    insts = []
    for k in range(n):
        N = nstr[k % len(nstr)]
        L = int(rng.integers(3, 25 if N < 32 else 12))
        g = rng.uniform(0.0, 0.9, L)
        dtau = np.clip(rng.lognormal(-2.0, 1.5, L), 1e-6, 20.0)
        inst = dict(num_streams=N, num_layers=L, num_phase_func_moments=0, delta_tau=dtau,
                    single_scat_albedo=rng.uniform(0.0, 0.95, L), phase_function_moments=workloads.hg_moments(g, N + 1),
                    temperature=200.0 + 100.0 * rng.random(L + 1), wavenumber_low=float(rng.uniform(300, 1500)),
                    surface_albedo=float(rng.uniform(0, 0.5)), temperature_bottom=300.0, temperature_top=50.0,
                    emissivity_top=0.9, direct_beam_flux=float(rng.uniform(0, 1)), direct_beam_mu=0.6,
                    mu_user=[-0.7, -0.2, 0.3, 0.9], phi_user=[0.0, 45.0])
        inst["wavenumber_high"] = inst["wavenumber_low"] * 1.02
        if user_tau:
            tot = workloads.column_total(dtau)
            inst["tau_user"] = [0.0, 0.37 * tot, tot]
        insts.append(inst)
    return insts


@pytest.mark.parametrize("extra", [0, capi.FLAG_INDEX_FROM_BOTTOM, capi.FLAG_DIFFUSION_LOWER_BC])
def test_general_jacobians_ragged_batch(extra):
    """A ragged batch of thermal (and beam) instances at 4-32 streams, outputs
    at user optical depths inside layers, intensities on (all azimuth modes
    run; the Jacobians come from mode 0)."""
    insts = general_thermal_mix(12, seed=90 + extra)
    general_check(insts, capi.FLAG_THERMAL | capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU | extra,
                  f"general Jacobians flags={extra}")


def test_general_jacobians_at_levels_and_64_streams():
    insts = general_thermal_mix(4, seed=95, nstr=(64, 8), user_tau=False)
    general_check(insts, capi.FLAG_THERMAL | capi.GFLAG_ONLY_FLUXES, "general Jacobians at the levels")
