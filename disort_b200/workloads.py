"""Seeded synthetic spectral workloads (numpy PCG64 streams).

The reference publishes no benchmark data set for this path, so the sweeps are
synthetic inputs with fixed seeds; the GPU engine, the CPU oracle and the CPU
baseline all consume the same arrays.

``beam_sweep``     1,024 bands of 10 cm^-1 (100..10,340 cm^-1), 4 layers, N=16,
                   beam pi at mu0=0.5, HG g=0.8, albedo 0.1, no thermal (seed 1).
``thermal_sweep``  20,000 bands of 0.14 cm^-1 (100..2,900 cm^-1), 60 layers, N=16,
                   lognormal(-3,2) optical depths clipped to [1e-6, 50], ssa U[0,0.99],
                   HG g U[0,0.9], one 61-level temperature profile 180..320 K with
                   +-10 K noise, albedo 0.05, thermal emission on, no beam (seed 2).
``general_mix``    the general solver's mixed batch: 65,536 instances, N in
                   {4, 8, 16, 32, 64} (weights .1 .2 .4 .2 .1), L uniform in 10..120,
                   optical depths and ssa as the thermal sweep, HG g U[0.5, 0.95] with
                   N+1 moments and delta-M+, beam F0 = 1 at mu0 U[0.1, 1], albedo
                   U[0, 0.6], no thermal; user taus {0, tau/2, tau}, user mu
                   {-0.5, -0.1, 0.1, 0.5, 1}, phi {0, 60, 120, 180}, all modes (seed 3).
"""
from __future__ import annotations

import numpy as np

from . import capi


def hg_moments(g: np.ndarray, count: int) -> np.ndarray:
    """Henyey-Greenstein moments g**k, k = 0..count-1 (PhaseFunction.cpp:6-19)."""
    g = np.asarray(g, dtype=np.float64)
    k = np.arange(count, dtype=np.float64)
    out = np.empty(g.shape + (count,), dtype=np.float64)
    out[..., 0] = 1.0
    for i in range(1, count):
        out[..., i] = out[..., i - 1] * g
    del k
    return out


def beam_sweep(n_bands: int = 1024, seed: int = 1) -> dict:
    rng = np.random.default_rng(seed)
    N, L = 16, 4
    lo = 100.0 + 10.0 * np.arange(n_bands)
    hi = lo + 10.0
    factor = rng.lognormal(0.0, 1.0, size=n_bands)
    base = np.array([0.1, 0.5, 1.0, 2.0])
    dtau = factor[:, None] * base[None, :]
    ssa = np.full(L, 0.9)
    pc = N + 1  # nmomNstr()+1 with nmom = 0
    pmom = hg_moments(np.full(L, 0.8), pc)
    return dict(
        name="beam_sweep_1024x4L_16str",
        n_inst=n_bands, num_streams=N, num_layers=L, num_phase_func_moments=0, pmom_count=pc,
        flags=0,
        arrays=dict(
            wavenumber_low=lo, wavenumber_high=hi, delta_tau=dtau, single_scat_albedo=ssa,
            phase_function_moments=pmom, surface_albedo=0.1, emissivity_top=1.0,
            direct_beam_flux=np.pi, direct_beam_mu=0.5, isotropic_flux_top=0.0,
            isotropic_flux_bottom=0.0, temperature_top=0.0, temperature_bottom=0.0,
        ),
    )


def thermal_sweep(n_bands: int = 20000, num_layers: int = 60, num_streams: int = 16, seed: int = 2) -> dict:
    rng = np.random.default_rng(seed)
    N, L = num_streams, num_layers
    lo = 100.0 + 0.14 * np.arange(n_bands)
    hi = 100.0 + 0.14 * (np.arange(n_bands) + 1)
    dtau = np.clip(rng.lognormal(-3.0, 2.0, size=(n_bands, L)), 1e-6, 50.0)
    ssa = rng.uniform(0.0, 0.99, size=(n_bands, L))
    g = rng.uniform(0.0, 0.9, size=(n_bands, L))
    lev = np.arange(L + 1, dtype=np.float64)
    temp = 180.0 + 140.0 * lev / L + rng.uniform(-10.0, 10.0, size=L + 1)
    pc = N + 1
    pmom = hg_moments(g, pc)
    return dict(
        name=f"thermal_sweep_{n_bands}x{L}L_{N}str",
        n_inst=n_bands, num_streams=N, num_layers=L, num_phase_func_moments=0, pmom_count=pc,
        flags=capi.FLAG_THERMAL, hg_g=g,
        arrays=dict(
            wavenumber_low=lo, wavenumber_high=hi, delta_tau=dtau, single_scat_albedo=ssa,
            phase_function_moments=pmom, temperature=temp, surface_albedo=0.05,
            emissivity_top=1.0, direct_beam_flux=0.0, direct_beam_mu=0.5,
            isotropic_flux_top=0.0, isotropic_flux_bottom=0.0, temperature_top=0.0,
            temperature_bottom=float(temp[-1]),
        ),
    )


def subset(w: dict, idx) -> dict:
    """The same workload restricted to instances `idx` (per-instance arrays sliced)."""
    idx = np.asarray(idx)
    n = w["n_inst"]
    out = dict(w)
    out["n_inst"] = int(idx.size)
    arrs = {}
    per_ndim = {"delta_tau": 1, "single_scat_albedo": 1, "phase_function_moments": 2, "temperature": 1,
                "level_altitudes": 1}
    for k, a in w["arrays"].items():
        if isinstance(a, np.ndarray):
            nd = per_ndim.get(k, 0)
            if a.ndim == nd + 1 and a.shape[0] == n and not (nd == 0 and n == 1):
                arrs[k] = np.ascontiguousarray(a[idx])
                continue
        arrs[k] = a
    out["arrays"] = arrs
    if isinstance(w.get("hg_g"), np.ndarray) and w["hg_g"].shape[0] == n:
        out["hg_g"] = np.ascontiguousarray(w["hg_g"][idx])
    return out


def as_hg(w: dict) -> dict:
    """The same workload through the Henyey-Greenstein fast path (DSP_FLAG_HG_G):
    one asymmetry factor per layer instead of the moments g**k."""
    out = dict(w)
    out["flags"] = w["flags"] | capi.FLAG_HG_G
    arrs = dict(w["arrays"])
    arrs["phase_function_moments"] = w["hg_g"]
    out["arrays"] = arrs
    out["name"] = w["name"] + "_hg"
    return out


def make_batch(w: dict, extra_flags: int = 0):
    return capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                w["num_phase_func_moments"], w["pmom_count"],
                                w["flags"] | extra_flags, w["arrays"])


GENERAL_NSTR = (4, 8, 16, 32, 64)
GENERAL_NSTR_WEIGHTS = (0.1, 0.2, 0.4, 0.2, 0.1)
GENERAL_MU = (-0.5, -0.1, 0.1, 0.5, 1.0)
GENERAL_PHI = (0.0, 60.0, 120.0, 180.0)


def column_total(dtau) -> float:
    """Total optical depth of a column as a user output depth: the smaller of
    the sequential top-down and bottom-up sums of delta_tau.  The solver sums
    the layers in its own (top-down) order, and with bottom-up indexing a user
    depth d becomes total - d, so a depth one rounding above either sum would
    fall outside the column."""
    down = up = 0.0
    for x in np.asarray(dtau, dtype=np.float64):
        down += float(x)
    for x in np.asarray(dtau, dtype=np.float64)[::-1]:
        up += float(x)
    return min(down, up)


def general_mix(n_inst: int = 65536, seed: int = 3, nstr=None, layers=(10, 120)) -> tuple[list, int]:
    """Instances of the general solver's mixed batch and its flags.

    `nstr` restricts the stream counts (same weights, renormalised); `layers` is
    the inclusive range of the uniform layer count."""
    rng = np.random.default_rng(seed)
    Ns = np.array(GENERAL_NSTR if nstr is None else nstr)
    w = np.array([GENERAL_NSTR_WEIGHTS[GENERAL_NSTR.index(x)] for x in Ns])
    w = w / w.sum()
    Nv = rng.choice(Ns, size=n_inst, p=w)
    Lv = rng.integers(layers[0], layers[1] + 1, size=n_inst)
    insts = []
    for k in range(n_inst):
        N, L = int(Nv[k]), int(Lv[k])
        dtau = np.clip(rng.lognormal(-3.0, 2.0, L), 1e-6, 50.0)
        g = rng.uniform(0.5, 0.95, L)
        tot = column_total(dtau)
        insts.append(dict(
            num_streams=N, num_layers=L, num_phase_func_moments=N + 1,
            delta_tau=dtau, single_scat_albedo=rng.uniform(0.0, 0.99, L),
            phase_function_moments=hg_moments(g, N + 2),
            direct_beam_flux=1.0, direct_beam_mu=float(rng.uniform(0.1, 1.0)), direct_beam_phi=0.0,
            surface_albedo=float(rng.uniform(0.0, 0.6)),
            tau_user=[0.0, tot / 2.0, tot], mu_user=list(GENERAL_MU), phi_user=list(GENERAL_PHI)))
    flags = capi.FLAG_DELTA_M_PLUS | capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU
    return insts, flags
