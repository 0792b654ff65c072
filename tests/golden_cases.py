"""Helpers that turn tests/golden/reference_goldens.json cases into flux batches."""
from __future__ import annotations

import json
import os

import numpy as np

from disort_b200 import capi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_goldens.json")


def load_cases() -> list:
    """The plane-parallel cases over a Lambertian surface (every solver path supports them)."""
    with open(GOLDEN) as f:
        return [c for c in json.load(f)["cases"]
                if not c.get("use_spherical_beam") and not c.get("brdf_type") and not c.get("intensity_corrected")
                and not c.get("special_bc")]


def load_special_cases() -> list:
    """The ibcnd = Special cases (albedo and transmissivity of the medium)."""
    with open(GOLDEN) as f:
        return [c for c in json.load(f)["cases"] if c.get("special_bc")]


def load_corrected_cases(engine_only: bool = False) -> list:
    """Lambertian cases run with the Nakajima-Tanaka intensity correction (general
    solver only); engine_only drops stream counts the engine does not take."""
    with open(GOLDEN) as f:
        cases = [c for c in json.load(f)["cases"] if c.get("intensity_corrected") and not c.get("brdf_type")]
    return [c for c in cases if not engine_only or c["num_streams"] in (4, 6, 8, 10, 12, 14, 16, 32, 64)]


def load_brdf_cases() -> list:
    """The cases over a bidirectional surface (general solver only)."""
    with open(GOLDEN) as f:
        return [c for c in json.load(f)["cases"] if c.get("brdf_type")]


def load_spherical_cases() -> list:
    """The pseudo-spherical beam cases (flux path)."""
    with open(GOLDEN) as f:
        return [c for c in json.load(f)["cases"] if c.get("use_spherical_beam")]


def flux_workload(c: dict) -> dict:
    L = c["num_layers"]
    pm = np.array(c["phase_function_moments"], dtype=np.float64)
    flags = 0
    if c["use_thermal_emission"]:
        flags |= capi.FLAG_THERMAL
    if c["use_delta_m_plus"]:
        flags |= capi.FLAG_DELTA_M_PLUS
    arrays = dict(
        wavenumber_low=c["wavenumber_low"], wavenumber_high=c["wavenumber_high"],
        delta_tau=np.array(c["delta_tau"], dtype=np.float64),
        single_scat_albedo=np.array(c["single_scat_albedo"], dtype=np.float64),
        phase_function_moments=pm,
        temperature=np.array(c["temperature"], dtype=np.float64) if c["use_thermal_emission"] else None,
        surface_albedo=c["surface_albedo"], emissivity_top=c["emissivity_top"],
        direct_beam_flux=c["direct_beam_flux"], direct_beam_mu=c["direct_beam_mu"],
        isotropic_flux_top=c["isotropic_flux_top"], isotropic_flux_bottom=0.0,
        temperature_top=c["temperature_top"], temperature_bottom=c["temperature_bottom"],
    )
    if c.get("use_spherical_beam"):
        flags |= capi.FLAG_SPHERICAL_BEAM
        arrays["level_altitudes"] = np.array(c["level_altitudes"], dtype=np.float64)
        arrays["bottom_radius"] = c["bottom_radius"]
    return dict(name=c["name"], n_inst=1, num_streams=c["num_streams"], num_layers=L,
                num_phase_func_moments=c["num_phase_func_moments"], pmom_count=pm.shape[1],
                flags=flags, arrays=arrays)


def level_of(c: dict, index: int):
    """Output level of expectation `index` (a user-tau index when tau_user is set)."""
    if c["tau_user"] is None:
        return index
    tau = c["tau_user"][index]
    cum = np.concatenate([[0.0], np.cumsum(c["delta_tau"])])
    hit = np.nonzero(np.abs(cum - tau) <= 1e-9 * max(1.0, abs(tau)))[0]
    return int(hit[0]) if hit.size else None


def general_instance(c: dict) -> tuple[dict, int]:
    """A golden case as one instance of the general batch, with its flags.

    Cases without user polar angles are fluxes-only runs (use_user_mu = false
    computes no intensities, so only the mode-0 fluxes are compared)."""
    flags = 0
    if c["use_thermal_emission"]:
        flags |= capi.FLAG_THERMAL
    if c["use_delta_m_plus"]:
        flags |= capi.FLAG_DELTA_M_PLUS
    inst = dict(
        num_streams=c["num_streams"], num_layers=c["num_layers"],
        num_phase_func_moments=c["num_phase_func_moments"],
        delta_tau=c["delta_tau"], single_scat_albedo=c["single_scat_albedo"],
        phase_function_moments=c["phase_function_moments"],
        temperature=c["temperature"] if c["use_thermal_emission"] else None,
        wavenumber_low=c["wavenumber_low"], wavenumber_high=c["wavenumber_high"],
        surface_albedo=c["surface_albedo"], emissivity_top=c["emissivity_top"],
        direct_beam_flux=c["direct_beam_flux"], direct_beam_mu=c["direct_beam_mu"],
        isotropic_flux_top=c["isotropic_flux_top"],
        temperature_top=c["temperature_top"], temperature_bottom=c["temperature_bottom"],
    )
    if c.get("intensity_corrected"):
        flags |= capi.GFLAG_INTENSITY_CORR
        if c.get("mu_phase_function"):  # a tabulated phase function: the Buras-Emde method
            flags |= capi.GFLAG_INTENSITY_CORR_BE
            inst["mu_phase_function"] = c["mu_phase_function"]
            inst["phase_function"] = c["phase_function"]
    if c.get("brdf_type"):
        inst["brdf_type"] = c["brdf_type"]
        inst["brdf_params"] = c["brdf_params"]
    if c.get("isotropic_flux_bottom"):
        inst["isotropic_flux_bottom"] = c["isotropic_flux_bottom"]
    if c["tau_user"] is not None:
        flags |= capi.GFLAG_USER_TAU
        inst["tau_user"] = c["tau_user"]
    if c["mu_user"] is not None:
        flags |= capi.GFLAG_USER_MU
        inst["mu_user"] = c["mu_user"]
        inst["phi_user"] = c["phi_user"]
    else:
        flags |= capi.GFLAG_ONLY_FLUXES
    return inst, flags
