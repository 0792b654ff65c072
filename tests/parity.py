"""The parity criterion between the GPU engine and the oracle.

Fluxes and mean intensities must agree within 1e-9 relative with a 1e-12
absolute floor: |gpu - oracle| <= 1e-9 * |oracle| + 1e-12, element by element.
"""
import numpy as np

from disort_b200 import capi

RTOL = 1e-9
ATOL = 1e-12


def worst(gpu: dict, ref: dict) -> tuple[float, str]:
    """Largest |diff| / (RTOL*|ref| + ATOL) over all outputs (<= 1 passes)."""
    w, where = 0.0, ""
    for f in capi.FLUX_OUT_FIELDS:
        a, b = np.asarray(gpu[f]), np.asarray(ref[f])
        both_nan = np.isnan(a) & np.isnan(b)
        r = np.where(both_nan, 0.0, np.abs(a - b) / (RTOL * np.abs(b) + ATOL))
        r = np.where(np.isnan(r), np.inf, r)
        k = float(r.max()) if r.size else 0.0
        if k > w:
            idx = np.unravel_index(int(np.argmax(r)), r.shape)
            w, where = k, f"{f}{tuple(int(x) for x in idx)} gpu={a[idx]!r} ref={b[idx]!r}"
    return w, where


def assert_parity(gpu: dict, ref: dict, label: str = ""):
    w, where = worst(gpu, ref)
    assert w <= 1.0, f"{label}: parity ratio {w:.3g} at {where}"
    return w


GENERAL_FIELDS = capi.FLUX_OUT_FIELDS + ("intensity", "intensity_azimuth_avg")


def worst_general(gpu: dict, ref: dict, rtol: float = RTOL, atol: float = ATOL) -> tuple[float, str]:
    """parity ratio of a general solve: fluxes element-wise as worst(); each
    instance's intensities against the largest |intensity| of that instance
    (the Fourier sum cancels, so single elements can be near zero)."""
    w, where = 0.0, ""
    for f in GENERAL_FIELDS:
        if f not in ref:  # a fluxes-only comparison
            continue
        a, b = np.asarray(gpu[f]), np.asarray(ref[f])
        if b.size == 0:
            continue
        if f.startswith("intensity"):
            flat = np.abs(np.where(np.isnan(b), 0.0, b)).reshape(b.shape[0], -1)
            scale = flat.max(axis=1).reshape((-1,) + (1,) * (b.ndim - 1))
            denom = rtol * np.maximum(np.abs(b), scale) + atol
        else:
            denom = rtol * np.abs(b) + atol
        both_nan = np.isnan(a) & np.isnan(b)
        r = np.where(both_nan, 0.0, np.abs(a - b) / denom)
        r = np.where(np.isnan(r), np.inf, r)
        k = float(r.max()) if r.size else 0.0
        if k > w:
            idx = np.unravel_index(int(np.argmax(r)), r.shape)
            w, where = k, f"{f}{tuple(int(x) for x in idx)} gpu={a[idx]!r} ref={b[idx]!r}"
    return w, where


def assert_parity_general(gpu: dict, ref: dict, label: str = "", rtol: float = RTOL, atol: float = ATOL):
    w, where = worst_general(gpu, ref, rtol, atol)
    assert w <= 1.0, f"{label}: parity ratio {w:.3g} at {where}"
    return w
