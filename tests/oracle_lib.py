"""Loader of the CPU oracle library (oracle/liboracle_disort.so) for tests.

The oracle is the checker: tests call it on the same dsp_flux_batch that the
GPU library receives and compare outputs.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int

import numpy as np

from disort_b200 import capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
_LIBS = {}


def load(native: bool = False, ext: bool = False):
    """Load (building if needed) the oracle shared library: the portable build,
    the -march=native build (native=True) or the extended-precision build
    (ext=True: x87 intermediates, the checker for ill-conditioned cases)."""
    key = "native" if native else ("ext" if ext else "all")
    if key in _LIBS and not native:
        return _LIBS[key]
    path = {"native": os.path.join(ORACLE_DIR, "_native", "liboracle_disort.so"),
            "ext": os.path.join(ORACLE_DIR, "liboracle_disort_ext.so"),
            "all": os.path.join(ORACLE_DIR, "liboracle_disort.so")}[key]
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, key], check=True)
    lib = ctypes.CDLL(path)
    lib.oracle_flux_bands_solve.restype = c_int
    lib.oracle_flux_bands_solve.argtypes = [POINTER(capi.FluxBatch), POINTER(capi.FluxOut), c_int]
    lib.oracle_quadrature.restype = c_int
    lib.oracle_quadrature.argtypes = [c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double)]
    lib.oracle_planck.restype = c_double
    lib.oracle_planck.argtypes = [c_double, c_double, c_double]
    lib.oracle_flux_bands_solve_jac.restype = c_int
    lib.oracle_flux_bands_solve_jac.argtypes = [POINTER(capi.FluxBatch), POINTER(capi.FluxOut),
                                                POINTER(capi.FluxJacOut), c_int]
    lib.oracle_general_bands_solve_jac.restype = c_int
    lib.oracle_general_bands_solve_jac.argtypes = [POINTER(capi.GeneralBatch), POINTER(capi.GeneralOut),
                                                   POINTER(capi.GeneralJacOut), c_int]
    lib.oracle_general_bands_solve.restype = c_int
    lib.oracle_general_bands_solve.argtypes = [POINTER(capi.GeneralBatch), POINTER(capi.GeneralOut), c_int]
    if not native:
        _LIBS[key] = lib
    return lib


def flux_solve(w: dict, nthreads: int = 0, extra_flags: int = 0, ext: bool = False):
    """Run the oracle on workload dict `w`; returns (outputs dict, status array)."""
    lib = load(ext=ext)
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags, w["arrays"])
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    o, keep2 = capi.make_flux_out(outs, status)
    lib.oracle_flux_bands_solve(ctypes.byref(batch), ctypes.byref(o), nthreads)
    return outs, status


def flux_solve_jac(w: dict, nthreads: int = 0, extra_flags: int = 0, ext: bool = False):
    """Flux solve with temperature Jacobians: (outputs, status, jacobians)."""
    lib = load(ext=ext)
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags, w["arrays"])
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    o, keep2 = capi.make_flux_out(outs, status)
    jac = capi.alloc_flux_jac_numpy(w["n_inst"], w["num_layers"])
    jo, keep3 = capi.make_flux_jac_out(jac)
    lib.oracle_flux_bands_solve_jac(ctypes.byref(batch), ctypes.byref(o), ctypes.byref(jo), nthreads)
    return outs, status, jac


def general_solve(d: dict, nthreads: int = 0, ext: bool = False):
    """Run the general oracle on a pack_general dict; returns the outputs dict."""
    lib = load(ext=ext)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    lib.oracle_general_bands_solve(ctypes.byref(batch), ctypes.byref(o), nthreads)
    return outs


def general_solve_jac(d: dict, nthreads: int = 0, ext: bool = False):
    """General solve with temperature Jacobians: (outputs, jacobians)."""
    lib = load(ext=ext)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    jac, jo, keep3 = capi.alloc_general_jac_numpy(d)
    lib.oracle_general_bands_solve_jac(ctypes.byref(batch), ctypes.byref(o), ctypes.byref(jo), nthreads)
    return outs, jac


def general_albtrans(d: dict, nthreads: int = 0, ext: bool = False):
    """ibcnd = Special through the oracle: albedo/transmissivity outputs dict."""
    lib = load(ext=ext)
    lib.oracle_general_bands_albtrans.restype = c_int
    lib.oracle_general_bands_albtrans.argtypes = [POINTER(capi.GeneralBatch), POINTER(capi.AlbTransOut), c_int]
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_albtrans_numpy(d)
    lib.oracle_general_bands_albtrans(ctypes.byref(batch), ctypes.byref(o), nthreads)
    return outs
