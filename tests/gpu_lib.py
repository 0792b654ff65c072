"""Calls into libdsp.so through its C ABI (ctypes), for the GPU parity tests."""
from __future__ import annotations

import numpy as np

from disort_b200 import capi

_CTX = None


def context() -> capi.Context:
    global _CTX
    if _CTX is None:
        _CTX = capi.Context(0)
    return _CTX


def flux_solve(w: dict, extra_flags: int = 0):
    """Host-pointer solve of workload `w`: returns (outputs dict, status, return code)."""
    ctx = context()
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags, w["arrays"])
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    o, keep2 = capi.make_flux_out(outs, status)
    rc = ctx.flux_bands_solve(batch, o)
    return outs, status, rc


def flux_solve_jac(w: dict, extra_flags: int = 0):
    """Host-pointer solve with temperature Jacobians: (outputs, status, jacobians, rc)."""
    ctx = context()
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags, w["arrays"])
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    o, keep2 = capi.make_flux_out(outs, status)
    jac = capi.alloc_flux_jac_numpy(w["n_inst"], w["num_layers"])
    jo, keep3 = capi.make_flux_jac_out(jac)
    rc = ctx.flux_bands_solve_jac(batch, o, jo)
    return outs, status, jac, rc


def flux_solve_jac_device(w: dict, extra_flags: int = 0):
    """Device-pointer solve with temperature Jacobians (torch CUDA tensors in and out)."""
    import torch
    ctx = context()
    dev_arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            dev_arrays[k] = None
        elif isinstance(a, np.ndarray):
            dev_arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        else:
            dev_arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device="cuda")
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags | capi.FLAG_DEVICE_POINTERS, dev_arrays)
    n, L = w["n_inst"], w["num_layers"]
    outs = {f: torch.full((n, L + 1), float("nan"), dtype=torch.float64, device="cuda")
            for f in capi.FLUX_OUT_FIELDS}
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    o, keep2 = capi.make_flux_out(outs, status)
    jac = {f: torch.full((n, L + 1, L + 2), float("nan"), dtype=torch.float64, device="cuda")
           for f in capi.JAC_FIELDS}
    jo, keep3 = capi.make_flux_jac_out(jac)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    rc = ctx.flux_bands_solve_jac(batch, o, jo)
    torch.cuda.synchronize()
    return ({k: v.cpu().numpy() for k, v in outs.items()}, status.cpu().numpy(),
            {k: v.cpu().numpy() for k, v in jac.items()}, rc)


def flux_solve_device(w: dict, extra_flags: int = 0):
    """Device-pointer solve (torch CUDA tensors in and out)."""
    import torch
    ctx = context()
    dev_arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            dev_arrays[k] = None
        elif isinstance(a, np.ndarray):
            dev_arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        else:
            dev_arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device="cuda")
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"],
                                       w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | extra_flags | capi.FLAG_DEVICE_POINTERS, dev_arrays)
    n, L = w["n_inst"], w["num_layers"]
    outs = {f: torch.full((n, L + 1), float("nan"), dtype=torch.float64, device="cuda")
            for f in capi.FLUX_OUT_FIELDS}
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    o, keep2 = capi.make_flux_out(outs, status)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    rc = ctx.flux_bands_solve(batch, o)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}, status.cpu().numpy(), rc


def general_solve(d: dict):
    """Host-pointer general solve of a pack_general dict: (outputs dict, return code)."""
    ctx = context()
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    rc = ctx.general_bands_solve(batch, o)
    return outs, rc


def general_solve_device(d: dict):
    """Device-pointer general solve: every batch array and output is a CUDA tensor."""
    import torch
    ctx = context()
    dd = dict(d)
    keep = []
    for k in ("num_streams", "num_layers", "layer_offset", "num_phase_func_moments", "delta_tau",
              "single_scat_albedo", "phase_function_moments", "temperature", "level_altitudes",
              "bottom_radius", "brdf_params", "phase_function") + capi.GENERAL_SCALAR_FIELDS:
        if k in d:
            dd[k] = torch.from_numpy(np.ascontiguousarray(d[k])).cuda()
    for k in ("tau_user", "mu_user", "phi_user", "mu_phase_function"):
        if k in d:
            a, stride = d[k]
            dd[k] = (torch.from_numpy(np.ascontiguousarray(a)).cuda(), stride)
    dd["flags"] = d["flags"] | capi.FLAG_DEVICE_POINTERS
    batch, keep = capi.make_general_batch(dd)
    n, nt, nu, nphi = d["n_inst"], d["ntau_out"], d["numu_out"], max(d["num_phi"], 0)
    outs = {f: torch.full((n, nt), float("nan"), dtype=torch.float64, device="cuda") for f in capi.FLUX_OUT_FIELDS}
    outs["intensity"] = torch.full((n, nt, nu, nphi), float("nan"), dtype=torch.float64, device="cuda")
    outs["intensity_azimuth_avg"] = torch.full((n, nt, nu), float("nan"), dtype=torch.float64, device="cuda")
    outs["status"] = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    o = capi.GeneralOut()
    import ctypes
    for k, f in enumerate(capi.FLUX_OUT_FIELDS):
        o.flux[k] = ctypes.cast(ctypes.c_void_p(outs[f].data_ptr()), ctypes.POINTER(ctypes.c_double))
    o.intensity = ctypes.cast(ctypes.c_void_p(outs["intensity"].data_ptr()), ctypes.POINTER(ctypes.c_double))
    o.intensity_azimuth_avg = ctypes.cast(ctypes.c_void_p(outs["intensity_azimuth_avg"].data_ptr()),
                                          ctypes.POINTER(ctypes.c_double))
    o.status = ctypes.cast(ctypes.c_void_p(outs["status"].data_ptr()), ctypes.POINTER(ctypes.c_int32))
    o.ntau_out, o.numu_out = nt, nu
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    rc = ctx.general_bands_solve(batch, o)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}, rc
