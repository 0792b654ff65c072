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
