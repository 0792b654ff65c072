"""Cycle accounting by phase of the flux boundary-value kernel (tracing build).

    python -m disort_b200.build --phase-clock
    python -m disort_b200.phase_profile [n_bands]

Solves the thermal sweep (20,000 bands x 60 layers x 16 streams by default)
twice through the tracing build of libdsp.so (lib/phase/libdsp.so) with device
pointers, and prints each phase's share of the boundary-value kernel's
warp-time and its cycles per instance.  The phases are the kernel's DSP_PHASE
markers (csrc/flux_bvp_reg.cuh): going down, per layer the new rows, per pivot
step the pivot search (with the previous step's row updates) and the pivot-row
broadcast, the last step's updates, the multiplier stores and the column phase;
going up, the wait for the records, the triangular solve, the next records'
prefetch and the fluxes.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

PHASES = [(0, "rows (new continuity / boundary rows)"), (7, "pivot search (+ previous step's updates)"),
          (8, "pivot row broadcast"), (1, "last step's updates"), (9, "multiplier stores"),
          (2, "column phase (x_{l+1} block, rhs)"), (4, "up: wait for records"), (5, "up: U x = c - V x_next"),
          (6, "up: record prefetch"), (3, "up: fluxes")]


def main(n_bands: int = 20000) -> None:
    import torch
    from disort_b200 import capi, workloads
    here = os.path.dirname(os.path.abspath(__file__))
    lib = capi.load_library(os.path.join(here, "lib", "phase", "libdsp.so"))
    capi._LIB = lib  # every context of this process uses the tracing build
    lib.dsp_phase_read.argtypes = [ctypes.c_void_p]
    w = workloads.thermal_sweep()
    if n_bands < w["n_inst"]:
        w = workloads.subset(w, np.arange(n_bands))
    n, L = w["n_inst"], w["num_layers"]
    ctx = capi.Context()
    arrays = {k: (None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda() if isinstance(a, np.ndarray)
                  else torch.tensor([float(a)], dtype=torch.float64, device="cuda")) for k, a in w["arrays"].items()}
    batch, keep = capi.make_flux_batch(n, w["num_streams"], L, w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | capi.FLAG_DEVICE_POINTERS, arrays)
    outs = {f: torch.empty((n, L + 1), dtype=torch.float64, device="cuda") for f in capi.FLUX_OUT_FIELDS}
    status = torch.empty(n, dtype=torch.int32, device="cuda")
    o, keep2 = capi.make_flux_out(outs, status)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    assert ctx.flux_bands_solve(batch, o) == 0
    torch.cuda.synchronize()
    lib.dsp_phase_reset()
    assert ctx.flux_bands_solve(batch, o) == 0
    torch.cuda.synchronize()
    buf = (ctypes.c_ulonglong * 16)()
    lib.dsp_phase_read(buf)
    v = np.array(list(buf)[:10], dtype=np.float64)
    tot = v.sum()
    print(f"flux boundary-value kernel, {n} bands x {L} layers x {w['num_streams']} streams: "
          f"{tot / n:,.0f} warp-cycles per instance")
    for k, name in PHASES:
        print(f"  {name:44s} {100.0 * v[k] / tot:6.2f} %  {v[k] / n:12,.0f} cycles/instance")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 20000)
