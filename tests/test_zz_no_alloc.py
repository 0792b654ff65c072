"""The allocation-free flux entry point, dsp_flux_bands_solve_noalloc.

Callers that cannot let a library allocate GPU memory (an application that owns
every byte of the device through its own pool, or one that forbids allocation
once it is running) use this entry point: its workspace is a fixed 32 MiB array
inside libdsp.so instead of memory obtained with cudaMalloc.  The test calls it
through the C ABI twice in a row on the same device buffers -- the array keeps
the previous call's contents, so the second call must not depend on them -- and
checks both results against the regular entry point, dsp_flux_bands_solve, at the
parity tolerance used by every other test (1e-9 relative, 1e-12 absolute).

This file is collected last on purpose, and it also passes when run alone.
"""
import ctypes

import numpy as np
import pytest

from disort_b200 import capi, workloads
from parity import assert_parity

pytestmark = pytest.mark.gpu


def _device_batch(w, torch):
    arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            arrays[k] = None
        elif isinstance(a, np.ndarray):
            arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        else:
            arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device="cuda")
    return capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"], w["num_phase_func_moments"],
                                w["pmom_count"], w["flags"] | capi.FLAG_DEVICE_POINTERS, arrays)


def _device_out(n, L, torch, with_status=True):
    outs = {f: torch.full((n, L + 1), float("nan"), dtype=torch.float64, device="cuda")
            for f in capi.FLUX_OUT_FIELDS}
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda") if with_status else None
    o, keep = capi.make_flux_out(outs, status)
    return outs, status, o, keep


def _compare_with_regular(w, calls, with_status=True):
    """Solve `w` with dsp_flux_bands_solve, then `calls` times with the no-alloc
    entry point on fresh outputs, each checked against the first result."""
    import torch
    lib = capi.load_library()
    n, L = w["n_inst"], w["num_layers"]
    batch, keep = _device_batch(w, torch)
    stream = torch.cuda.current_stream()
    ctx = capi.Context(0, stream.cuda_stream)
    ref, ref_status, o_ref, k1 = _device_out(n, L, torch)
    assert ctx.flux_bands_solve(batch, o_ref) == capi.DSP_OK, ctx.last_error()
    torch.cuda.synchronize()
    ref_np = {f: v.cpu().numpy() for f, v in ref.items()}
    assert int((ref_status != 0).sum()) == 0
    for call in range(calls):
        got, got_status, o_got, k2 = _device_out(n, L, torch, with_status)
        rc = lib.dsp_flux_bands_solve_noalloc(ctypes.byref(batch), ctypes.byref(o_got),
                                              ctypes.c_void_p(stream.cuda_stream))
        assert rc == capi.DSP_OK
        torch.cuda.synchronize()
        if with_status:
            assert int((got_status != 0).sum()) == 0
        assert_parity({f: v.cpu().numpy() for f, v in got.items()}, ref_np,
                      f"no-alloc N={w['num_streams']} call {call + 1}")
    ctx.close()


def test_noalloc_matches_regular_entry_point_twice():
    # 600 bands of the 60-layer thermal sweep: more than one pass through the 32 MiB array
    w = workloads.subset(workloads.thermal_sweep(), np.arange(0, 20000, 33)[:600])
    _compare_with_regular(w, calls=2)


def _deep_beam_column(N, L, n, seed):
    rng = np.random.default_rng(seed)
    pc = N + 2
    g = rng.uniform(0.5, 0.9, (n, L))
    return dict(name=f"deep_beam_N{N}", n_inst=n, num_streams=N, num_layers=L, num_phase_func_moments=N + 1,
                pmom_count=pc, flags=capi.FLAG_DELTA_M_PLUS,
                arrays=dict(delta_tau=np.clip(rng.lognormal(-3, 2, (n, L)), 1e-6, 50),
                            single_scat_albedo=rng.uniform(0, 0.99, (n, L)),
                            phase_function_moments=np.stack([workloads.hg_moments(g[i], pc) for i in range(n)]),
                            surface_albedo=rng.uniform(0, 0.6, n), direct_beam_flux=1.0,
                            direct_beam_mu=rng.uniform(0.1, 1.0, n)))


def test_noalloc_tile_path_in_several_launches():
    # 64 streams x 100 layers: about 10 MB of workspace per instance, three fit in
    # the array, so seven instances take three launches (the 32/64-stream kernels,
    # whose shared-memory attribute this entry point sets itself)
    _compare_with_regular(_deep_beam_column(64, 100, 7, seed=11), calls=2)
    # 32 streams, 90 layers, 20 instances: two launches
    _compare_with_regular(_deep_beam_column(32, 90, 20, seed=12), calls=1)


def test_noalloc_without_status_array():
    # out->status == NULL: the status words live in the array itself
    w = workloads.subset(workloads.thermal_sweep(), np.arange(0, 20000, 97)[:120])
    _compare_with_regular(w, calls=2, with_status=False)


def test_noalloc_rejects_instances_larger_than_its_array():
    import torch
    lib = capi.load_library()
    assert lib.dsp_noalloc_scratch_bytes() == 32 << 20
    # one 64-stream instance with 600 layers needs about 61 MB of workspace: refused before any launch
    N, L = 64, 600
    pc = N + 1
    w = dict(n_inst=1, num_streams=N, num_layers=L, num_phase_func_moments=0, pmom_count=pc, flags=0,
             arrays=dict(delta_tau=np.full(L, 0.01), single_scat_albedo=np.full(L, 0.5),
                         phase_function_moments=workloads.hg_moments(np.full(L, 0.5), pc),
                         direct_beam_flux=1.0, direct_beam_mu=0.5))
    batch, keep = _device_batch(w, torch)
    got, got_status, o_got, k2 = _device_out(1, L, torch)
    rc = lib.dsp_flux_bands_solve_noalloc(ctypes.byref(batch), ctypes.byref(o_got), None)
    assert rc == capi.DSP_ERR_NO_MEMORY
    # host pointers cannot be staged without allocating: refused
    hbatch, hkeep = workloads.make_batch(workloads.beam_sweep(8))
    rc = lib.dsp_flux_bands_solve_noalloc(ctypes.byref(hbatch), ctypes.byref(o_got), None)
    assert rc == capi.DSP_ERR_INVALID_INPUT
