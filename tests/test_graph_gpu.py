"""A flux spectral loop captured as one CUDA graph (dsp_flux_graph_create):
replays re-read the device inputs and give the same outputs, bit for bit, as
direct solves of the same inputs."""
import numpy as np
import pytest

import gpu_lib
from disort_b200 import capi, workloads

pytestmark = pytest.mark.gpu


def _device(w):
    import torch
    arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            arrays[k] = None
        elif isinstance(a, np.ndarray):
            arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).cuda()
        else:
            arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device="cuda")
    n, L = w["n_inst"], w["num_layers"]
    batch, keep = capi.make_flux_batch(n, w["num_streams"], L, w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | capi.FLAG_DEVICE_POINTERS, arrays)
    outs = {f: torch.full((n, L + 1), float("nan"), dtype=torch.float64, device="cuda") for f in capi.FLUX_OUT_FIELDS}
    status = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    out, keep2 = capi.make_flux_out(outs, status)
    return batch, out, arrays, outs, status, (keep, keep2)


@pytest.mark.parametrize("kind", ["beam", "thermal"])
def test_graph_replay_matches_direct_solves(kind):
    import torch
    w = workloads.beam_sweep(1024) if kind == "beam" else workloads.subset(workloads.thermal_sweep(),
                                                                           np.arange(0, 20000, 20))
    batch, out, arrays, outs, status, keep = _device(w)
    ctx = gpu_lib.context()
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    assert ctx.flux_bands_solve(batch, out) == 0
    torch.cuda.synchronize()
    direct = {f: outs[f].clone() for f in outs}
    g = capi.FluxGraph(batch, out)
    try:
        for f in outs:
            outs[f].fill_(float("nan"))
        assert g.launch(stream.cuda_stream) == 0
        torch.cuda.synchronize()
        for f in outs:
            assert torch.equal(outs[f], direct[f]), f
        assert int((status != 0).sum()) == 0
        # new inputs in place: the replay solves them
        arrays["delta_tau"].mul_(1.37)
        assert g.launch(stream.cuda_stream) == 0
        torch.cuda.synchronize()
        replay = {f: outs[f].clone() for f in outs}
        assert ctx.flux_bands_solve(batch, out) == 0
        torch.cuda.synchronize()
        for f in outs:
            assert torch.equal(outs[f], replay[f]), f
        assert not torch.equal(replay["flux_up"], direct["flux_up"])
    finally:
        torch.cuda.synchronize()
        g.close()


def test_graph_rejects_host_pointers():
    w = workloads.beam_sweep(8)
    batch, keep = capi.make_flux_batch(w["n_inst"], w["num_streams"], w["num_layers"], w["num_phase_func_moments"],
                                       w["pmom_count"], w["flags"], w["arrays"])
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    out, keep2 = capi.make_flux_out(outs, status)
    with pytest.raises(RuntimeError, match="INVALID_INPUT"):
        capi.FluxGraph(batch, out)
