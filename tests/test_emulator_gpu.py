"""GPU tests of the emulator's tensor-core kernels (libdsp_emu.so).

1. The tcgen05 BF16 GEMM against an FP64 product of the same BF16 operands.
2. One forward + backward pass against the CPU FP64 MLP oracle
   (oracle/mlp_oracle.py) on the same BF16 data and weights: every parameter
   block's gradient within 2e-2 relative Frobenius error (BF16 activations and
   gradients are re-rounded on both sides; the rest is accumulation order).
3. The training loop (fused loss gradient, tensor-core backward, fused Adam,
   cosine schedule) tracks a plain PyTorch FP32 run from the same initial weights.
4. A bounded device wait that runs out returns DSP_ERR_TIMEOUT to the host.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def torch_bf16(bits: np.ndarray):
    import torch
    return torch.from_numpy(bits.view(np.int16)).cuda().view(torch.bfloat16)


@pytest.fixture(scope="module")
def emu_small():
    from disort_b200.emu import Emulator
    e = Emulator(n_in=165, hidden=128, n_hidden_layers=2, n_out=82, n_heads=2, batch=256, seed=3)
    yield e
    e.close()


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (256, 192, 192), (384, 512, 512), (200, 128, 136)])
def test_tc_gemm_matches_fp64(emu_small, M, N, K):
    import torch
    rng = np.random.default_rng(M + N + K)
    a = rng.standard_normal((M, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    A, B = torch_bf16(mlp_oracle.bf16_bits(a)), torch_bf16(mlp_oracle.bf16_bits(b))
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    emu_small.gemm(A, B, C)
    torch.cuda.synchronize()
    ref = mlp_oracle.bf16_round(a) @ mlp_oracle.bf16_round(b).T
    got = C.cpu().numpy().astype(np.float64)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


def test_bounded_wait_times_out_and_the_emulator_stays_usable(emu_small):
    """A device wait on an mbarrier that nothing arrives on (no copy or MMA in
    flight) gives up after its cycle limit; the host reads DSP_ERR_TIMEOUT from
    the GEMMs' error flag, and the context and the emulator keep working."""
    from disort_b200 import capi
    assert emu_small.wait_selftest(1 << 20) == capi.DSP_ERR_TIMEOUT
    assert "ran out" in emu_small.last_error()
    assert emu_small.wait_selftest(0) == capi.DSP_ERR_INVALID_INPUT
    test_tc_gemm_matches_fp64(emu_small, 128, 64, 64)


def make_data(rng, n, n_in, in_pad, n_out, n_heads):
    x = np.zeros((n, in_pad), dtype=np.float32)
    x[:, :n_in] = rng.standard_normal((n, n_in))
    w = rng.standard_normal((n_in, n_out)) / np.sqrt(n_in)
    y = np.tanh(x[:, :n_in] @ w).astype(np.float32)
    hw = (rng.random((n, n_heads)) < 0.7).astype(np.float32)
    return x, y, hw


def test_gradients_match_cpu_oracle(emu_small):
    import torch
    e = emu_small
    rng = np.random.default_rng(11)
    n = 512
    x, y, hw = make_data(rng, n, 165, e.in_stride, 82, 2)
    xb = mlp_oracle.bf16_bits(x)
    e.set_data(torch_bf16(xb), torch.from_numpy(y).cuda(), torch.from_numpy(hw).cuda())
    npar = e.param_count()
    grads = torch.zeros(npar, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    e.gradients(grads, loss)
    torch.cuda.synchronize()
    flat = np.zeros(npar, dtype=np.float32)
    e.get_params(flat)
    dims = e.layer_dims()
    params = mlp_oracle.unpack_params(flat, dims)
    B = 256
    xv = mlp_oracle.bf16_round(x[:B])
    ref_loss, ref = mlp_oracle.forward_backward(params, xv, y[:B].astype(np.float64), hw[:B].astype(np.float64), 82, 2)
    got = mlp_oracle.unpack_params(grads.cpu().numpy(), dims)
    assert abs(float(loss.item()) - ref_loss) <= 1e-3 * abs(ref_loss)
    for i, ((gW, gb), (rW, rb)) in enumerate(zip(got, ref)):
        eW = np.linalg.norm(gW - rW) / np.linalg.norm(rW)
        eb = np.linalg.norm(gb - rb) / max(np.linalg.norm(rb), 1e-30)
        assert eW < 2e-2, (i, "W", eW)
        assert eb < 2e-2, (i, "b", eb)


def test_forward_matches_cpu_oracle(emu_small):
    import torch
    e = emu_small
    rng = np.random.default_rng(13)
    x = np.zeros((300, e.in_stride), dtype=np.float32)
    x[:, :165] = rng.standard_normal((300, 165))
    preds = torch.zeros((300, 164), dtype=torch.float32, device="cuda")
    e.forward(torch_bf16(mlp_oracle.bf16_bits(x)), preds)
    torch.cuda.synchronize()
    flat = np.zeros(e.param_count(), dtype=np.float32)
    e.get_params(flat)
    ref = mlp_oracle.forward(mlp_oracle.unpack_params(flat, e.layer_dims()), x)[:, :164]
    got = preds.cpu().numpy()
    assert np.abs(got - ref).max() <= 2e-2 * np.abs(ref).max()


def torch_reference_loss(flat, dims, x, y, epochs, batch, lr, lr_min):
    """Mean epoch loss of a plain PyTorch FP32 MLP with the same initial weights,
    architecture, loss and Adam schedule (its own shuffling)."""
    import math
    import torch
    params = mlp_oracle.unpack_params(flat, dims)
    Ws = [torch.tensor(W, dtype=torch.float32, device="cuda", requires_grad=True) for W, _ in params]
    bs = [torch.tensor(b, dtype=torch.float32, device="cuda", requires_grad=True) for _, b in params]
    opt = torch.optim.Adam(Ws + bs, lr=lr, eps=1e-8)
    X = torch.tensor(x, device="cuda")
    Y = torch.tensor(y, device="cuda")
    n = X.shape[0]
    nb = n // batch
    total = nb * epochs
    g = torch.Generator(device="cpu").manual_seed(0)
    step, losses = 0, []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).cuda()
        tot = 0.0
        for b in range(nb):
            for group in opt.param_groups:
                group["lr"] = lr_min + (lr - lr_min) * 0.5 * (1 + math.cos(math.pi * step / total))
            idx = perm[b * batch:(b + 1) * batch]
            h = X[idx]
            for i in range(len(Ws) - 1):
                h = torch.nn.functional.gelu(h @ Ws[i].T + bs[i])
            p = h @ Ws[-1].T + bs[-1]
            yy = Y[idx]
            l = ((p[:, :82] - yy) ** 2).sum() + ((p[:, 82:164] - yy) ** 2).sum()
            loss = l / (82 * batch)
            opt.zero_grad()
            loss.backward()
            with torch.no_grad():  # padding rows/columns stay zero, as on the GPU
                Ws[0].grad[:, 165:] = 0
                Ws[-1].grad[164:] = 0
                bs[-1].grad[164:] = 0
            opt.step()
            tot += float(l)
            step += 1
        losses.append(tot / (nb * batch))
    return losses


def test_training_follows_torch_fp32():
    """The tensor-core training loop tracks a PyTorch FP32 run from the same initial weights."""
    import torch
    from disort_b200.emu import Emulator
    e = Emulator(n_in=165, hidden=128, n_hidden_layers=2, n_out=82, n_heads=2, batch=256, seed=5)
    rng = np.random.default_rng(12)
    x = np.zeros((4096, e.in_stride), dtype=np.float32)
    x[:, :165] = rng.standard_normal((4096, 165))
    w = rng.standard_normal((165, 82)) / np.sqrt(165)
    y = (0.8 * np.tanh(x[:, :165] @ w)).astype(np.float32)
    flat = np.zeros(e.param_count(), dtype=np.float32)
    e.get_params(flat)
    xq = mlp_oracle.bf16_round(x).astype(np.float32)
    e.set_data(torch_bf16(mlp_oracle.bf16_bits(x)), torch.from_numpy(y).cuda())
    losses = e.train(20, lr=2e-3, lr_min=1e-4, seed=1)
    ref = torch_reference_loss(flat, e.layer_dims(), xq, y, 20, 256, 2e-3, 1e-4)
    assert losses[-1] < 0.5 * losses[0], (losses, ref)
    assert abs(losses[-1] - ref[-1]) <= 0.15 * ref[-1], (losses, ref)
    preds = torch.zeros((4096, 164), dtype=torch.float32, device="cuda")
    e.forward(torch_bf16(mlp_oracle.bf16_bits(x)), preds)
    torch.cuda.synchronize()
    p = preds.cpu().numpy()
    mse = float(np.mean((p[:, :82] - y) ** 2))
    ref_mse = ref[-1] / (2 * 82)  # the reference's last epoch loss per head and output
    assert mse < 1.3 * ref_mse + 1e-3, (mse, ref_mse)
    e.close()
