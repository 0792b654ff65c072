"""GPU test of the gated emulator pipeline (disort_b200/surrogate.py).

The emulator corrects a 4-stream FP64 solve toward the 16-stream one; it is
trained on columns labelled by the FP64 GPU solver, then used on column x band
instances with some columns pushed out of the training envelope.  Checked here:
- what the network gains over the method without it: the corrected solve's
  held-out errors are a fraction of the 4-stream solve's;
- what the gate guarantees: a gated instance carries the 16-stream FP64 result
  itself, and every out-of-envelope instance is gated at any disagreement
  tolerance, while the emulator alone carries the in-envelope instances when
  the disagreement test is switched off.
The network is trained at the bench leg's scale; the throughput at each gate
tolerance is measured by bench.py's surrogate leg.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    import torch
    from disort_b200 import capi, surrogate
    ctx = capi.Context(0, torch.cuda.current_stream().cuda_stream)
    # the bench leg's scale: 2^20 solver-labelled columns, 50 epochs (about 20 s)
    sur, rep = surrogate.train(ctx, n_columns=1 << 20, epochs=50, log=lambda *a: None)
    yield ctx, sur, rep
    sur.emu.close()
    ctx.close()


def test_training_on_solver_labels(trained):
    ctx, sur, rep = trained
    assert rep["bad_label_status"] == 0
    assert rep["last_loss"] < 0.35 * rep["first_loss"], rep


def test_network_gain_over_the_cheap_solve(trained):
    """The network's correction cuts the 4-stream solve's held-out median error
    at least in half and its p99 error by at least 30 %, and brings the median
    under 1 %."""
    ctx, sur, rep = trained
    four = rep["four_stream_alone"]
    print(f"held-out median/p99: corrected {rep['holdout_median_rel_err']:.4g}/{rep['holdout_p99_rel_err']:.4g}, "
          f"4-stream alone {four['median_rel_err']:.4g}/{four['p99_rel_err']:.4g}")
    assert rep["holdout_median_rel_err"] < 0.5 * four["median_rel_err"], rep
    assert rep["holdout_p99_rel_err"] < 0.7 * four["p99_rel_err"], rep
    assert rep["holdout_median_rel_err"] < 1e-2, rep


def test_gate_bounds_error_and_catches_out_of_envelope(trained):
    import torch
    from disort_b200 import surrogate as s
    ctx, sur, rep = trained
    columns = 32
    n = columns * s.NBANDS
    d = s.sample(n, 21, columns=columns, ooe_columns=0.125)
    arrays = s.device_inputs(d)
    F_ref, st = s.solve_fp64(ctx, arrays, n)
    assert int((st != 0).sum()) == 0
    # strict gate: every gated instance carries the FP64 result itself
    F, k, fb = s.gated_run(ctx, sur, arrays, n, s.GATE_TOL)
    fbm = fb.bool()
    assert int(fbm.sum()) == k
    assert torch.equal(F[fbm], F_ref[fbm])
    e = s.rel_err(F, F_ref).amax(dim=1)
    print(f"strict gate: fallback {k / n:.3f}, max rel err {float(e.max()):.3g}")
    # envelope-only gate: the emulator carries every in-envelope instance; the
    # pushed columns are still solved in FP64
    ooe = torch.from_numpy(d["ooe"]).cuda()
    Fo, ko, fbo = s.gated_run(ctx, sur, arrays, n, 1e30)
    assert bool(fbo.bool()[ooe].all())
    assert torch.equal(Fo[ooe], F_ref[ooe])
    assert ko <= int(ooe.sum()) + n // 100, (ko, int(ooe.sum()))
    eo = s.rel_err(Fo, F_ref).amax(dim=1)[~ooe]
    print(f"envelope-only gate: fallback {ko / n:.3f}, in-envelope p50/p99 rel err {float(eo.median()):.3g}/"
          f"{float(torch.quantile(eo.float(), 0.99)):.3g}")
    assert float(eo.median()) < 2e-2


def test_save_and_load_give_the_same_predictions(trained, tmp_path):
    import torch
    from disort_b200 import surrogate as s
    ctx, sur, rep = trained
    p = str(tmp_path / "emulator")
    s.save(sur, p)
    sur2 = s.load(p)
    try:
        d = s.sample(512, 33)
        arrays = s.device_inputs(d)
        raw, pa, *_ = s.emulate(ctx, sur, arrays, 512)
        raw2, pb, *_ = s.emulate(ctx, sur2, arrays, 512)
        assert torch.equal(raw, raw2) and torch.equal(pa, pb)
        for k in ("fmean", "fstd", "lo", "hi", "mu", "sd"):
            assert torch.equal(getattr(sur, k), getattr(sur2, k))
    finally:
        sur2.emu.close()
