"""Launch schedules on the GPU: every form a schedule can pick solves the same
problem (dsp_context_set_schedule / dsp_context_load_schedule_file).

- flux path, N <= 16: the team layer stage and the three-launch stage at 64 and
  128 threads per CTA all match the oracle at 1e-9; the two CTA sizes run the
  same per-thread code, so their outputs are bit-identical;
- general path: the persistent boundary-value kernel (instances taken from the
  queue by descending layer count) gives bit-identical outputs to one CTA or
  team per instance;
- table files: the committed table loads; malformed files and out-of-range
  entries are rejected.
"""
import os

import numpy as np
import pytest

import gpu_lib
import oracle_lib
from disort_b200 import capi, workloads
from parity import assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture()
def ctx():
    c = gpu_lib.context()
    yield c
    if os.path.exists(capi.TUNING_FILE):
        assert c.load_schedule_file(capi.TUNING_FILE) == 0
    else:
        c.set_schedule([])


@pytest.mark.parametrize("nstr", [4, 8, 12, 16])
def test_flux_layer_stage_forms(ctx, nstr):
    w = workloads.thermal_sweep(n_bands=300, num_layers=23, num_streams=nstr, seed=40 + nstr)
    ref, rst = oracle_lib.flux_solve(w)
    got = {}
    for stage, cta in ((1, 128), (1, 64), (2, 0)):
        assert ctx.set_schedule([(nstr, 1, 1000, stage, cta, 0)]) == 0
        out, st, rc = gpu_lib.flux_solve(w)
        assert rc == 0 and np.all(st == 0) and np.all(rst == 0)
        assert_parity(out, ref, f"N={nstr} stage={stage} cta={cta}")
        got[(stage, cta)] = out
    for f in capi.FLUX_OUT_FIELDS:
        np.testing.assert_array_equal(got[(1, 128)][f], got[(1, 64)][f], err_msg=f)


def test_flux_schedule_applies_by_layer_range(ctx):
    """An entry covers only its layer range: outside it the built-in choice runs."""
    w = workloads.thermal_sweep(n_bands=200, num_layers=30, num_streams=16, seed=3)
    assert ctx.set_schedule([]) == 0
    base, _, _ = gpu_lib.flux_solve(w)
    assert ctx.set_schedule([(16, 1, 29, 2, 0, 0), (16, 31, 100, 2, 0, 0)]) == 0
    out, _, _ = gpu_lib.flux_solve(w)
    for f in capi.FLUX_OUT_FIELDS:
        np.testing.assert_array_equal(base[f], out[f], err_msg=f)


@pytest.mark.parametrize("nstr", [(4, 8), (16,), (32,), (64,)])
def test_general_persistent_queue_is_bit_identical(ctx, nstr):
    n = 4 if 64 in nstr else 24
    insts, flags = workloads.general_mix(n, seed=70, nstr=nstr, layers=(2, 30 if 64 not in nstr else 8))
    d = capi.pack_general(insts, flags)
    outs = []
    for pm in (2, 1):
        assert ctx.set_schedule([(N, 1, 1000, 0, 0, pm) for N in nstr]) == 0
        got, rc = gpu_lib.general_solve(d)
        assert rc == 0 and np.all(got["status"] == 0), ctx.last_error()
        outs.append(got)
    for k in outs[0]:
        np.testing.assert_array_equal(outs[0][k], outs[1][k], err_msg=k)


def test_schedule_files_and_entry_checks(ctx, tmp_path):
    if os.path.exists(capi.TUNING_FILE):
        assert ctx.load_schedule_file(capi.TUNING_FILE) == 0 and ctx.schedule_count() > 0
    bad = tmp_path / "bad.txt"
    bad.write_text("16 1 24 1 128\n")
    assert ctx.load_schedule_file(str(bad)) == capi.DSP_ERR_INVALID_INPUT
    assert "line 1" in ctx.last_error()
    assert ctx.load_schedule_file(str(tmp_path / "missing.txt")) == capi.DSP_ERR_INVALID_INPUT
    assert ctx.set_schedule([(16, 1, 24, 3, 0, 0)]) == capi.DSP_ERR_INVALID_INPUT
    assert ctx.set_schedule([(16, 1, 24, 1, 96, 0)]) == capi.DSP_ERR_INVALID_INPUT
    assert ctx.set_schedule([(16, 30, 24, 1, 64, 0)]) == capi.DSP_ERR_INVALID_INPUT
    good = tmp_path / "good.txt"
    good.write_text("# table\n16 1 24 1 64 0\n\n64 1 1000000 0 0 1  # persistent\n")
    assert ctx.load_schedule_file(str(good)) == 0 and ctx.schedule_count() == 2
