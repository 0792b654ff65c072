"""Multi-GPU host logic (disort_b200/replicas.py) as world-size-2 gloo ranks on CPU.

Runs are replicas: each rank solves its own instances and the only cross-rank
steps are barriers and the maximum of the timed durations.  The test checks
that the slowest rank's time is what every rank reports, that the whole-job
rate counts every rank's instances, that ranks draw distinct instances, and
that a rank which never joins ends the others' wait with an error instead of
a hang.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    from disort_b200 import replicas, workloads
    try:
        replicas.init("gloo", 30.0)
        r, local, w = replicas.rank_env()
        replicas.barrier()
        ms = 10.0 + 5.0 * r  # rank 1 is the slow one
        ms_max = replicas.max_over_ranks(ms)
        rate = replicas.job_rate(1000, 4, w, ms_max)
        wl = workloads.thermal_sweep(seed=replicas.replica_seed(2, r), n_bands=8)
        q.put((r, w, ms_max, rate, float(wl["arrays"]["delta_tau"].sum())))
        replicas.finish()
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(len(x) == 5 for x in res), res
    (r0, w0, m0, rate0, s0), (r1, w1, m1, rate1, s1) = res
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert m0 == m1 == 15.0
    assert rate0 == rate1 == pytest.approx(1000 * 4 * 2 / 0.015)
    assert s0 != s1


def _lonely_rank(port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", LOCAL_RANK="0", WORLD_SIZE="2")
    from disort_b200 import replicas
    try:
        replicas.init("gloo", 3.0)  # rank 1 never joins
        q.put("joined")
    except Exception as e:
        q.put(type(e).__name__)


def test_missing_rank_times_out():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely_rank, args=(_free_port(), q))
    p.start()
    out = q.get(timeout=120)
    p.join(timeout=60)
    assert out != "joined"


def test_single_process_is_a_no_op():
    from disort_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(20000, 10, 1, 290.0) == pytest.approx(20000 * 10 / 0.29)
    replicas.barrier()
