"""Autotuner of the engine's launch schedules, per (stream count, layer range).

The engine has more than one way to launch some of its stages; which is faster
depends on the stream count N and the layer count L of the instances:
  - flux path, N <= 16: the layer stage as three one-thread-per-task launches
    (eigensolver in registers; 64 or 128 threads per CTA) or as one team per
    layer task (eigensolver in shared memory);
  - general path: the boundary-value kernel as one CTA or team per instance in
    index order, or persistent (a resident grid taking instances from a queue
    sorted by descending layer count, the size classes).
`tune()` times every candidate on synthetic instances of each (N, layer range)
through the C ABI with CUDA events and keeps the fastest; `write_table` stores
the result in the text format `dsp_context_load_schedule_file` reads:
    N min_layers max_layers layer_stage layer_cta persistent
The committed table (capi.TUNING_FILE) is loaded by every capi.Context and by
the C++ solver objects.  Run on the target GPU:
    python -m disort_b200.autotune --out disort_b200/tuning/b200.txt
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import capi, workloads

# layer ranges the table distinguishes (inclusive)
LAYER_BUCKETS = ((1, 24), (25, 60), (61, 120), (121, 1000000))
FLUX_N = (4, 6, 8, 10, 12, 14, 16)
GENERAL_N = (4, 8, 16, 32, 64)
# (layer_stage, layer_cta) candidates of the flux path at N <= 16
FLUX_CANDIDATES = ((1, 128), (1, 64), (2, 0))
# persistent candidates of the general path
GENERAL_CANDIDATES = (2, 1)


def write_table(path: str, entries: list, notes: list | None = None) -> None:
    """entries: (N, min_layers, max_layers, layer_stage, layer_cta, persistent)."""
    with open(path, "w") as f:
        f.write("# N min_layers max_layers layer_stage layer_cta persistent\n")
        for line in notes or []:
            f.write(f"# {line}\n")
        for e in entries:
            f.write(" ".join(str(int(v)) for v in e) + "\n")


def read_table(path: str) -> list:
    """The entries of a table file; ValueError on a malformed line."""
    out = []
    with open(path) as f:
        for k, line in enumerate(f, 1):
            body = line.split("#", 1)[0].split()
            if not body:
                continue
            if len(body) != 6:
                raise ValueError(f"{path}: line {k} is not 'N min_layers max_layers layer_stage layer_cta persistent'")
            out.append(tuple(int(v) for v in body))
    return out


def lookup(entries: list, N: int, L: int) -> tuple:
    """The entry the engine applies to (N, L): the first match, else zeros."""
    for e in entries:
        if e[0] == N and e[1] <= L <= e[2]:
            return tuple(e)
    return (N, 0, 0, 0, 0, 0)


def _device_flux(w: dict, dev):
    """A flux batch of workload w on the device: (batch, out, keep)."""
    import torch
    arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            arrays[k] = None
        elif isinstance(a, np.ndarray):
            arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        else:
            arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device=dev)
    n, L = w["n_inst"], w["num_layers"]
    batch, keep = capi.make_flux_batch(n, w["num_streams"], L, w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | capi.FLAG_DEVICE_POINTERS, arrays)
    outs = {f: torch.empty((n, L + 1), dtype=torch.float64, device=dev) for f in capi.FLUX_OUT_FIELDS}
    status = torch.empty((n,), dtype=torch.int32, device=dev)
    out, keep2 = capi.make_flux_out(outs, status)
    return batch, out, (keep, keep2, arrays, outs, status)


def _time(fn, reps: int) -> float:
    """Median ms of `reps` runs of fn() on the current stream (CUDA events), after one warm-up."""
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def time_flux(ctx, N: int, L: int, n: int, stage: int, cta: int, reps: int = 3) -> float:
    """ms of one device-resident thermal-sweep solve of n instances (N streams, L layers) under a schedule."""
    import torch
    w = workloads.thermal_sweep(n_bands=n, num_layers=L, num_streams=N, seed=11)
    batch, out, keep = _device_flux(w, torch.device("cuda", torch.cuda.current_device()))
    assert ctx.set_schedule([(N, 1, 1000000, stage, cta, 0)]) == 0, ctx.last_error()

    def run():
        rc = ctx.flux_bands_solve(batch, out)
        if rc != 0:
            raise RuntimeError(f"flux solve: {capi.STATUS_NAMES.get(rc, rc)}: {ctx.last_error()}")
    return _time(run, reps)


def time_general(ctx, N: int, lo: int, hi: int, n: int, persistent: int, reps: int = 1) -> float:
    """ms of one general solve of n mixed-batch instances (N streams, lo..hi layers) under a schedule."""
    insts, flags = workloads.general_mix(n, seed=13, nstr=(N,), layers=(lo, hi))
    d = capi.pack_general(insts, flags)
    batch, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    assert ctx.set_schedule([(N, 1, 1000000, 0, 0, persistent)]) == 0, ctx.last_error()

    def run():
        rc = ctx.general_bands_solve(batch, o)
        if rc != 0:
            raise RuntimeError(f"general solve: {capi.STATUS_NAMES.get(rc, rc)}: {ctx.last_error()}")
    return _time(run, reps)


def _mid(lo: int, hi: int) -> int:
    return (lo + min(hi, 160)) // 2


def tune(ctx, flux_instances: int = 32768, quick: bool = False, log=print) -> tuple[list, list]:
    """Time every candidate per (N, layer range); returns (entries, notes)."""
    buckets = LAYER_BUCKETS[:2] if quick else LAYER_BUCKETS
    best = {}  # (N, lo, hi) -> [layer_stage, layer_cta, persistent]
    notes = []
    for N in FLUX_N:
        for lo, hi in buckets:
            L = _mid(lo, hi)
            n = max(256, flux_instances * 60 // max(L, 1) // (1 if N <= 8 else 2))
            times = {c: time_flux(ctx, N, L, n, *c, reps=5) for c in FLUX_CANDIDATES}
            c = min(times, key=times.get)
            best[(N, lo, hi)] = [c[0], c[1], 0]
            line = f"flux N={N} L={L} n={n}: " + ", ".join(f"stage {a} cta {b}: {t:.3f} ms" for (a, b), t in times.items())
            notes.append(line)
            log(line)
    for N in GENERAL_N:
        for lo, hi in buckets:
            glo, ghi = max(lo, 2), min(hi, 160)
            n = {4: 4096, 8: 4096, 16: 2048, 32: 1024, 64: 256}[N] // (4 if quick else 1)
            times = {pm: time_general(ctx, N, glo, ghi, n, pm, reps=3) for pm in GENERAL_CANDIDATES}
            pm = min(times, key=times.get)
            best.setdefault((N, lo, hi), [0, 0, 0])[2] = pm
            line = f"general N={N} L={glo}-{ghi} n={n}: " + ", ".join(
                f"{'persistent' if k == 1 else 'per-instance'}: {t:.1f} ms" for k, t in times.items())
            notes.append(line)
            log(line)
    entries = [(N, lo, hi, *v) for (N, lo, hi), v in sorted(best.items())]
    return entries, notes


def main() -> None:
    import torch
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=capi.TUNING_FILE)
    ap.add_argument("--quick", action="store_true", help="two layer ranges, smaller general batches")
    ap.add_argument("--flux-instances", type=int, default=32768)
    a = ap.parse_args()
    ctx = capi.Context(0, torch.cuda.current_stream().cuda_stream, tuned=False)
    t0 = time.time()
    entries, notes = tune(ctx, a.flux_instances, a.quick)
    notes.append(f"{torch.cuda.get_device_name()}: tuned in {time.time() - t0:.0f} s")
    write_table(a.out, entries, notes)
    print(f"wrote {len(entries)} entries to {a.out}")


if __name__ == "__main__":
    main()
