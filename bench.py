"""Benchmark of the B200 DISORT flux path: solves/s on the 60-layer, 16-stream,
20,000-band thermal sweep (one spectral loop per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload thermal|beam|general]

Prints one JSON line (rank 0).  A step is one dsp_flux_bands_solve over the whole
sweep with inputs resident in HBM (`value`); `e2e` repeats the step through the
same C ABI with pinned host buffers, host<->device copies inside the timed region.
`--impl reference` times the CPU restatement of the reference solver (oracle/,
OpenMP over all host threads, the reference loop's structure) on a bounded
sample of the same sweep.  Multi-GPU runs are replicas: every rank solves its own
20,000-band sweep (weak scaling), no collective on the data path.

`--workload general` measures the general solver (dsp_general_bands_solve,
DisortSolver::solve) on the mixed batch of workloads.general_mix: 4,096 instances
by default (`--bands` sets the count), N 4..64, 10..120 layers, delta-M+, beam,
3 optical depths x 5 polar angles x 4 azimuths, every azimuth mode.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from disort_b200 import capi, flops, replicas, workloads  # noqa: E402

METRIC = "solves/s (60 lyr,16 str): plain GPU vs gated surrogate at ≤0.5% flux err"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["thermal", "beam", "general", "emulator"], default="thermal")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target CPU-baseline sample time")
    ap.add_argument("--bands", type=int, default=0, help="profiling: solve only the first N bands")
    ap.add_argument("--no-cpu", action="store_true", help="profiling: skip the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true", help="profiling: skip the host-buffer pass")
    ap.add_argument("--no-graph", action="store_true", help="profiling: skip the CUDA-graph replay pass")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the gated-emulator leg (solver-labelled training + gated inference)")
    ap.add_argument("--no-general", action="store_true",
                    help="skip the general-solver leg (65,536-instance mixed batch)")
    ap.add_argument("--general-instances", type=int, default=65536)
    return ap.parse_args()


def make_workload(kind: str, rank: int):
    if kind == "beam":
        return workloads.beam_sweep()
    w = workloads.thermal_sweep(seed=2 + rank)
    if rank:
        off = 0.14 * 20000 * rank
        w["arrays"]["wavenumber_low"] = w["arrays"]["wavenumber_low"] + off
        w["arrays"]["wavenumber_high"] = w["arrays"]["wavenumber_high"] + off
    return w


def config_of(w, args, world):
    return {
        "workload": w["name"], "bands_per_gpu": w["n_inst"], "num_layers": w["num_layers"],
        "num_streams": w["num_streams"], "thermal": bool(w["flags"] & capi.FLAG_THERMAL),
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "l2": "inputs (pmom 163 MB) and workspace (5.7 GB) larger than L2; no flush needed",
    }


# ---------------------------------------------------------------------------
# CPU baseline (oracle restatement of the reference solver, OpenMP)
# ---------------------------------------------------------------------------
def cpu_oracle():
    sys.path.insert(0, os.path.join(REPO, "tests"))
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "native"], check=True)
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "_native", "liboracle_disort.so"))
    lib.oracle_flux_bands_solve.restype = ctypes.c_int
    lib.oracle_flux_bands_solve.argtypes = [ctypes.POINTER(capi.FluxBatch), ctypes.POINTER(capi.FluxOut),
                                            ctypes.c_int]
    return lib


def cpu_time(lib, w, threads, keep_outputs=False):
    batch, keep = workloads.make_batch(w)
    outs, status = capi.alloc_flux_out_numpy(w["n_inst"], w["num_layers"])
    o, keep2 = capi.make_flux_out(outs, status)
    t0 = time.perf_counter()
    lib.oracle_flux_bands_solve(ctypes.byref(batch), ctypes.byref(o), threads)
    t = time.perf_counter() - t0
    return (t, outs, status) if keep_outputs else t


def cpu_baseline(w, target_s: float):
    """The oracle on the host's threads over the whole sweep when that takes at
    most a few times `target_s` (else an evenly spaced sample sized to it).
    Returns (cpu_baseline dict, band indices solved, oracle outputs)."""
    lib = cpu_oracle()
    threads = os.cpu_count() or 1
    probe = workloads.subset(w, np.arange(0, w["n_inst"], max(1, w["n_inst"] // (4 * threads)))[: 4 * threads])
    cpu_time(lib, probe, threads)  # warm-up
    t = cpu_time(lib, probe, threads)
    rate = probe["n_inst"] / t
    m = w["n_inst"] if w["n_inst"] / rate <= 4 * target_s else int(max(threads, rate * target_s))
    idx = np.linspace(0, w["n_inst"] - 1, m).astype(np.int64)
    sample = workloads.subset(w, idx) if m < w["n_inst"] else w
    t, outs, status = cpu_time(lib, sample, threads, keep_outputs=True)
    what = "all" if m == w["n_inst"] else f"{m} of"
    return dict(value=m / t, unit="solves/s", cores=threads, kind="port",
                sample=f"{what} {w['n_inst']} bands{'' if m == w['n_inst'] else ' evenly spaced across the sweep'}, "
                       f"oracle built -march=native, {threads} OpenMP threads, {t:.1f} s"), idx, (outs, status)


def parity_of(gpu_outs: dict, idx, ref, rtol=1e-9, atol=1e-12) -> dict:
    """Element-wise |gpu - oracle| / (rtol |oracle| + atol) over the solved bands
    (<= 1 passes), every FluxResult field."""
    outs, status = ref
    worst, where = 0.0, None
    for f in capi.FLUX_OUT_FIELDS:
        a, b = np.asarray(gpu_outs[f])[idx], np.asarray(outs[f])
        r = np.abs(a - b) / (rtol * np.abs(b) + atol)
        r = np.where(np.isnan(a) & np.isnan(b), 0.0, np.where(np.isnan(r), np.inf, r))
        k = float(r.max())
        if k > worst:
            worst, where = k, f + str(tuple(int(x) for x in np.unravel_index(int(np.argmax(r)), r.shape)))
    return {"max_ratio": worst, "at": where, "rtol": rtol, "atol": atol, "bands_compared": int(len(idx)),
            "fields": list(capi.FLUX_OUT_FIELDS), "oracle_bad_status": int((np.asarray(status) != 0).sum()),
            "passes": worst <= 1.0}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = make_workload(args.workload, 0)
    lib = cpu_oracle()
    threads = os.cpu_count() or 1
    probe = workloads.subset(w, np.arange(0, w["n_inst"], max(1, w["n_inst"] // (4 * threads)))[: 4 * threads])
    cpu_time(lib, probe, threads)
    rate = probe["n_inst"] / cpu_time(lib, probe, threads)
    per_step = max(1.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    m = int(min(w["n_inst"], max(threads, rate * per_step)))
    sample = workloads.subset(w, np.linspace(0, w["n_inst"] - 1, m).astype(np.int64))
    for _ in range(args.warmup):
        cpu_time(lib, sample, threads)
    ts = [cpu_time(lib, sample, threads) for _ in range(args.steps)]
    value = m * len(ts) / sum(ts)
    desc = (f"{m} of {w['n_inst']} bands per step (evenly spaced), CPU restatement of "
            f"DisortFluxSolver<16> (oracle/, -march=native), {threads} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(ts),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": config_of(w, args, 1),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.fh = None

    def start(self):
        self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.fh.flush()
        self.fh.seek(0)
        rows = [r.strip().split(", ") for r in self.fh.read().splitlines() if r.strip()]
        os.unlink(self.fh.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                smax.append(float(r[1]))
                for k, nm in enumerate(names):
                    if r[4 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def fp64_peak_tflops() -> float | None:
    try:
        lib = ctypes.CDLL(os.path.join(REPO, "disort_b200", "lib", "libdsp_bench.so"))
        lib.dsp_bench_fp64_tflops.restype = ctypes.c_double
        lib.dsp_bench_fp64_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
        import torch
        v = lib.dsp_bench_fp64_tflops(torch.cuda.current_device(), 5)
        return v if v > 0 else None
    except OSError:
        return None


def committed_traffic(workload_name: str, kernel: str):
    """DRAM bytes per launch of `kernel` on this workload, from the committed ncu summary."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        entry = json.load(open(p)).get(workload_name) or {}
        return entry.get(kernel)
    except (ValueError, OSError):
        return None


def general_traffic(kernel: str, n: int, launches: int):
    """Average DRAM bytes per launch of the general path's boundary-value kernel
    on n instances, from the committed per-instance ncu figure."""
    if kernel != "gen_bvp_kernel" or launches <= 0:
        return None
    per = committed_traffic("general_mix", "gen_bvp_kernel_bytes_per_instance")
    return None if per is None else per * n / launches


def run_e2e(args, ctx, w, douts, stream, dev, world):
    """Same solve through the C ABI with pinned host buffers: inputs up, results
    down, inside the timed region.  Returns (solves/s, h2d bytes, d2h bytes,
    results equal to the device-resident run)."""
    import torch
    n, L, N = w["n_inst"], w["num_layers"], w["num_streams"]
    host_arrays = {}
    h2d = 0
    for k, a in w["arrays"].items():
        if isinstance(a, np.ndarray):
            ta = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            host_arrays[k] = ta
            h2d += ta.numel() * 8
        else:
            host_arrays[k] = a
            if a is not None:
                h2d += 8
    hbatch, hkeep = capi.make_flux_batch(n, N, L, w["num_phase_func_moments"], w["pmom_count"], w["flags"],
                                         host_arrays)
    houts = {f: torch.empty((n, L + 1), dtype=torch.float64).pin_memory() for f in capi.FLUX_OUT_FIELDS}
    hstatus = torch.empty((n,), dtype=torch.int32).pin_memory()
    hout, hkeep2 = capi.make_flux_out(houts, hstatus)
    d2h = 8 * n * (L + 1) * 8 + 4 * n

    def hstep():
        rc = ctx.flux_bands_solve(hbatch, hout)
        if rc != 0:
            raise RuntimeError(f"host-pointer solve: {ctx.last_error()}")

    for _ in range(max(1, args.warmup)):
        hstep()
    replicas.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        hstep()
    e3.record(stream)
    torch.cuda.synchronize()
    replicas.barrier()
    e2e_value = replicas.job_rate(n, args.steps, world, replicas.max_over_ranks(e2.elapsed_time(e3), dev))
    # host results must equal the device-resident results
    same = all(torch.equal(houts[f], douts[f].cpu()) for f in capi.FLUX_OUT_FIELDS)

    return e2e_value, h2d, d2h, same


def run_ours(args):
    import torch
    rank, local, world = replicas.rank_env()
    torch.cuda.set_device(local)
    replicas.init("nccl", 120.0)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()

    w = make_workload(args.workload, rank)
    if args.bands:
        w = workloads.subset(w, np.arange(min(args.bands, w["n_inst"])))
        w["name"] += f"_first{w['n_inst']}"
    n, L, N = w["n_inst"], w["num_layers"], w["num_streams"]
    ctx = capi.Context(local, stream.cuda_stream)

    # device-resident inputs/outputs
    dev_arrays = {}
    for k, a in w["arrays"].items():
        if a is None:
            dev_arrays[k] = None
        elif isinstance(a, np.ndarray):
            dev_arrays[k] = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        else:
            dev_arrays[k] = torch.tensor([float(a)], dtype=torch.float64, device=dev)
    batch, keep = capi.make_flux_batch(n, N, L, w["num_phase_func_moments"], w["pmom_count"],
                                       w["flags"] | capi.FLAG_DEVICE_POINTERS, dev_arrays)
    douts = {f: torch.empty((n, L + 1), dtype=torch.float64, device=dev) for f in capi.FLUX_OUT_FIELDS}
    dstatus = torch.empty((n,), dtype=torch.int32, device=dev)
    out, keep2 = capi.make_flux_out(douts, dstatus)

    def step():
        rc = ctx.flux_bands_solve(batch, out)
        if rc != 0:
            raise RuntimeError(f"dsp_flux_bands_solve: {capi.STATUS_NAMES.get(rc, rc)}: {ctx.last_error()}")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    bad = int((dstatus != 0).sum())

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
    except Exception:
        uuid = str(local)
    clocks = ClockSampler(uuid)

    # ---- timed region: device-resident inputs --------------------------------
    ctx.set_timing(True)
    ctx.timing_reset()
    replicas.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ktimes = ctx.timings()
    ctx.set_timing(False)
    ms_max = replicas.max_over_ranks(ms, dev)
    value = replicas.job_rate(n, args.steps, world, ms_max)

    # ---- e2e: through the C ABI with pinned host buffers ----------------------
    # the headline e2e sends one Henyey-Greenstein g per layer (DSP_FLAG_HG_G; the
    # engine forms the moments on the device, bit-identical results); the same
    # call with the full [L][17] moment array is reported beside it
    if args.no_e2e:
        e2e_value, h2d, d2h, same, e2e_mom = None, 0, 0, None, None
    else:
        w_e2e = workloads.as_hg(w) if "hg_g" in w else w
        e2e_value, h2d, d2h, same = run_e2e(args, ctx, w_e2e, douts, stream, dev, world)
        e2e_mom = None
        if w_e2e is not w:
            v, h, d, sm = run_e2e(args, ctx, w, douts, stream, dev, world)
            e2e_mom = {"value": v, "unit": "solves/s", "h2d_bytes_per_step": h, "d2h_bytes_per_step": d,
                       "matches_device_result": sm, "inputs": "full phase-function moments [L][17]"}

    # ---- the same device-resident step replayed as one CUDA graph ---------------
    graph = None if args.no_graph else graph_leg(batch, out, stream, local, n, args)

    # ---- roofline of the dominant kernel -----------------------------------
    beam = bool(np.any(np.asarray(w["arrays"]["direct_beam_flux"]) > 0))
    thermal = bool(w["flags"] & capi.FLAG_THERMAL)
    fl = flops.flux_solve_flops(N, L, beam, thermal)
    dom = max((k for k in ktimes if k in fl), key=lambda k: ktimes[k][0])
    dom_ms, dom_launches = ktimes[dom]
    achieved = fl[dom] * n * args.steps / (dom_ms / 1000.0) / 1e12
    peak = fp64_peak_tflops()
    roofline = {
        "bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
        "frac": (achieved / peak) if peak else None,
        "peak_source": "measured on this GPU by disort_b200/csrc/fp64_peak.cu (FP64 FMA chains, burst)",
        "flops_per_solve": fl[dom], "avg_launch_ms": dom_ms / max(1, dom_launches),
        "traffic": committed_traffic(w["name"], dom),
        "traffic_source": "profiles/traffic.json (ncu dram bytes of one 4,000-band launch, scaled to the sweep)",
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
    }

    if rank == 0:
        cpu, parity = None, None
        if not args.no_cpu:
            cpu, idx, ref = cpu_baseline(w, args.cpu_seconds)
            parity = parity_of({f: v.cpu().numpy() for f, v in douts.items()}, idx, ref)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
            "config": config_of(w, args, world),
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "matches_device_result": same,
                    "inputs": "one HG asymmetry factor per layer (DSP_FLAG_HG_G)" if "hg_g" in w else "moments"},
            "e2e_full_moments": e2e_mom,
            "graph": graph,
            "gpu_launches": int(sum(v[1] for v in ktimes.values())),
            "roofline": roofline, "cpu_baseline": cpu, "parity": parity, "clocks": clk,
            "bad_status_instances": bad,
        }
        if not args.no_surrogate and world == 1:
            line["surrogate"] = surrogate_leg(ctx)
        if not args.no_general and world == 1:
            line["general"] = general_leg(ctx, stream, dev, args)
        print(json.dumps(line), flush=True)
    ctx.close()
    replicas.finish()


def graph_leg(batch, out, stream, device, n, args) -> dict:
    """The device-resident step as one CUDA graph (dsp_flux_graph_create),
    replayed `steps` times after `warmup` replays; CUDA events on the stream."""
    import torch
    g = capi.FluxGraph(batch, out, device)
    try:
        for _ in range(max(1, args.warmup)):
            g.launch(stream.cuda_stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            rc = g.launch(stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(f"dsp_graph_launch: {capi.STATUS_NAMES.get(rc, rc)}")
        b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
    finally:
        torch.cuda.synchronize()
        g.close()
    return {"value": n * args.steps / (ms / 1000.0), "unit": "solves/s", "ms_per_step": ms / args.steps,
            "note": "the same device-resident solve replayed as one CUDA graph"}


def surrogate_leg(ctx) -> dict:
    """The gated emulator on this GPU: 2^20 solver-labelled columns (40 layers,
    16 streams, thermal + solar), 50 epochs of tensor-core training, then 4,096
    columns x 256 bands (1,048,576 solves, 5 % of the columns out of envelope)
    emulated and gated, against the plain FP64 solve of the same instances."""
    try:
        from disort_b200 import surrogate
        sur, rep = surrogate.train(ctx, log=lambda *a: None)
        ev = surrogate.evaluate(ctx, sur)
        sur.emu.close()
        return {"metric": "gated surrogate solves/s vs plain FP64 GPU solves/s, same instances",
                "workload": "4096 columns x 256 bands, 40 layers, 16 streams, thermal + solar", "training": rep,
                "inference": ev}
    except Exception as e:  # the plain-solver line stands on its own
        return {"error": f"{type(e).__name__}: {e}"}


def general_leg(ctx, stream, dev, args) -> dict:
    """The general solver (DisortSolver) on the 65,536-instance mixed batch
    (N 4-64, L 10-120, all azimuth modes, intensities): one warm-up and one
    timed solve with inputs in HBM, the oracle on an evenly spaced sample (CPU
    baseline and parity, the parity also against the extended-precision
    oracle build, the checker of the 64-stream instances)."""
    try:
        return measure_general(ctx, stream, dev, args.general_instances, 3, 1, 1, e2e=False,
                               cpu_seconds=None if args.no_cpu else args.cpu_seconds, ext_parity=True)
    except Exception as e:  # the plain-solver line stands on its own
        return {"error": f"{type(e).__name__}: {e}"}


# ---------------------------------------------------------------------------
# general solver (DisortSolver) on the mixed batch
# ---------------------------------------------------------------------------
GENERAL_METRIC = "solves/s (general mix: N 4-64, L 10-120, DM+, beam, 3 tau x 5 mu x 4 phi, all modes)"


def general_batch(n: int, seed: int):
    insts, flags = workloads.general_mix(n, seed=seed)
    d = capi.pack_general(insts, flags)
    fl = {"gen_layer_kernel": 0.0, "gen_bvp_kernel": 0.0, "gen_intensity_kernel": 0.0, "total": 0.0}
    for c in insts:
        ncut = flops.absorption_cut(c["delta_tau"], c["single_scat_albedo"], False)
        modes = 1 if abs(1.0 - c["direct_beam_mu"]) < 1e-5 else c["num_streams"]
        f = flops.general_solve_flops(c["num_streams"], c["num_layers"], ncut, modes, 5, 3, True, False)
        for k in fl:
            fl[k] += f[k]
    return insts, d, fl


def general_oracle_lib(ext: bool = False):
    """The oracle built for this host (-march=native), or its extended-precision build."""
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ext" if ext else "native"], check=True)
    lib = ctypes.CDLL(os.path.join(REPO, "oracle", "liboracle_disort_ext.so") if ext else
                      os.path.join(REPO, "oracle", "_native", "liboracle_disort.so"))
    lib.oracle_general_bands_solve.restype = ctypes.c_int
    lib.oracle_general_bands_solve.argtypes = [ctypes.POINTER(capi.GeneralBatch), ctypes.POINTER(capi.GeneralOut),
                                               ctypes.c_int]
    return lib


ULP_COPIES = 2  # one-ulp-perturbed copies of the sample behind the FP64 spread


def general_cpu_time(lib, insts, flags, threads, keep_outputs=False):
    d = capi.pack_general(insts, flags, pmom_count=66)
    b, keep = capi.make_general_batch(d)
    outs, o, keep2 = capi.alloc_general_out_numpy(d)
    t0 = time.perf_counter()
    lib.oracle_general_bands_solve(ctypes.byref(b), ctypes.byref(o), threads)
    t = time.perf_counter() - t0
    return (t, outs) if keep_outputs else t


def ulp_perturbed(inst: dict, rng) -> dict:
    """A copy of a general instance whose layer optical depths, single-
    scattering albedos and phase-function moments past the zeroth each move one
    ulp up or down at random (zeros stay, albedos stay <= 1); user depths at the
    half and the full column follow its new total.  The double oracle's spread
    over such copies is how closely the FP64-representable inputs determine an
    instance's outputs."""
    p = dict(inst)
    for k in ("delta_tau", "single_scat_albedo", "phase_function_moments"):
        a = np.asarray(inst[k], dtype=np.float64)
        up = rng.integers(0, 2, a.shape).astype(bool)
        b = np.where(up, np.nextafter(a, np.inf), np.nextafter(a, -np.inf))
        b = np.where(a == 0.0, a, b)
        if k == "single_scat_albedo":
            b = np.where(a <= 1.0, np.minimum(b, 1.0), b)
        if k == "phase_function_moments":
            b[..., 0] = a[..., 0]
        p[k] = b
    if inst.get("tau_user") is not None:
        t0 = workloads.column_total(np.asarray(inst["delta_tau"], dtype=np.float64))
        t1 = workloads.column_total(p["delta_tau"])
        p["tau_user"] = [t1 if t == t0 else t1 / 2.0 if t == t0 / 2.0 else t for t in inst["tau_user"]]
    return p


def general_parity(gpu: dict, idx, ref: dict, rtol=1e-9, atol=1e-12, floor_ref=None) -> dict:
    """Fluxes element-wise; intensities against max(|value|, the instance's
    largest |intensity|) (a Fourier sum whose terms cancel); <= 1 passes.

    With `floor_ref` (FP64 evaluations when `ref` is the extended-precision
    build: one output dict or a list of them, the double build on the given
    inputs and on one-ulp-perturbed copies) an element's allowance widens to
    twice the instance's FP64 spread when that is larger: the largest distance
    from `ref` of any of those evaluations over the instance's values of the
    field, in units of the same plain allowance (instances an evaluation did not
    solve left out).  That spread belongs to the formulation, which no FP64
    solver (the reference included) is held below."""
    floor_refs = [] if floor_ref is None else [floor_ref] if isinstance(floor_ref, dict) else list(floor_ref)
    worst, where, spread_max = 0.0, None, 0.0
    for f in capi.FLUX_OUT_FIELDS + ("intensity", "intensity_azimuth_avg"):
        a = np.asarray(gpu[f])[idx]
        b = np.asarray(ref[f])
        if f.startswith("intensity"):
            flat = np.abs(np.nan_to_num(b)).reshape(b.shape[0], -1)
            scale = flat.max(axis=1).reshape((-1,) + (1,) * (b.ndim - 1))
            denom = rtol * np.maximum(np.abs(b), scale) + atol
        else:
            denom = rtol * np.abs(b) + atol
        if floor_refs:
            spread = np.zeros(b.shape[0])
            for fr in floor_refs:
                rf = (np.abs(np.nan_to_num(np.asarray(fr[f]) - b)) / denom).reshape(b.shape[0], -1)
                sp = rf.max(axis=1) if rf.size else np.zeros(b.shape[0])
                if "status" in fr:
                    sp = np.where(np.asarray(fr["status"]).reshape(-1) == 0, sp, 0.0)
                spread = np.maximum(spread, sp)
            spread_max = max(spread_max, float(spread.max()) if spread.size else 0.0)
            denom = denom * np.maximum(1.0, 2.0 * spread).reshape((-1,) + (1,) * (b.ndim - 1))
        r = np.abs(a - b) / denom
        r = np.where(np.isnan(a) & np.isnan(b), 0.0, np.where(np.isnan(r), np.inf, r))
        k = float(r.max()) if r.size else 0.0
        if k > worst:
            worst, where = k, f + str(tuple(int(x) for x in np.unravel_index(int(np.argmax(r)), r.shape)))
    out = {"max_ratio": worst, "at": where, "rtol": rtol, "atol": atol, "instances_compared": int(len(idx)),
           "passes": worst <= 1.0}
    if floor_refs:
        out["fp64_spread_max"] = spread_max
    return out


def general_cpu_sample(insts, target_s: float):
    """An evenly spaced sample of the batch sized to about target_s of CPU time."""
    lib = general_oracle_lib()
    threads = os.cpu_count() or 1
    flags = capi.FLAG_DELTA_M_PLUS | capi.GFLAG_USER_TAU | capi.GFLAG_USER_MU
    n = len(insts)
    probe = [insts[k] for k in np.linspace(0, n - 1, min(n, 2 * threads)).astype(int)]
    t = general_cpu_time(lib, probe, flags, threads)
    m = int(min(n, max(threads, len(probe) * target_s / max(t, 1e-6))))
    idx = np.linspace(0, n - 1, m).astype(int)
    return lib, [insts[k] for k in idx], flags, threads, idx


def run_general(args):
    import torch
    rank, local, world = replicas.rank_env()
    n = args.bands or 4096
    if args.impl == "reference":
        if rank != 0:
            return
        insts, flags = workloads.general_mix(n, seed=3)
        lib, sample, flags, threads, _ = general_cpu_sample(insts, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
        for _ in range(args.warmup):
            general_cpu_time(lib, sample, flags, threads)
        ts = [general_cpu_time(lib, sample, flags, threads) for _ in range(args.steps)]
        value = len(sample) * len(ts) / sum(ts)
        desc = (f"{len(sample)} of {n} instances per step (evenly spaced), CPU restatement of DisortSolver "
                f"(oracle/, -march=native), {threads} OpenMP threads")
        print(json.dumps({
            "impl": "reference", "metric": GENERAL_METRIC, "value": value, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": f"general_mix_{n}", "instances_per_gpu": n},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    torch.cuda.set_device(local)
    replicas.init("nccl", 300.0)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ctx = capi.Context(local, stream.cuda_stream)
    line = measure_general(ctx, stream, dev, n, replicas.replica_seed(3, rank), args.steps, args.warmup,
                           world, rank, e2e=not args.no_e2e, cpu_seconds=None if args.no_cpu else args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    replicas.finish()


def measure_general(ctx, stream, dev, n, seed, steps, warmup, world=1, rank=0, e2e=True, cpu_seconds=10.0,
                    ext_parity=False):
    """The general solver on n instances of the mixed batch: device-resident
    solves/s over `steps` timed solves (CUDA events), optionally the host-buffer
    e2e rate, the oracle on an evenly spaced CPU sample (baseline and parity)
    and the roofline of the dominant kernel.  Returns the bench line."""
    import torch
    from types import SimpleNamespace
    args = SimpleNamespace(steps=steps, warmup=warmup, no_e2e=not e2e, no_cpu=cpu_seconds is None,
                           cpu_seconds=cpu_seconds)
    insts, d, fl = general_batch(n, seed)
    dd = dict(d)
    for k in ("num_streams", "num_layers", "layer_offset", "num_phase_func_moments", "delta_tau",
              "single_scat_albedo", "phase_function_moments", "temperature") + capi.GENERAL_SCALAR_FIELDS:
        dd[k] = torch.from_numpy(np.ascontiguousarray(d[k])).to(dev)
    for k in ("tau_user", "mu_user", "phi_user"):
        a, stride = d[k]
        dd[k] = (torch.from_numpy(np.ascontiguousarray(a)).to(dev), stride)
    dd["flags"] = d["flags"] | capi.FLAG_DEVICE_POINTERS
    batch, keep = capi.make_general_batch(dd)
    nt, nu, nphi = d["ntau_out"], d["numu_out"], d["num_phi"]

    def make_out(device, pin):
        mk = (lambda *shape, dt=torch.float64: torch.empty(shape, dtype=dt, device=device)) if device != "cpu" else \
            (lambda *shape, dt=torch.float64: torch.empty(shape, dtype=dt).pin_memory())
        outs = {f: mk(n, nt) for f in capi.FLUX_OUT_FIELDS}
        outs["intensity"] = mk(n, nt, nu, nphi)
        outs["intensity_azimuth_avg"] = mk(n, nt, nu)
        outs["status"] = mk(n, dt=torch.int32)
        o = capi.GeneralOut()
        for k, f in enumerate(capi.FLUX_OUT_FIELDS):
            o.flux[k] = ctypes.cast(ctypes.c_void_p(outs[f].data_ptr()), ctypes.POINTER(ctypes.c_double))
        o.intensity = ctypes.cast(ctypes.c_void_p(outs["intensity"].data_ptr()), ctypes.POINTER(ctypes.c_double))
        o.intensity_azimuth_avg = ctypes.cast(ctypes.c_void_p(outs["intensity_azimuth_avg"].data_ptr()),
                                              ctypes.POINTER(ctypes.c_double))
        o.status = ctypes.cast(ctypes.c_void_p(outs["status"].data_ptr()), ctypes.POINTER(ctypes.c_int32))
        o.ntau_out, o.numu_out = nt, nu
        return outs, o

    douts, dout = make_out(dev, False)

    def step(b, o):
        rc = ctx.general_bands_solve(b, o)
        if rc != 0:
            raise RuntimeError(f"dsp_general_bands_solve: {capi.STATUS_NAMES.get(rc, rc)}: {ctx.last_error()}")

    for _ in range(args.warmup):
        step(batch, dout)
    torch.cuda.synchronize()
    bad = int((douts["status"] != 0).sum())
    clocks = ClockSampler(str(dev.index if dev.index is not None else 0))
    ctx.set_timing(True)
    ctx.timing_reset()
    replicas.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step(batch, dout)
    e1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ktimes = ctx.timings()
    ctx.set_timing(False)
    ms_max = replicas.max_over_ranks(ms, dev)
    value = replicas.job_rate(n, args.steps, world, ms_max)
    e2e = None
    if not args.no_e2e:
        hb, hkeep = capi.make_general_batch(d)
        houts, hout = make_out("cpu", True)
        h2d = sum(int(np.asarray(d[k]).nbytes) for k in ("num_streams", "num_layers", "layer_offset",
                                                          "num_phase_func_moments", "delta_tau", "single_scat_albedo",
                                                          "phase_function_moments") + capi.GENERAL_SCALAR_FIELDS)
        h2d += sum(int(np.asarray(d[k][0]).nbytes) for k in ("tau_user", "mu_user", "phi_user"))
        d2h = sum(int(v.numel() * v.element_size()) for v in houts.values())
        step(hb, hout)
        torch.cuda.synchronize()
        replicas.barrier()
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            step(hb, hout)
        e3.record(stream)
        torch.cuda.synchronize()
        replicas.barrier()
        te_max = replicas.max_over_ranks(e2.elapsed_time(e3), dev)
        same = all(torch.equal(houts[f], douts[f].cpu()) for f in houts)
        e2e = {"value": replicas.job_rate(n, args.steps, world, te_max), "unit": "solves/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "matches_device_result": same}
    dom = max((k for k in ktimes if k in fl), key=lambda k: ktimes[k][0])
    dom_ms, dom_launches = ktimes[dom]
    achieved = fl[dom] * args.steps / (dom_ms / 1000.0) / 1e12
    peak = fp64_peak_tflops()
    roofline = {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None,
                "peak_source": "measured on this GPU by disort_b200/csrc/fp64_peak.cu (FP64 FMA chains, burst)",
                "flops_per_step": fl[dom], "flops_total_per_step": fl["total"],
                "avg_launch_ms": dom_ms / max(1, dom_launches),
                "traffic": general_traffic(dom, n, dom_launches),
                "traffic_source": "profiles/traffic.json (ncu DRAM bytes per instance-solve of the boundary-value "
                                  "kernels on a 512-instance mix, x instances / launches)",
                "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
                "all_kernels_tflops": fl["total"] * args.steps / (ms_max / 1000.0) / 1e12}
    cpu, parity = None, None
    if rank == 0:
        if not args.no_cpu:
            lib, sample, flags, threads, idx = general_cpu_sample(insts, args.cpu_seconds)
            tcpu, ref = general_cpu_time(lib, sample, flags, threads, keep_outputs=True)
            cpu = {"value": len(sample) / tcpu, "unit": "solves/s", "cores": threads, "kind": "port",
                   "sample": f"{len(sample)} of {n} instances evenly spaced, oracle -march=native, "
                             f"{threads} OpenMP threads, {tcpu:.1f} s"}
            got = {k: v.cpu().numpy() for k, v in douts.items()}
            vs_double = general_parity(got, idx, ref)
            vs_double["checker"] = "oracle (double)"
            parity = vs_double
            if ext_parity:
                # the checker of record: the extended-precision build, each
                # element allowed 1e-9 rel + 1e-12 times max(1, twice the
                # instance's FP64 spread: the farthest of the double build on
                # the given inputs and on one-ulp-perturbed copies, in units of
                # that allowance); the plain comparisons with both builds beside it
                _, ref_ext = general_cpu_time(general_oracle_lib(ext=True), sample, flags, threads, keep_outputs=True)
                floor_refs = [ref]
                for copy_no in range(ULP_COPIES):
                    rng = np.random.default_rng(1000 + copy_no)
                    floor_refs.append(general_cpu_time(lib, [ulp_perturbed(c, rng) for c in sample], flags,
                                                       threads, keep_outputs=True)[1])
                parity = general_parity(got, idx, ref_ext, floor_ref=floor_refs)
                parity["checker"] = ("oracle (extended precision), allowance (1e-9 rel + 1e-12 abs) x max(1, twice "
                                     "the instance's FP64 spread: the largest distance from it, in those units, of "
                                     f"the double build on the given inputs and on {ULP_COPIES} copies with every "
                                     "layer input moved one ulp)")
                parity["vs_extended_precision_oracle"] = general_parity(got, idx, ref_ext)
                parity["vs_double_oracle"] = vs_double
    return {
            "metric": GENERAL_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
            "config": {"workload": f"general_mix_{n}", "instances_per_gpu": n,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "workspace larger than L2; no flush needed"},
            "e2e": e2e, "gpu_launches": int(sum(v[1] for v in ktimes.values())), "roofline": roofline,
            "cpu_baseline": cpu, "parity": parity, "clocks": clk, "bad_status_instances": bad}




# ---------------------------------------------------------------------------
# emulator training step on the tensor cores
# ---------------------------------------------------------------------------
def measured_bf16_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        j = json.load(open(p))
        return float(j["bf16_tflops"]), float(j["bf16_tflops_sustained"]), "MEASURED_PEAKS.json (measured)"
    except (OSError, ValueError, KeyError):
        return 1590.0, 1400.0, "fallback figure of this GPU pool"


def run_emulator(args):
    """Training throughput of the emulator MLP (494 -> 4 x 512 GELU -> 2 x 82, batch 4,096):
    one step = forward, loss gradient, backward and Adam over one batch; each epoch
    is 16 steps over a 65,536-row synthetic set."""
    import torch
    from disort_b200.emu import Emulator
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    B, rows = 4096, 65536
    e = Emulator(n_in=494, hidden=512, n_hidden_layers=4, n_out=82, n_heads=2, batch=B, seed=1, device=local,
                 stream=stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.zeros((rows, e.in_stride), dtype=torch.float32, device="cuda")
    x[:, :494] = torch.randn((rows, 494), generator=g, device="cuda")
    y = torch.randn((rows, 82), generator=g, device="cuda")
    e.set_data(x.to(torch.bfloat16), y)
    dims = e.layer_dims()
    fwd = sum(2.0 * B * a * b for a, b in dims)
    bwd_w = fwd
    bwd_x = sum(2.0 * B * a * b for a, b in dims[1:])
    step_flops = fwd + bwd_w + bwd_x
    steps_per_epoch = rows // B
    e.train(max(1, args.warmup), lr=1e-3, lr_min=1e-3)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(str(local))
    clocks.start()
    ev0.record(stream)
    e.train(args.steps, lr=1e-3, lr_min=1e-3)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    nsteps = args.steps * steps_per_epoch
    tflops = step_flops * nsteps / (ms / 1000.0) / 1e12
    peak, peak_sus, src = measured_bf16_peak()
    # the same kernel on one large GEMM (C = A B^T, 8192^3), where latency does not dominate
    Mg = 8192
    A = torch.randn((Mg, Mg), generator=g, device="cuda").to(torch.bfloat16)
    Bm = torch.randn((Mg, Mg), generator=g, device="cuda").to(torch.bfloat16)
    C = torch.empty((Mg, Mg), dtype=torch.float32, device="cuda")
    e.gemm(A, Bm, C)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(5):
        e.gemm(A, Bm, C)
    ev1.record(stream)
    torch.cuda.synchronize()
    big_tf = 5 * 2.0 * Mg ** 3 / (ev0.elapsed_time(ev1) / 1000.0) / 1e12
    ref = (A[:256].float() @ Bm[:256].float().T)
    big_err = float((C[:256, :256] - ref[:, :256]).abs().max() / ref[:, :256].abs().max())
    if rank == 0:
        print(json.dumps({
            "metric": "emulator training steps/s (BF16 tcgen05 GEMMs, batch 4096, 494-4x512-164)",
            "value": nsteps / (ms / 1000.0), "unit": "steps/s", "n_gpus": 1, "steps": nsteps,
            "warmup": args.warmup * steps_per_epoch, "ms_per_step": ms / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (fp32 accumulate)", "data": "synthetic",
            "config": {"workload": "emulator_train_step_b4096", "layers": dims},
            "roofline": {"bound": "tensor", "kernel": "all GEMMs of a training step (with epilogues, Adam, "
                         "transposes)", "achieved": tflops, "peak": peak_sus, "unit": "TFLOP/s",
                         "frac": tflops / peak_sus, "peak_source": src + ", sustained bf16 (kernel timed inside a "
                         "long loop)", "flops_per_step": step_flops},
            "large_gemm": {"shape": [Mg, Mg, Mg], "tflops": big_tf, "frac_of_burst_peak": big_tf / peak,
                           "burst_peak": peak, "max_rel_err_vs_fp32": big_err,
                           "note": "one tcgen05 GEMM with an FP32 store epilogue (includes the 256 MB C write)"},
            "clocks": clk}), flush=True)
    e.close()


def main():
    args = parse()
    if args.workload == "emulator":
        run_emulator(args)
    elif args.workload == "general":
        run_general(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
