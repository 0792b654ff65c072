"""The gated flux emulator: data from the GPU FP64 solver, tensor-core training,
and inference that routes doubtful instances back to the FP64 solve.

Instances are 40-layer, 16-stream thermal + solar columns.  Per (column, band):
  delta_tau  lognormal(-3, 2) clipped to [1e-6, 50], ssa U[0, 0.99], HG g U[0, 0.9]
  level T    linear from T_top U[180, 220] to T_surf U[280, 320] plus U(-10, 10)
  albedo U[0, 0.6], beam F0 = 1 at mu0 U[0.1, 1], emissivity_top 1, T_top 0 K,
  T_bottom = T_surf level, and one of 256 contiguous bands over 100-2,900 cm^-1.

The emulator corrects a cheap physical solve instead of predicting fluxes from
scratch: every instance is first solved in FP64 on the GPU with 4 streams
(about ten times faster than 16), and the network predicts the difference
between the 16-stream and the 4-stream fluxes.  A network trained to predict
the fluxes themselves from the same inputs (same architecture, same data)
reaches a held-out MSE of 0.007 per standardised output -- and the plain
PyTorch FP32 training of that network reaches the same -- but that leaves
~25 % median per-instance maximum error: the map from 40 layers of optical
properties to 82 fluxes is too sharp for the network to reach the 0.5 % bar.
The 4-stream solve carries the physics; the network learns its smooth bias.

Features (165 + 82 + 82): log delta_tau, ssa, g (40 each), the 41 level
temperatures, albedo, mu0, and the band edges nu_lo, nu_hi; physics features
computed from the same inputs: log cumulative optical depth at levels 1..40,
the level Planck fluxes pi B(T) / S and the thermal share of S, where
S = pi B(T_surface) + mu0 F0 is the instance's flux scale (B: band Planck
radiance, midpoint rule); and the 4-stream solution t4 = log(x4 + 1e-3) for the
82 fluxes x4 (flux_up and the diffuse downward flux at the 41 levels, over S).
Targets (82): t16 - t4, t16 the same transform of the 16-stream solution,
standardised per output.  The standardised features enter the network as
hi/lo BF16 pairs (x_hi = bf16(x), x_lo = bf16(x - x_hi)), 658 inputs carrying
about 16 mantissa bits.  The direct beam mu0 F0 exp(-tau/mu0) is exact and
added back, so the emulated total downward flux is direct + S * diffuse.

Relative flux error: |F - F_ref| / max(|F_ref|, 1e-3 max_k |F_ref,k|) over the
82 fluxes of an instance (flux_up and direct + diffuse down); the floor keeps
near-zero fluxes of an instance from dominating its error.

The gate sends an instance to the 16-stream FP64 solver when a raw feature
lies outside the training envelope or the two heads disagree by more than
0.2 % in the same floored relative measure.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import capi

L, N = 40, 16
N_LOW = 4  # streams of the cheap physical solve the network corrects
NLEV = L + 1
N_OUT = 2 * NLEV  # 82
N_RAW = 3 * L + NLEV + 4  # 165 input features
N_IN = N_RAW + L + NLEV + 1 + N_OUT  # + physics features + the 4-stream solution = 329
NBANDS = 256
BAND_W = 2800.0 / NBANDS
FLOOR_FRAC = 1e-3
GATE_TOL = 2e-3
EPS = 1e-3
C1, C2 = 1.191042e-8, 1.4387769  # W m^-2 sr^-1 (cm^-1)^-4, cm K


def band_edges(k):
    lo = 100.0 + BAND_W * np.asarray(k, dtype=np.float64)
    return lo, lo + BAND_W


def sample(n: int, seed: int, columns: int | None = None, ooe_columns: float = 0.0) -> dict:
    """n instances.  With `columns`, instances are column-major (column c, band b):
    temperature, albedo and mu0 belong to the column, optical properties to the
    instance, and a fraction `ooe_columns` of the columns is pushed out of the
    training envelope (delta_tau x 100, g = 0.98)."""
    rng = np.random.default_rng(seed)
    d = {}
    d["dtau"] = np.clip(rng.lognormal(-3.0, 2.0, (n, L)), 1e-6, 50.0)
    d["ssa"] = rng.uniform(0.0, 0.99, (n, L))
    d["g"] = rng.uniform(0.0, 0.9, (n, L))
    if columns is None:
        ncol, col = n, np.arange(n)
        d["band"] = rng.integers(0, NBANDS, n)
    else:
        ncol = columns
        col = np.arange(n) // NBANDS
        d["band"] = np.arange(n) % NBANDS
    ttop = rng.uniform(180.0, 220.0, ncol)
    tsurf = rng.uniform(280.0, 320.0, ncol)
    lev = np.arange(NLEV) / L
    T = ttop[:, None] + (tsurf - ttop)[:, None] * lev[None, :] + rng.uniform(-10.0, 10.0, (ncol, NLEV))
    d["T"] = T[col]
    d["albedo"] = rng.uniform(0.0, 0.6, ncol)[col]
    d["mu0"] = rng.uniform(0.1, 1.0, ncol)[col]
    d["ooe"] = np.zeros(n, dtype=bool)
    if columns is not None and ooe_columns > 0:
        pushed = rng.choice(ncol, size=int(round(ooe_columns * ncol)), replace=False)
        mask = np.isin(col, pushed)
        d["dtau"][mask] *= 100.0
        d["g"][mask] = 0.98
        d["ooe"] = mask
    d["wlo"], d["whi"] = band_edges(d["band"])
    return d


def device_inputs(d: dict, rows=None, dev="cuda") -> dict:
    """Per-instance flux-batch arrays on the device (all 40-layer, 16-stream)."""
    import torch
    sel = (lambda a: a) if rows is None else (lambda a: a[rows])
    g = sel(d["g"])
    pm = np.empty(g.shape + (N + 1,), dtype=np.float64)
    pm[..., 0] = 1.0
    for k in range(1, N + 1):
        pm[..., k] = pm[..., k - 1] * g
    T = sel(d["T"])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    c = lambda v: torch.tensor([v], dtype=torch.float64, device=dev)  # shared scalar (stride 0)
    return dict(wavenumber_low=t(sel(d["wlo"])), wavenumber_high=t(sel(d["whi"])), delta_tau=t(sel(d["dtau"])),
                single_scat_albedo=t(sel(d["ssa"])), phase_function_moments=t(pm), temperature=t(T),
                surface_albedo=t(sel(d["albedo"])), emissivity_top=c(1.0), direct_beam_flux=c(1.0),
                direct_beam_mu=t(sel(d["mu0"])), isotropic_flux_top=c(0.0), isotropic_flux_bottom=c(0.0),
                temperature_top=c(0.0), temperature_bottom=t(T[:, -1]))


def physics(arrays: dict):
    """Per-instance flux scale S [n], direct beam [n][41] and the physics features."""
    import torch
    n = arrays["delta_tau"].shape[0]
    tcum = torch.cumsum(arrays["delta_tau"], dim=1)
    mu0 = arrays["direct_beam_mu"].reshape(n, 1)
    fdir = torch.cat([mu0, mu0 * torch.exp(-tcum / mu0)], dim=1)
    nu = 0.5 * (arrays["wavenumber_low"] + arrays["wavenumber_high"]).reshape(n, 1)
    dnu = (arrays["wavenumber_high"] - arrays["wavenumber_low"]).reshape(n, 1)
    B = C1 * nu ** 3 * dnu / torch.expm1(C2 * nu / arrays["temperature"])
    sth = math.pi * B[:, -1:]
    S = sth + mu0
    feats = torch.cat([torch.log(tcum), math.pi * B / S, sth / S], dim=1)
    return S.reshape(n), fdir, feats


def log_diffuse(F, S, fdir):
    """t = log(diffuse / S + 1e-3) of fluxes [n][82] (the direct beam removed)."""
    import torch
    diffuse = F.clone()
    diffuse[:, NLEV:] -= fdir
    return torch.log((diffuse / S.reshape(-1, 1)).clamp_min(0.0) + EPS)


def features_device(arrays: dict, t4):
    """The 329 features from the device flux-batch arrays and the 4-stream
    solution t4 [n][82] (float32 [n][329])."""
    import torch
    n = arrays["delta_tau"].shape[0]
    pm = arrays["phase_function_moments"]
    cols = [torch.log(arrays["delta_tau"]), arrays["single_scat_albedo"], pm[:, :, 1], arrays["temperature"],
            arrays["surface_albedo"].reshape(n, 1), arrays["direct_beam_mu"].reshape(n, 1),
            arrays["wavenumber_low"].reshape(n, 1), arrays["wavenumber_high"].reshape(n, 1), physics(arrays)[2],
            t4]
    return torch.cat(cols, dim=1).float().contiguous()


def reconstruct(y, mu, sd, S, fdir, t4):
    """Fluxes [n][82] from the standardised correction predicted by one head."""
    import torch
    x = torch.exp(t4.double() + y.double() * sd.double() + mu.double()) - EPS
    F = S.double().reshape(-1, 1) * x
    F[:, NLEV:] += fdir
    return F


def solve_fp64(ctx: capi.Context, arrays: dict, n: int, chunk: int = 262144, nstr: int = N):
    """FP64 GPU solves of n instances with `nstr` streams: fluxes [n][82]
    (flux_up, direct + diffuse down)."""
    import torch
    dev = arrays["delta_tau"].device
    out = torch.empty((n, N_OUT), dtype=torch.float64, device=dev)
    st_all = torch.empty((n,), dtype=torch.int32, device=dev)
    for r0 in range(0, n, chunk):
        m = min(chunk, n - r0)
        part = {}
        for k, v in arrays.items():
            part[k] = v[r0:r0 + m] if hasattr(v, "shape") and v.dim() >= 1 and v.shape[0] == n else v
        # the moment array holds N + 1 = 17 moments; a 4-stream solve reads the first 5
        batch, keep = capi.make_flux_batch(m, nstr, L, 0, N + 1, capi.FLAG_THERMAL | capi.FLAG_DEVICE_POINTERS,
                                           part)
        outs = {f: torch.empty((m, NLEV), dtype=torch.float64, device=dev) for f in capi.FLUX_OUT_FIELDS}
        st = torch.empty((m,), dtype=torch.int32, device=dev)
        o, keep2 = capi.make_flux_out(outs, st)
        rc = ctx.flux_bands_solve(batch, o)
        if rc != 0:
            raise RuntimeError(f"flux solve: {ctx.last_error()}")
        out[r0:r0 + m, :NLEV] = outs["flux_up"]
        out[r0:r0 + m, NLEV:] = outs["flux_direct_beam"] + outs["flux_down"]
        st_all[r0:r0 + m] = st
    return out, st_all


def rel_err(F, R):
    """Floored relative error per flux (torch tensors [n][82])."""
    import torch
    floor = FLOOR_FRAC * R.abs().amax(dim=1, keepdim=True)
    return (F - R).abs() / torch.maximum(R.abs(), floor)


class Surrogate:
    """Normalisation, envelope and the trained emulator."""

    def __init__(self, emu, fmean, fstd, lo, hi, mu, sd):
        self.emu, self.fmean, self.fstd, self.lo, self.hi, self.mu, self.sd = emu, fmean, fstd, lo, hi, mu, sd

    def encode(self, raw):
        """Standardised features as hi/lo BF16 pairs [n][in_stride] for the emulator."""
        import torch
        z = (raw - self.fmean) / self.fstd
        hi = z.to(torch.bfloat16)
        lo = (z - hi.float()).to(torch.bfloat16)
        x = torch.zeros((raw.shape[0], self.emu.in_stride), dtype=torch.bfloat16, device=raw.device)
        x[:, :N_IN] = hi
        x[:, N_IN:2 * N_IN] = lo
        return x


def train(ctx: capi.Context, n_columns: int = 1 << 20, epochs: int = 50, batch: int = 4096, seed: int = 4,
          holdout: float = 0.05, log=print):
    """Generate solver labels on the GPU, train the emulator; returns (Surrogate, report)."""
    import torch
    from .emu import Emulator
    t0 = time.perf_counter()
    d = sample(n_columns, seed)
    arrays = device_inputs(d)
    F, st = solve_fp64(ctx, arrays, n_columns)
    F4, st4 = solve_fp64(ctx, arrays, n_columns, nstr=N_LOW)
    torch.cuda.synchronize()
    t_label = time.perf_counter() - t0
    bad = int((st != 0).sum()) + int((st4 != 0).sum())
    S, fdir, _ = physics(arrays)
    t4 = log_diffuse(F4, S, fdir)
    raw = features_device(arrays, t4)
    ntr = int(n_columns * (1.0 - holdout)) // batch * batch
    t = log_diffuse(F, S, fdir) - t4
    mu = t[:ntr].mean(dim=0)
    sd = t[:ntr].std(dim=0).clamp_min(1e-6)
    y = ((t - mu) / sd).float()
    fmean = raw[:ntr].mean(dim=0)
    fstd = raw[:ntr].std(dim=0).clamp_min(1e-6)
    # training envelope, widened by 1 % of each feature's range
    lo = raw[:ntr].amin(dim=0)
    hi = raw[:ntr].amax(dim=0)
    span = hi - lo
    lo, hi = lo - 0.01 * span, hi + 0.01 * span
    emu = Emulator(n_in=2 * N_IN, hidden=512, n_hidden_layers=4, n_out=N_OUT, n_heads=2, batch=batch, seed=seed)
    sur = Surrogate(emu, fmean, fstd, lo, hi, mu.float(), sd.float())
    X = sur.encode(raw)
    # bagging: each head sees every training instance with a Poisson(1) weight
    hw = torch.from_numpy(np.random.default_rng(seed + 1).poisson(1.0, (ntr, 2)).astype(np.float32)).cuda()
    emu.set_data(X[:ntr].contiguous(), y[:ntr].contiguous(), hw)
    t1 = time.perf_counter()
    losses = emu.train(epochs, lr=1e-3, lr_min=1e-5, seed=seed + 2)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    # held-out error of the corrected solve (head mean) and of the 4-stream solve alone
    Xh = X[ntr:].contiguous()
    preds = torch.empty((Xh.shape[0], 2 * N_OUT), dtype=torch.float32, device="cuda")
    emu.forward(Xh, preds)
    Sh, fh, t4h = S[ntr:], fdir[ntr:], t4[ntr:]
    Fe = 0.5 * (reconstruct(preds[:, :N_OUT], mu, sd, Sh, fh, t4h) + reconstruct(preds[:, N_OUT:], mu, sd, Sh, fh, t4h))
    emax = rel_err(Fe, F[ntr:]).amax(dim=1)
    e4 = rel_err(F4[ntr:], F[ntr:]).amax(dim=1)
    per_out = 1.0 / (2 * N_OUT)  # the training loss sums the squared errors of 82 outputs over 2 heads
    report = dict(columns=n_columns, train_columns=ntr, holdout_columns=n_columns - ntr, epochs=epochs, batch=batch,
                  label_seconds=t_label, train_seconds=t_train, bad_label_status=bad, first_loss=losses[0],
                  last_loss=losses[-1], last_loss_per_output=losses[-1] * per_out,
                  holdout_max_rel_err=float(emax.max()),
                  holdout_p99_rel_err=float(torch.quantile(emax.float(), 0.99)),
                  holdout_median_rel_err=float(emax.median()),
                  four_stream_alone=dict(max_rel_err=float(e4.max()),
                                         p99_rel_err=float(torch.quantile(e4.float(), 0.99)),
                                         median_rel_err=float(e4.median())))
    log(f"emulator: labels {t_label:.1f} s, training {t_train:.1f} s, loss {losses[0]:.4g} -> {losses[-1]:.4g}, "
        f"held-out max/p99/median rel err {report['holdout_max_rel_err']:.3g}/{report['holdout_p99_rel_err']:.3g}/"
        f"{report['holdout_median_rel_err']:.3g} (4-stream alone: median {report['four_stream_alone']['median_rel_err']:.3g})")
    return sur, report


def emulate(ctx: capi.Context, sur: Surrogate, arrays: dict, n: int):
    """The 4-stream solve, the features and both heads' predictions, shifted so
    that pred * sd + mu is the corrected log flux (t4 folded in).  Returns
    (raw features, predictions [n][164], S, direct beam, t4)."""
    import torch
    S, fdir, _ = physics(arrays)
    F4, _ = solve_fp64(ctx, arrays, n, nstr=N_LOW)
    t4 = log_diffuse(F4, S, fdir)
    raw = features_device(arrays, t4)
    X = sur.encode(raw)
    preds = torch.empty((n, 2 * N_OUT), dtype=torch.float32, device="cuda")
    sur.emu.forward(X, preds)
    shift = (t4 / sur.sd).float()
    preds[:, :N_OUT] += shift
    preds[:, N_OUT:] += shift
    return raw, preds, S, fdir, t4


def gated_run(ctx: capi.Context, sur: Surrogate, arrays: dict, n: int, tol: float = GATE_TOL):
    """Emulate every instance, re-solve the gated ones in FP64, merge.  Returns the
    fluxes [n][82], the fallback count and the fallback flags [n] (int32)."""
    import torch
    raw, preds, S, fdir, _ = emulate(ctx, sur, arrays, n)
    add = torch.zeros((n, N_OUT), dtype=torch.float32, device="cuda")
    add[:, NLEV:] = fdir
    flux = torch.empty((n, N_OUT), dtype=torch.float32, device="cuda")
    fb = torch.empty((n,), dtype=torch.int32, device="cuda")
    idx = torch.empty((n,), dtype=torch.int32, device="cuda")
    cnt = torch.zeros((1,), dtype=torch.int32, device="cuda")
    # the envelope test reads the first n_in raw values of each row: raw features twice (hi and lo share it)
    raw2 = torch.cat([raw, raw], dim=1).contiguous()
    lo2, hi2 = torch.cat([sur.lo, sur.lo]), torch.cat([sur.hi, sur.hi])
    sur.emu.gate(raw2, lo2, hi2, preds, sur.mu, sur.sd, S.float().contiguous(), add, EPS, tol, FLOOR_FRAC,
                 flux, fb, idx, cnt)
    k = int(cnt.item())
    out = flux.double()
    if k:
        rows = idx[:k].long()
        sub = {key: (v.index_select(0, rows) if hasattr(v, "shape") and v.dim() >= 1 and v.shape[0] == n else v)
               for key, v in arrays.items()}
        Fk, _ = solve_fp64(ctx, sub, k)
        out.index_copy_(0, rows, Fk)
    return out, k, fb


def evaluate(ctx: capi.Context, sur: Surrogate, columns: int = 4096, seed: int = 5, ooe: float = 0.05,
             repeats: int = 3, tols=(5e-3, 1e-2, 2e-2, 5e-2)) -> dict:
    """Gated inference against the plain FP64 solve on columns x 256 bands (timed on the device)."""
    import torch
    n = columns * NBANDS
    d = sample(n, seed, columns=columns, ooe_columns=ooe)
    arrays = device_inputs(d)
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    F_ref, _ = solve_fp64(ctx, arrays, n)
    torch.cuda.synchronize()
    a, b = ev()
    a.record()
    for _ in range(repeats):
        F_ref, st = solve_fp64(ctx, arrays, n)
    b.record()
    torch.cuda.synchronize()
    t_plain = a.elapsed_time(b) / 1000.0 / repeats
    # gated: 4-stream solve -> features -> emulator -> gate -> 16-stream FP64 solve of the fallback instances
    F_g, k, _ = gated_run(ctx, sur, arrays, n)
    torch.cuda.synchronize()
    a, b = ev()
    a.record()
    for _ in range(repeats):
        F_g, k, _ = gated_run(ctx, sur, arrays, n)
    b.record()
    torch.cuda.synchronize()
    t_gated = a.elapsed_time(b) / 1000.0 / repeats
    e = rel_err(F_g, F_ref).amax(dim=1)
    ooe_mask = torch.from_numpy(d["ooe"]).cuda()
    res = dict(instances=n, columns=columns, bands=NBANDS, out_of_envelope_instances=int(ooe_mask.sum()),
               plain_solves_per_s=n / t_plain, gated_solves_per_s=n / t_gated, speedup=t_plain / t_gated,
               gate_tol=GATE_TOL, fallback_instances=k, fallback_fraction=k / n, max_rel_err=float(e.max()),
               p99_rel_err=float(torch.quantile(e.float(), 0.99)), median_rel_err=float(e.median()),
               plain_seconds=t_plain, gated_seconds=t_gated, bad_status=int((st != 0).sum()))
    # the trade-off of looser gates (one timed run each)
    sweep = []
    for tol in tols:
        a, b = ev()
        a.record()
        F_t, k_t, _ = gated_run(ctx, sur, arrays, n, tol)
        b.record()
        torch.cuda.synchronize()
        tt = a.elapsed_time(b) / 1000.0
        et = rel_err(F_t, F_ref).amax(dim=1)
        sweep.append(dict(gate_tol=tol, fallback_fraction=k_t / n, speedup=t_plain / tt,
                          max_rel_err=float(et.max()), p99_rel_err=float(torch.quantile(et.float(), 0.99))))
    res["gate_sweep"] = sweep
    # the corrected solve alone (no gate) on the in-envelope instances, beside the
    # 4-stream solve it corrects: what the network gains
    raw, preds, S, fdir, t4 = emulate(ctx, sur, arrays, n)
    zero = torch.zeros_like(t4)
    Fe = 0.5 * (reconstruct(preds[:, :N_OUT], sur.mu, sur.sd, S, fdir, zero) +
                reconstruct(preds[:, N_OUT:], sur.mu, sur.sd, S, fdir, zero))
    ee = rel_err(Fe, F_ref).amax(dim=1)[~ooe_mask]
    F4, _ = solve_fp64(ctx, arrays, n, nstr=N_LOW)
    e4 = rel_err(F4, F_ref).amax(dim=1)[~ooe_mask]
    res["emulator_only_in_envelope"] = dict(max_rel_err=float(ee.max()), p99_rel_err=float(torch.quantile(ee.float(), 0.99)),
                                            median_rel_err=float(ee.median()))
    res["four_stream_alone_in_envelope"] = dict(max_rel_err=float(e4.max()),
                                                p99_rel_err=float(torch.quantile(e4.float(), 0.99)),
                                                median_rel_err=float(e4.median()))
    # the 4-stream solve's own rate on these instances (the floor of the gated path's cost)
    a, b = ev()
    a.record()
    solve_fp64(ctx, arrays, n, nstr=N_LOW)
    b.record()
    torch.cuda.synchronize()
    res["four_stream_solves_per_s"] = n / (a.elapsed_time(b) / 1000.0)
    return res


# ---------------------------------------------------------------------------
# save / load: a JSON header and one little-endian binary blob
# ---------------------------------------------------------------------------
SAVE_FORMAT = "disort_b200.surrogate"
SAVE_VERSION = 1
_VECTORS = ("fmean", "fstd", "lo", "hi", "mu", "sd")


def write_blob(path: str, header: dict, blocks: list) -> None:
    """`path`.json holds `header` plus the list of blocks (name, dtype, shape,
    byte offset); `path`.bin holds the blocks back to back, little-endian."""
    import json
    meta, off = [], 0
    with open(path + ".bin", "wb") as f:
        for name, a in blocks:
            a = np.ascontiguousarray(a)
            a = a.astype(a.dtype.newbyteorder("<"), copy=False)
            f.write(a.tobytes())
            meta.append(dict(name=name, dtype=a.dtype.str, shape=list(a.shape), offset=off, nbytes=a.nbytes))
            off += a.nbytes
    h = dict(header)
    h["blocks"] = meta
    h["blob_bytes"] = off
    with open(path + ".json", "w") as f:
        json.dump(h, f, indent=1)


def read_blob(path: str, fmt: str, version: int) -> tuple[dict, dict]:
    """Header and {name: array} of a write_blob pair; ValueError when the format,
    version or blob size does not match."""
    import json
    with open(path + ".json") as f:
        h = json.load(f)
    if h.get("format") != fmt or h.get("version") != version:
        raise ValueError(f"{path}.json: format {h.get('format')!r} version {h.get('version')!r}, "
                         f"expected {fmt!r} version {version}")
    with open(path + ".bin", "rb") as f:
        raw = f.read()
    if len(raw) != h["blob_bytes"]:
        raise ValueError(f"{path}.bin: {len(raw)} bytes, header says {h['blob_bytes']}")
    out = {}
    for b in h["blocks"]:
        a = np.frombuffer(raw, dtype=np.dtype(b["dtype"]), count=int(np.prod(b["shape"], dtype=np.int64)),
                          offset=b["offset"])
        out[b["name"]] = a.reshape(b["shape"]).copy()
    return h, out


def save(sur: Surrogate, path: str) -> None:
    """The trained emulator's FP32 master weights, its configuration and the
    normalisation and envelope vectors, to `path`.json + `path`.bin."""
    e = sur.emu
    params = np.empty(e.param_count(), dtype=np.float32)
    e.get_params(params)
    c = e.cfg
    header = dict(format=SAVE_FORMAT, version=SAVE_VERSION,
                  emulator=dict(n_in=c.n_in, hidden=c.hidden, n_hidden_layers=c.n_hidden_layers, n_out=c.n_out,
                                n_heads=c.n_heads, batch=c.batch, seed=c.seed),
                  layer_dims=[list(d) for d in e.layer_dims()],
                  instances=dict(layers=L, streams=N, low_streams=N_LOW, features=N_IN, outputs=N_OUT,
                                 bands=NBANDS, floor_frac=FLOOR_FRAC, gate_tol=GATE_TOL, eps=EPS))
    blocks = [("params", params)] + [(k, getattr(sur, k).detach().cpu().numpy()) for k in _VECTORS]
    write_blob(path, header, blocks)


def load(path: str, device: int = 0, stream: int = 0) -> Surrogate:
    """A Surrogate from a save() pair: a new emulator with the stored weights."""
    import torch
    from .emu import Emulator
    h, b = read_blob(path, SAVE_FORMAT, SAVE_VERSION)
    inst = h["instances"]
    if (inst["layers"], inst["streams"], inst["low_streams"], inst["features"], inst["outputs"]) != \
            (L, N, N_LOW, N_IN, N_OUT):
        raise ValueError(f"{path}.json: saved for a different instance layout ({inst})")
    c = h["emulator"]
    emu = Emulator(n_in=c["n_in"], hidden=c["hidden"], n_hidden_layers=c["n_hidden_layers"], n_out=c["n_out"],
                   n_heads=c["n_heads"], batch=c["batch"], seed=c["seed"], device=device, stream=stream)
    if emu.param_count() != b["params"].size or [list(d) for d in emu.layer_dims()] != h["layer_dims"]:
        emu.close()
        raise ValueError(f"{path}: parameter layout does not match the emulator's")
    emu.set_params(np.ascontiguousarray(b["params"], dtype=np.float32))
    dev = torch.device("cuda", device)
    vec = {k: torch.from_numpy(b[k]).to(dev) for k in _VECTORS}
    return Surrogate(emu, vec["fmean"], vec["fstd"], vec["lo"], vec["hi"], vec["mu"], vec["sd"])
