"""ctypes mirror of include/dsp.h.

This is the thin binding a ctypes user of the C ABI writes: the structures of
dsp.h, the prototypes of the entry points, and a helper that packs per-instance
arrays into a ``dsp_flux_batch``.  The same structures are passed to the CPU
oracle library in tests, so both sides see byte-identical inputs.

Arrays may be numpy arrays (host memory) or torch tensors (host or device); an
array of one instance's shape is shared by all instances (stride 0), an array
with a leading ``n_inst`` axis is per instance.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int32, c_int64, c_uint32, c_void_p

import numpy as np

DSP_OK = 0
DSP_ERR_INVALID_INPUT = 1
DSP_ERR_SINGULAR = 2
DSP_ERR_NONFINITE = 3
DSP_ERR_TIMEOUT = 4
DSP_ERR_CUDA = 5
DSP_ERR_UNSUPPORTED = 6
DSP_ERR_NO_MEMORY = 7
DSP_ERR_EIGEN = 8
DSP_ERR_NOT_INITIALIZED = 9

STATUS_NAMES = {
    0: "OK", 1: "INVALID_INPUT", 2: "SINGULAR", 3: "NONFINITE", 4: "TIMEOUT",
    5: "CUDA_ERROR", 6: "UNSUPPORTED", 7: "NO_MEMORY", 8: "EIGEN", 9: "NOT_INITIALIZED",
}

FLAG_THERMAL = 1 << 0
FLAG_DELTA_M_PLUS = 1 << 1
FLAG_DIFFUSION_LOWER_BC = 1 << 2
FLAG_INDEX_FROM_BOTTOM = 1 << 3
FLAG_DEVICE_POINTERS = 1 << 4
FLAG_SPHERICAL_BEAM = 1 << 5
FLAG_TEMPERATURE_JAC = 1 << 6
FLAG_HG_G = 1 << 7

DEBUG_POISON_SCRATCH = 1  # dsp_context_set_debug

GFLAG_USER_TAU = 1 << 8
GFLAG_USER_MU = 1 << 9
GFLAG_ONLY_FLUXES = 1 << 10
GFLAG_INTENSITY_CORR = 1 << 11
GFLAG_INTENSITY_CORR_BE = 1 << 12

SUPPORTED_NSTR = (4, 6, 8, 10, 12, 14, 16, 32, 64)


class DArray(ctypes.Structure):
    _fields_ = [("ptr", c_void_p), ("stride", c_int64)]


FLUX_ARRAY_FIELDS = (
    "wavenumber_low", "wavenumber_high", "delta_tau", "single_scat_albedo",
    "phase_function_moments", "temperature", "surface_albedo", "emissivity_top",
    "direct_beam_flux", "direct_beam_mu", "isotropic_flux_top", "isotropic_flux_bottom",
    "temperature_top", "temperature_bottom", "level_altitudes", "bottom_radius",
)

FLUX_OUT_FIELDS = (
    "flux_direct_beam", "flux_down", "flux_up", "flux_tau_divergence",
    "mean_intensity", "mean_intensity_down", "mean_intensity_up", "mean_intensity_direct_beam",
)


class FluxBatch(ctypes.Structure):
    _fields_ = [
        ("n_inst", c_int32), ("num_streams", c_int32), ("num_layers", c_int32),
        ("num_phase_func_moments", c_int32), ("pmom_count", c_int32), ("flags", c_uint32),
    ] + [(f, DArray) for f in FLUX_ARRAY_FIELDS]


class FluxOut(ctypes.Structure):
    _fields_ = [(f, POINTER(c_double)) for f in FLUX_OUT_FIELDS] + [("status", POINTER(c_int32))]


# dsp_flux_jac_out: temperature Jacobians, each [n_inst][L+1][L+2]
JAC_FIELDS = ("flux_up", "flux_down", "mean_intensity", "mean_intensity_down", "mean_intensity_up",
              "flux_divergence")
# the FluxResult output each Jacobian differentiates
JAC_OF = dict(zip(JAC_FIELDS, ("flux_up", "flux_down", "mean_intensity", "mean_intensity_down",
                               "mean_intensity_up", "flux_tau_divergence")))


class FluxJacOut(ctypes.Structure):
    _fields_ = [(f, POINTER(c_double)) for f in JAC_FIELDS]


def make_flux_jac_out(arrays: dict) -> tuple[FluxJacOut, list]:
    o = FluxJacOut()
    keep = []
    for f in JAC_FIELDS:
        a = arrays[f]
        keep.append(a)
        setattr(o, f, ctypes.cast(c_void_p(_ptr(a)), POINTER(c_double)))
    return o, keep


def alloc_flux_jac_numpy(n_inst: int, num_layers: int) -> dict:
    return {f: np.full((n_inst, num_layers + 1, num_layers + 2), np.nan) for f in JAC_FIELDS}


def _ptr(a) -> int:
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor


def _darray(a, per_inst_ndim: int, n_inst: int, keep: list) -> DArray:
    """Stride 0 if `a` has one instance's shape, else the per-instance element count."""
    if a is None:
        return DArray(0, 0)
    if isinstance(a, (int, float)):
        a = np.array([float(a)], dtype=np.float64)
    if isinstance(a, np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
    keep.append(a)
    ndim = a.ndim if isinstance(a, np.ndarray) else a.dim()
    if ndim == per_inst_ndim + 1 and a.shape[0] == n_inst and per_inst_ndim >= 0:
        per = 1
        for s in a.shape[1:]:
            per *= int(s)
        return DArray(_ptr(a), per)
    return DArray(_ptr(a), 0)


def make_flux_batch(n_inst: int, num_streams: int, num_layers: int, num_phase_func_moments: int,
                    pmom_count: int, flags: int, arrays: dict) -> tuple[FluxBatch, list]:
    """Pack arrays into a dsp_flux_batch.  Returns (batch, keepalive list)."""
    keep: list = []
    per_ndim = {  # dimensions of one instance's value
        "delta_tau": 1, "single_scat_albedo": 1, "phase_function_moments": 2, "temperature": 1,
        "level_altitudes": 1,
    }
    if flags & FLAG_HG_G:  # one asymmetry factor per layer instead of moments
        per_ndim["phase_function_moments"] = 1
    b = FluxBatch()
    b.n_inst = n_inst
    b.num_streams = num_streams
    b.num_layers = num_layers
    b.num_phase_func_moments = num_phase_func_moments
    b.pmom_count = pmom_count
    b.flags = flags
    for f in FLUX_ARRAY_FIELDS:
        a = arrays.get(f)
        nd = per_ndim.get(f, 0)
        if nd == 0 and a is not None and not isinstance(a, (int, float)):
            # scalar field: shape () or (1,) shared, (n_inst,) per instance
            if isinstance(a, np.ndarray):
                a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
                if a.shape[0] == n_inst and n_inst > 1:
                    keep.append(a)
                    setattr(b, f, DArray(_ptr(a), 1))
                    continue
                a = a[:1].copy()
            else:  # torch
                a = a.reshape(-1)
                if a.shape[0] == n_inst and n_inst > 1:
                    keep.append(a)
                    setattr(b, f, DArray(_ptr(a), 1))
                    continue
        setattr(b, f, _darray(a, nd, n_inst, keep))
    return b, keep


def make_flux_out(arrays: dict, status=None) -> tuple[FluxOut, list]:
    o = FluxOut()
    keep = []
    for f in FLUX_OUT_FIELDS:
        a = arrays[f]
        keep.append(a)
        setattr(o, f, ctypes.cast(c_void_p(_ptr(a)), POINTER(c_double)))
    o.status = ctypes.cast(c_void_p(_ptr(status)), POINTER(c_int32)) if status is not None else None
    keep.append(status)
    return o, keep


GENERAL_SCALAR_FIELDS = (
    "wavenumber_low", "wavenumber_high", "surface_albedo", "emissivity_top", "direct_beam_flux",
    "direct_beam_mu", "direct_beam_phi", "isotropic_flux_top", "isotropic_flux_bottom",
    "temperature_top", "temperature_bottom",
)
GENERAL_SCALAR_DEFAULTS = dict(wavenumber_low=0.0, wavenumber_high=0.0, surface_albedo=0.0,
                               emissivity_top=1.0, direct_beam_flux=0.0, direct_beam_mu=0.5,
                               direct_beam_phi=0.0, isotropic_flux_top=0.0, isotropic_flux_bottom=0.0,
                               temperature_top=0.0, temperature_bottom=0.0)


# surface models (dsp.h DSP_BRDF_*; the BrdfType enum of the reference)
BRDF_LAMBERTIAN, BRDF_RPV, BRDF_COX_MUNK, BRDF_AMBRALS, BRDF_HAPKE = 0, 1, 2, 3, 4
BRDF_PARAMS = 8


class GeneralBatch(ctypes.Structure):
    _fields_ = [
        ("n_inst", c_int32), ("flags", c_uint32),
        ("num_streams", c_void_p), ("num_layers", c_void_p), ("layer_offset", c_void_p),
        ("num_phase_func_moments", c_void_p), ("pmom_count", c_int32),
        ("num_user_tau", c_int32), ("num_user_mu", c_int32), ("num_phi", c_int32),
        ("accuracy_fourier_series", c_double),
        ("delta_tau", c_void_p), ("single_scat_albedo", c_void_p), ("phase_function_moments", c_void_p),
        ("temperature", c_void_p),
        ("tau_user", DArray), ("mu_user", DArray), ("phi_user", DArray),
    ] + [(f, DArray) for f in GENERAL_SCALAR_FIELDS] + [("level_altitudes", c_void_p), ("bottom_radius", DArray),
                                                        ("brdf_type", c_int32), ("brdf_params", DArray),
                                                        ("num_phase_func_angles", c_int32),
                                                        ("mu_phase_function", DArray), ("phase_function", c_void_p)]


class GeneralOut(ctypes.Structure):
    _fields_ = [("flux", POINTER(c_double) * 8), ("intensity", POINTER(c_double)),
                ("intensity_azimuth_avg", POINTER(c_double)), ("status", POINTER(c_int32)),
                ("ntau_out", c_int32), ("numu_out", c_int32)]


def _user_list(insts, key, n):
    """(array, stride): stride 0 when every instance carries the same list."""
    vals = [np.asarray(c.get(key), dtype=np.float64).reshape(-1) for c in insts]
    if any(v.size != n for v in vals):
        raise ValueError(f"{key}: every instance needs {n} values")
    if all(np.array_equal(v, vals[0]) for v in vals):
        return np.ascontiguousarray(vals[0]), 0
    return np.ascontiguousarray(np.stack(vals)), n


def pack_general(insts: list, flags: int, accuracy_fourier_series: float = 0.0,
                 pmom_count: int | None = None) -> dict:
    """Pack per-instance dicts into host arrays for a dsp_general_batch.

    Each instance dict carries num_streams, num_layers, num_phase_func_moments,
    delta_tau [L], single_scat_albedo [L], phase_function_moments [L][>= nmomNstr+1],
    temperature [L+1] (thermal), the scalar fields of GENERAL_SCALAR_FIELDS
    (defaults as DisortConfig) and, as the flags ask, tau_user, mu_user, phi_user.
    Returns a dict of numpy arrays and dimensions (see make_general_batch)."""
    n = len(insts)
    N = np.array([c["num_streams"] for c in insts], dtype=np.int32)
    L = np.array([c["num_layers"] for c in insts], dtype=np.int32)
    nmom = np.array([c.get("num_phase_func_moments", 0) for c in insts], dtype=np.int32)
    off = np.zeros(n + 1, dtype=np.int64)
    off[1:] = np.cumsum(L)
    if pmom_count is None:
        pmom_count = int(max(len(np.asarray(c["phase_function_moments"])[0]) for c in insts))
    tot = int(off[-1])
    dtau = np.zeros(tot)
    ssa = np.zeros(tot)
    pm = np.zeros((tot, pmom_count))
    temp = np.zeros(tot + n)
    for i, c in enumerate(insts):
        a, b = off[i], off[i + 1]
        dtau[a:b] = c["delta_tau"]
        ssa[a:b] = c["single_scat_albedo"]
        m = np.asarray(c["phase_function_moments"], dtype=np.float64)
        pm[a:b, :m.shape[1]] = m[:, :pmom_count]
        t = c.get("temperature")
        if t is not None and len(t):
            temp[a + i:b + i + 1] = t
    d = dict(n_inst=n, flags=flags, num_streams=N, num_layers=L, layer_offset=off,
             num_phase_func_moments=nmom, pmom_count=pmom_count, accuracy=float(accuracy_fourier_series),
             delta_tau=dtau, single_scat_albedo=ssa, phase_function_moments=pm, temperature=temp)
    if flags & FLAG_SPHERICAL_BEAM:  # level altitudes [L+1] per instance (like temperature), radius per instance
        zalt = np.zeros(tot + n)
        for i, c in enumerate(insts):
            za = c.get("level_altitudes")
            if za is not None:
                zalt[off[i] + i:off[i + 1] + i + 1] = za
        d["level_altitudes"] = zalt
        d["bottom_radius"] = np.array([float(c.get("bottom_radius", 0.0)) for c in insts])
    for f in GENERAL_SCALAR_FIELDS:
        d[f] = np.array([float(c.get(f, GENERAL_SCALAR_DEFAULTS[f])) for c in insts])
    ntau = numu = nphi = 0
    if flags & GFLAG_USER_TAU:
        ntau = len(insts[0]["tau_user"])
        d["tau_user"] = _user_list(insts, "tau_user", ntau)
    if flags & GFLAG_USER_MU:
        numu = len(insts[0]["mu_user"])
        d["mu_user"] = _user_list(insts, "mu_user", numu)
    if not (flags & GFLAG_ONLY_FLUXES) or insts[0].get("phi_user") is not None:
        if insts[0].get("phi_user") is not None:
            nphi = len(insts[0]["phi_user"])
            d["phi_user"] = _user_list(insts, "phi_user", nphi)
    d["num_user_tau"], d["num_user_mu"], d["num_phi"] = ntau, numu, nphi
    # bidirectional surface: one type for the batch, parameters per instance
    types = {int(c.get("brdf_type", BRDF_LAMBERTIAN)) for c in insts}
    if len(types) != 1:
        raise ValueError("brdf_type: one surface model per batch")
    d["brdf_type"] = types.pop()
    if d["brdf_type"] != BRDF_LAMBERTIAN:
        bp = np.zeros((n, BRDF_PARAMS))
        for i, c in enumerate(insts):
            v = np.asarray(c.get("brdf_params", ()), dtype=np.float64).reshape(-1)
            bp[i, :v.size] = v
        d["brdf_params"] = bp
    # tabulated phase function (Buras-Emde correction): angles shared or per instance,
    # values per layer like delta_tau
    if insts[0].get("mu_phase_function") is not None:
        na = len(insts[0]["mu_phase_function"])
        d["num_phase_func_angles"] = na
        d["mu_phase_function"] = _user_list(insts, "mu_phase_function", na)
        pf = np.zeros((tot, na))
        for i, c in enumerate(insts):
            pf[off[i]:off[i + 1]] = np.asarray(c["phase_function"], dtype=np.float64).reshape(-1, na)
        d["phase_function"] = pf
    d["ntau_out"] = ntau if flags & GFLAG_USER_TAU else int(L.max()) + 1
    d["numu_out"] = numu if (flags & GFLAG_USER_MU and not flags & GFLAG_ONLY_FLUXES) else int(N.max())
    return d


def make_general_batch(d: dict) -> tuple[GeneralBatch, list]:
    """dsp_general_batch over the arrays of pack_general (host pointers, or
    CUDA tensors in place of every array with FLAG_DEVICE_POINTERS)."""
    if d["flags"] & FLAG_DEVICE_POINTERS:
        host = [k for k, v in d.items() if isinstance(v, np.ndarray) or
                (isinstance(v, tuple) and v and isinstance(v[0], np.ndarray))]
        host = [k for k in host if k not in ("ntau_out", "numu_out")]
        if host:
            raise ValueError(f"FLAG_DEVICE_POINTERS with host arrays: {host}")
    keep = [d]
    b = GeneralBatch()
    b.n_inst = d["n_inst"]
    b.flags = d["flags"]
    for f in ("num_streams", "num_layers", "layer_offset", "num_phase_func_moments",
              "delta_tau", "single_scat_albedo", "phase_function_moments", "temperature"):
        setattr(b, f, _ptr(d[f]))
    b.pmom_count = d["pmom_count"]
    b.num_user_tau, b.num_user_mu, b.num_phi = d["num_user_tau"], d["num_user_mu"], d["num_phi"]
    b.accuracy_fourier_series = d["accuracy"]
    for f in ("tau_user", "mu_user", "phi_user"):
        if f in d:
            a, stride = d[f]
            setattr(b, f, DArray(_ptr(a), stride))
    for f in GENERAL_SCALAR_FIELDS:
        a = d[f]
        setattr(b, f, DArray(_ptr(a), 1 if a.shape[0] > 1 else 0))
    if "level_altitudes" in d:
        b.level_altitudes = _ptr(d["level_altitudes"])
        a = d["bottom_radius"]
        b.bottom_radius = DArray(_ptr(a), 1 if a.shape[0] > 1 else 0)
    b.brdf_type = d.get("brdf_type", BRDF_LAMBERTIAN)
    if "mu_phase_function" in d:
        b.num_phase_func_angles = d["num_phase_func_angles"]
        a, stride = d["mu_phase_function"]
        b.mu_phase_function = DArray(_ptr(a), stride)
        b.phase_function = _ptr(d["phase_function"])
    if "brdf_params" in d:
        a = d["brdf_params"]
        b.brdf_params = DArray(_ptr(a), BRDF_PARAMS if a.shape[0] > 1 else 0)
    return b, keep


def alloc_general_out_numpy(d: dict) -> tuple[dict, GeneralOut, list]:
    """NaN-filled host outputs for the batch of pack_general and the dsp_general_out over them."""
    n, nt, nu, nphi = d["n_inst"], d["ntau_out"], d["numu_out"], max(d["num_phi"], 0)
    outs = {f: np.full((n, nt), np.nan) for f in FLUX_OUT_FIELDS}
    outs["intensity"] = np.full((n, nt, nu, nphi), np.nan)
    outs["intensity_azimuth_avg"] = np.full((n, nt, nu), np.nan)
    outs["status"] = np.full(n, -1, dtype=np.int32)
    o = GeneralOut()
    for k, f in enumerate(FLUX_OUT_FIELDS):
        o.flux[k] = ctypes.cast(c_void_p(_ptr(outs[f])), POINTER(c_double))
    o.intensity = ctypes.cast(c_void_p(_ptr(outs["intensity"])), POINTER(c_double))
    o.intensity_azimuth_avg = ctypes.cast(c_void_p(_ptr(outs["intensity_azimuth_avg"])), POINTER(c_double))
    o.status = ctypes.cast(c_void_p(_ptr(outs["status"])), POINTER(c_int32))
    o.ntau_out, o.numu_out = nt, nu
    return outs, o, [outs]


class AlbTransOut(ctypes.Structure):
    """dsp_albtrans_out (ibcnd = Special)."""
    _fields_ = [("albedo_medium", POINTER(c_double)), ("transmissivity_medium", POINTER(c_double)),
                ("spherical_albedo", POINTER(c_double)), ("spherical_transmissivity", POINTER(c_double)),
                ("status", POINTER(c_int32)), ("numu_out", c_int32)]


def alloc_albtrans_numpy(d: dict) -> tuple[dict, AlbTransOut, list]:
    """NaN-filled host outputs of dsp_general_bands_albtrans for a pack_general batch."""
    n = d["n_inst"]
    nu = d["num_user_mu"] if d["flags"] & GFLAG_USER_MU else int(d["num_streams"].max()) // 2
    outs = {"albedo_medium": np.full((n, nu), np.nan), "transmissivity_medium": np.full((n, nu), np.nan),
            "spherical_albedo": np.full(n, np.nan), "spherical_transmissivity": np.full(n, np.nan),
            "status": np.full(n, -1, dtype=np.int32)}
    o = AlbTransOut()
    for f in ("albedo_medium", "transmissivity_medium", "spherical_albedo", "spherical_transmissivity"):
        setattr(o, f, ctypes.cast(c_void_p(_ptr(outs[f])), POINTER(c_double)))
    o.status = ctypes.cast(c_void_p(_ptr(outs["status"])), POINTER(c_int32))
    o.numu_out = nu
    return outs, o, [outs]


class GeneralJacOut(ctypes.Structure):
    _fields_ = [(f, POINTER(c_double)) for f in JAC_FIELDS] + [("ndof_out", c_int32)]


def alloc_general_jac_numpy(d: dict) -> tuple[dict, GeneralJacOut, list]:
    """NaN-filled Jacobian outputs [n][ntau_out][max L + 2] for a pack_general batch."""
    n, nt = d["n_inst"], d["ntau_out"]
    ndof = int(np.max(d["num_layers"])) + 2 if n else 2
    jac = {f: np.full((n, nt, ndof), np.nan) for f in JAC_FIELDS}
    o = GeneralJacOut()
    for f in JAC_FIELDS:
        setattr(o, f, ctypes.cast(c_void_p(_ptr(jac[f])), POINTER(c_double)))
    o.ndof_out = ndof
    return jac, o, [jac]


def alloc_flux_out_numpy(n_inst: int, num_layers: int) -> tuple[dict, np.ndarray]:
    outs = {f: np.full((n_inst, num_layers + 1), np.nan) for f in FLUX_OUT_FIELDS}
    status = np.full(n_inst, -1, dtype=np.int32)
    return outs, status


# ---------------------------------------------------------------------------
# libdsp.so (the product library)
# ---------------------------------------------------------------------------
class Schedule(ctypes.Structure):
    """dsp_schedule: a launch schedule for instances with N streams and
    min_layers..max_layers layers (0 fields: the built-in choice)."""
    _fields_ = [("num_streams", c_int32), ("min_layers", c_int32), ("max_layers", c_int32),
                ("layer_stage", c_int32), ("layer_cta", c_int32), ("persistent", c_int32)]


# the schedule table measured by disort_b200/autotune.py on this GPU model
TUNING_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.txt")

_LIB = None


def lib_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libdsp.so")


def load_library(path: str | None = None):
    """Load libdsp.so and declare its prototypes.  Raises OSError if it is missing."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or lib_path()
    if not os.path.exists(p):
        raise OSError(f"libdsp.so not built: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    lib.dsp_api_version.restype = c_int32
    lib.dsp_status_string.restype = ctypes.c_char_p
    lib.dsp_status_string.argtypes = [c_int32]
    lib.dsp_context_create.restype = c_int32
    lib.dsp_context_create.argtypes = [c_int32, c_void_p, POINTER(c_void_p)]
    lib.dsp_context_destroy.restype = c_int32
    lib.dsp_context_destroy.argtypes = [c_void_p]
    lib.dsp_context_set_stream.restype = c_int32
    lib.dsp_context_set_stream.argtypes = [c_void_p, c_void_p]
    lib.dsp_context_last_error.restype = ctypes.c_char_p
    lib.dsp_general_bands_albtrans.restype = c_int32
    lib.dsp_general_bands_albtrans.argtypes = [c_void_p, POINTER(GeneralBatch), POINTER(AlbTransOut)]
    lib.dsp_context_last_error.argtypes = [c_void_p]
    lib.dsp_flux_workspace_bytes.restype = c_int64
    lib.dsp_flux_workspace_bytes.argtypes = [POINTER(FluxBatch)]
    lib.dsp_context_set_schedule.restype = c_int32
    lib.dsp_context_set_schedule.argtypes = [c_void_p, POINTER(Schedule), c_int32]
    lib.dsp_context_load_schedule_file.restype = c_int32
    lib.dsp_context_load_schedule_file.argtypes = [c_void_p, ctypes.c_char_p]
    lib.dsp_context_schedule_count.restype = c_int32
    lib.dsp_context_schedule_count.argtypes = [c_void_p]
    lib.dsp_flux_graph_create.restype = c_int32
    lib.dsp_flux_graph_create.argtypes = [c_int32, POINTER(FluxBatch), POINTER(FluxOut), POINTER(c_void_p)]
    lib.dsp_graph_launch.restype = c_int32
    lib.dsp_graph_launch.argtypes = [c_void_p, c_void_p]
    lib.dsp_graph_destroy.restype = c_int32
    lib.dsp_graph_destroy.argtypes = [c_void_p]
    lib.dsp_context_set_debug.restype = c_int32
    lib.dsp_context_set_debug.argtypes = [c_void_p, c_uint32]
    lib.dsp_context_set_timing.restype = c_int32
    lib.dsp_context_set_timing.argtypes = [c_void_p, c_int32]
    lib.dsp_context_timing_reset.restype = c_int32
    lib.dsp_context_timing_reset.argtypes = [c_void_p]
    lib.dsp_context_timing_count.restype = c_int32
    lib.dsp_context_timing_count.argtypes = [c_void_p]
    lib.dsp_context_timing_get.restype = c_int32
    lib.dsp_context_timing_get.argtypes = [c_void_p, c_int32, POINTER(ctypes.c_char_p),
                                           POINTER(c_double), POINTER(c_int64)]
    lib.dsp_flux_bands_solve.restype = c_int32
    lib.dsp_flux_bands_solve.argtypes = [c_void_p, POINTER(FluxBatch), POINTER(FluxOut)]
    lib.dsp_flux_bands_solve_jac.restype = c_int32
    lib.dsp_flux_bands_solve_jac.argtypes = [c_void_p, POINTER(FluxBatch), POINTER(FluxOut), POINTER(FluxJacOut)]
    lib.dsp_general_bands_solve.restype = c_int32
    lib.dsp_general_bands_solve.argtypes = [c_void_p, POINTER(GeneralBatch), POINTER(GeneralOut)]
    lib.dsp_general_bands_solve_jac.restype = c_int32
    lib.dsp_general_bands_solve_jac.argtypes = [c_void_p, POINTER(GeneralBatch), POINTER(GeneralOut),
                                                POINTER(GeneralJacOut)]
    lib.dsp_noalloc_scratch_bytes.restype = c_int64
    lib.dsp_noalloc_scratch_bytes.argtypes = []
    lib.dsp_flux_bands_solve_noalloc.restype = c_int32
    lib.dsp_flux_bands_solve_noalloc.argtypes = [POINTER(FluxBatch), POINTER(FluxOut), c_void_p]
    if path is None:
        _LIB = lib
    return lib


class Context:
    """RAII wrapper of a dsp_context."""

    def __init__(self, device: int = 0, stream: int = 0, lib=None, tuned: bool = True):
        """tuned: load the committed schedule table (TUNING_FILE) when present."""
        self.lib = lib or load_library()
        h = c_void_p()
        st = self.lib.dsp_context_create(device, c_void_p(stream), ctypes.byref(h))
        if st != DSP_OK:
            raise RuntimeError(f"dsp_context_create failed: {STATUS_NAMES.get(st, st)}")
        self.h = h
        if tuned and os.path.exists(TUNING_FILE):
            st = self.load_schedule_file(TUNING_FILE)
            if st != DSP_OK:
                raise RuntimeError(f"{TUNING_FILE}: {self.last_error()}")

    def set_schedule(self, entries) -> int:
        """entries: (N, min_layers, max_layers, layer_stage, layer_cta, persistent) tuples."""
        arr = (Schedule * max(1, len(entries)))(*[Schedule(*e) for e in entries])
        return int(self.lib.dsp_context_set_schedule(self.h, arr, len(entries)))

    def load_schedule_file(self, path: str) -> int:
        return int(self.lib.dsp_context_load_schedule_file(self.h, path.encode()))

    def schedule_count(self) -> int:
        return int(self.lib.dsp_context_schedule_count(self.h))

    def set_stream(self, stream: int):
        self.lib.dsp_context_set_stream(self.h, c_void_p(stream))

    def last_error(self) -> str:
        s = self.lib.dsp_context_last_error(self.h)
        return s.decode() if s else ""

    def flux_bands_solve(self, batch: FluxBatch, out: FluxOut) -> int:
        return self.lib.dsp_flux_bands_solve(self.h, ctypes.byref(batch), ctypes.byref(out))

    def flux_bands_solve_jac(self, batch: FluxBatch, out: FluxOut, jac: FluxJacOut) -> int:
        return self.lib.dsp_flux_bands_solve_jac(self.h, ctypes.byref(batch), ctypes.byref(out), ctypes.byref(jac))

    def general_bands_solve(self, batch: GeneralBatch, out: GeneralOut) -> int:
        return self.lib.dsp_general_bands_solve(self.h, ctypes.byref(batch), ctypes.byref(out))

    def general_bands_solve_jac(self, batch: GeneralBatch, out: GeneralOut, jac: GeneralJacOut) -> int:
        return self.lib.dsp_general_bands_solve_jac(self.h, ctypes.byref(batch), ctypes.byref(out), ctypes.byref(jac))

    def general_bands_albtrans(self, batch: GeneralBatch, out: AlbTransOut) -> int:
        """ibcnd = Special: albedo and transmissivity of the medium (host pointers)."""
        return self.lib.dsp_general_bands_albtrans(self.h, ctypes.byref(batch), ctypes.byref(out))

    def set_debug(self, flags: int) -> int:
        """DSP_DEBUG_* flags (DEBUG_POISON_SCRATCH: NaN-filled workspace before each chunk)."""
        return int(self.lib.dsp_context_set_debug(self.h, flags))

    def set_timing(self, enable: bool):
        self.lib.dsp_context_set_timing(self.h, 1 if enable else 0)

    def timing_reset(self):
        self.lib.dsp_context_timing_reset(self.h)

    def timings(self) -> dict:
        """{kernel name: (total ms, launches)} accumulated since the last reset."""
        out = {}
        for k in range(self.lib.dsp_context_timing_count(self.h)):
            name = ctypes.c_char_p()
            ms = c_double()
            cnt = c_int64()
            self.lib.dsp_context_timing_get(self.h, k, ctypes.byref(name), ctypes.byref(ms), ctypes.byref(cnt))
            out[name.value.decode()] = (ms.value, cnt.value)
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.dsp_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FluxGraph:
    """A device-pointer flux solve captured as a CUDA graph (dsp_flux_graph_create);
    launch() replays it on a stream; the batch's arrays are re-read on every launch."""

    def __init__(self, batch: FluxBatch, out: FluxOut, device: int = 0, lib=None):
        self.lib = lib or load_library()
        self._keep = (batch, out)
        h = c_void_p()
        st = self.lib.dsp_flux_graph_create(device, ctypes.byref(batch), ctypes.byref(out), ctypes.byref(h))
        if st != DSP_OK:
            raise RuntimeError(f"dsp_flux_graph_create: {STATUS_NAMES.get(st, st)}")
        self.h = h

    def launch(self, stream: int = 0) -> int:
        return int(self.lib.dsp_graph_launch(self.h, c_void_p(stream)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.dsp_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
