"""ctypes binding of libdsp_emu.so (include/dsp_emu.h): the flux emulator's MLP.

Arrays are torch CUDA tensors on the emulator's device.  BF16 features are
passed as torch.bfloat16 tensors (their bit patterns are the uint16_t of the C ABI).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int32, c_int64, c_uint64, c_void_p

from . import capi

_LIB = None


class EmuConfig(ctypes.Structure):
    _fields_ = [("n_in", c_int32), ("hidden", c_int32), ("n_hidden_layers", c_int32), ("n_out", c_int32),
                ("n_heads", c_int32), ("batch", c_int32), ("seed", c_uint64)]


def lib_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libdsp_emu.so")


def load_library():
    global _LIB
    if _LIB is not None:
        return _LIB
    p = lib_path()
    if not os.path.exists(p):
        raise OSError(f"libdsp_emu.so not built: {p} (run __graft_entry__.build())")
    lib = ctypes.CDLL(p)
    lib.dsp_emu_create.restype = c_int32
    lib.dsp_emu_create.argtypes = [c_int32, c_void_p, POINTER(EmuConfig), POINTER(c_void_p)]
    lib.dsp_emu_destroy.restype = c_int32
    lib.dsp_emu_destroy.argtypes = [c_void_p]
    lib.dsp_emu_last_error.restype = c_char_p
    lib.dsp_emu_last_error.argtypes = [c_void_p]
    lib.dsp_emu_input_stride.restype = c_int32
    lib.dsp_emu_input_stride.argtypes = [c_void_p]
    lib.dsp_emu_set_data.restype = c_int32
    lib.dsp_emu_set_data.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int64]
    lib.dsp_emu_train.restype = c_int32
    lib.dsp_emu_train.argtypes = [c_void_p, c_int32, c_float, c_float, c_uint64, POINTER(c_float)]
    lib.dsp_emu_forward.restype = c_int32
    lib.dsp_emu_forward.argtypes = [c_void_p, c_void_p, c_int64, c_void_p]
    lib.dsp_emu_gradients.restype = c_int32
    lib.dsp_emu_gradients.argtypes = [c_void_p, c_void_p, c_void_p]
    lib.dsp_emu_param_count.restype = c_int64
    lib.dsp_emu_param_count.argtypes = [c_void_p]
    lib.dsp_emu_layer_dims.restype = c_int32
    lib.dsp_emu_layer_dims.argtypes = [c_void_p, c_int32, POINTER(c_int32), POINTER(c_int32)]
    lib.dsp_emu_get_params.restype = c_int32
    lib.dsp_emu_get_params.argtypes = [c_void_p, c_void_p]
    lib.dsp_emu_set_params.restype = c_int32
    lib.dsp_emu_set_params.argtypes = [c_void_p, c_void_p]
    lib.dsp_emu_gemm_bf16.restype = c_int32
    lib.dsp_emu_gemm_bf16.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32]
    lib.dsp_emu_wait_selftest.restype = c_int32
    lib.dsp_emu_wait_selftest.argtypes = [c_void_p, c_int64]
    lib.dsp_emu_gate.restype = c_int32
    lib.dsp_emu_gate.argtypes = [c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p, c_void_p, c_float, c_float, c_float, c_int64, c_void_p, c_void_p,
                                 c_void_p, c_void_p]
    _LIB = lib
    return lib


def _p(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class Emulator:
    """Owner of one dsp_emu handle."""

    def __init__(self, n_in=247, hidden=512, n_hidden_layers=4, n_out=82, n_heads=2, batch=4096, seed=1,
                 device=0, stream=0):
        self.lib = load_library()
        self.cfg = EmuConfig(n_in, hidden, n_hidden_layers, n_out, n_heads, batch, seed)
        h = c_void_p()
        st = self.lib.dsp_emu_create(device, c_void_p(stream), ctypes.byref(self.cfg), ctypes.byref(h))
        if st != 0:
            raise RuntimeError(f"dsp_emu_create: {capi.STATUS_NAMES.get(st, st)}")
        self.h = h
        self.in_stride = self.lib.dsp_emu_input_stride(h)

    def _check(self, st, what):
        if st != 0:
            raise RuntimeError(f"{what}: {capi.STATUS_NAMES.get(st, st)}: {self.last_error()}")

    def last_error(self) -> str:
        s = self.lib.dsp_emu_last_error(self.h)
        return s.decode() if s else ""

    def set_data(self, feats, targets, head_weights=None):
        self._check(self.lib.dsp_emu_set_data(self.h, _p(feats), _p(targets), _p(head_weights), feats.shape[0]),
                    "dsp_emu_set_data")

    def train(self, epochs, lr=1e-3, lr_min=1e-5, seed=7):
        losses = (c_float * max(1, epochs))()
        self._check(self.lib.dsp_emu_train(self.h, epochs, lr, lr_min, seed, losses), "dsp_emu_train")
        return [losses[i] for i in range(epochs)]

    def forward(self, feats, out):
        self._check(self.lib.dsp_emu_forward(self.h, _p(feats), feats.shape[0], _p(out)), "dsp_emu_forward")

    def gradients(self, grads, loss):
        self._check(self.lib.dsp_emu_gradients(self.h, _p(grads), _p(loss)), "dsp_emu_gradients")

    def param_count(self) -> int:
        return int(self.lib.dsp_emu_param_count(self.h))

    def layer_dims(self):
        dims = []
        k = 0
        while True:
            a, b = c_int32(), c_int32()
            if self.lib.dsp_emu_layer_dims(self.h, k, ctypes.byref(a), ctypes.byref(b)) != 0:
                return dims
            dims.append((a.value, b.value))
            k += 1

    def get_params(self, host):
        self._check(self.lib.dsp_emu_get_params(self.h, host.ctypes.data), "dsp_emu_get_params")

    def set_params(self, host):
        self._check(self.lib.dsp_emu_set_params(self.h, host.ctypes.data), "dsp_emu_set_params")

    def gemm(self, A, B, C):
        self._check(self.lib.dsp_emu_gemm_bf16(self.h, _p(A), _p(B), _p(C), A.shape[0], B.shape[0], A.shape[1]),
                    "dsp_emu_gemm_bf16")

    def wait_selftest(self, cycles: int) -> int:
        """Status of the bounded-wait self-test (DSP_ERR_TIMEOUT when the wait ran out)."""
        return int(self.lib.dsp_emu_wait_selftest(self.h, cycles))

    def gate(self, raw, lo, hi, preds, mu, sd, scale, add, eps, rel_tol, floor_frac, flux, fallback, idx, count):
        self._check(self.lib.dsp_emu_gate(self.h, _p(raw), raw.shape[1], _p(lo), _p(hi), _p(preds), _p(mu), _p(sd),
                                          _p(scale), _p(add), eps, rel_tol, floor_frac, raw.shape[0], _p(flux),
                                          _p(fallback), _p(idx), _p(count)), "dsp_emu_gate")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dsp_emu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
