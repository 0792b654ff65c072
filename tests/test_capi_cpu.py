"""CPU-side checks of the C ABI: each library loads and exports every entry point its header declares
(include/dsp.h -> libdsp.so, include/dsp_emu.h -> libdsp_emu.so)."""
import os
import re

import pytest

from disort_b200 import capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header: str = "dsp.h"):
    txt = open(os.path.join(REPO, "include", header)).read()
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(dsp_\w+)\s*\(", txt, re.M)))


def test_every_header_has_a_library():
    headers = sorted(h for h in os.listdir(os.path.join(REPO, "include")) if h.endswith(".h"))
    assert headers == ["dsp.h", "dsp_emu.h"], headers


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("dsp_context_create", "dsp_context_destroy", "dsp_flux_bands_solve"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(capi.lib_path()):
        pytest.skip("libdsp.so not built")
    lib = capi.load_library()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.dsp_api_version() == 3
    assert lib.dsp_status_string(capi.DSP_ERR_SINGULAR) == b"SINGULAR"


def test_emulator_library_exports_every_declared_symbol():
    from disort_b200 import emu
    if not os.path.exists(emu.lib_path()):
        pytest.skip("libdsp_emu.so not built")
    lib = emu.load_library()
    names = declared_functions("dsp_emu.h")
    assert "dsp_emu_gemm_bf16" in names and "dsp_emu_train" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_workspace_query_without_gpu():
    if not os.path.exists(capi.lib_path()):
        pytest.skip("libdsp.so not built")
    import ctypes
    lib = capi.load_library()
    b = capi.FluxBatch()
    b.n_inst, b.num_streams, b.num_layers, b.pmom_count = 1000, 16, 60, 17
    assert lib.dsp_flux_workspace_bytes(ctypes.byref(b)) > 1000 * 60 * 16 * 16 * 8
    b.num_streams = 18
    assert lib.dsp_flux_workspace_bytes(ctypes.byref(b)) == -1
