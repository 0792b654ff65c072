"""CPU-side checks of the C ABI: the library loads and exports every entry point of dsp.h."""
import os
import re

import pytest

from disort_b200 import capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(REPO, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(REPO, "include", h)).read()
            names += re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(dsp_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


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
    assert lib.dsp_api_version() == 1
    assert lib.dsp_status_string(capi.DSP_ERR_SINGULAR) == b"SINGULAR"


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
