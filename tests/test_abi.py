"""The C-ABI boundary without a GPU: the library loads, exports exactly the
declared entry points, and fails cleanly (error code, no crash) when no device
is usable."""
import ctypes as C
import os
import subprocess

import pytest

from dragonfly_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib_path = _lib.LIB_PATH
    assert os.path.exists(lib_path), "libdfgpu.so not built"
    declared = set(_lib.header_symbols())
    assert len(declared) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert declared <= exported, sorted(declared - exported)
    # nothing else leaks out of the library
    assert {s for s in exported if not s.startswith("dfg_")} == set()
    # the Python binding declares a signature for each entry point
    assert declared == set(_lib._SIGS), sorted(declared ^ set(_lib._SIGS))


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert lib.dfg_version().startswith(b"dragonfly_b200")
    assert lib.dfg_phase_name(0) == b"slice"
    assert lib.dfg_phase_name(99) == b""


def test_null_context_is_rejected():
    lib = _lib.load()
    assert lib.dfg_set_detector(None, 0, None, None, None) == _lib.DFG_ERR_ARG
    assert lib.dfg_maximize(None, None, None) == _lib.DFG_ERR_ARG
    assert lib.dfg_last_error(None) == b"null context"
    lib.dfg_destroy(None)


def test_create_without_usable_device_fails_cleanly():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.dfg_create(0, C.byref(h)) == _lib.DFG_ERR_CUDA
    assert not h.value
    with pytest.raises(_lib.DFGError):
        _lib.Context(0)
