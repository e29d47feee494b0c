"""The C-ABI library loads and exports every symbol the header declares (CPU only)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "cusnarks_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "sizeof")))


def test_header_declares_reference_entry_points():
    names = _declared_functions()
    assert "ec_jacreduce_server_h" in names
    assert "cs_msm" in names


def test_library_exports_every_declared_symbol():
    path = os.path.join(ROOT, "cusnarks_b200", "libcusnarks_b200.so")
    if not os.path.exists(path):
        pytest.fail("libcusnarks_b200.so not built (python -m cusnarks_b200.build)")
    lib = ctypes.CDLL(path)  # loading needs no GPU
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from cusnarks_b200 import exported_symbols
    assert set(exported_symbols()) == set(_declared_functions())


def test_no_device_reports_error_instead_of_exiting():
    """Without a GPU the context API returns an error code; it never exits the process."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cusnarks_b200 import lib
    L = lib()
    h = ctypes.c_void_p()
    assert L.cs_ctx_create(0, ctypes.byref(h)) != 0


def test_server_refuses_without_device():
    """The prove server needs a CUDA device: without one it fails loudly (no CPU path)."""
    import ctypes
    from cusnarks_b200 import lib
    from cusnarks_b200._lib import CS_ERR_NODEVICE
    from tests.gpu_common import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert lib().cs_server_create(0, 2, 0, ctypes.byref(h)) == CS_ERR_NODEVICE
    assert not h.value
