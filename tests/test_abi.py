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


def test_reference_cython_module_links_this_library():
    """Where it was built (the reference tree present at build time), the reference's own
    Cython module loads against this library on a machine without a GPU: every symbol it
    binds resolves to libcusnarks_b200.so."""
    import importlib
    import subprocess
    import sys
    from cusnarks_b200 import refcython
    path = refcython.module_path()
    if path is None:
        pytest.skip("pycusnarks not built here (no reference tree at build time)")
    need = subprocess.run(["ldd", path], capture_output=True, text=True).stdout
    assert "not found" not in need
    lines = [ln for ln in need.splitlines() if "libcusnarks_b200.so =>" in ln]
    assert len(lines) == 1
    resolved = lines[0].split("=>")[1].split("(")[0].strip()
    assert os.path.realpath(resolved) == os.path.join(ROOT, "cusnarks_b200", "libcusnarks_b200.so")
    d = os.path.dirname(path)
    sys.path.insert(0, d)
    try:
        mod = importlib.import_module("pycusnarks")
    finally:
        sys.path.remove(d)
    for name in ("ec_jacreduce_h", "ntt_h", "intt_h", "ntt_interpolandmul_h", "mpoly_eval_h"):
        assert callable(getattr(mod, name))


def test_window_and_workspace_queries_need_no_device():
    """The sizing queries are host arithmetic: windows by the cost models (G1 for 2n
    GLV half-scalars, G2 for full scalars), scratch bytes for each, and the allocation-free
    entry point's term limit, which stays at or above 2^16 terms."""
    from cusnarks_b200 import lib
    L = lib()
    assert L.cs_msm_default_window(1 << 20, 0) == 16   # G1: 2^21 half-scalars of 8 windows
    assert L.cs_msm_num_windows(16) == 16               # a full scalar: 254 / 16 + 1
    for n in (1 << 10, 1 << 16, 1 << 20):
        for ec2 in (0, 1):
            assert L.cs_msm_workspace_bytes(n, ec2, 0) > 0
            assert L.cs_msm_fixed_workspace_bytes(n, ec2, 0) > 0
    assert L.cs_msm_noalloc_scratch_bytes() == 32 << 20
    assert L.cs_msm_g1_noalloc_max_terms() >= 1 << 16
