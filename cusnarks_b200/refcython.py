"""Builds the reference's own Cython module, ``pycusnarks``, against this library.

    python -m cusnarks_b200.refcython [--ref DIR]      (DIR: $CUSNARKS_REF by default)

The reference's Python prover reaches the hot path through ``pycusnarks``, compiled from
src/cython/_cusnarks_kernel.pyx over the C++ declarations of src/cython/_utils_host.pxd.
This script builds that module unchanged, in its CPU configuration (CUDA_DEF False,
src/cython/setup.py:180), with one edit to the binding file: every ``cdef extern from
"../cuda/<x>.h"`` in _utils_host.pxd names ``cusnarks_b200.h`` instead, so the calls the
wrappers make (ec_jacreduce_server_h, ntt_h, intt_h, ntt_interpolandmul_server_h,
mpoly_eval_server_h, ...) resolve to this library's C entry points.  The reference's
types.h still supplies the argument structs (the header then leaves out its own copies:
CS_REFERENCE_TYPES), and the module links libcusnarks_b200.so with an rpath to it.

The reference files are copied to a temporary directory and edited there; only the built
module lands in the repository, in ``cusnarks_b200/_refcy/`` (not version-controlled),
together with ``constants.py``: the seven layout constants the module imports at start-up
from the reference's Python package (limbs per element, coordinates per point, the thread
cap), written out as values so the module imports where the reference tree is absent.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import sys
import tempfile

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "_refcy")
CYTHON_FILES = ("_cusnarks_kernel.pyx", "_types.pxd", "_utils_host.pxd", "_cusnarks_kernel.pxd", "_zpoly_host.pxd")
CONSTANTS = ("NWORDS_256BIT", "ECP_JAC_INDIMS", "ECP_JAC_OUTDIMS", "ECP2_JAC_INDIMS", "ECP2_JAC_OUTDIMS",
             "MAX_NCORES_OMP", "MAX_R1CSPOLY_NWORDS")


def default_ref() -> str | None:
    return os.environ.get("CUSNARKS_REF") or None


def module_path() -> str | None:
    """The built module, or None."""
    if not os.path.isdir(OUT):
        return None
    for f in sorted(os.listdir(OUT)):
        if f.startswith("pycusnarks") and f.endswith(".so"):
            return os.path.join(OUT, f)
    return None


def _edit_binding(text: str) -> str:
    """_utils_host.pxd with its C++ headers replaced by this library's C header."""
    new, n = re.subn(r'cdef extern from "\.\./cuda/[A-Za-z_]+\.h"', 'cdef extern from "cusnarks_b200.h"', text)
    if n == 0:
        raise RuntimeError("no reference header includes found in _utils_host.pxd")
    return new


def _constants_module(ref: str) -> str:
    sys.path.insert(0, os.path.join(ref, "src", "python"))
    try:
        import importlib
        c = importlib.import_module("constants")
        vals = {k: getattr(c, k) for k in CONSTANTS}
    finally:
        sys.path.pop(0)
        sys.modules.pop("constants", None)
    lines = ['"""Layout constants the reference\'s pycusnarks module imports at start-up (values of',
             'the reference\'s src/python/constants.py)."""']
    lines += [f"{k} = {v!r}" for k, v in vals.items()]
    return "\n".join(lines) + "\n"


def build(ref: str | None = None, verbose: bool = False, force: bool = False) -> str:
    ref = ref or default_ref()
    if not ref:
        raise RuntimeError("the reference tree is needed: pass --ref DIR or set CUSNARKS_REF")
    cy = os.path.join(ref, "src", "cython")
    inc_ref = os.path.join(ref, "src", "cuda")
    lib = os.path.join(PKG, "libcusnarks_b200.so")
    if not os.path.exists(lib):
        raise RuntimeError(f"{lib} is missing: build the library first")
    have = module_path()
    deps = [lib, __file__, os.path.join(ROOT, "include", "cusnarks_b200.h")] + [os.path.join(cy, f) for f in CYTHON_FILES]
    if (not force and have and os.path.exists(os.path.join(OUT, "constants.py"))
            and os.path.getmtime(have) >= max(os.path.getmtime(d) for d in deps)):
        return have
    import contextlib
    import io
    import numpy
    from Cython.Build import cythonize
    from setuptools import Extension
    from setuptools.dist import Distribution
    work = tempfile.mkdtemp(prefix="pycusnarks_")
    try:
        for f in CYTHON_FILES:
            shutil.copy(os.path.join(cy, f), os.path.join(work, f))
        p = os.path.join(work, "_utils_host.pxd")
        with open(p) as fh:
            text = fh.read()
        with open(p, "w") as fh:
            fh.write(_edit_binding(text))
        ext = Extension(
            "pycusnarks", sources=[os.path.join(work, "_cusnarks_kernel.pyx")], language="c++",
            include_dirs=[numpy.get_include(), inc_ref, os.path.join(ROOT, "include")],
            define_macros=[("CS_REFERENCE_TYPES", "1")],
            libraries=["cusnarks_b200"], library_dirs=[PKG], runtime_library_dirs=["$ORIGIN/.."],
            extra_compile_args=["-w", "-O2"])
        cwd = os.getcwd()
        os.chdir(work)
        try:
            sink = io.StringIO()
            with contextlib.redirect_stdout(sink if not verbose else sys.stdout), \
                    contextlib.redirect_stderr(sink if not verbose else sys.stderr):
                exts = cythonize([ext], compile_time_env={"CUDA_DEF": False}, include_path=[work],
                                 language_level=3, quiet=not verbose)
            dist = Distribution({"name": "pycusnarks", "ext_modules": exts})
            cmd = dist.get_command_obj("build_ext")
            cmd.build_lib = os.path.join(work, "lib")
            cmd.build_temp = os.path.join(work, "tmp")
            cmd.ensure_finalized()
            cmd.run()
        finally:
            os.chdir(cwd)
        built = [os.path.join(dp, f) for dp, _, fs in os.walk(os.path.join(work, "lib")) for f in fs
                 if f.startswith("pycusnarks") and f.endswith(".so")]
        if not built:
            raise RuntimeError("pycusnarks was not built")
        os.makedirs(OUT, exist_ok=True)
        for f in os.listdir(OUT):
            if f.startswith("pycusnarks"):
                os.remove(os.path.join(OUT, f))
        dst = os.path.join(OUT, os.path.basename(built[0]))
        shutil.copy(built[0], dst)
        with open(os.path.join(OUT, "constants.py"), "w") as fh:
            fh.write(_constants_module(ref))
        return dst
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=default_ref())
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.ref, a.verbose, a.force))
