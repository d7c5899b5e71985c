"""The C-ABI libraries load and export every symbol include/b200ode.h and
include/b200ode_io.h declare (no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from hpc_ode_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(b200ode_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(native.LIB_PATH)
    syms = declared_symbols("b200ode.h")
    assert "b200ode_integrate" in syms and "b200ode_create" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(native.EXPORTED) == syms


def test_host_library_exports_the_io_symbols():
    build.build()
    from hpc_ode_b200 import io
    lib = ctypes.CDLL(io.HOST_LIB_PATH)
    syms = declared_symbols("b200ode_io.h")
    assert "b200ode_csv_read" in syms
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_loader_fails_loudly_without_library(tmp_path):
    import pytest
    saved = native._lib
    native._lib = None
    try:
        with pytest.raises(native.NativeLibraryError):
            native.load(str(tmp_path / "missing.so"))
    finally:
        native._lib = saved


def test_version_and_defaults():
    lib = native.load()
    assert b"sm_100a" in lib.b200ode_version()
    o = native.default_options()
    assert (o.reltol, o.abstol, o.max_steps, o.max_order) == (1e-6, 1e-10, 10000, 5)
    assert o.precision == native.B200ODE_MIXED and o.persistent == 1
