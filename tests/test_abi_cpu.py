"""The C-ABI library loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re

import pytest

from pastix_b200 import native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = []
    for h in ("pastix_b200.h",):
        txt = open(os.path.join(REPO, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        syms += re.findall(r"\b(b200_\w+)\s*\(", txt)
    return sorted(set(syms))


@pytest.mark.skipif(not os.path.exists(native.LIBPATH), reason="library not built")
def test_library_exports_header_symbols():
    lib = ctypes.CDLL(native.LIBPATH)
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_python_binding_covers_header():
    assert sorted(native.SYMBOLS) == sorted(s for s in declared_symbols() if s in native.SYMBOLS)
    missing = set(declared_symbols()) - set(native.SYMBOLS)
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(native.LIBPATH), reason="library not built")
def test_strerror_without_gpu():
    lib = native.lib()
    assert lib.b200_strerror(0) == b"success"
    assert b"bad parameter" in lib.b200_strerror(7)


@pytest.mark.skipif(not os.path.exists(native.LIBPATH), reason="library not built")
def test_null_arguments_rejected_without_gpu():
    lib = native.lib()
    assert lib.b200_solver_create(None, 0, 0, None, None) == 7
    assert lib.b200_numfact(None, 0.0, None) == 7
    assert lib.b200_solve(None, 1, None, 1) == 7
