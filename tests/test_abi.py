"""The C ABI: every symbol that include/*.h declares is exported by its
libraries, and the reference's lib_ipm symbol set is complete."""
import ctypes
import os
import re

import pytest

from irs_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", txt)) - {"if", "while", "for", "return"})


@pytest.mark.parametrize("kind,dbl", [("ipm", False), ("ipm", True), ("irs", False), ("irs", True)])
def test_library_exports_header_symbols(kind, dbl):
    lib = ctypes.CDLL(_lib.lib_path(kind, dbl))
    names = declared(f"lib_{kind}.h")
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("dbl", [False, True])
def test_reference_ipm_symbol_set(dbl):
    lib = ctypes.CDLL(_lib.lib_path("ipm", dbl))
    missing = [n for n in _lib.REFERENCE_IPM_SYMBOLS if not hasattr(lib, n)]
    assert not missing, missing
    assert len(_lib.REFERENCE_IPM_SYMBOLS) == 63  # src/lib_ipm.cu:15-81


def test_loads_and_binds_all():
    for kind in ("ipm", "irs"):
        for dbl in (False, True):
            lib = _lib.load(kind, dbl)
            obj = lib.init()
            assert obj
            lib.set_kappa_tot(obj, 0.5)
            assert abs(lib.get_kappa_tot(obj) - 0.5) < 1e-7
            lib.set_mass_function(obj, b"kroupa")
            assert lib.get_mass_function(obj) == b"kroupa"
            lib.destroy(obj)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIBDIR", str(tmp_path))
    monkeypatch.setattr(_lib, "_cache", {})
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load("ipm", False)
