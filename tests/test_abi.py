"""The C-ABI library loads and exports every symbol include/blond_b200.h
declares (no compute call: this runs without a GPU)."""
import ctypes as ct
import os
import re

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "blond_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(blond_\w+)\s*\(", src)))


def test_library_builds_and_exports_every_declared_symbol():
    from blond_b200.build import build
    lib_path = build()
    lib = ct.CDLL(lib_path)
    declared = _declared()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_annotates_every_declared_symbol():
    from blond_b200 import _lib
    lib = _lib.load()
    assert set(_declared()) == set(_lib.exported_symbols())
    assert lib.blond_b200_version() >= 100


def test_status_codes_match_header():
    from blond_b200 import _lib
    src = open(os.path.join(ROOT, "include", "blond_b200.h")).read()
    codes = dict((int(v), k) for k, v in re.findall(r"#define BLOND_(ERR_\w+) (\d+)", src))
    assert set(codes) == set(_lib.ERR_NAMES)


def test_no_cpu_fallback_when_library_missing(tmp_path):
    """Loading from a path without the library raises instead of falling back."""
    import pytest
    from blond_b200 import _lib
    saved = _lib._lib
    _lib._lib = None
    try:
        with pytest.raises(ImportError):
            _lib.load(str(tmp_path / "missing.so"))
    finally:
        _lib._lib = saved
