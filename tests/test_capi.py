"""The C-ABI library loads and exports every entry point include/phs.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

from pyheartsim_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "phs.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(phs_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "phs_simulate" in names and "phs_electrogram" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in include/phs.h but not exported"


def test_bindings_cover_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_struct_layouts_match_c():
    # sizes fixed by include/phs.h (natural alignment, 64-bit)
    assert ctypes.sizeof(_lib.InstanceDesc) == 224
    assert ctypes.sizeof(_lib.InstanceInfo) == 64
    assert ctypes.sizeof(_lib.OperatorTablesArgs) == 184


def test_status_strings_without_gpu():
    lib = _lib.lib()
    assert lib.phs_version() >= 100
    assert b"converge" in lib.phs_status_string(_lib.PHS_WARN_NO_CONVERGE)
    assert lib.phs_status_string(12345) == b"unknown status"


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    try:
        _lib.lib()
    except RuntimeError as e:
        assert "missing" in str(e)
    else:
        raise AssertionError("expected a RuntimeError")
