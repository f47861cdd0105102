"""The C ABI library loads and exports every entry point include/bsmpo.h declares
(no compute call: this runs without a GPU)."""
import os
import re

from bosonsampling_b200 import _capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "bsmpo.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bsmpo_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    assert "bsmpo_bs_update" in names and "bsmpo_create" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    for name in declared():
        assert hasattr(lib, name), name


def test_binding_covers_every_declared_symbol():
    assert set(declared()) <= set(_capi.SIGNATURES), set(declared()) - set(_capi.SIGNATURES)


def test_version_string():
    assert b"sm_100a" in _capi.lib().bsmpo_version()
