"""The C-ABI library builds, loads without a GPU and exports every entry
point that include/rkb200.h declares (no compute calls here)."""
import ctypes
import os
import re

from conftest import ROOT


def _declared():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(rkb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared()
    assert "rkb_yk_flat" in names and "rkb_table_contract_fp64" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    from atomx_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_table_matches_header():
    from atomx_b200 import _native
    assert sorted(_native._SIGNATURES) == _declared()


def test_version_string_without_gpu():
    from atomx_b200 import build
    lib = ctypes.CDLL(build.build())
    lib.rkb_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.rkb_version()
