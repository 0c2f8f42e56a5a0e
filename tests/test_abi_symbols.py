"""libp3m_b200.so loads (no GPU needed) and exports every entry point that
include/p3m_b200.h declares; the Python binding covers them all."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "p3m_b200.h")
LIB = os.path.join(ROOT, "md-force-routines_b200", "libp3m_b200.so")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(p3m_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_header():
    lib = ctypes.CDLL(LIB)
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from p3m_b200._lib import SIGNATURES

    assert sorted(SIGNATURES) == declared()
