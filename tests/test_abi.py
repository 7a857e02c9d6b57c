"""The C-ABI library: it loads, and it exports every entry point include/qfb.h
declares, each bound by the Python layer.  No compute call is made here."""

import ctypes
import os
import re
import subprocess

import pytest

from qforte_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"QFB_API\s+[\w\s\*]+?\b(qfb_\w+)\s*\(", txt))
    return names


def test_library_loads_and_exports_all_declared_symbols():
    L = _lib.lib()
    declared = _declared()
    assert len(declared) >= 30
    for name in sorted(declared):
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r" T (qfb_\w+)", out))
    assert declared <= exported
    # nothing beyond the declared ABI leaks out of the library
    assert exported <= declared


def test_every_declared_symbol_has_a_binding():
    assert _declared() <= set(_lib.SIGNATURES)


def test_version_and_error_plumbing():
    L = _lib.lib()
    assert L.qfb_version() >= 10000
    # an argument error is reported without touching a device
    h = ctypes.c_void_p()
    rc = L.qfb_state_create(0, 1, ctypes.byref(h))
    assert rc == _lib.QFB_EINVAL and not h.value
    assert "nqubit" in _lib.last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)
    rc = L.qfb_prog_create(None, None, None, 1, 0, ctypes.byref(h))
    assert rc == _lib.QFB_EINVAL
