"""The C-ABI library loads and exports every function include/dndsb.h declares (no GPU needed)."""
import ctypes
import os
import re

import pytest

from dndsr_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "dndsb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dndsb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_bound_functions():
    assert set(_declared()) == set(capi.SIGNATURES)


def test_library_exports_every_declared_symbol():
    build.build()
    lib = ctypes.CDLL(capi.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_device():
    L = capi.load(require_device=False)
    assert L.dndsb_version() == 1
    # argument checks run before any device work
    h = ctypes.c_void_p()
    rc = L.dndsb_vr_create(ctypes.byref(h), None, None)
    assert rc == -1 and b"null" in L.dndsb_last_error()
