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


def _mesh_args(nCell, nFace, nf=4, dim=3, nvert=4, nfv=3, nNode=4):
    """dndsb_mesh_create arguments with valid (non-null) host arrays of the given sizes."""
    import numpy as np
    D = ctypes.POINTER(ctypes.c_double)
    I64 = ctypes.POINTER(ctypes.c_int64)
    I32 = ctypes.POINTER(ctypes.c_int32)
    keep = dict(coords=np.zeros((max(nNode, 1), 3)), c2n=np.zeros((max(nCell, 1), nvert), np.int64), cs=np.zeros((max(nCell, 1), nvert, 3)),
                f2n=np.zeros((max(nFace, 1), nfv), np.int64), fs=np.zeros((max(nFace, 1), nfv, 3)), f2c=np.zeros((max(nFace, 1), 2), np.int64),
                fz=np.zeros(max(nFace, 1), np.int32), fp=np.zeros((max(nFace, 1), 3)), c2f=np.zeros((max(nCell, 1), max(nf, 1)), np.int64))
    p = lambda a, t: a.ctypes.data_as(t)
    args = [dim, 4, 3, nNode, p(keep["coords"], D), nCell, nvert, p(keep["c2n"], I64), p(keep["cs"], D), nFace, nfv, p(keep["f2n"], I64),
            p(keep["fs"], D), p(keep["f2c"], I64), p(keep["fz"], I32), p(keep["fp"], D), nf, p(keep["c2f"], I64)]
    return args, keep


@pytest.mark.parametrize("nCell, nFace, nf, code, word", [(0, 4, 4, -1, b"bad sizes"), (1, 0, 4, -1, b"bad sizes"),
                                                          (1, 4, 7, -1, b"bad sizes"), (1 << 30, 4, 4, -5, b"too large")])
def test_mesh_sizes_are_checked_before_device_work(nCell, nFace, nf, code, word):
    """Empty meshes, more than six faces per cell and meshes beyond the 32-bit device indices are rejected
    by the host with a status code, before any device work."""
    L = capi.load(require_device=False)
    h = ctypes.c_void_p()
    args, keep = _mesh_args(min(nCell, 1) if nCell >= (1 << 30) else nCell, nFace, nf)
    args[5] = nCell
    rc = L.dndsb_mesh_create(ctypes.byref(h), *args)
    assert rc == code and word in L.dndsb_last_error(), (rc, L.dndsb_last_error())
