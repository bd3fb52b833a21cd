"""Test harness for the LabVIEW binding: builds the fake LabVIEW run-time (tests/lv_fake), loads it
with RTLD_GLOBAL so that libqtrk_b200_lv.so resolves NumericArrayResize/MoveBlock from it, and
converts between numpy arrays and LabVIEW handles."""
import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

from qtrk_b200 import abi
from qtrk_b200.tracker import load_library

ROOT = Path(__file__).resolve().parent.parent
LV_LIB = ROOT / "qtrk_b200" / "libqtrk_b200_lv.so"
_fake = None
_lv = None

CODES = {np.dtype(np.float32): 9, np.dtype(np.int32): 3, np.dtype(np.uint32): 7, np.dtype(np.uint16): 6,
         np.dtype(np.uint8): 5}


class ErrorCluster(C.Structure):
    _fields_ = [("status", C.c_uint8), ("code", C.c_int32), ("message", C.c_void_p)]


def fake_runtime():
    global _fake
    if _fake is None:
        out = Path(tempfile.mkdtemp(prefix="fake_lv_")) / "libfake_labview.so"
        subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", str(out), str(ROOT / "tests" / "lv_fake" / "fake_labview.c")],
                       check=True)
        _fake = C.CDLL(str(out), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
        _fake.fake_lv_new.restype = C.c_void_p
        _fake.fake_lv_new.argtypes = [C.c_int32, C.c_int32, C.c_void_p]
        _fake.fake_lv_free.argtypes = [C.c_void_p]
    return _fake


def lv_library():
    global _lv
    if _lv is None:
        load_library()  # the core library first, from its in-tree path
        fake_runtime()
        _lv = C.CDLL(str(LV_LIB), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    return _lv


def handle(a: np.ndarray) -> int:
    """A new LabVIEW handle holding a copy of a (any number of dimensions)."""
    a = np.ascontiguousarray(a)
    dims = np.array(a.shape if a.ndim else (1,), np.int32)
    h = fake_runtime().fake_lv_new(CODES[a.dtype], len(dims), dims.ctypes.data)
    assert h
    if a.size:
        C.memmove(_data_ptr(h, len(dims), a.dtype), a.ctypes.data, a.nbytes)
    return h


def empty_handle(dtype, ndims: int) -> int:
    return handle(np.zeros((0,) * ndims, dtype))


def _data_ptr(h: int, ndims: int, dtype) -> int:
    block = C.cast(h, C.POINTER(C.c_void_p))[0]
    hdr = 4 * ndims
    al = min(np.dtype(dtype).itemsize, 8)
    hdr = (hdr + al - 1) // al * al
    return block + hdr


def read(h: int, ndims: int, dtype) -> np.ndarray:
    block = C.cast(h, C.POINTER(C.c_void_p))[0]
    dims = tuple(np.ctypeslib.as_array(C.cast(block, C.POINTER(C.c_int32)), shape=(ndims,)))
    n = int(np.prod(dims)) if dims else 0
    out = np.zeros(n, dtype)
    if n:
        C.memmove(out.ctypes.data, _data_ptr(h, ndims, dtype), out.nbytes)
    return out.reshape(dims)


def free(h: int) -> None:
    fake_runtime().fake_lv_free(h)


def lstr(h: int) -> str:
    if not h:
        return ""
    block = C.cast(h, C.POINTER(C.c_void_p))[0]
    n = C.cast(block, C.POINTER(C.c_int32))[0]
    return C.string_at(block + 4, n).decode(errors="replace")


def new_lstr(text: str = "") -> int:
    b = np.frombuffer(text.encode(), np.uint8) if text else np.zeros(0, np.uint8)
    return handle(b)
