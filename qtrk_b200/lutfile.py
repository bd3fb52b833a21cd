"""Z-LUT files (``.radialzlut``) through the library's C ABI.

Layout (the one ``cputrack/utils.cpp:680-710`` ReadLUTFile reads): int32 count, planes,
radialsteps, then ``count*planes*radialsteps`` float32 in [bead][plane][bin] order.
``read_bead("file.radialzlut#k")`` returns bead k's LUT min-max normalised to [0, 1], as
ReadLUTFile does (``normalize``, cputrack/utils.h:23-34).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .tracker import last_error, load_library


def read(path: str | os.PathLike) -> np.ndarray:
    """The whole table, shape (count, planes, radialsteps) float32."""
    lib = load_library()
    c, p, r = C.c_int(), C.c_int(), C.c_int()
    if lib.QTrkB200ReadRadialZLUTFile(os.fsencode(path), None, C.byref(c), C.byref(p), C.byref(r)) != 0:
        raise OSError(last_error())
    out = np.zeros((c.value, p.value, r.value), np.float32)
    if lib.QTrkB200ReadRadialZLUTFile(os.fsencode(path), out.ctypes.data_as(C.c_void_p), C.byref(c), C.byref(p),
                                      C.byref(r)) != 0:
        raise OSError(last_error())
    return out


def write(path: str | os.PathLike, lut: np.ndarray) -> None:
    lut = np.ascontiguousarray(lut, np.float32)
    if lut.ndim == 2:
        lut = lut[None]
    lib = load_library()
    if lib.QTrkB200WriteRadialZLUTFile(os.fsencode(path), lut.ctypes.data_as(C.c_void_p), *lut.shape) != 0:
        raise OSError(last_error())


def read_bead(spec: str) -> np.ndarray:
    """``path#k``: bead k's (planes, radialsteps) LUT, min-max normalised."""
    path, _, idx = str(spec).rpartition("#")
    lut = read(path)[int(idx)]
    mn, mx = lut.min(), lut.max()
    return ((lut - mn) / (mx - mn)).astype(np.float32)
