"""Python host binding of libqtrk_b200.so, mirroring QTrkDotNet's ``QTrkInstance``.

``QTrkInstance`` keeps the method names and argument meaning of
``QTrkDotNet/QTrkInstance.cs:13-190`` (BeginLUT/BuildLUT/FinalizeLUT, SetLocalizationMode,
ScheduleLocalization, Flush, GetResultCount, GetResults, IsIdle, GetQueueLength, ...), with
numpy arrays in place of the .NET image types. Every call goes through the C ABI of
``include/qtrk_c_api.h``. The library must be built (``python -m qtrk_b200.build``); there
is no CPU fallback: creating an instance without a B200 raises ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from pathlib import Path

import numpy as np

from . import abi

LIB_PATH = Path(__file__).resolve().parent / "libqtrk_b200.so"
_lib: C.CDLL | None = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load (once) and bind the compiled library. Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} not found: build it with `python -m qtrk_b200.build`")
    lib = abi.bind(C.CDLL(str(p)), extensions=True)
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    lib = load_library()
    buf = C.create_string_buffer(4096)
    lib.QTrkB200GetLastError(buf, len(buf))
    return buf.value.decode(errors="replace")


def computed_config(settings: abi.QTrkSettings) -> abi.QTrkComputedConfig:
    cc = abi.QTrkComputedConfig()
    load_library().QTrkGetComputedConfig(C.byref(settings), C.byref(cc))
    return cc


class QTrkInstance:
    """One tracker instance on one GPU (QTrkDotNet/QTrkInstance.cs:13)."""

    def __init__(self, settings: abi.QTrkSettings, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.settings = settings
        self.handle = self.lib.QTrkCreateInstance(C.byref(settings))
        if not self.handle:
            raise RuntimeError("QTrkCreateInstance failed: " + last_error())
        self.config = abi.QTrkComputedConfig()
        self.lib.QTrkGetComputedConfig(C.byref(settings), C.byref(self.config))
        self._async_stacks: list = []  # stacks handed to BuildLUTAsync, kept alive until FinalizeLUT

    # -- lifecycle --
    def Destroy(self) -> None:
        if self.handle:
            self.lib.QTrkFreeInstance(self.handle)
            self.handle = None
        self._async_stacks = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Destroy()

    def __del__(self):
        try:
            self.Destroy()
        except Exception:
            pass

    # -- configuration --
    def SetLocalizationMode(self, mode: int) -> None:
        self.lib.QTrkSetLocalizationMode(self.handle, int(mode))

    def SetRadialZLUT(self, lut: np.ndarray | None, count: int | None = None, planes: int | None = None) -> None:
        if lut is None:
            self.lib.QTrkSetRadialZLUT(self.handle, None, int(count), int(planes))
            return
        lut = np.ascontiguousarray(lut, np.float32)
        self.lib.QTrkSetRadialZLUT(self.handle, lut.ctypes.data_as(C.c_void_p), lut.shape[0], lut.shape[1])

    def SetRadialZLUTSize(self, nbeads: int, planes: int) -> None:
        self.SetRadialZLUT(None, nbeads, planes)

    def GetRadialZLUTSize(self) -> tuple[int, int, int]:
        c, p, r = C.c_int(), C.c_int(), C.c_int()
        self.lib.QTrkGetRadialZLUTSize(self.handle, C.byref(c), C.byref(p), C.byref(r))
        return c.value, p.value, r.value

    def GetRadialZLUT(self) -> np.ndarray:
        c, p, r = self.GetRadialZLUTSize()
        out = np.zeros((c, p, r), np.float32)
        if out.size:
            self.lib.QTrkGetRadialZLUT(self.handle, out.ctypes.data_as(C.c_void_p))
        return out

    def SetRadialWeights(self, w: np.ndarray | None) -> None:
        if w is None:
            self.lib.QTrkSetRadialWeights(self.handle, None)
        else:
            w = np.ascontiguousarray(w, np.float32)
            self.lib.QTrkSetRadialWeights(self.handle, w.ctypes.data_as(C.c_void_p))

    def SetPixelCalibrationImages(self, offset: np.ndarray | None, gain: np.ndarray | None) -> None:
        o = None if offset is None else np.ascontiguousarray(offset, np.float32)
        g = None if gain is None else np.ascontiguousarray(gain, np.float32)
        self.lib.QTrkSetPixelCalibrationImages(self.handle, None if o is None else o.ctypes.data_as(C.c_void_p),
                                               None if g is None else g.ctypes.data_as(C.c_void_p))

    def SetPixelCalibrationFactors(self, offset_factor: float, gain_factor: float) -> None:
        """Scale factors of this instance's calibration images (1, 1 by default)."""
        self.lib.QTrkB200SetPixelCalibrationFactors(self.handle, float(offset_factor), float(gain_factor))

    # -- LUT building (QTrkInstance.cs:51-60, 95-98) --
    def BeginLUT(self, flags: int | bool = abi.BUILDLUT_NORMALIZE) -> None:
        if isinstance(flags, bool):
            flags = abi.BUILDLUT_NORMALIZE if flags else 0
        self.lib.QTrkBeginLUT(self.handle, int(flags))

    def BuildLUT(self, stack: np.ndarray, plane: int, known_pos: np.ndarray | None = None) -> None:
        """stack: (nbeads, H, W) ROIs of one plane (u8/u16/f32)."""
        stack = np.ascontiguousarray(stack)
        pdt = abi.NUMPY_PDT[stack.dtype]
        kp = None if known_pos is None else np.ascontiguousarray(known_pos, np.float32)
        self.lib.QTrkBuildLUT(self.handle, stack.ctypes.data_as(C.c_void_p), stack.shape[2] * stack.itemsize, pdt,
                              int(plane), None if kp is None else kp.ctypes.data_as(C.c_void_p))

    def BuildLUTAsync(self, stack: np.ndarray, plane: int, known_pos: np.ndarray | None = None) -> None:
        """BuildLUT that does not wait for the plane's copy: `stack` (nbeads, H, W), contiguous and in
        pinned memory for the copy to be asynchronous, must stay unchanged until FinalizeLUT returns
        (the instance holds a reference to it until then, so it stays alive)."""
        if not stack.flags.c_contiguous:
            raise ValueError("BuildLUTAsync needs a contiguous stack (it is read after the call returns)")
        self._async_stacks.append(stack)
        pdt = abi.NUMPY_PDT[stack.dtype]
        kp = None if known_pos is None else np.ascontiguousarray(known_pos, np.float32)
        self.lib.QTrkB200BuildLUTAsync(self.handle, stack.ctypes.data_as(C.c_void_p), stack.shape[2] * stack.itemsize,
                                       pdt, int(plane), None if kp is None else kp.ctypes.data_as(C.c_void_p))

    def FinalizeLUT(self) -> None:
        self.lib.QTrkFinalizeLUT(self.handle)
        self._async_stacks = []

    # -- scheduling --
    def ScheduleLocalization(self, img: np.ndarray, frame: int = 0, zlut: int = 0, timestamp: int = 0) -> None:
        img = np.ascontiguousarray(img)
        job = abi.LocalizationJob()
        job.frame, job.timestamp, job.zlutIndex = frame, timestamp, zlut
        self.lib.QTrkScheduleLocalization(self.handle, img.ctypes.data_as(C.c_void_p), img.shape[1] * img.itemsize,
                                          abi.NUMPY_PDT[img.dtype], C.byref(job))

    def ScheduleStack(self, rois: np.ndarray, zlut_index: np.ndarray | None = None, first_frame: int = 0) -> None:
        """Schedule a (N, H, W) stack, ROI i as job frame first_frame+i."""
        rois = np.ascontiguousarray(rois)
        pdt = abi.NUMPY_PDT[rois.dtype]
        pitch = rois.shape[2] * rois.itemsize
        job = abi.LocalizationJob()
        base = rois.ctypes.data
        step = rois.strides[0]
        for i in range(rois.shape[0]):
            job.frame = first_frame + i
            job.zlutIndex = int(zlut_index[i]) if zlut_index is not None else 0
            self.lib.QTrkScheduleLocalization(self.handle, C.c_void_p(base + i * step), pitch, pdt, C.byref(job))

    def ScheduleFrame(self, frame: np.ndarray, positions: np.ndarray, frame_no: int = 0, zlut_base: int = 0) -> int:
        frame = np.ascontiguousarray(frame) if not frame.flags.c_contiguous else frame
        pos = np.ascontiguousarray(positions, np.int32)
        job = abi.LocalizationJob()
        job.frame, job.zlutIndex = frame_no, zlut_base
        return self.lib.QTrkScheduleFrame(self.handle, frame.ctypes.data_as(C.c_void_p), frame.strides[0],
                                          frame.shape[1], frame.shape[0], pos.ctypes.data_as(C.c_void_p),
                                          pos.shape[0], abi.NUMPY_PDT[frame.dtype], C.byref(job))

    def Flush(self) -> None:
        self.lib.QTrkFlush(self.handle)

    # -- results --
    def GetResultCount(self) -> int:
        return self.lib.QTrkGetResultCount(self.handle)

    def GetResults(self, max_results: int | None = None) -> np.ndarray:
        n = max_results if max_results is not None else self.GetResultCount()
        buf = (abi.LocalizationResult * max(n, 1))()
        got = self.lib.QTrkFetchResults(self.handle, buf, n)
        return abi.results_to_numpy(buf, got)

    def ClearResults(self) -> None:
        self.lib.QTrkClearResults(self.handle)

    def IsIdle(self) -> bool:
        return bool(self.lib.QTrkIsIdle(self.handle))

    def GetQueueLength(self) -> int:
        m = C.c_int()
        return self.lib.QTrkGetQueueLength(self.handle, C.byref(m))

    def GetMaxQueueLength(self) -> int:
        m = C.c_int()
        self.lib.QTrkGetQueueLength(self.handle, C.byref(m))
        return m.value

    def GetWarnings(self) -> str:
        buf = C.create_string_buffer(65536)
        self.lib.QTrkGetWarnings(self.handle, buf, len(buf))
        return buf.value.decode(errors="replace")

    def GetProfileReport(self) -> str:
        buf = C.create_string_buffer(8192)
        self.lib.QTrkGetProfileReport(self.handle, buf, len(buf))
        return buf.value.decode(errors="replace")

    def KernelLaunchCount(self) -> int:
        return int(self.lib.QTrkB200GetKernelLaunchCount(self.handle))

    # -- convenience --
    def WaitForResults(self, n: int, timeout_s: float = 120.0) -> np.ndarray:
        """Flush, wait until n results are available and return them sorted by job frame."""
        self.Flush()
        deadline = time.monotonic() + timeout_s
        while self.GetResultCount() < n:
            if time.monotonic() > deadline:
                raise TimeoutError(f"only {self.GetResultCount()} of {n} results after {timeout_s} s; "
                                   f"warnings: {self.GetWarnings()}")
            time.sleep(0.0002)
        res = self.GetResults(n)
        return res[np.argsort(res["frame"], kind="stable")]

    def Localize(self, rois: np.ndarray, zlut_index: np.ndarray | None = None, timeout_s: float = 120.0) -> np.ndarray:
        self.ScheduleStack(rois, zlut_index)
        return self.WaitForResults(rois.shape[0], timeout_s)

    def LocalizeDevice(self, d_pixels: int, pitch: int, roi_stride: int, pdt: int, count: int,
                       d_results: int, d_jobs: int = 0, stream: int = 0) -> None:
        """Device-resident batch (pointers are device addresses, e.g. torch data_ptr())."""
        rc = self.lib.QTrkB200LocalizeDevice(self.handle, C.c_void_p(d_pixels), pitch, roi_stride, pdt, count,
                                             C.c_void_p(d_jobs) if d_jobs else None, C.c_void_p(d_results),
                                             C.c_void_p(stream) if stream else None)
        if rc != 0:
            raise RuntimeError(f"QTrkB200LocalizeDevice failed ({rc}): {self.GetWarnings()}")
