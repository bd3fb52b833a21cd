"""Python binding of the request server (``QTrkB200Server*`` in ``include/qtrk_c_api.h``).

A ``Server`` serves frames of several ``QTrkInstance`` objects on one GPU: frames are
submitted as they arrive and their results polled per frame; the native dispatcher batches
waiting frames of one instance into a single CUDA-graph launch. No counterpart in the
reference, whose callers keep one ``QueuedTracker`` per camera
(``QTrkDotNet/QTrkInstance.cs:13``) and schedule with ``ScheduleFrame``
(``cputrack/QueuedTracker.cpp:91-111``); a frame's results here are the ones
``ScheduleFrame`` gives for it.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import abi
from .tracker import QTrkInstance, last_error, load_library


class Server:
    def __init__(self, device: int = 0, memory_budget: int = 1 << 30, lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.handle = self.lib.QTrkB200ServerCreate(device, memory_budget)
        if not self.handle:
            raise RuntimeError("QTrkB200ServerCreate failed: " + last_error())
        self._frames: dict[int, np.ndarray] = {}  # keeps submitted frames alive until polled

    def close(self) -> None:
        if self.handle:
            self.lib.QTrkB200ServerDestroy(self.handle)
            self.handle = None
            self._frames.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def attach(self, inst: QTrkInstance) -> int:
        idx = self.lib.QTrkB200ServerAttach(self.handle, inst.handle)
        if idx < 0:
            raise RuntimeError("QTrkB200ServerAttach failed: " + last_error())
        return idx

    def submit(self, instance: int, frame: np.ndarray, positions: np.ndarray, frame_no: int = 0,
               zlut_base: int = 0) -> int:
        """Submit one frame (2-D u8/u16/f32 array) with its ROI corners (n x 2 int32)."""
        if frame.ndim != 2 or frame.strides[1] != frame.itemsize:
            frame = np.ascontiguousarray(frame)
        pos = np.ascontiguousarray(positions, np.int32).reshape(-1, 2)
        job = abi.LocalizationJob()
        job.frame, job.zlutIndex = frame_no, zlut_base
        rid = self.lib.QTrkB200ServerSubmitFrame(self.handle, instance, frame.ctypes.data_as(C.c_void_p),
                                                 frame.strides[0], frame.shape[1], frame.shape[0],
                                                 pos.ctypes.data_as(C.c_void_p), pos.shape[0],
                                                 abi.NUMPY_PDT[frame.dtype], C.byref(job))
        if rid < 0:
            raise RuntimeError("QTrkB200ServerSubmitFrame failed: " + last_error())
        self._frames[rid] = frame
        return rid

    def poll(self, request: int, max_results: int = 8192) -> np.ndarray | None:
        """The request's results (structured array), or None while it is pending."""
        buf = (abi.LocalizationResult * max(max_results, 1))()
        n = self.lib.QTrkB200ServerPoll(self.handle, request, buf, max_results)
        if n == -1:
            return None
        self._frames.pop(request, None)
        if n == -2:
            raise KeyError(f"unknown request {request}")
        if n == -3:
            raise RuntimeError("request failed: " + last_error())
        return abi.results_to_numpy(buf, n)

    def wait(self, request: int, timeout_s: float = 120.0, max_results: int = 8192) -> np.ndarray:
        t0 = time.monotonic()
        while True:
            r = self.poll(request, max_results)
            if r is not None:
                return r
            if time.monotonic() - t0 > timeout_s:
                raise TimeoutError(f"request {request} not done after {timeout_s} s")
            time.sleep(0.0002)

    def hold(self, on: bool = True) -> None:
        """While held, submitted frames wait; releasing batches them together."""
        self.lib.QTrkB200ServerHold(self.handle, 1 if on else 0)

    def reset_stats(self) -> None:
        self.lib.QTrkB200ServerResetStats(self.handle)

    def stats(self) -> dict:
        s = abi.QTrkB200ServeStats()
        self.lib.QTrkB200ServerGetStats(self.handle, C.byref(s))
        return {name: getattr(s, name) for name, _ in s._fields_ if name != "reserved"}
