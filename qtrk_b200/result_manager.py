"""Python binding of the ResultManager C ABI (``RM*`` in ``include/qtrk_c_api.h``), with the
method names of ``QTrkDotNet/ResultManager.cs:8-80`` (SetTracker, StoreFrameInfo, GetBeadResults,
GetFrameCounters, Flush, GetResults, RemoveBead, GetConfig, Dispose)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .tracker import last_error, load_library


def config(num_beads: int, num_frame_info_columns: int = 0, scaling=(1.0, 1.0, 1.0), offset=(0.0, 0.0, 0.0),
           write_interval: int = 1, max_frames_in_memory: int = 0, binary_output: bool = False):
    c = abi.ResultManagerConfig()
    c.numBeads, c.numFrameInfoColumns = num_beads, num_frame_info_columns
    c.scaling = abi.vector3f(*scaling)
    c.offset = abi.vector3f(*offset)
    c.writeInterval, c.maxFramesInMemory, c.binaryOutput = write_interval, max_frames_in_memory, int(binary_output)
    return c


class ResultManager:
    def __init__(self, file: str, frame_info_file: str, cfg, colnames=(), lib: C.CDLL | None = None):
        self.lib = lib or load_library()
        self.cfg = cfg
        names = ";".join(colnames).encode()
        self.handle = self.lib.RMCreate(file.encode() if file else b"", frame_info_file.encode() if frame_info_file else b"",
                                        C.byref(cfg), names)
        if not self.handle:
            raise RuntimeError("RMCreate failed: " + last_error())

    def SetTracker(self, trk) -> None:
        self.lib.RMSetTracker(self.handle, trk.handle if trk is not None else None)

    def StoreFrameInfo(self, frame: int, timestamp: float, cols=None) -> None:
        a = np.ascontiguousarray(cols if cols is not None else np.zeros(max(self.cfg.numFrameInfoColumns, 1)),
                                 np.float32)
        self.lib.RMStoreFrameInfo(self.handle, frame, timestamp, a.ctypes.data_as(C.c_void_p))

    def StoreResults(self, results: np.ndarray, roi_width: int, roi_height: int) -> None:
        """Results from another source (e.g. the request server), as a RESULT_DTYPE array."""
        r = np.ascontiguousarray(results, abi.RESULT_DTYPE)
        self.lib.QTrkB200RMStoreResults(self.handle, r.ctypes.data_as(C.c_void_p), len(r), roi_width, roi_height)

    def GetBeadResults(self, start: int, num_frames: int, bead: int) -> np.ndarray:
        buf = (abi.LocalizationResult * max(num_frames, 1))()
        n = self.lib.RMGetBeadResults(self.handle, start, num_frames, bead, buf)
        return abi.results_to_numpy(buf, max(n, 0))

    def GetFrameCounters(self) -> dict:
        c = abi.RMFrameCounters()
        self.lib.RMGetFrameCounters(self.handle, C.byref(c))
        return {n: getattr(c, n) for n, _ in c._fields_}

    def Flush(self) -> None:
        self.lib.RMFlush(self.handle)

    def GetResults(self, start_frame: int, num_frames: int) -> np.ndarray:
        n_b = self.cfg.numBeads
        buf = (abi.LocalizationResult * max(num_frames * n_b, 1))()
        n = self.lib.RMGetResults(self.handle, start_frame, num_frames, buf)
        return abi.results_to_numpy(buf, n * n_b).reshape(n, n_b) if n else abi.results_to_numpy(buf, 0)

    def RemoveBead(self, bead: int) -> None:
        self.lib.RMRemoveBead(self.handle, bead)

    def GetConfig(self):
        c = abi.ResultManagerConfig()
        self.lib.RMGetConfig(self.handle, C.byref(c))
        return c

    def Dispose(self) -> None:
        if self.handle:
            self.lib.RMDestroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Dispose()

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass
