"""Python access to the two oracles.

TEST INFRASTRUCTURE ONLY — the checker, never the thing measured or shipped. Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this.

* ``RefOracle``: the reference's own CPU tracker (``cputrack/QueuedCPUTracker.cpp`` +
  ``cputrack/cpu_tracker.cpp``), compiled from its sources by ``oracle/build.py`` into
  ``oracle/_ref/libqtrk_ref.so`` and driven through its unmodified C ABI
  (``cputrack/qtrk_c_api.cpp``) plus the stage entry points of
  ``oracle/ref_stage_exports.cpp``.
* ``PortOracle``: the FP64 restatement in ``oracle/qtrk_oracle.c``.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

from qtrk_b200 import abi  # noqa: E402  (struct layouts shared by both libraries)

REF_LIB = HERE / "_ref" / "libqtrk_ref.so"
PORT_LIB = HERE / "liboracle_port.so"

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def ref_available() -> bool:
    return REF_LIB.exists()


def port_available() -> bool:
    return PORT_LIB.exists()


class RefOracle:
    """The reference CPU tracker through its own C ABI."""

    def __init__(self, path: Path | str = REF_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing: run python oracle/build.py where the reference tree exists")
        self.lib = abi.bind(C.CDLL(str(path)))
        L = self.lib
        for name, args in {
            "ref_stage_com": [_f32p, C.c_int, C.c_int, C.c_float, _f32p],
            "ref_stage_qi": [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float,
                             C.c_float, C.c_float, C.c_void_p, _f32p],
            "ref_stage_quadrant_profile": [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_float, C.c_float, C.c_void_p, _f32p],
            "ref_stage_radial_profile": [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
                                         C.c_float, C.c_int, _f32p],
            "ref_stage_lut_compare": [_f32p, _f32p, C.c_int, C.c_int, C.c_void_p, C.c_void_p],
            "ref_stage_gauss2d": [_f32p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_float, _f32p],
            "ref_stage_radial_bin_window": [C.c_int, _f32p],
            "ref_stage_erf": [C.c_float],
        }.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = None
        L.ref_stage_lut_compare.restype = C.c_float
        L.ref_stage_erf.restype = C.c_float

    # ---- configuration ----
    def computed_config(self, s: abi.QTrkSettings) -> abi.QTrkComputedConfig:
        cc = abi.QTrkComputedConfig()
        self.lib.QTrkGetComputedConfig(C.byref(s), C.byref(cc))
        return cc

    # ---- whole pipeline through the reference's QueuedCPUTracker ----
    def track(self, s: abi.QTrkSettings, mode: int, rois: np.ndarray, lut: np.ndarray | None = None,
              zlut_index: np.ndarray | None = None, weights: np.ndarray | None = None,
              calib: tuple | None = None, timeout_s: float = 600.0, return_seconds: bool = False):
        """Localize a stack of ROIs (N,H,W; u8/u16/f32). Returns results sorted by job.frame.
        calib = (offset, gain): per-bead pixel calibration images ([beads][H][W] float32 or None),
        installed after the Z-LUT as QueuedCPUTracker::SetPixelCalibrationImages requires."""
        L = self.lib
        rois = np.ascontiguousarray(rois)
        n, h, w = rois.shape
        pdt = abi.NUMPY_PDT[rois.dtype]
        trk = L.QTrkCreateInstance(C.byref(s))
        try:
            if lut is not None:
                lut = np.ascontiguousarray(lut, dtype=np.float32)
                L.QTrkSetRadialZLUT(trk, _ptr(lut), lut.shape[0], lut.shape[1])
            if weights is not None:
                weights = np.ascontiguousarray(weights, dtype=np.float32)
                L.QTrkSetRadialWeights(trk, _ptr(weights))
            if calib is not None:
                off, gain = (None if a is None else np.ascontiguousarray(a, dtype=np.float32) for a in calib)
                L.ref_set_pixel_calibration.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
                L.ref_set_pixel_calibration(trk, None if off is None else off.ctypes.data,
                                            None if gain is None else gain.ctypes.data)
            L.QTrkSetLocalizationMode(trk, mode)
            job = abi.LocalizationJob()
            pitch = w * rois.itemsize
            t0 = time.perf_counter()
            for i in range(n):
                job.frame = i
                job.zlutIndex = int(zlut_index[i]) if zlut_index is not None else 0
                L.QTrkScheduleLocalization(trk, rois[i].ctypes.data_as(C.c_void_p), pitch, pdt, C.byref(job))
            L.QTrkFlush(trk)
            deadline = time.monotonic() + timeout_s
            while L.QTrkGetResultCount(trk) < n:
                if time.monotonic() > deadline:
                    raise TimeoutError("reference tracker did not finish")
                time.sleep(0.0005)
            dt = time.perf_counter() - t0
            buf = (abi.LocalizationResult * n)()
            got = L.QTrkFetchResults(trk, buf, n)
            res = abi.results_to_numpy(buf, got)
            while not L.QTrkIsIdle(trk):
                time.sleep(0.001)
        finally:
            L.QTrkFreeInstance(trk)
        res = res[np.argsort(res["frame"], kind="stable")]
        return (res, dt) if return_seconds else res

    def build_lut(self, s: abi.QTrkSettings, planes_stack: np.ndarray, flags: int = abi.BUILDLUT_NORMALIZE,
                  known_pos: np.ndarray | None = None, finalize: bool = True) -> np.ndarray:
        """BeginLUT/BuildLUT per plane/FinalizeLUT; planes_stack = (planes, nbeads, H, W)."""
        L = self.lib
        stack = np.ascontiguousarray(planes_stack)
        planes, nbeads, h, w = stack.shape
        pdt = abi.NUMPY_PDT[stack.dtype]
        trk = L.QTrkCreateInstance(C.byref(s))
        try:
            L.QTrkSetRadialZLUT(trk, None, nbeads, planes)
            L.QTrkBeginLUT(trk, flags)
            kp = None
            if known_pos is not None:
                kp = np.ascontiguousarray(known_pos, dtype=np.float32)
            for p in range(planes):
                L.QTrkBuildLUT(trk, stack[p].ctypes.data_as(C.c_void_p), w * stack.itemsize, pdt, p, _ptr(kp))
            if finalize:
                L.QTrkFinalizeLUT(trk)
            cnt, pl, rs = C.c_int(), C.c_int(), C.c_int()
            L.QTrkGetRadialZLUTSize(trk, C.byref(cnt), C.byref(pl), C.byref(rs))
            out = np.zeros((cnt.value, pl.value, rs.value), np.float32)
            L.QTrkGetRadialZLUT(trk, _ptr(out))
        finally:
            L.QTrkFreeInstance(trk)
        return out

    # ---- single stages ----
    def com(self, img: np.ndarray, bgcorr: float = 0.0) -> np.ndarray:
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(4, np.float32)
        self.lib.ref_stage_com(img, img.shape[1], img.shape[0], bgcorr, out)
        return out

    def qi(self, img, init, iterations, nr, angpq, factor, minr, maxr, weights=None) -> np.ndarray:
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(3, np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        self.lib.ref_stage_qi(img, img.shape[1], img.shape[0], init[0], init[1], iterations, nr, angpq, factor, minr,
                              maxr, _ptr(w), out)
        return out

    def radial_profile(self, img, center, nbins, angsteps, minr, maxr, normalize) -> np.ndarray:
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(nbins, np.float32)
        self.lib.ref_stage_radial_profile(img, img.shape[1], img.shape[0], center[0], center[1], nbins, angsteps,
                                          minr, maxr, int(normalize), out)
        return out

    def lut_compare(self, prof, lut, weights=None):
        prof = np.ascontiguousarray(prof, np.float32)
        lut = np.ascontiguousarray(lut, np.float32)
        scores = np.zeros(lut.shape[0], np.float32)
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        z = self.lib.ref_stage_lut_compare(prof, lut, lut.shape[0], lut.shape[1], _ptr(w), _ptr(scores))
        return z, scores

    def gauss2d(self, img, init, iterations, sigma) -> np.ndarray:
        img = np.ascontiguousarray(img, np.float32)
        out = np.zeros(4, np.float32)
        self.lib.ref_stage_gauss2d(img, img.shape[1], img.shape[0], init[0], init[1], iterations, sigma, out)
        return out

    def radial_bin_window(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.float32)
        self.lib.ref_stage_radial_bin_window(n, out)
        return out


class PortOracle:
    """FP64 restatement (oracle/qtrk_oracle.c)."""

    def __init__(self, path: Path | str = PORT_LIB):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} missing: run python oracle/build.py")
        L = self.lib = C.CDLL(str(path))
        P = C.c_void_p
        sig = {
            "oracle_nearest_pow2": (C.c_int, [C.c_int]),
            "oracle_update_config": (None, [P]),
            "oracle_radial_bin_window": (None, [C.c_int, _f64p]),
            "oracle_com": (None, [_f64p, C.c_int, C.c_int, C.c_double, _f64p]),
            "oracle_max_interp7": (C.c_double, [_f64p, C.c_int, _f64p]),
            "oracle_qi": (None, [_f64p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                 C.c_int, C.c_double, C.c_double, C.c_double, P, _f64p]),
            "oracle_normalize_profile": (None, [_f64p, C.c_int]),
            "oracle_radial_profile": (None, [_f64p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                             C.c_int, C.c_double, C.c_double, C.c_int, _f64p]),
            "oracle_lut_compare": (C.c_double, [_f64p, _f32p, C.c_int, C.c_int, P, P]),
            "oracle_erf_as": (C.c_double, [C.c_double]),
            "oracle_gauss2d": (None, [_f64p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                      C.c_double, _f64p]),
            "oracle_localize": (None, [P, C.c_int, _f64p, P, C.c_int, P, _f64p]),
            "oracle_build_lut_bead": (None, [P, _f64p, C.c_int, C.c_double, C.c_double, C.c_int, _f64p]),
            "oracle_gauss5": (None, [_f64p, C.c_int, C.c_int, _f64p, C.c_int, _f64p, P]),
            "oracle_zcost_grad": (C.c_double, [_f64p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                                 C.c_double, _f32p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                 P, C.c_int, _f64p, P]),
            "oracle_joint_refine": (None, [_f64p, C.c_int, C.c_int, C.c_double, _f64p, _f32p, C.c_int, C.c_int,
                                           C.c_int, C.c_double, C.c_double, P, C.c_int, C.c_int]),
            "oracle_set_joint_prior_scale": (None, [C.c_double]),
            "oracle_zlut_bias_correct": (C.c_double, [C.c_double, C.c_int, _f32p, C.c_int, C.c_int, C.c_int]),
            "oracle_gauss_nll_grad": (C.c_double, [_f64p, C.c_int, C.c_int, _f64p, _f64p]),
            "oracle_find_beads": (C.c_int, [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                            C.c_float, P, C.c_int, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args

    def computed_config(self, s: abi.QTrkSettings) -> abi.QTrkComputedConfig:
        cc = abi.QTrkComputedConfig()
        C.memmove(C.byref(cc), C.byref(s), C.sizeof(s))
        self.lib.oracle_update_config(C.byref(cc))
        return cc

    def com(self, img, bgcorr=0.0):
        img = np.ascontiguousarray(img, np.float64)
        out = np.zeros(4)
        self.lib.oracle_com(img, img.shape[1], img.shape[0], bgcorr, out)
        return out

    def qi(self, img, mean, init, iterations, nr, angpq, factor, minr, maxr, weights=None):
        img = np.ascontiguousarray(img, np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        out = np.zeros(3)
        self.lib.oracle_qi(img, img.shape[1], img.shape[0], mean, init[0], init[1], iterations, nr, angpq, factor,
                           minr, maxr, _ptr(w), out)
        return out

    def radial_profile(self, img, mean, center, nbins, angsteps, minr, maxr, normalize):
        img = np.ascontiguousarray(img, np.float64)
        out = np.zeros(nbins)
        self.lib.oracle_radial_profile(img, img.shape[1], img.shape[0], mean, center[0], center[1], nbins, angsteps,
                                       minr, maxr, int(normalize), out)
        return out

    def lut_compare(self, prof, lut, weights=None):
        prof = np.ascontiguousarray(prof, np.float64)
        lut = np.ascontiguousarray(lut, np.float32)
        scores = np.zeros(lut.shape[0])
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        z = self.lib.oracle_lut_compare(prof, lut, lut.shape[0], lut.shape[1], _ptr(w), _ptr(scores))
        return z, scores

    def gauss2d(self, img, mean, init, iterations, sigma):
        img = np.ascontiguousarray(img, np.float64)
        out = np.zeros(4)
        self.lib.oracle_gauss2d(img, img.shape[1], img.shape[0], mean, init[0], init[1], iterations, sigma, out)
        return out

    def gauss5(self, img, init, iterations, with_fisher=False):
        img = np.ascontiguousarray(img, np.float64)
        out = np.zeros(5)
        fisher = np.zeros(25) if with_fisher else None
        self.lib.oracle_gauss5(img, img.shape[1], img.shape[0], np.ascontiguousarray(init, np.float64), iterations,
                               out, _ptr(fisher))
        return (out, fisher.reshape(5, 5)) if with_fisher else out

    def zlut_bias_correct(self, z, planes, table, bead):
        table = np.ascontiguousarray(table, np.float32)
        return self.lib.oracle_zlut_bias_correct(float(z), planes, table, table.shape[1], table.shape[0], int(bead))

    def radial_bin_window(self, n):
        out = np.zeros(n)
        self.lib.oracle_radial_bin_window(n, out)
        return out

    def localize(self, cc: abi.QTrkComputedConfig, mode: int, rois: np.ndarray, lut: np.ndarray | None = None,
                 zlut_index: np.ndarray | None = None, weights: np.ndarray | None = None) -> np.ndarray:
        """Per-ROI pipeline of QueuedCPUTracker::ProcessJob in FP64. Returns (N, 7):
        x, y, z, com_x, com_y, error, imageMean."""
        n = rois.shape[0]
        out = np.zeros((n, 7))
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        o = np.zeros(7)
        for i in range(n):
            img = np.ascontiguousarray(rois[i], np.float64).copy()
            lp = None
            planes = 0
            if lut is not None:
                b = int(zlut_index[i]) if zlut_index is not None else 0
                lb = np.ascontiguousarray(lut[b], np.float32)
                lp, planes = lb, lb.shape[0]
            self.lib.oracle_localize(C.byref(cc), mode, img, _ptr(lp), planes, _ptr(w), o)
            out[i] = o
        return out

    def build_lut(self, cc: abi.QTrkComputedConfig, planes_stack: np.ndarray, flags: int,
                  known_pos: np.ndarray | None = None, finalize: bool = True) -> np.ndarray:
        planes, nbeads = planes_stack.shape[:2]
        nb = cc.zlut_radialsteps
        lut = np.zeros((nbeads, planes, nb))
        norm = int((flags & abi.BUILDLUT_NORMALIZE) != 0)
        for p in range(planes):
            for b in range(nbeads):
                img = np.ascontiguousarray(planes_stack[p, b], np.float64)
                row = lut[b, p]
                has = known_pos is not None
                kx, ky = (float(known_pos[b, 0]), float(known_pos[b, 1])) if has else (0.0, 0.0)
                tmp = np.ascontiguousarray(row.copy())
                self.lib.oracle_build_lut_bead(C.byref(cc), img, int(has), kx, ky, norm, tmp)
                lut[b, p] = tmp
        if finalize:
            for b in range(nbeads):
                for p in range(planes):
                    r = np.ascontiguousarray(lut[b, p])
                    self.lib.oracle_normalize_profile(r, nb)
                    lut[b, p] = r
        return lut

    def zcost_grad(self, img, mean, xyz, lut, angsteps, minr, maxr, weights=None, normalize=True,
                   want_lut_grad=False):
        """(cost, grad xyz (3,), grad LUT (planes, bins) or None) of the radial-profile/LUT cost."""
        img = np.ascontiguousarray(img, np.float64)
        lut = np.ascontiguousarray(lut, np.float32)
        planes, nb = lut.shape
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        grad = np.zeros(3)
        glut = np.zeros((planes, nb)) if want_lut_grad else None
        c = self.lib.oracle_zcost_grad(img, img.shape[1], img.shape[0], mean, xyz[0], xyz[1], xyz[2], lut, planes,
                                       nb, angsteps, minr, maxr, _ptr(w), int(normalize), grad,
                                       glut.ctypes.data if glut is not None else None)
        return c, grad, glut

    def joint_refine(self, img, mean, xyz, lut, angsteps, minr, maxr, weights=None, normalize=True, steps=5):
        img = np.ascontiguousarray(img, np.float64)
        lut = np.ascontiguousarray(lut, np.float32)
        io = np.ascontiguousarray(np.array(xyz, np.float64))
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        self.lib.oracle_joint_refine(img, img.shape[1], img.shape[0], mean, io, lut, lut.shape[0], lut.shape[1],
                                     angsteps, minr, maxr, _ptr(w), int(normalize), steps)
        return io

    def gauss_nll_grad(self, img, params):
        """(NLL, gradient (5,)) of the integrated-Gaussian Poisson model at params (x, y, I0, bg, sigma)."""
        img = np.ascontiguousarray(img, np.float64)
        p = np.ascontiguousarray(params, np.float64)
        g = np.zeros(5)
        return self.lib.oracle_gauss_nll_grad(img, img.shape[1], img.shape[0], p, g), g

    def find_beads(self, img, sample_corner, roi, rel_dist, similarity, return_conv=False):
        """QTrkFindBeads restated (FP64 convolution); returns (n, 2) int ROI corners [, conv map]."""
        img = np.ascontiguousarray(img, np.float32)
        h, w = img.shape
        out = np.zeros((4096, 2), np.int32)
        w2, h2 = 1 << max(0, (w - 1).bit_length()), 1 << max(0, (h - 1).bit_length())
        conv = np.zeros((h2, w2)) if return_conv else None
        n = self.lib.oracle_find_beads(img, w, h, int(sample_corner[0]), int(sample_corner[1]), roi, rel_dist,
                                       similarity, out.ctypes.data, len(out),
                                       conv.ctypes.data if conv is not None else None)
        pos = out[:min(n, len(out))].copy()
        return (pos, conv) if return_conv else pos


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
