"""ctypes mirror of the QTrk C ABI (``include/qtrk_c_api.h``).

The struct layouts and prototypes are those of the reference's ``cputrack/qtrk_c_api.h``
(packed structs, cdecl), so the same binding drives any library that exports that ABI:
``libqtrk_b200.so`` (this package's GPU tracker) and, in the tests, the reference's own
CPU tracker compiled into ``oracle/_ref/libqtrk_ref.so``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# Localization modes, cputrack/qtrk_c_api.h:5-20
LT_OnlyCOM = 0
LT_XCor1D = 1
LT_QI = 2
LT_Gaussian2D = 4
LT_ZLUTAlign = 8
LT_LocalizeZ = 16
LT_NormalizeProfile = 64
LT_ClearFirstFourPixels = 128
LT_FourierLUT = 256
LT_LocalizeZWeighted = 512
# Extensions of libqtrk_b200 (no reference counterpart)
LT_B200_ZMatchBF16 = 1 << 20
LT_B200_JointRefine = 1 << 21
LT_B200_Gaussian5P = 1 << 22
LT_B200_ZMatchTF32 = 1 << 23

# Pixel data types, cputrack/qtrk_c_api.h:24-29
QTrkU8, QTrkU16, QTrkFloat = 0, 1, 2
PDT_BYTES = {QTrkU8: 1, QTrkU16: 2, QTrkFloat: 4}
PDT_NUMPY = {QTrkU8: np.uint8, QTrkU16: np.uint16, QTrkFloat: np.float32}
NUMPY_PDT = {np.dtype(np.uint8): QTrkU8, np.dtype(np.uint16): QTrkU16, np.dtype(np.float32): QTrkFloat}

# BuildLUT flags, cputrack/QueuedTracker.h:305-308
BUILDLUT_IMAGELUT = 1
BUILDLUT_FOURIER = 2
BUILDLUT_NORMALIZE = 4
BUILDLUT_BIASCORRECT = 8

QTrkCUDA_UseList, QTrkCUDA_UseAll, QTrkCUDA_UseBest = -3, -2, -1


class vector2f(C.Structure):
    _pack_ = 4
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class vector3f(C.Structure):
    _pack_ = 4
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class ImageData(C.Structure):
    """TImageData<float>, cputrack/utils.h:79-136 (pack(4)): data, w, h."""

    _pack_ = 4
    _fields_ = [("data", C.POINTER(C.c_float)), ("w", C.c_int), ("h", C.c_int)]


class LocalizationJob(C.Structure):
    """24 bytes, cputrack/qtrk_c_api.h:34-45."""

    _pack_ = 1
    _fields_ = [("frame", C.c_uint32), ("timestamp", C.c_uint32), ("zlutIndex", C.c_int32),
                ("initialPos", vector3f)]


class LocalizationResult(C.Structure):
    """52 bytes, cputrack/qtrk_c_api.h:49-57."""

    _pack_ = 1
    _fields_ = [("job", LocalizationJob), ("pos", vector3f), ("firstGuess", vector2f), ("error", C.c_uint32),
                ("imageMean", C.c_float)]


class QTrkSettings(C.Structure):
    """84 bytes, cputrack/qtrk_c_api.h:59-114."""

    _pack_ = 1
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int), ("numThreads", C.c_int), ("cuda_device", C.c_int),
        ("com_bgcorrection", C.c_float),
        ("zlut_minradius", C.c_float), ("zlut_radial_coverage", C.c_float), ("zlut_angular_coverage", C.c_float),
        ("zlut_roi_coverage", C.c_float),
        ("qi_iterations", C.c_int), ("qi_minradius", C.c_float), ("qi_radial_coverage", C.c_float),
        ("qi_angular_coverage", C.c_float), ("qi_roi_coverage", C.c_float), ("qi_angstep_factor", C.c_float),
        ("xc1_profileLength", C.c_int), ("xc1_profileWidth", C.c_int), ("xc1_iterations", C.c_int),
        ("gauss2D_iterations", C.c_int), ("gauss2D_sigma", C.c_float),
        ("downsample", C.c_int),
    ]


class QTrkComputedConfig(C.Structure):
    """108 bytes, cputrack/qtrk_c_api.h:123-138 (QTrkSettings followed by the derived fields)."""

    _pack_ = 1
    _fields_ = QTrkSettings._fields_ + [
        ("zlut_radialsteps", C.c_int), ("zlut_angularsteps", C.c_int), ("zlut_maxradius", C.c_float),
        ("qi_radialsteps", C.c_int), ("qi_angstepspq", C.c_int), ("qi_maxradius", C.c_float),
    ]


class ROIPosition(C.Structure):
    """8 bytes, cputrack/qtrk_c_api.h:116-119."""

    _pack_ = 1
    _fields_ = [("x", C.c_int), ("y", C.c_int)]


class ResultManagerConfig(C.Structure):
    """41 bytes, cputrack/qtrk_c_api.h:211-219."""

    _pack_ = 1
    _fields_ = [("numBeads", C.c_int), ("numFrameInfoColumns", C.c_int), ("scaling", vector3f),
                ("offset", vector3f), ("writeInterval", C.c_int), ("maxFramesInMemory", C.c_uint32),
                ("binaryOutput", C.c_uint8)]


class RMFrameCounters(C.Structure):
    """28 bytes, cputrack/qtrk_c_api.h:220-229."""

    _pack_ = 1
    _fields_ = [(n, C.c_int) for n in ("startFrame", "processedFrames", "lastSaveFrame", "capturedFrames",
                                       "localizationsDone", "lostFrames", "fileError")]


class QTrkB200ServeStats(C.Structure):
    """Request-server statistics (library extension; 80 bytes)."""

    _fields_ = [
        ("frames", C.c_int64), ("rois", C.c_int64), ("launches", C.c_int64), ("graphs", C.c_int64),
        ("waits_for_memory", C.c_int64), ("lanes", C.c_int32), ("reserved", C.c_int32),
        ("elapsed_s", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
    ]


assert C.sizeof(QTrkB200ServeStats) == 80
assert C.sizeof(ResultManagerConfig) == 41
assert C.sizeof(RMFrameCounters) == 28
assert C.sizeof(LocalizationJob) == 24
assert C.sizeof(LocalizationResult) == 52
assert C.sizeof(QTrkSettings) == 84
assert C.sizeof(QTrkComputedConfig) == 108
assert C.sizeof(ROIPosition) == 8

RESULT_DTYPE = np.dtype([
    ("frame", "<u4"), ("timestamp", "<u4"), ("zlutIndex", "<i4"), ("init", "<f4", 3),
    ("pos", "<f4", 3), ("firstGuess", "<f4", 2), ("error", "<u4"), ("imageMean", "<f4"),
])
JOB_DTYPE = np.dtype([("frame", "<u4"), ("timestamp", "<u4"), ("zlutIndex", "<i4"), ("init", "<f4", 3)])
assert RESULT_DTYPE.itemsize == 52 and JOB_DTYPE.itemsize == 24

_P = C.c_void_p
_TRK = C.c_void_p

# name -> (restype, argtypes); the prototypes of cputrack/qtrk_c_api.h and cputrack/utils.h
PROTOTYPES = {
    "TestDLLCallConv": (None, [C.c_int]),
    "QTrkGetDefaultConfig": (None, [C.POINTER(QTrkSettings)]),
    "QTrkGetComputedConfig": (None, [C.POINTER(QTrkSettings), C.POINTER(QTrkComputedConfig)]),
    "QTrkCreateInstance": (_TRK, [C.POINTER(QTrkSettings)]),
    "QTrkFreeInstance": (None, [_TRK]),
    "QTrkSetLocalizationMode": (None, [_TRK, C.c_int]),
    "QTrkSetPixelCalibrationImages": (None, [_TRK, _P, _P]),
    "QTrkSetPixelCalibrationFactors": (None, [C.c_float, C.c_float]),
    "QTrkScheduleLocalization": (None, [_TRK, _P, C.c_int, C.c_int, C.POINTER(LocalizationJob)]),
    "QTrkClearResults": (None, [_TRK]),
    "QTrkFlush": (None, [_TRK]),
    "QTrkScheduleFrame": (C.c_int, [_TRK, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_int,
                                    C.POINTER(LocalizationJob)]),
    "QTrkEnableRadialZLUTCompareProfile": (None, [C.c_bool]),
    "QTrkGetRadialZLUTCompareProfile": (None, [_P]),
    "QTrkSetRadialZLUT": (None, [_TRK, _P, C.c_int, C.c_int]),
    "QTrkGetRadialZLUT": (None, [_TRK, _P]),
    "QTrkGetRadialZLUTSize": (None, [_TRK, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "QTrkSetRadialWeights": (None, [_TRK, _P]),
    "QTrkBeginLUT": (None, [_TRK, C.c_uint]),
    "QTrkBuildLUT": (None, [_TRK, _P, C.c_int, C.c_int, C.c_int, _P]),
    "QTrkBuildLUTFromFrame": (None, [_TRK, C.POINTER(ImageData), C.c_int, _P, C.c_int]),
    "QTrkFinalizeLUT": (None, [_TRK]),
    "QTrkGetResultCount": (C.c_int, [_TRK]),
    "QTrkFetchResults": (C.c_int, [_TRK, _P, C.c_int]),
    "QTrkGetQueueLength": (C.c_int, [_TRK, C.POINTER(C.c_int)]),
    "QTrkIsIdle": (C.c_bool, [_TRK]),
    "QTrkGetProfileReport": (None, [_TRK, C.c_char_p, C.c_int]),
    "QTrkGetWarnings": (None, [_TRK, C.c_char_p, C.c_int]),
    "ComputeRadialProfile": (None, [_P, C.c_int, C.c_int, C.c_float, C.c_float, vector2f, C.POINTER(ImageData),
                                    C.c_float, C.c_bool]),
    "NormalizeRadialProfile": (None, [_P, C.c_int]),
    "NormalizeImage": (None, [C.POINTER(ImageData)]),
    "ApplyPoissonNoise": (None, [C.POINTER(ImageData), C.c_float, C.c_float]),
    "ApplyGaussianNoise": (None, [C.POINTER(ImageData), C.c_float]),
    "QTrkFindBeads": (_P, [C.POINTER(ImageData), C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                           C.POINTER(C.c_int), C.POINTER(ImageData)]),
    "QTrkFreeROIPositions": (None, [_P]),
    "RMCreate": (_P, [C.c_char_p, C.c_char_p, C.POINTER(ResultManagerConfig), C.c_char_p]),
    "RMSetTracker": (None, [_P, _TRK]),
    "RMDestroy": (None, [_P]),
    "RMStoreFrameInfo": (None, [_P, C.c_int, C.c_double, _P]),
    "RMGetBeadResults": (C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P]),
    "RMGetFrameCounters": (None, [_P, C.POINTER(RMFrameCounters)]),
    "RMFlush": (None, [_P]),
    "RMGetResults": (C.c_int, [_P, C.c_int, C.c_int, _P]),
    "RMRemoveBead": (None, [_P, C.c_int]),
    "RMGetConfig": (None, [_P, C.POINTER(ResultManagerConfig)]),
    "GenerateImageFromLUT": (None, [C.POINTER(ImageData), C.POINTER(ImageData), C.c_float, C.c_float, vector3f,
                                    C.c_bool, C.c_int]),
    "GenerateGaussianSpotImage": (None, [C.POINTER(ImageData), vector2f, C.c_float, C.c_float, C.c_float]),
}

# Extensions exported by libqtrk_b200 only.
B200_PROTOTYPES = {
    "QTrkB200GetLastError": (C.c_int, [C.c_char_p, C.c_int]),
    "QTrkB200GetKernelLaunchCount": (C.c_int64, [_TRK]),
    "QTrkB200SetZLUTBiasTable": (None, [_TRK, _P, C.c_int, C.c_int]),
    "QTrkB200ComputeZLUTBiasTable": (None, [_TRK, C.c_int, _P, C.c_int, C.c_int]),
    "QTrkB200LocalizeDevice": (C.c_int, [_TRK, _P, C.c_int, C.c_int64, C.c_int, C.c_int, _P, _P, _P]),
    "QTrkB200BuildLUTAsync": (None, [_TRK, _P, C.c_int, C.c_int, C.c_int, _P]),
    "QTrkB200ZLUTCostGradient": (C.c_int, [_TRK, _P, C.c_int, C.c_int64, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]),
    "QTrkB200GaussianNLLGradient": (C.c_int, [_TRK, _P, C.c_int, C.c_int64, C.c_int, C.c_int, _P, _P, _P, _P]),
    "QTrkB200RefineZLUT": (None, [_TRK, _P, C.c_int, C.c_int64, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_float,
                                  _P, _P]),
    "QTrkB200LocalizeDeviceNoAlloc": (C.c_int, [_TRK, _P, C.c_int, C.c_int64, C.c_int, C.c_int, _P, _P, _P]),
    "QTrkB200RMStoreResults": (None, [_P, _P, C.c_int, C.c_int, C.c_int]),
    "QTrkB200SetPixelCalibrationFactors": (None, [_TRK, C.c_float, C.c_float]),
    "QTrkB200ReadRadialZLUTFile": (C.c_int, [C.c_char_p, _P, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int)]),
    "QTrkB200WriteRadialZLUTFile": (C.c_int, [C.c_char_p, _P, C.c_int, C.c_int, C.c_int]),
    "QTrkB200ServerCreate": (_P, [C.c_int, C.c_int64]),
    "QTrkB200ServerDestroy": (None, [_P]),
    "QTrkB200ServerAttach": (C.c_int, [_P, _TRK]),
    "QTrkB200ServerSubmitFrame": (C.c_int64, [_P, C.c_int, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_int, _P]),
    "QTrkB200ServerPoll": (C.c_int, [_P, C.c_int64, _P, C.c_int]),
    "QTrkB200ServerGetStats": (None, [_P, _P]),
    "QTrkB200ServerHold": (None, [_P, C.c_int]),
    "QTrkB200ServerResetStats": (None, [_P]),
}


def bind(lib: C.CDLL, extensions: bool = False) -> C.CDLL:
    """Attach restype/argtypes to every ABI function that ``lib`` exports."""
    protos = dict(PROTOTYPES)
    if extensions:
        protos.update(B200_PROTOTYPES)
    for name, (res, args) in protos.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


def settings(**overrides) -> QTrkSettings:
    """QTrkSettings with the reference defaults (cputrack/qtrk_c_api.h:60-80), then overrides."""
    s = QTrkSettings()
    s.width = s.height = 150
    s.numThreads = -1
    s.xc1_profileLength = 128
    s.xc1_profileWidth = 32
    s.xc1_iterations = 2
    s.zlut_minradius = 1.0
    s.zlut_angular_coverage = 0.7
    s.zlut_radial_coverage = 3.0
    s.zlut_roi_coverage = 1.0
    s.qi_iterations = 4
    s.qi_minradius = 1
    s.qi_angular_coverage = 0.7
    s.qi_radial_coverage = 3.0
    s.qi_roi_coverage = 1.0
    s.qi_angstep_factor = 1.0
    s.cuda_device = -2
    s.com_bgcorrection = 0.0
    s.gauss2D_iterations = 6
    s.gauss2D_sigma = 4
    s.downsample = 0
    for k, v in overrides.items():
        setattr(s, k, v)
    return s


def results_to_numpy(buf, n: int) -> np.ndarray:
    return np.frombuffer(buf, dtype=RESULT_DTYPE, count=n).copy()
