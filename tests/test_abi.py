"""C-ABI checks that need no GPU: exports, struct layouts, host-side entry points."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from qtrk_b200 import abi, synth

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "qtrk_c_api.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"QTRK_API\s+[\w\s\*]+?QTRK_CALLCONV\s+(\w+)\s*\(", text)))


def test_header_declares_the_reference_abi():
    names = declared_symbols()
    # every entry point QTrkDotNet binds for the tracker path (QTrkDLL.cs:244-328)
    for n in ["TestDLLCallConv", "QTrkGetDefaultConfig", "QTrkGetComputedConfig", "QTrkCreateInstance",
              "QTrkFreeInstance", "QTrkSetLocalizationMode", "QTrkSetPixelCalibrationImages",
              "QTrkSetPixelCalibrationFactors", "QTrkScheduleLocalization", "QTrkClearResults", "QTrkFlush",
              "QTrkScheduleFrame", "QTrkEnableRadialZLUTCompareProfile", "QTrkGetRadialZLUTCompareProfile",
              "QTrkSetRadialZLUT", "QTrkGetRadialZLUT", "QTrkGetRadialZLUTSize", "QTrkSetRadialWeights",
              "QTrkBeginLUT", "QTrkBuildLUT", "QTrkFinalizeLUT", "QTrkGetResultCount", "QTrkFetchResults",
              "QTrkGetQueueLength", "QTrkIsIdle", "QTrkGetProfileReport", "QTrkGetWarnings", "ComputeRadialProfile",
              "NormalizeRadialProfile", "GenerateImageFromLUT", "NormalizeImage"]:
        assert n in names, n


def test_library_exports_every_declared_symbol(qlib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(Path(qlib._name))], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, missing
    # nothing but the ABI is exported
    extra = [n for n in exported if not (n in declared_symbols() or n.startswith("_"))]
    assert not extra, extra


def test_struct_layouts_compiled_from_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "qtrk_c_api.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(LocalizationJob), sizeof(LocalizationResult),
         sizeof(QTrkSettings), sizeof(QTrkComputedConfig), sizeof(ROIPosition),
         offsetof(LocalizationResult, pos), offsetof(LocalizationResult, firstGuess),
         offsetof(LocalizationResult, error), offsetof(LocalizationResult, imageMean),
         offsetof(QTrkComputedConfig, zlut_radialsteps));
  return 0; }
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    # sizes measured on the reference (qtrk_c_api.h packing) and offsets of qtrk_c_api.h:50-57
    assert vals == [24, 52, 84, 108, 8, 24, 36, 44, 48, 84]
    assert C.sizeof(abi.LocalizationResult) == 52 and abi.LocalizationResult.pos.offset == 24


def test_computed_config_matches_reference(qlib, ref):
    for s in [synth.settings_roi60(), synth.settings_roi100(), abi.settings(), abi.settings(width=37, height=37)]:
        a = abi.QTrkComputedConfig()
        qlib.QTrkGetComputedConfig(C.byref(s), C.byref(a))
        b = ref.computed_config(s)
        assert bytes(a) == bytes(b)


def test_default_config_matches_reference(qlib, ref):
    a, b = abi.QTrkSettings(), abi.QTrkSettings()
    qlib.QTrkGetDefaultConfig(C.byref(a))
    ref.lib.QTrkGetDefaultConfig(C.byref(b))
    assert bytes(a) == bytes(b)


def test_normalize_radial_profile_matches_reference(qlib, ref):
    rng = np.random.default_rng(0)
    for n in (8, 40, 64):
        p = rng.normal(3, 2, n).astype(np.float32)
        a, b = p.copy(), p.copy()
        qlib.NormalizeRadialProfile(a.ctypes.data_as(C.c_void_p), n)
        ref.lib.NormalizeRadialProfile(b.ctypes.data_as(C.c_void_p), n)
        np.testing.assert_array_equal(a, b)


def _img(a):
    return abi.ImageData(a.ctypes.data_as(C.POINTER(C.c_float)), a.shape[1], a.shape[0])


def test_image_generators_match_reference(qlib, ref):
    a = np.zeros((20, 24), np.float32)
    b = np.zeros_like(a)
    qlib.GenerateGaussianSpotImage(C.byref(_img(a)), abi.vector2f(11.3, 9.7), 1.7, 1000.0, 12.0)
    ref.lib.GenerateGaussianSpotImage(C.byref(_img(b)), abi.vector2f(11.3, 9.7), 1.7, 1000.0, 12.0)
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-3)
    rng = np.random.default_rng(1)
    lut = rng.normal(size=(30, 40)).astype(np.float32)
    for spline in (False, True):
        for z in (0.0, 7.3, 28.9):
            a = np.zeros((50, 50), np.float32)
            b = np.zeros_like(a)
            qlib.GenerateImageFromLUT(C.byref(_img(a)), C.byref(_img(lut)), 2.0, 22.0, abi.vector3f(24.6, 25.2, z),
                                      spline, 2)
            ref.lib.GenerateImageFromLUT(C.byref(_img(b)), C.byref(_img(lut)), 2.0, 22.0,
                                         abi.vector3f(24.6, 25.2, z), spline, 2)
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-5)


def test_noise_utilities_match_reference(qlib, ref):
    """ApplyPoissonNoise / ApplyGaussianNoise draw from libc rand(): same srand seed, same image."""
    libc = C.CDLL(None)
    base = np.abs(np.sin(np.arange(64 * 48, dtype=np.float32) * 0.37)).reshape(48, 64).astype(np.float32)
    base[0, :8] = [0, 0.001, 0.01, 0.05, 0.2, 0.6, 0.9, 1.0]
    for fn, args in (("ApplyPoissonNoise", (40.0, 255.0)), ("ApplyPoissonNoise", (3000.0, 3000.0)),
                     ("ApplyGaussianNoise", (0.25,))):
        a, b = base.copy(), base.copy()
        libc.srand(1234)
        getattr(qlib, fn)(C.byref(_img(a)), *args)
        libc.srand(1234)
        getattr(ref.lib, fn)(C.byref(_img(b)), *args)
        assert np.array_equal(a, b), fn
        assert not np.array_equal(a, base)
    # the Poisson sampler's moments (both branches): mean and variance of lambda
    for lam in (2.5, 400.0):
        img = np.full((200, 250), lam / 1000.0, np.float32)
        libc.srand(7)
        qlib.ApplyPoissonNoise(C.byref(_img(img)), 1000.0, 1000.0)
        assert abs(img.mean() - lam) < 0.03 * lam + 0.05
        assert abs(img.var() - lam) < 0.08 * lam + 0.1


def _gpu_present() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU failure path")
def test_create_without_gpu_fails_cleanly(qlib):
    from qtrk_b200 import tracker

    s = synth.settings_roi60()
    h = qlib.QTrkCreateInstance(C.byref(s))
    assert not h
    assert "CUDA" in tracker.last_error() or "device" in tracker.last_error()
    with pytest.raises(RuntimeError):
        tracker.QTrkInstance(s)
    # calls on a null instance are rejected, not crashed
    qlib.QTrkFlush(None)
    assert qlib.QTrkGetResultCount(None) == 0
    # the request server needs a GPU too
    assert not qlib.QTrkB200ServerCreate(0, 1 << 30)
    assert "QTrkB200ServerCreate" in tracker.last_error()
    assert qlib.QTrkB200ServerPoll(None, 1, None, 0) == -2
    assert qlib.QTrkB200ServerSubmitFrame(None, 0, None, 0, 0, 0, None, 0, 0, None) == -1
    assert qlib.QTrkB200ServerAttach(None, None) == -1
    # so does the bead finder's convolution: NULL, no beads, an error message
    frame = np.ones((64, 64), np.float32)
    n = C.c_int(5)
    assert not qlib.QTrkFindBeads(C.byref(_img(frame)), 0, 0, 16, 1.0, 0.5, C.byref(n), None)
    assert n.value == 0 and "QTrkFindBeads" in tracker.last_error()
