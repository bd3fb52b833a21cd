"""Pixel calibration (offset and gain images per bead) against the reference CPU tracker.

QueuedCPUTracker::ApplyOffsetGain (QueuedCPUTracker.cpp:258-271, CPUTracker::ApplyOffsetGain at
cpu_tracker.cpp:98-112) rewrites each ROI pixel before the COM: v + o, v * g or (v + o) * g,
with the images of bead job.zlutIndex, after LT_ClearFirstFourPixels (QueuedCPUTracker.cpp:279-284).
The reference's C ABI declares QTrkSetPixelCalibrationImages without a body, so the reference side
goes through QueuedTracker::SetPixelCalibrationImages directly (oracle/ref_stage_exports.cpp).
Tolerances as in test_gpu_parity.py: COM 1e-4 px, QI 1e-3 px, Z 0.01 plane, flags identical.
"""
import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance
from test_gpu_parity import check_results

pytestmark = pytest.mark.gpu

BEADS = 3


def _calibration(shape, seed):
    """Per-bead offset (about +-2 counts, smooth plus pixel noise) and gain (0.85..1.15)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h, w = shape
    yy, xx = np.mgrid[0:h, 0:w]
    off = np.empty((BEADS, h, w), np.float32)
    gain = np.empty((BEADS, h, w), np.float32)
    for b in range(BEADS):
        off[b] = 1.5 * np.sin(xx / (7.0 + b)) * np.cos(yy / 11.0) + rng.normal(0, 0.5, (h, w))
        gain[b] = 1.0 + 0.1 * np.cos((xx + 2 * yy) / (9.0 + b)) + rng.uniform(-0.05, 0.05, (h, w))
    return off, gain


def _ours(settings, mode, lut, rois, idx, off, gain, factors=None):
    with QTrkInstance(settings) as t:
        t.SetRadialZLUT(lut)
        t.SetLocalizationMode(mode)
        t.SetPixelCalibrationImages(off, gain)
        if factors is not None:
            t.SetPixelCalibrationFactors(*factors)
        return t.Localize(rois, zlut_index=idx)


@pytest.fixture(scope="module")
def roi60(ref):
    wl = synth.roi60_f32(90, seed=41)
    lut1 = ref.build_lut(wl.settings, wl.lut_stack, abi.BUILDLUT_NORMALIZE, known_pos=wl.lut_known_pos)
    lut = np.ascontiguousarray(np.concatenate([lut1] * BEADS))
    idx = np.arange(len(wl.rois)) % BEADS
    return wl, lut, idx


@pytest.mark.parametrize("which", ["offset", "gain", "both"])
def test_calibration_images_match_reference(ref, roi60, which):
    wl, lut, idx = roi60
    off, gain = _calibration(wl.rois.shape[1:], 42)
    off = off if which in ("offset", "both") else None
    gain = gain if which in ("gain", "both") else None
    r_ref = ref.track(wl.settings, wl.mode, wl.rois, lut, zlut_index=idx, calib=(off, gain))
    r = _ours(wl.settings, wl.mode, lut, wl.rois, idx, off, gain)
    check_results(r, r_ref["pos"], r_ref["firstGuess"], r_ref["error"], r_ref["imageMean"],
                      lut_planes=lut.shape[1])
    # the calibration must have changed the answer, or the comparison proves nothing
    plain = ref.track(wl.settings, wl.mode, wl.rois, lut, zlut_index=idx)
    assert np.abs(plain["imageMean"] - r_ref["imageMean"]).max() > 1e-3


def test_calibration_u16_and_clear_first_four(ref):
    """u16 ROIs (converted before calibration) and LT_ClearFirstFourPixels (cleared, then
    calibrated: the first four pixels become (0 + o) * g)."""
    wl = synth.roi100_u16(60, seed=43)
    lut1 = ref.build_lut(wl.settings, wl.lut_stack, abi.BUILDLUT_NORMALIZE, known_pos=wl.lut_known_pos)
    lut = np.ascontiguousarray(np.concatenate([lut1] * BEADS))
    idx = (np.arange(len(wl.rois)) * 2) % BEADS
    off, gain = _calibration(wl.rois.shape[1:], 44)
    off *= 40.0  # the u16 workload's background is 200 counts
    for mode in (wl.mode, wl.mode | abi.LT_ClearFirstFourPixels):
        r_ref = ref.track(wl.settings, mode, wl.rois, lut, zlut_index=idx, calib=(off, gain))
        r = _ours(wl.settings, mode, lut, wl.rois, idx, off, gain)
        check_results(r, r_ref["pos"], r_ref["firstGuess"], r_ref["error"], r_ref["imageMean"],
                      lut_planes=lut.shape[1])


def test_calibration_factors_scale_the_images(ref, roi60):
    """The reference's tracker fixes both factors at 1 (QueuedCPUTracker.cpp:266). Factors of 2 and
    0.5 on images o, g must equal factors of 1 on images 2o, g/2: powers of two scale exactly, so
    the reference with the pre-scaled images is the oracle."""
    wl, lut, idx = roi60
    off, gain = _calibration(wl.rois.shape[1:], 45)
    r_ref = ref.track(wl.settings, wl.mode, wl.rois, lut, zlut_index=idx, calib=(off * 2.0, gain * 0.5))
    r = _ours(wl.settings, wl.mode, lut, wl.rois, idx, off, gain, factors=(2.0, 0.5))
    check_results(r, r_ref["pos"], r_ref["firstGuess"], r_ref["error"], r_ref["imageMean"],
                      lut_planes=lut.shape[1])


def test_removing_calibration_restores_plain_results(roi60):
    """A null image removes it (QueuedCPUTracker.cpp:174-186): results equal an uncalibrated run."""
    wl, lut, idx = roi60
    off, gain = _calibration(wl.rois.shape[1:], 46)
    with QTrkInstance(wl.settings) as t:
        t.SetRadialZLUT(lut)
        t.SetLocalizationMode(wl.mode)
        plain = t.Localize(wl.rois, zlut_index=idx)
        t.SetPixelCalibrationImages(off, gain)
        cal = t.Localize(wl.rois, zlut_index=idx)
        t.SetPixelCalibrationImages(None, None)
        again = t.Localize(wl.rois, zlut_index=idx)
    assert not np.array_equal(cal["pos"], plain["pos"])
    for f in ("pos", "firstGuess", "error", "imageMean"):
        assert np.array_equal(again[f], plain[f]), f


def test_calibration_through_schedule_frame_equals_per_roi(roi60):
    """Frame path (ROIs cropped from frame rows at a pitch on the device) with calibration images
    gives the same results as queuing the same ROIs one by one: ScheduleFrame gives ROI i the
    images of bead i (zlutIndex = i, QueuedTracker.cpp:105)."""
    wl, lut1, _ = roi60
    n = 12
    rois = wl.rois[:n]
    off, gain = _calibration(rois.shape[1:], 47)
    off = np.ascontiguousarray(np.concatenate([off] * 4))[:n]
    gain = np.ascontiguousarray(np.concatenate([gain] * 4))[:n]
    lut = np.ascontiguousarray(np.concatenate([lut1[:1]] * n))
    gap, h, w = 3, rois.shape[1], rois.shape[2]
    frame = np.zeros((3 * (h + gap) + gap, 4 * (w + gap) + gap), np.float32)
    pos = []
    for i in range(n):
        y, x = gap + (i // 4) * (h + gap), gap + (i % 4) * (w + gap)
        frame[y:y + h, x:x + w] = rois[i]
        pos.append((x, y))
    with QTrkInstance(wl.settings) as t:
        t.SetRadialZLUT(lut)
        t.SetLocalizationMode(wl.mode)
        t.SetPixelCalibrationImages(off, gain)
        assert t.ScheduleFrame(frame, np.array(pos, np.int32)) == n
        fr = t.WaitForResults(n)
        fr = fr[np.argsort(fr["zlutIndex"])]
        single = t.Localize(rois, zlut_index=np.arange(n))
    for f in ("pos", "firstGuess", "error", "imageMean"):
        assert np.array_equal(fr[f], single[f]), f
