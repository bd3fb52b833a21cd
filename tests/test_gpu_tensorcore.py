"""Tensor-core (tcgen05, BF16 operands, FP32 accumulate) Z match against the plain FP32 path.

The BF16 cross terms only rank the planes; the best kTopK are re-scored exactly and the
7-point fit runs on exact scores, so z must equal the plain path's (|dz| < 1e-6 plane) on
every ROI whose exact argmax is among the BF16 top candidates. The test counts argmax flips
(|dz| > 0.01 plane) and requires none on these inputs.
"""
import numpy as np
import pytest

from golden_io import load
from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu

TC = abi.LT_B200_ZMatchBF16


def run(settings, mode, lut, rois, zlut_index=None, weights=None):
    with QTrkInstance(settings) as t:
        t.SetRadialZLUT(lut)
        if weights is not None:
            t.SetRadialWeights(weights)
        t.SetLocalizationMode(mode)
        r = t.Localize(rois, zlut_index=zlut_index)
        warn = t.GetWarnings()
        launches = t.KernelLaunchCount()
    assert "timed out" not in warn, warn
    return r, launches


def compare(plain, tc):
    assert np.array_equal(plain["pos"][:, :2], tc["pos"][:, :2])   # same localization kernel
    dz = np.abs(plain["pos"][:, 2] - tc["pos"][:, 2])
    flips = int((dz > 0.01).sum())
    assert flips == 0, f"{flips} argmax flips"
    assert dz.max() < 1e-4, dz.max()


def gpu_lut(wl):
    with QTrkInstance(wl.settings) as t:
        planes = wl.lut_stack.shape[0]
        t.SetRadialZLUTSize(1, planes)
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(planes):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        return t.GetRadialZLUT()


def test_tensor_core_matches_plain_roi100():
    wl = synth.roi100_u16(3000, seed=31)
    lut = gpu_lut(wl)
    plain, n0 = run(wl.settings, wl.mode, lut, wl.rois)
    tc, n1 = run(wl.settings, wl.mode | TC, lut, wl.rois)
    compare(plain, tc)
    assert n1 > n0   # the Z-match kernel (and the BF16 LUT preparation) ran


def test_tensor_core_golden_roi100():
    g = load("roi100_u16.npz")
    tc, _ = run(g["settings"], int(g["mode"]) | TC, g["lut"], g["rois"])
    assert np.abs(tc["pos"][:, 2] - g["pos"][:, 2]).max() < 0.01
    assert np.abs(tc["pos"][:, :2] - g["pos"][:, :2]).max() < 1e-3


def test_tensor_core_per_bead_groups_and_invalid_bead():
    wl = synth.roi60_f32(900, seed=32)
    lut1 = gpu_lut(wl)
    lut = np.ascontiguousarray(np.concatenate([lut1, lut1[:, ::-1], 0.5 * lut1 + 0.1, lut1[:, ::2].repeat(2, 1)[:, :50]]))
    idx = np.random.default_rng(3).integers(-1, 5, 900)   # -1 and 4 are outside the 4-bead LUT
    plain, _ = run(wl.settings, wl.mode, lut, wl.rois, zlut_index=idx)
    tc, _ = run(wl.settings, wl.mode | TC, lut, wl.rois, zlut_index=idx)
    compare(plain, tc)
    assert (tc["pos"][(idx < 0) | (idx > 3), 2] == 0).all()


def test_tensor_core_many_planes_and_weights():
    # 300 planes -> two N chunks of the MMA; 40 bins -> K padded to 48
    wl = synth.roi60_f32(600, seed=33)
    lut50 = gpu_lut(wl)
    zz = np.linspace(0, 49, 300)
    i0 = np.minimum(zz.astype(int), 48)
    f = (zz - i0)[:, None]
    lut = ((1 - f) * lut50[0, i0] + f * lut50[0, i0 + 1])[None].astype(np.float32)
    w = np.linspace(0.2, 1.0, lut.shape[2]).astype(np.float32)
    plain, _ = run(wl.settings, wl.mode, lut, wl.rois, weights=w)
    tc, _ = run(wl.settings, wl.mode | TC, lut, wl.rois, weights=w)
    compare(plain, tc)


def test_tensor_core_device_entry():
    import torch

    wl = synth.roi100_u16(1000, seed=34)
    lut = gpu_lut(wl)
    out = {}
    for name, mode in (("plain", wl.mode), ("tc", wl.mode | TC)):
        with QTrkInstance(wl.settings) as t:
            t.SetRadialZLUT(lut)
            t.SetLocalizationMode(mode)
            d = torch.from_numpy(wl.rois.view(np.int16).copy()).cuda()
            res = torch.zeros(1000 * 52, dtype=torch.uint8, device="cuda")
            t.LocalizeDevice(d.data_ptr(), 200, 20000, abi.QTrkU16, 1000, res.data_ptr(),
                             stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            out[name] = np.frombuffer(res.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)
            assert "timed out" not in t.GetWarnings()
    compare(out["plain"], out["tc"])
