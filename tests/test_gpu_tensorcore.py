"""Tensor-core (tcgen05, FP32 accumulate) Z match against the plain path, with BF16 (hi/lo split)
and TF32 operands.

The tensor-core cross terms only rank the planes: every plane whose score can still be the best
under the provable error bound is re-scored exactly with the plain path's per-plane function, and
the argmax and 7-point fit run on those exact scores, so z must equal the plain path's bit for
bit on every ROI.
"""
import numpy as np
import pytest

from golden_io import load
from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu

TC_MODES = {"bf16": abi.LT_B200_ZMatchBF16, "tf32": abi.LT_B200_ZMatchTF32}


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
    assert np.array_equal(plain["pos"][:, 2], tc["pos"][:, 2]), np.abs(plain["pos"][:, 2] - tc["pos"][:, 2]).max()
    assert np.array_equal(plain["error"], tc["error"])


def gpu_lut(wl):
    with QTrkInstance(wl.settings) as t:
        planes = wl.lut_stack.shape[0]
        t.SetRadialZLUTSize(1, planes)
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(planes):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        return t.GetRadialZLUT()


@pytest.mark.parametrize("kind", TC_MODES)
def test_tensor_core_matches_plain_roi100(kind):
    wl = synth.roi100_u16(3000, seed=31)
    lut = gpu_lut(wl)
    plain, n0 = run(wl.settings, wl.mode, lut, wl.rois)
    tc, n1 = run(wl.settings, wl.mode | TC_MODES[kind], lut, wl.rois)
    compare(plain, tc)
    assert n1 > n0   # the Z-match kernel (and the tensor-core LUT preparation) ran


@pytest.mark.parametrize("kind", TC_MODES)
def test_tensor_core_golden_roi100(kind):
    g = load("roi100_u16.npz")
    tc, _ = run(g["settings"], int(g["mode"]) | TC_MODES[kind], g["lut"], g["rois"])
    assert np.abs(tc["pos"][:, 2] - g["pos"][:, 2]).max() < 0.01
    assert np.abs(tc["pos"][:, :2] - g["pos"][:, :2]).max() < 1e-3


@pytest.mark.parametrize("kind", TC_MODES)
def test_tensor_core_per_bead_groups_and_invalid_bead(kind):
    wl = synth.roi60_f32(900, seed=32)
    lut1 = gpu_lut(wl)
    lut = np.ascontiguousarray(np.concatenate([lut1, lut1[:, ::-1], 0.5 * lut1 + 0.1, lut1[:, ::2].repeat(2, 1)[:, :50]]))
    idx = np.random.default_rng(3).integers(-1, 5, 900)   # -1 and 4 are outside the 4-bead LUT
    plain, _ = run(wl.settings, wl.mode, lut, wl.rois, zlut_index=idx)
    tc, _ = run(wl.settings, wl.mode | TC_MODES[kind], lut, wl.rois, zlut_index=idx)
    compare(plain, tc)
    assert (tc["pos"][(idx < 0) | (idx > 3), 2] == 0).all()


@pytest.mark.parametrize("kind", TC_MODES)
def test_tensor_core_many_planes_and_weights(kind):
    # 300 planes -> two N chunks of the MMA; 40 bins -> K padded to 48
    wl = synth.roi60_f32(600, seed=33)
    lut50 = gpu_lut(wl)
    zz = np.linspace(0, 49, 300)
    i0 = np.minimum(zz.astype(int), 48)
    f = (zz - i0)[:, None]
    lut = ((1 - f) * lut50[0, i0] + f * lut50[0, i0 + 1])[None].astype(np.float32)
    w = np.linspace(0.2, 1.0, lut.shape[2]).astype(np.float32)
    plain, _ = run(wl.settings, wl.mode, lut, wl.rois, weights=w)
    tc, _ = run(wl.settings, wl.mode | TC_MODES[kind], lut, wl.rois, weights=w)
    compare(plain, tc)


@pytest.mark.parametrize("kind", TC_MODES)
def test_tensor_core_device_entry(kind):
    import torch

    wl = synth.roi100_u16(1000, seed=34)
    lut = gpu_lut(wl)
    out = {}
    for name, mode in (("plain", wl.mode), ("tc", wl.mode | TC_MODES[kind])):
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
