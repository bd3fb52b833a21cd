"""Z-LUT refinement from a calibration stack (QTrkB200RefineZLUT) on a stack whose stage positions
are off by N(0, 0.3) planes: the objective decreases, the recovered plane offsets follow the true
ones, and held-out ROIs are located more consistently with the refined LUT."""
import ctypes as C

import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu


def build_lut(t, stack):
    planes, nbeads = stack.shape[:2]
    t.SetRadialZLUTSize(nbeads, planes)
    t.BeginLUT(abi.BUILDLUT_NORMALIZE)
    for k in range(planes):
        t.BuildLUT(stack[k], k)
    t.FinalizeLUT()


def z_spread(t, cal, mode):
    """Median absolute deviation of the held-out z errors (and the share within 3 planes)."""
    t.SetLocalizationMode(mode)
    r = t.Localize(cal["test"], zlut_index=cal["test_bead"].astype(np.int32))
    e = r["pos"][:, 2] - cal["test_z"]
    ok = np.abs(e) < 3
    return np.median(np.abs(e[ok] - np.median(e[ok]))), ok.mean()


def refine(t, stack, iters, smoothness):
    import torch

    planes, nbeads, h, w = stack.shape
    d_stack = torch.from_numpy(stack.reshape(-1, h, w).view(np.int16)).cuda()
    plane_z = np.zeros(planes, np.float32)
    hist = np.zeros(iters + 1, np.float32)
    t.lib.QTrkB200RefineZLUT(t.handle, d_stack.data_ptr(), w * 2, h * w * 2, abi.QTrkU16, nbeads, planes, None, iters,
                             C.c_float(smoothness), plane_z.ctypes.data_as(C.c_void_p), hist.ctypes.data_as(C.c_void_p))
    return plane_z, hist


def test_refine_lut_recovers_stage_offsets():
    cal = synth.calibration_stack(nbeads=16, planes=60, jitter=0.3)
    s, stack = cal["settings"], cal["stack"]
    planes = stack.shape[0]
    mode = synth.MODE_QI_Z
    iters = 20
    with QTrkInstance(s) as t:
        t.SetLocalizationMode(mode)
        build_lut(t, stack)
        spread0, ok0 = z_spread(t, cal, mode)
        l0 = t.KernelLaunchCount()
        plane_z, hist = refine(t, stack, iters, SMOOTHNESS)
        assert "RefineZLUT" not in t.GetWarnings(), t.GetWarnings()
        assert t.KernelLaunchCount() - l0 == iters + 2  # positions + one adjoint launch per evaluation
        spread1, ok1 = z_spread(t, cal, mode)
    print("objective", hist[0], "->", hist[-1], "; held-out z spread", spread0, "->", spread1)
    assert hist[-1] < 0.7 * hist[0]
    k = np.arange(planes)
    true = cal["offsets"] - np.polyval(np.polyfit(k, cal["offsets"], 1), k)
    est = plane_z - k
    assert abs(est.mean()) < 1e-4
    assert np.corrcoef(est, true)[0, 1] > 0.8
    assert spread1 < SPREAD_GAIN * spread0 and ok1 >= ok0 - 0.01


# smoothness 3 over 20 iterations measured on a B200: objective 54.2 -> 1.67, held-out z spread
# 0.189 -> 0.176 planes, offset correlation 0.87 (0.3: 0.185, 0.75; 10: 0.177, 0.88)
SMOOTHNESS = 3.0
SPREAD_GAIN = 0.97
