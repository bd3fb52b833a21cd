"""GPU tests of the Z-LUT bias correction and the Gaussian MLE forms against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from golden_io import load
from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu


def test_zlut_bias_table(port):
    """QueuedTracker::ZLUTBiasCorrection (QueuedTracker.cpp:115-140) applied on the device."""
    g = load("roi60_f32.npz")
    rois = g["rois"].astype(np.float32)
    planes = g["lut"].shape[1]
    rng = np.random.default_rng(5)
    table = np.ascontiguousarray(rng.uniform(-0.8, 0.8, (1, 37)).astype(np.float32))
    for extra in (0, abi.LT_B200_ZMatchBF16):
        with QTrkInstance(g["settings"]) as t:
            t.SetRadialZLUT(g["lut"])
            t.SetLocalizationMode(int(g["mode"]) | extra)
            plain = t.Localize(rois)
            t.lib.QTrkB200SetZLUTBiasTable(t.handle, table.ctypes.data_as(C.c_void_p), 37, 1)
            corr = t.Localize(rois)
            t.lib.QTrkB200SetZLUTBiasTable(t.handle, None, 0, 0)
            back = t.Localize(rois)
        expect = np.array([port.zlut_bias_correct(z, planes, table, 0) for z in plain["pos"][:, 2]])
        assert np.abs(corr["pos"][:, 2] - expect).max() < 1e-4
        assert np.array_equal(back["pos"][:, 2], plain["pos"][:, 2])
        assert np.array_equal(corr["pos"][:, :2], plain["pos"][:, :2])


def test_gaussian_4p_cta_kernel_matches_reference(ref):
    """ROIs above 32x32 take the CTA kernel's MLE: same results as the reference's
    CPUTracker::Compute2DGaussianMLE (cpu_tracker.cpp:514-589) on every ROI where that
    diagonal-Newton iteration has converged (last step < 1e-5 px; where it has not, the
    reference's float iteration is ill-conditioned and even an FP64 restatement departs from it)."""
    rng = np.random.Generator(np.random.PCG64(53))
    n, w, it = 128, 36, 12
    cx = 18 + rng.uniform(-2, 2, n)
    cy = 18 + rng.uniform(-2, 2, n)
    ph = np.exp(rng.uniform(np.log(20000), np.log(60000), n))
    imgs = rng.poisson(synth.gaussian_spots(n, w, cx, cy, 3.0, ph, 10.0)).astype(np.float32)
    s = abi.settings(width=w, height=w, gauss2D_sigma=3.0, gauss2D_iterations=it, qi_minradius=1, zlut_minradius=1)
    with QTrkInstance(s) as t:
        t.SetLocalizationMode(abi.LT_Gaussian2D)
        cta = t.Localize(imgs)
    r = np.array([ref.gauss2d(im, ref.com(im)[:2], it, 3.0) for im in imgs])
    r1 = np.array([ref.gauss2d(im, ref.com(im)[:2], it - 1, 3.0) for im in imgs])
    conv = np.abs(r[:, :2] - r1[:, :2]).max(1) < 1e-5
    assert conv.mean() > 0.75
    assert np.abs(cta["pos"][conv, :2] - r[conv, :2]).max() < 1e-3
    assert np.abs(cta["firstGuess"] - np.array([ref.com(im)[:2] for im in imgs])).max() < 1e-4


def test_gaussian_5p_matches_fp64_oracle_and_crlb(port):
    """5-parameter (x, y, I0, bg, sigma) full-Newton MLE vs the FP64 oracle and the Cramer-Rao bound."""
    wl = synth.gauss16_f32(600, seed=52)
    s = wl.settings
    s.gauss2D_iterations = 10
    with QTrkInstance(s) as t:
        t.SetLocalizationMode(abi.LT_Gaussian2D | abi.LT_B200_Gaussian5P)
        r = t.Localize(wl.rois)
    dx, crlb = [], []
    for i in range(600):
        img = wl.rois[i].astype(np.float64)
        com = port.com(img)
        init = np.array([r["firstGuess"][i, 0], r["firstGuess"][i, 1], com[2] * 0.5 * 256, com[2] * 0.5, 1.5])
        o, fisher = port.gauss5(img, init, 10, with_fisher=True)
        dx.append(max(abs(r["pos"][i, 0] - o[0]), abs(r["pos"][i, 1] - o[1])))
        assert abs(r["pos"][i, 2] - o[4]) < 1e-3          # sigma is returned in pos.z
        crlb.append(np.sqrt(np.diag(np.linalg.inv(fisher)))[:2])
    assert max(dx) < 1e-3, max(dx)
    # errors about the truth, each divided by that ROI's Cramer-Rao bound, have unit scatter
    # for an efficient estimator (600 ROIs: the sample std is within a few percent of 1)
    err = np.stack([r["pos"][:, 0] - wl.true_xyz[:, 0], r["pos"][:, 1] - wl.true_xyz[:, 1]], 1)
    ratio = (err / np.array(crlb)).std(0)
    assert (ratio > 0.8).all() and (ratio < 1.25).all(), ratio


@pytest.mark.parametrize("roi,seed,noise", [(32, 6, 2.0), (24, 7, 4.0), (40, 8, 1.0)])
def test_find_beads_matches_reference(ref, port, roi, seed, noise):
    """QTrkFindBeads (GPU convolution + host search) gives the reference's bead list."""
    import ctypes as C

    from qtrk_b200.tracker import load_library

    lib = load_library()
    frame, centres = synth.bead_frame(300, 220, 10, roi, seed=seed, noise=noise)
    corner = (int(centres[0][0] - roi / 2), int(centres[0][1] - roi / 2))
    img = abi.ImageData(frame.ctypes.data_as(C.POINTER(C.c_float)), frame.shape[1], frame.shape[0])
    for rel, acc in ((1.0, 0.3), (1.0, 0.6), (0.8, 0.45)):
        outs = []
        for L in (lib, ref.lib):
            n = C.c_int()
            smp = np.zeros((roi, roi), np.float32)
            smp_img = abi.ImageData(smp.ctypes.data_as(C.POINTER(C.c_float)), roi, roi)
            p = L.QTrkFindBeads(C.byref(img), corner[0], corner[1], roi, rel, acc, C.byref(n), C.byref(smp_img))
            assert p
            outs.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int)), shape=(2 * n.value,)).reshape(-1, 2).copy())
            L.QTrkFreeROIPositions(p)
            assert np.array_equal(smp, frame[corner[1]:corner[1] + roi, corner[0]:corner[0] + roi])
        assert np.array_equal(outs[0], outs[1]), (rel, acc)
        assert np.array_equal(outs[0], port.find_beads(frame, corner, roi, rel, acc))


def test_find_beads_large_frame():
    """A 2048 x 2048 frame with a 100 px sample: every planted bead found, within a ROI's reach."""
    import ctypes as C
    import time

    from qtrk_b200.tracker import load_library

    lib = load_library()
    roi = 100
    frame, centres = synth.bead_frame(2048, 2048, 120, roi, seed=9, noise=2.0)
    corner = (int(centres[0][0] - roi / 2), int(centres[0][1] - roi / 2))
    img = abi.ImageData(frame.ctypes.data_as(C.POINTER(C.c_float)), 2048, 2048)
    n = C.c_int()
    t0 = time.perf_counter()
    p = lib.QTrkFindBeads(C.byref(img), corner[0], corner[1], roi, 1.0, 0.5, C.byref(n), None)
    dt = time.perf_counter() - t0
    assert p
    pos = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int)), shape=(2 * n.value,)).reshape(-1, 2).copy()
    lib.QTrkFreeROIPositions(p)
    found = pos + roi / 2
    inside = (centres[:, 0] > roi) & (centres[:, 1] > roi) & (centres[:, 0] < 2048 - roi) & (centres[:, 1] < 2048 - roi)
    d = np.hypot(centres[inside, None, 0] - found[None, :, 0], centres[inside, None, 1] - found[None, :, 1]).min(1)
    assert (d < 3).all(), d.max()
    print(f"FindBeads 2048x2048, roi {roi}: {n.value} beads in {dt * 1e3:.1f} ms")


@pytest.mark.parametrize("spline,smp", [(1, 4), (0, 2)])
def test_compute_zlut_bias_table_matches_reference(ref, spline, smp):
    """QTrkB200ComputeZLUTBiasTable (images rendered and localized on the GPU) against the
    reference's QueuedTracker::ComputeZBiasCorrection; the table is installed as the bias table."""
    g = load("roi60_f32.npz")
    s, lut = g["settings"], np.ascontiguousarray(g["lut"], np.float32)
    two = np.ascontiguousarray(np.concatenate([lut, lut[:, ::-1]]))  # 2 beads, the second reversed in z
    bias_planes = 100
    L = ref.lib
    L.ref_compute_zbias.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int]
    L.ref_compute_zbias.restype = None
    trk = L.QTrkCreateInstance(C.byref(s))
    try:
        L.QTrkSetRadialZLUT(trk, two.ctypes.data_as(C.c_void_p), 2, two.shape[1])
        L.QTrkSetLocalizationMode(trk, int(g["mode"]))
        want = np.zeros(2 * bias_planes, np.float32)
        L.ref_compute_zbias(trk, bias_planes, want.ctypes.data, smp, spline)
    finally:
        L.QTrkFreeInstance(trk)
    rois = g["rois"].astype(np.float32)[:64]
    with QTrkInstance(s) as t:
        t.SetRadialZLUT(two)
        t.SetLocalizationMode(int(g["mode"]))
        got = np.zeros(2 * bias_planes, np.float32)
        t.lib.QTrkB200ComputeZLUTBiasTable(t.handle, bias_planes, got.ctypes.data_as(C.c_void_p), smp, spline)
        assert "QTrkB200ComputeZLUTBiasTable" not in t.GetWarnings()
        with_table = t.Localize(rois)
        t.lib.QTrkB200SetZLUTBiasTable(t.handle, got.ctypes.data_as(C.c_void_p), bias_planes, 2)
        again = t.Localize(rois)
        t.lib.QTrkB200SetZLUTBiasTable(t.handle, None, 0, 0)
        plain = t.Localize(rois)
    assert np.abs(got - want).max() < 0.01, np.abs(got - want).max()
    assert np.array_equal(with_table["pos"], again["pos"])
    assert not np.array_equal(with_table["pos"][:, 2], plain["pos"][:, 2])


def test_buildlut_pinned_and_pageable_agree():
    """BuildLUT from a pinned stack (DMA on the copy stream, overlapping the previous plane's
    kernel) gives the LUT that the same stack from pageable memory gives; the buffer may be reused
    as soon as the call returns."""
    import torch

    s, stack, centres = synth.calib_stack_80x80(nbeads=8, planes=30, seed=15)
    pinned = torch.empty(stack.shape, dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    luts = []
    for src in ("pageable", "pinned"):
        with QTrkInstance(s) as t:
            t.SetRadialZLUTSize(8, 30)
            t.BeginLUT(abi.BUILDLUT_NORMALIZE)
            for k in range(30):
                if src == "pinned":
                    pinned[0] = stack[k]  # one pinned plane buffer, overwritten after every call
                    t.BuildLUT(pinned[0], k, known_pos=centres if k % 2 else None)
                else:
                    t.BuildLUT(stack[k].copy(), k, known_pos=centres if k % 2 else None)
            t.FinalizeLUT()
            luts.append(t.GetRadialZLUT())
    assert np.array_equal(luts[0], luts[1])


def test_buildlut_async_equals_buildlut():
    """QTrkB200BuildLUTAsync over a whole pinned stack (the copies of successive planes queued
    without waiting; the stack untouched until FinalizeLUT returns) gives the LUT that QTrkBuildLUT
    gives, bit for bit; a pageable stack through the async entry as well."""
    import torch

    s, stack, centres = synth.calib_stack_80x80(nbeads=8, planes=30, seed=16)
    pinned = torch.empty(stack.shape, dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    pinned[:] = stack
    luts = []
    for form in ("sync", "async_pinned", "async_pageable"):
        with QTrkInstance(s) as t:
            t.SetRadialZLUTSize(8, 30)
            t.BeginLUT(abi.BUILDLUT_NORMALIZE)
            for k in range(30):
                kp = centres if k % 3 else None
                if form == "sync":
                    t.BuildLUT(stack[k], k, known_pos=kp)
                elif form == "async_pinned":
                    t.BuildLUTAsync(pinned[k], k, known_pos=kp)
                else:
                    t.BuildLUTAsync(stack[k], k, known_pos=kp)
            t.FinalizeLUT()
            luts.append(t.GetRadialZLUT())
    assert np.array_equal(luts[0], luts[1])
    assert np.array_equal(luts[0], luts[2])
