"""Pin the FP64 restatement (oracle/qtrk_oracle.c) to the reference CPU tracker.

The reference itself runs here from oracle/_ref/libqtrk_ref.so (compiled from its own
cputrack/ sources); where that library is absent, the committed fixtures in tests/golden/
(outputs of the same reference build) pin the port instead.
"""
import ctypes as C

import numpy as np
import pytest

from golden_io import load
from qtrk_b200 import abi, synth

# Tolerances of the reference (float, KISS FFT) against the FP64 port: the reference's own
# single-precision arithmetic is the error being bounded here.
TOL_COM = 1e-4    # px
TOL_QI = 1e-3     # px
TOL_Z = 0.01      # planes


def _settings_grid():
    yield synth.settings_roi60()
    yield synth.settings_roi100()
    yield synth.calib_stack_80x80(1, 1)[0]
    for w in (16, 31, 40, 64, 100, 128, 150):
        for cov in (0.5, 0.7, 1.0, 3.0):
            yield abi.settings(width=w, height=w, qi_radial_coverage=cov * 1.3, qi_angular_coverage=cov,
                               zlut_radial_coverage=cov, zlut_angular_coverage=cov * 0.9, qi_minradius=1 + cov,
                               zlut_minradius=cov, qi_roi_coverage=0.9, zlut_roi_coverage=0.8)


def test_computed_config_matches_reference(ref, port):
    """QTrkComputedConfig::Update (QueuedTracker.cpp:6-21): bit-exact step counts and radii."""
    n = 0
    for s in _settings_grid():
        a, b = ref.computed_config(s), port.computed_config(s)
        for f in ("zlut_radialsteps", "zlut_angularsteps", "qi_radialsteps", "qi_angstepspq"):
            assert getattr(a, f) == getattr(b, f), (f, s.width)
        for f in ("zlut_maxradius", "qi_maxradius"):
            assert np.float32(getattr(a, f)) == np.float32(getattr(b, f))
        n += 1
    assert n > 20


def test_nearest_pow2(port):
    # utils.cpp:644-652: ties go down (fabsf(r-v) < fabsf(r/2-v) is strict)
    expect = {1: 1, 2: 2, 3: 2, 5: 4, 6: 4, 7: 8, 12: 8, 13: 16, 40: 32, 48: 32, 49: 64, 61: 64, 100: 128}
    for v, e in expect.items():
        assert port.lib.oracle_nearest_pow2(v) == e, v


def test_radial_bin_window(ref, port):
    for n in (8, 32, 40, 64):
        np.testing.assert_allclose(port.radial_bin_window(n), ref.radial_bin_window(n), atol=1e-6)


def test_com_matches_reference(ref, port):
    wl = synth.roi60_f32(16, seed=7)
    for bg in (0.0, 0.5, 1.5):
        for img in wl.rois[:8]:
            a = ref.com(img, bg)
            b = port.com(img, bg)
            assert abs(a[0] - b[0]) < TOL_COM and abs(a[1] - b[1]) < TOL_COM
            assert abs(a[2] - b[2]) < 1e-4 * max(1.0, abs(b[2]))


def test_qi_matches_reference(ref, port):
    wl = synth.roi60_f32(12, seed=8)
    cc = port.computed_config(wl.settings)
    w = ref.radial_bin_window(cc.qi_radialsteps)
    for img in wl.rois:
        com = ref.com(img)
        for weights in (None, w):
            a = ref.qi(img, com[:2], 4, cc.qi_radialsteps, cc.qi_angstepspq, 1.0, 3.0, cc.qi_maxradius, weights)
            b = port.qi(img, float(com[2]), com[:2].astype(float), 4, cc.qi_radialsteps, cc.qi_angstepspq, 1.0, 3.0,
                        cc.qi_maxradius, weights)
            assert np.abs(a[:2] - b[:2]).max() < TOL_QI
            assert a[2] == b[2]


def test_qi_angstep_factor_quirk(ref, port):
    """qi_angstep_factor != 1 exercises the truncated stride of cpu_tracker.cpp:655-657."""
    wl = synth.roi60_f32(4, seed=9)
    cc = port.computed_config(wl.settings)
    for f in (1.5, 2.0, 0.8):
        for img in wl.rois:
            com = ref.com(img)
            a = ref.qi(img, com[:2], 3, cc.qi_radialsteps, cc.qi_angstepspq, f, 3.0, cc.qi_maxradius)
            b = port.qi(img, float(com[2]), com[:2].astype(float), 3, cc.qi_radialsteps, cc.qi_angstepspq, f, 3.0,
                        cc.qi_maxradius)
            assert np.abs(a[:2] - b[:2]).max() < TOL_QI


@pytest.mark.parametrize("normalize", [False, True])
def test_radial_profile_matches_reference(ref, port, normalize):
    wl = synth.roi100_u16(4, seed=10)
    cc = port.computed_config(wl.settings)
    img = wl.rois[0].astype(np.float32)
    com = ref.com(img)
    # centres inside, near an edge (sparse bins fall back to the mean) and outside
    for c in ([50.3, 49.7], [8.2, 50.0], [97.5, 3.1], [-5.0, 20.0]):
        a = ref.radial_profile(img, c, cc.zlut_radialsteps, cc.zlut_angularsteps, 3.0, cc.zlut_maxradius, normalize)
        b = port.radial_profile(img, float(com[2]), c, cc.zlut_radialsteps, cc.zlut_angularsteps, 3.0,
                                cc.zlut_maxradius, normalize)
        if not normalize:
            np.testing.assert_allclose(a, b, rtol=2e-6, atol=2e-3)
        elif np.all(np.isfinite(a)):
            np.testing.assert_allclose(a, b, atol=2e-5)


def test_lut_compare_matches_reference(ref, port):
    rng = np.random.default_rng(11)
    lut = rng.normal(size=(80, 48)).astype(np.float32)
    for _ in range(10):
        k = rng.integers(0, 80)
        prof = (lut[k] + 0.3 * rng.normal(size=48)).astype(np.float32)
        w = rng.uniform(0.2, 1.0, 48).astype(np.float32)
        for weights in (None, w):
            za, sa = ref.lut_compare(prof, lut, weights)
            zb, sb = port.lut_compare(prof.astype(float), lut, None if weights is None else weights.astype(float))
            np.testing.assert_allclose(sa, sb, rtol=1e-6, atol=1e-4)
            assert abs(za - zb) < 1e-4


def test_gauss2d_matches_reference(ref, port):
    wl = synth.gauss16_f32(16, seed=12)
    for img in wl.rois:
        com = ref.com(img)
        a = ref.gauss2d(img, com[:2], 8, 1.5)
        b = port.gauss2d(img, float(com[2]), com[:2].astype(float), 8, 1.5)
        assert np.abs(a[:2] - b[:2]).max() < 1e-3


def test_pipeline_matches_reference(ref, port):
    """QueuedCPUTracker::ProcessJob end to end (QI + Z, normalised profiles)."""
    wl = synth.roi60_f32(60, seed=13)
    cc = port.computed_config(wl.settings)
    lut = ref.build_lut(wl.settings, wl.lut_stack, abi.BUILDLUT_NORMALIZE, known_pos=wl.lut_known_pos)
    r = ref.track(wl.settings, wl.mode, wl.rois, lut)
    p = port.localize(cc, wl.mode, wl.rois, lut)
    # ROIs whose QI lost the bead (walked > 5 px from the COM) are ill-conditioned in the
    # reference's float arithmetic; they are held to 0.05 px (see tests/test_gpu_parity.py).
    ok = np.hypot(r["pos"][:, 0] - r["firstGuess"][:, 0], r["pos"][:, 1] - r["firstGuess"][:, 1]) <= 5.0
    assert ok.mean() > 0.9
    assert np.abs(r["pos"][ok, 0] - p[ok, 0]).max() < TOL_QI
    assert np.abs(r["pos"][ok, 1] - p[ok, 1]).max() < TOL_QI
    assert np.abs(r["pos"][ok, 2] - p[ok, 2]).max() < TOL_Z
    assert np.abs(r["pos"][~ok, :2] - p[~ok, :2]).max(initial=0) < 0.05
    assert np.abs(r["firstGuess"][:, 0] - p[:, 3]).max() < TOL_COM
    assert (r["error"] == p[:, 5]).all()


def test_build_lut_matches_reference(ref, port):
    s, stack, centres = synth.calib_stack_80x80(nbeads=2, planes=6, seed=14)
    cc = port.computed_config(s)
    for known in (None, centres):
        a = ref.build_lut(s, stack, abi.BUILDLUT_NORMALIZE, known_pos=known)
        b = port.build_lut(cc, stack, abi.BUILDLUT_NORMALIZE, known_pos=known)
        assert np.abs(a - b).max() < 2e-3


# ---- golden fixtures (outputs of the reference build, committed) ----

def test_port_reproduces_golden_roi60(port):
    g = load("roi60_f32.npz")
    cc = port.computed_config(g["settings"])
    p = port.localize(cc, int(g["mode"]), g["rois"].astype(np.float32), g["lut"])
    assert np.abs(g["pos"][:, :2] - p[:, :2]).max() < TOL_QI
    assert np.abs(g["pos"][:, 2] - p[:, 2]).max() < TOL_Z
    assert np.abs(g["com"][:, 0] - p[:, 3]).max() < TOL_COM
    assert (g["error"] == p[:, 5]).all()
    pc = port.localize(cc, abi.LT_OnlyCOM, g["rois"].astype(np.float32))
    assert np.abs(g["com_only_pos"][:, :2] - pc[:, :2]).max() < TOL_COM


def test_port_reproduces_golden_roi100(port):
    g = load("roi100_u16.npz")
    cc = port.computed_config(g["settings"])
    p = port.localize(cc, int(g["mode"]), g["rois"], g["lut"])
    assert np.abs(g["pos"][:, :2] - p[:, :2]).max() < TOL_QI
    assert np.abs(g["pos"][:, 2] - p[:, 2]).max() < TOL_Z


def test_port_reproduces_golden_gauss(port):
    g = load("gauss16_f32.npz")
    cc = port.computed_config(g["settings"])
    p = port.localize(cc, int(g["mode"]), g["rois"].astype(np.float32))
    assert np.abs(g["pos"][:, :2] - p[:, :2]).max() < 1e-3


def test_port_reproduces_golden_buildlut(port):
    g = load("buildlut_80x80_u16.npz")
    cc = port.computed_config(g["settings"])
    lut = port.build_lut(cc, g["stack"], abi.BUILDLUT_NORMALIZE)
    assert np.abs(lut - g["lut"]).max() < 2e-3


def _ref_find_beads(ref, frame, corner, roi, rel, acc):
    img = abi.ImageData(frame.ctypes.data_as(C.POINTER(C.c_float)), frame.shape[1], frame.shape[0])
    n = C.c_int()
    p = ref.lib.QTrkFindBeads(C.byref(img), int(corner[0]), int(corner[1]), roi, rel, acc, C.byref(n), None)
    out = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int)), shape=(2 * n.value,)).reshape(-1, 2).copy() \
        if n.value else np.zeros((0, 2), np.int32)
    ref.lib.QTrkFreeROIPositions(p)
    return out


@pytest.mark.parametrize("roi,seed,noise", [(32, 6, 2.0), (24, 7, 4.0), (40, 8, 1.0)])
def test_bead_finder_oracle_matches_reference(ref, port, roi, seed, noise):
    """oracle_find_beads (direct FP64 convolution) gives the reference's bead list (KISS FFT)."""
    frame, centres = synth.bead_frame(300, 220, 10, roi, seed=seed, noise=noise)
    corner = (int(centres[0][0] - roi / 2), int(centres[0][1] - roi / 2))
    for rel, acc in ((1.0, 0.3), (1.0, 0.6), (0.8, 0.45)):
        a = _ref_find_beads(ref, frame, corner, roi, rel, acc)
        b = port.find_beads(frame, corner, roi, rel, acc)
        assert np.array_equal(a, b), (rel, acc)
        assert len(a) >= 6
