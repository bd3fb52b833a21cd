"""LabVIEW binding on the GPU (fake LabVIEW run-time): the qtrk_* calls give the results of the
C ABI calls they stand for, on the same inputs."""
import ctypes as C
import time

import numpy as np
import pytest

import lv_helpers as lv
from golden_io import load
from qtrk_b200 import abi, synth
from qtrk_b200 import result_manager as rmm
from qtrk_b200.tracker import QTrkInstance, load_library

pytestmark = pytest.mark.gpu


def _create(L, s):
    L.qtrk_create.restype = C.c_void_p
    e = lv.ErrorCluster()
    warn = lv.new_lstr()
    t = L.qtrk_create(C.byref(s), C.c_void_p(warn), C.byref(e))
    assert t and e.status == 0, lv.lstr(e.message)
    lv.free(warn)
    return t


def _wait(L, t, n):
    e = lv.ErrorCluster()
    L.qtrk_flush(C.c_void_p(t), C.byref(e))
    deadline = time.monotonic() + 60
    while L.qtrk_resultcount(C.c_void_p(t), C.byref(e)) < n:
        assert time.monotonic() < deadline
        time.sleep(0.001)
    buf = (abi.LocalizationResult * n)()
    assert L.qtrk_get_results(C.c_void_p(t), buf, n, 1, C.byref(e)) == n
    return abi.results_to_numpy(buf, n)


def test_queue_and_results_match_c_abi():
    L = lv.lv_library()
    g = load("roi60_f32.npz")
    s, lut, mode = g["settings"], np.ascontiguousarray(g["lut"], np.float32), int(g["mode"])
    rois = g["rois"].astype(np.float32)  # 24 ROIs
    t = _create(L, s)
    e = lv.ErrorCluster()
    try:
        cc = abi.QTrkComputedConfig()
        L.qtrk_get_computed_config(C.c_void_p(t), C.byref(cc), C.byref(e))
        assert cc.zlut_radialsteps == lut.shape[2]
        lut_h, win_h = lv.handle(lut), lv.empty_handle(np.float32, 1)
        L.qtrk_set_ZLUT(C.c_void_p(t), C.c_void_p(lut_h), C.c_void_p(win_h), 0, C.byref(e))
        L.qtrk_set_localization_mode(C.c_void_p(t), mode, C.byref(e))
        back = lv.empty_handle(np.float32, 3)
        L.qtrk_get_ZLUT(C.c_void_p(t), C.c_void_p(back), C.byref(e))
        assert np.array_equal(lv.read(back, 3, np.float32), lut)
        job = abi.LocalizationJob()
        for i, r in enumerate(rois):
            h = lv.handle(r)
            job.frame = i
            L.qtrk_queue_float(C.c_void_p(t), C.byref(e), C.c_void_p(h), C.byref(job))
            lv.free(h)
        assert e.status == 0, lv.lstr(e.message)
        got = _wait(L, t, len(rois))
        assert L.qtrk_idle(C.c_void_p(t), C.byref(e)) in (0, 1)
        # a wrong image size is an argument error, nothing queued
        bad = lv.handle(np.zeros((10, 12), np.float32))
        L.qtrk_queue_float(C.c_void_p(t), C.byref(e), C.c_void_p(bad), C.byref(job))
        assert e.status == 1 and "wrong size (12,10)" in lv.lstr(e.message)
        for h in (lut_h, win_h, back, bad):
            lv.free(h)
    finally:
        L.qtrk_destroy(C.c_void_p(t), C.byref(lv.ErrorCluster()))
    with QTrkInstance(s) as ti:
        ti.SetRadialZLUT(lut)
        ti.SetLocalizationMode(mode)
        want = ti.Localize(rois)
    assert np.array_equal(got["pos"], want["pos"]) and np.array_equal(got["frame"], want["frame"])


def test_build_lut_bias_table_and_find_beads():
    L = lv.lv_library()
    wl = synth.roi100_u16(1, seed=23)
    s = wl.settings
    t = _create(L, s)
    e = lv.ErrorCluster()
    try:
        planes = wl.lut_stack.shape[0]
        nb = abi.QTrkComputedConfig()
        L.qtrk_get_computed_config(C.c_void_p(t), C.byref(nb), C.byref(e))
        empty = lv.handle(np.zeros((1, planes, nb.zlut_radialsteps), np.float32))
        L.qtrk_set_ZLUT(C.c_void_p(t), C.c_void_p(empty), C.c_void_p(lv.empty_handle(np.float32, 1)), 0, C.byref(e))
        lib = load_library()
        lib.QTrkBeginLUT(C.c_void_p(t), abi.BUILDLUT_NORMALIZE)
        for p in range(planes):
            h = lv.handle(wl.lut_stack[p].astype(np.float32))
            L.qtrk_build_lut_plane(C.c_void_p(t), C.c_void_p(h), 0, p, C.byref(e))
            lv.free(h)
        L.qtrk_finalize_lut(C.c_void_p(t), C.byref(e))
        assert e.status == 0, lv.lstr(e.message)
        out = lv.empty_handle(np.float32, 3)
        L.qtrk_get_ZLUT(C.c_void_p(t), C.c_void_p(out), C.byref(e))
        lut_lv = lv.read(out, 3, np.float32)
        tbl = lv.empty_handle(np.float32, 2)
        L.qtrk_compute_zlut_bias_table(C.c_void_p(t), 50, C.c_void_p(tbl), 2, 1, C.byref(e))
        table = lv.read(tbl, 2, np.float32)
        assert table.shape == (1, 50) and np.isfinite(table).all()
    finally:
        L.qtrk_destroy(C.c_void_p(t), C.byref(lv.ErrorCluster()))
    with QTrkInstance(s) as ti:
        ti.SetRadialZLUTSize(1, planes)
        ti.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(planes):
            ti.BuildLUT(wl.lut_stack[p].astype(np.float32), p)
        ti.FinalizeLUT()
        want = ti.GetRadialZLUT()
        t2 = np.zeros(50, np.float32)
        ti.lib.QTrkB200ComputeZLUTBiasTable(ti.handle, 50, t2.ctypes.data_as(C.c_void_p), 2, 1)
    assert np.array_equal(lut_lv, want)
    assert np.array_equal(table[0], t2)
    # bead finder on a u8 frame: the same list as QTrkFindBeads on its float copy
    frame, centres = synth.bead_frame(300, 220, 10, 32, seed=6)
    f8 = np.clip(frame * 2, 0, 255).astype(np.uint8)
    corner = np.array([int(centres[0][0] - 16), int(centres[0][1] - 16)], np.int32)
    outh = lv.empty_handle(np.uint32, 2)
    L.qtrk_find_beads(f8.ctypes.data_as(C.c_void_p), 300, 300, 220, corner.ctypes.data_as(C.c_void_p), 32,
                      C.c_float(1.0), C.c_float(0.5), C.c_void_p(outh))
    lvpos = lv.read(outh, 2, np.uint32).astype(np.int32)
    ff = f8.astype(np.float32)
    img = abi.ImageData(ff.ctypes.data_as(C.POINTER(C.c_float)), 300, 220)
    n = C.c_int()
    p = lib.QTrkFindBeads(C.byref(img), int(corner[0]), int(corner[1]), 32, 1.0, 0.5, C.byref(n), None)
    want_pos = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int)), shape=(2 * n.value,)).reshape(-1, 2).copy()
    lib.QTrkFreeROIPositions(p)
    assert len(want_pos) >= 5 and np.array_equal(lvpos, want_pos)


def test_result_manager_and_device_info(tmp_path):
    L = lv.lv_library()
    e = lv.ErrorCluster()
    assert L.qtrkcuda_device_count(C.byref(e)) >= 1 and e.status == 0

    class DevInfo(C.Structure):
        _fields_ = [("name", C.c_void_p), ("clockRate", C.c_int), ("multiProcCount", C.c_int), ("major", C.c_int),
                    ("minor", C.c_int)]

    di = DevInfo()
    di.name = lv.new_lstr()
    L.qtrkcuda_get_device(0, C.byref(di), C.byref(e))
    assert di.major == 10 and di.multiProcCount >= 100 and "B200" in lv.lstr(di.name)
    g = load("roi60_f32.npz")
    s = g["settings"]
    rois = g["rois"].astype(np.float32)[:24]  # the fixture's 24 ROIs: 8 frames of 3 beads
    t = _create(L, s)
    L.rm_create.restype = C.c_void_p
    cfg = rmm.config(3, 0, write_interval=2)
    rm = L.rm_create(str(tmp_path / "r.txt").encode(), b"", C.byref(cfg), None)
    try:
        L.qtrk_set_localization_mode(C.c_void_p(t), abi.LT_QI, C.byref(e))
        L.rm_set_tracker(C.c_void_p(rm), C.c_void_p(t), C.byref(e))
        job = abi.LocalizationJob()
        for i, r in enumerate(rois):
            job.frame, job.zlutIndex = i // 3, i % 3
            L.qtrk_queue_pitchedmem(C.c_void_p(t), r.ctypes.data_as(C.c_void_p), 240, abi.QTrkFloat, C.byref(job))
        L.qtrk_flush(C.c_void_p(t), C.byref(e))
        deadline = time.monotonic() + 60
        counters = [C.c_int() for _ in range(6)]
        while True:
            L.rm_getframecounters(C.c_void_p(rm), *[C.byref(c) for c in counters], C.byref(e))
            if counters[2].value == 8:
                break
            assert time.monotonic() < deadline
            time.sleep(0.002)
        L.rm_flush(C.c_void_p(rm), C.byref(e))
        assert counters[4].value == 24
        e = lv.ErrorCluster()
        L.rm_removebead(C.c_void_p(rm), 0, C.byref(e))  # tracker attached: reported, bead removed
        assert e.status == 1 and "tracking in progress" in lv.lstr(e.message)
    finally:
        L.rm_destroy(C.c_void_p(rm), C.byref(lv.ErrorCluster()))
        L.qtrk_destroy(C.c_void_p(t), C.byref(lv.ErrorCluster()))
    assert len((tmp_path / "r.txt").read_text().splitlines()) == 8
    # simulate_tracking on a fresh instance with the golden LUT
    e = lv.ErrorCluster()
    t = _create(L, s)
    try:
        lut_h = lv.handle(np.ascontiguousarray(g["lut"], np.float32))
        L.qtrk_set_ZLUT(C.c_void_p(t), C.c_void_p(lut_h), C.c_void_p(lv.empty_handle(np.float32, 1)), 0, C.byref(e))
        L.qtrk_set_localization_mode(C.c_void_p(t), int(g["mode"]), C.byref(e))
        bias, scatter = abi.vector3f(), abi.vector3f()
        L.qtrk_simulate_tracking(C.c_void_p(t), 50, 0, C.byref(abi.vector3f(29.5, 29.5, 20)),
                                 C.byref(abi.vector3f(1, 1, 5)), C.byref(bias), C.byref(scatter), C.c_float(10000.0),
                                 C.byref(e))
        assert e.status == 0, lv.lstr(e.message)
        assert np.isfinite([bias.x, bias.y, bias.z, scatter.x, scatter.y, scatter.z]).all()
        assert scatter.x > 0 and scatter.z > 0
    finally:
        L.qtrk_destroy(C.c_void_p(t), C.byref(lv.ErrorCluster()))
