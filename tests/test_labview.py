"""LabVIEW binding (libqtrk_b200_lv.so) on the CPU, with the fake LabVIEW run-time: exports,
error clusters, array handles, the ResultManager functions, image generators and the Fisher
matrix against the reference's own code (cputrack/lv_queuetrk_api.cpp, FisherMatrix.h)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import lv_helpers as lv
from qtrk_b200 import abi, synth
from qtrk_b200 import result_manager as rmm

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    text = (ROOT / "include" / "qtrk_lv_api.h").read_text()
    return sorted(set(re.findall(r"QTRK_LV_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)))


def test_binding_exports_every_declared_function():
    names = _declared()
    assert len(names) >= 50
    L = lv.lv_library()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing


def _gpu_present():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU error path")
def test_create_without_gpu_fills_error_cluster():
    L = lv.lv_library()
    L.qtrk_create.restype = C.c_void_p
    e = lv.ErrorCluster()
    warn = lv.new_lstr()
    s = synth.settings_roi60()
    t = L.qtrk_create(C.byref(s), C.c_void_p(warn), C.byref(e))
    assert not t and e.status == 1 and e.code == 5000 and "CUDA" in lv.lstr(e.message)
    e2 = lv.ErrorCluster()
    assert L.qtrkcuda_device_count(C.byref(e2)) == 0 and e2.status == 1


def test_invalid_handles_are_reported():
    L = lv.lv_library()
    e = lv.ErrorCluster()
    L.qtrk_flush(C.c_void_p(0x1234), C.byref(e))
    assert e.status == 1 and e.code == 1
    assert "QTrk C++ function flush called with invalid tracker pointer" in lv.lstr(e.message)
    e = lv.ErrorCluster()
    L.rm_flush(C.c_void_p(0x5678), C.byref(e))
    assert e.status == 1 and lv.lstr(e.message) == "Invalid ResultManager instance passed."
    e = lv.ErrorCluster()
    L.qtrk_destroy(C.c_void_p(0x1234), C.byref(e))
    assert "qtrk_destroy with invalid qtrk pointer" in lv.lstr(e.message)


def test_array_passing_pattern():
    L = lv.lv_library()
    hs = [lv.empty_handle(np.float32, 1), lv.empty_handle(np.float32, 2), lv.empty_handle(np.int32, 1),
          lv.empty_handle(np.int32, 2)]
    n = 6
    L.test_array_passing(n, *[C.c_void_p(h) for h in hs])
    f1, f2, i1, i2 = lv.read(hs[0], 1, np.float32), lv.read(hs[1], 2, np.float32), lv.read(hs[2], 1, np.int32), \
        lv.read(hs[3], 2, np.int32)
    assert np.array_equal(i1, [(i + 1) * i for i in range(n)])
    assert np.allclose(f1, np.sqrt(np.arange(n)))
    jj, ii = np.meshgrid(np.arange(n // 2), np.arange(n), indexing="ij")
    assert np.array_equal(i2, jj * 2 + ii) and np.array_equal(f2, (jj * 2 + ii).astype(np.float32))
    for h in hs:
        lv.free(h)


def test_read_timestamp():
    L = lv.lv_library()
    L.qtrk_read_timestamp.restype = C.c_uint32
    img = np.array([0x78, 0x56, 0x34, 0x12, 9, 9], np.uint8)
    assert L.qtrk_read_timestamp(img.ctypes.data_as(C.c_void_p), 3, 2) == 0x12345678
    assert L.qtrk_read_timestamp(img.ctypes.data_as(C.c_void_p), 1, 3) == 0


def test_image_generators_match_reference(ref):
    L = lv.lv_library()
    g = np.load(ROOT / "tests" / "golden" / "roi60_f32.npz")
    lut = np.ascontiguousarray(g["lut"][0], np.float32)
    img_h, lut_h = lv.handle(np.zeros((60, 60), np.float32)), lv.handle(lut)
    radii = np.array([3.0, 28.0], np.float32)
    pos = abi.vector2f(30.3, 29.6)
    L.qtrk_generate_image_from_lut(C.c_void_p(img_h), C.c_void_p(lut_h), radii.ctypes.data_as(C.c_void_p), C.byref(pos),
                                   C.c_float(17.4), C.c_float(1.0), C.c_float(0.0))
    ours = lv.read(img_h, 2, np.float32)
    want = np.zeros((60, 60), np.float32)
    im = abi.ImageData(want.ctypes.data_as(C.POINTER(C.c_float)), 60, 60)
    lim = abi.ImageData(lut.ctypes.data_as(C.POINTER(C.c_float)), lut.shape[1], lut.shape[0])
    ref.lib.GenerateImageFromLUT(C.byref(im), C.byref(lim), 3.0, 28.0, abi.vector3f(30.3, 29.6, 17.4), True, 4)
    np.testing.assert_allclose(ours, want, rtol=1e-5, atol=1e-5)
    spot_h = lv.handle(np.zeros((16, 16), np.float32))
    L.qtrk_generate_gaussian_spot(C.c_void_p(spot_h), C.byref(abi.vector2f(7.2, 8.9)), C.c_float(1.5),
                                  C.c_float(1000.0), C.c_float(10.0), 0)
    spot = np.zeros((16, 16), np.float32)
    ref.lib.GenerateGaussianSpotImage(C.byref(abi.ImageData(spot.ctypes.data_as(C.POINTER(C.c_float)), 16, 16)),
                                      abi.vector2f(7.2, 8.9), C.c_float(1.5), C.c_float(1000.0), C.c_float(10.0))
    np.testing.assert_allclose(lv.read(spot_h, 2, np.float32), spot, rtol=1e-5, atol=1e-4)
    for h in (img_h, lut_h, spot_h):
        lv.free(h)


def test_compute_fisher_matches_reference(ref):
    """Same libc rand() seed: the same sample positions, the same averaged Fisher matrix."""
    L = lv.lv_library()
    libc = C.CDLL(None)
    g = np.load(ROOT / "tests" / "golden" / "roi60_f32.npz")
    lut = np.ascontiguousarray(g["lut"][0], np.float32)
    s = synth.settings_roi60()
    cc = abi.QTrkComputedConfig()
    ref.lib.QTrkGetComputedConfig(C.byref(s), C.byref(cc))
    fis, inv = lv.empty_handle(np.float32, 2), lv.empty_handle(np.float32, 2)
    var = abi.vector3f()
    lut_h = lv.handle(lut)
    libc.srand(99)
    L.qtrk_compute_fisher(C.c_void_p(lut_h), C.byref(s), C.byref(abi.vector3f(30, 30, 20)), C.c_void_p(fis),
                          C.c_void_p(inv), C.byref(var), 4, C.c_float(1000.0))
    F, Fi = lv.read(fis, 2, np.float32), lv.read(inv, 2, np.float32)
    L2 = ref.lib
    L2.ref_average_fisher.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, C.c_int,
                                      C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, C.c_void_p]
    want = np.zeros(9, np.float32)
    libc.srand(99)
    L2.ref_average_fisher(lut.ctypes.data, lut.shape[1], lut.shape[0], s.zlut_minradius, cc.zlut_maxradius, 60, 60,
                          30, 30, 20, 4, 1000.0, want.ctypes.data)
    want = want.reshape(3, 3)
    np.testing.assert_allclose(F, want, rtol=2e-3, atol=1e-3 * np.abs(want).max())
    assert F.shape == (3, 3) and np.allclose(F, F.T)
    np.testing.assert_allclose(Fi @ F, np.eye(3), atol=1e-3)
    assert np.allclose([var.x, var.y, var.z], np.diag(Fi))
    for h in (fis, inv, lut_h):
        lv.free(h)


def test_result_manager_functions(tmp_path, qlib):
    L = lv.lv_library()
    L.rm_create.restype = C.c_void_p
    names = [lv.new_lstr("motorA"), lv.new_lstr("motorB")]
    arr = (C.c_void_p * 2)(*names)
    cfg = rmm.config(3, 2, write_interval=1, binary_output=True)
    rm = L.rm_create(str(tmp_path / "r.bin").encode(), b"", C.byref(cfg), arr)
    assert rm
    e = lv.ErrorCluster()
    for f in range(4):
        L.rm_store_frame_info(C.c_void_p(rm), f, C.c_double(f * 0.5), np.array([f, -f], np.float32).ctypes.data_as(C.c_void_p),
                              C.byref(e))
    res = np.zeros(12, abi.RESULT_DTYPE)
    res["frame"] = np.repeat(np.arange(4), 3)
    res["zlutIndex"] = np.tile(np.arange(3), 4)
    res["pos"][:, 0] = 30 + res["frame"]
    qlib.QTrkB200RMStoreResults(C.c_void_p(rm), res.ctypes.data_as(C.c_void_p), 12, 60, 60)
    counters = [C.c_int() for _ in range(6)]
    L.rm_getframecounters(C.c_void_p(rm), *[C.byref(c) for c in counters], C.byref(e))
    assert [c.value for c in counters] == [0, 4, 4, 4, 12, 0] and e.status == 0
    out = (abi.LocalizationResult * 12)()
    assert L.rm_getresults(C.c_void_p(rm), 0, 4, out, C.byref(e)) == 4
    got = abi.results_to_numpy(out, 12)
    assert np.allclose(got["pos"][:, 0], np.repeat(np.arange(4), 3))
    bead = (abi.LocalizationResult * 4)()
    assert L.rm_getbeadresults(C.c_void_p(rm), 0, 4, 7, bead, C.byref(e)) == 0
    assert "Invalid bead index: 7" in lv.lstr(e.message)
    e = lv.ErrorCluster()
    assert L.rm_getbeadresults(C.c_void_p(rm), 1, 3, 2, bead, C.byref(e)) == 3 and e.status == 0
    got_cfg = abi.ResultManagerConfig()
    L.rm_getconfig(C.c_void_p(rm), C.byref(got_cfg), C.byref(e))
    assert bytes(got_cfg) == bytes(cfg)
    L.rm_destroy(C.c_void_p(rm), C.byref(e))
    assert e.status == 0
    data = (tmp_path / "r.bin").read_bytes()
    assert data[16:30] == b"motorA\0motorB\0"  # names as given (no separator prefix on this path)
    for h in names:
        lv.free(h)
