"""ResultManager (RM* C ABI) against the reference's own ResultManager (cputrack/ResultManager.cpp
compiled in oracle/_ref), on the CPU: the reference manager fetches from the reference CPU
tracker; this library's manager is given the same results through QTrkB200RMStoreResults.
Binned results, counters and the written files must be identical (the binary header's data
offset is a 32-bit int here; the reference's Linux build writes an 8-byte long over the first
4 bytes of the column names, so those 4 bytes are excluded)."""
import ctypes as C
import time

import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200 import result_manager as rmm

N_BEADS, N_FRAMES = 4, 12


def _rois():
    wl = synth.roi60_f32(N_BEADS * N_FRAMES, seed=41)
    return wl.settings, wl.rois  # ROI f*N_BEADS + b is bead b of frame f


def _schedule(L, trk, rois):
    job = abi.LocalizationJob()
    for f in range(N_FRAMES):
        for b in range(N_BEADS):
            job.frame, job.zlutIndex = f, b
            img = rois[f * N_BEADS + b]
            L.QTrkScheduleLocalization(trk, img.ctypes.data_as(C.c_void_p), img.strides[0], abi.QTrkFloat,
                                       C.byref(job))
    L.QTrkFlush(trk)


def _ref_results(ref, s, rois):
    L = ref.lib
    trk = L.QTrkCreateInstance(C.byref(s))
    try:
        L.QTrkSetLocalizationMode(trk, abi.LT_QI)
        _schedule(L, trk, rois)
        n = N_BEADS * N_FRAMES
        deadline = time.monotonic() + 120
        while L.QTrkGetResultCount(trk) < n:
            assert time.monotonic() < deadline
            time.sleep(0.001)
        buf = (abi.LocalizationResult * n)()
        assert L.QTrkFetchResults(trk, buf, n) == n
        while not L.QTrkIsIdle(trk):
            time.sleep(0.001)
    finally:
        L.QTrkFreeInstance(trk)
    return abi.results_to_numpy(buf, n)


def _info(f):
    return np.array([0.5 * f, -1.25 * f], np.float32)


def _run_reference_rm(ref, s, rois, out, info, cfg):
    L = ref.lib
    rm = L.RMCreate(str(out).encode(), str(info).encode(), C.byref(cfg), b"motorA;motorB")
    trk = L.QTrkCreateInstance(C.byref(s))
    try:
        for f in range(N_FRAMES):
            L.RMStoreFrameInfo(rm, f, 0.01 * f + 0.5, _info(f).ctypes.data_as(C.c_void_p))
        L.QTrkSetLocalizationMode(trk, abi.LT_QI)
        L.RMSetTracker(rm, trk)
        _schedule(L, trk, rois)
        cnt = abi.RMFrameCounters()
        deadline = time.monotonic() + 120
        while True:
            L.RMGetFrameCounters(rm, C.byref(cnt))
            if cnt.processedFrames == N_FRAMES and cnt.localizationsDone == N_BEADS * N_FRAMES:
                break
            assert time.monotonic() < deadline, "reference ResultManager did not complete"
            time.sleep(0.005)
        L.RMFlush(rm)
        return _collect(L, rm)
    finally:
        L.RMDestroy(rm)
        L.QTrkFreeInstance(trk)


def _collect(L, rm):
    allr = (abi.LocalizationResult * (N_FRAMES * N_BEADS))()
    n = L.RMGetResults(rm, 0, N_FRAMES, allr)
    bead = (abi.LocalizationResult * 5)()
    nb = L.RMGetBeadResults(rm, 2, 5, 1, bead)
    none = (abi.LocalizationResult * 4)()
    n_bad = L.RMGetResults(rm, 5, N_FRAMES, none)  # past the processed frames: nothing
    cnt = abi.RMFrameCounters()
    L.RMGetFrameCounters(rm, C.byref(cnt))
    cfg = abi.ResultManagerConfig()
    L.RMGetConfig(rm, C.byref(cfg))
    return (n, abi.results_to_numpy(allr, N_FRAMES * N_BEADS), nb, abi.results_to_numpy(bead, 5), n_bad,
            {k: getattr(cnt, k) for k, _ in cnt._fields_}, bytes(cfg))


def _run_our_rm(qlib, results, out, info, cfg, w, h):
    rm = qlib.RMCreate(str(out).encode(), str(info).encode(), C.byref(cfg), b"motorA;motorB")
    assert rm
    try:
        for f in range(N_FRAMES):
            qlib.RMStoreFrameInfo(rm, f, 0.01 * f + 0.5, _info(f).ctypes.data_as(C.c_void_p))
        r = np.ascontiguousarray(results)
        qlib.QTrkB200RMStoreResults(rm, r.ctypes.data_as(C.c_void_p), len(r), w, h)
        qlib.RMFlush(rm)
        return _collect(qlib, rm)
    finally:
        qlib.RMDestroy(rm)


@pytest.mark.parametrize("binary", [False, True])
def test_result_manager_matches_reference(ref, qlib, tmp_path, binary):
    s, rois = _rois()
    cfg = rmm.config(N_BEADS, 2, scaling=(0.1, 0.2, 1.5), offset=(1.0, 2.0, 3.0), write_interval=5,
                     binary_output=binary)
    a = _run_reference_rm(ref, s, rois, tmp_path / "ref.out", tmp_path / "ref.info", cfg)
    results = _ref_results(ref, s, rois)
    # arrival order must not matter: shuffle the results this manager is given
    results = results[np.random.default_rng(3).permutation(len(results))]
    b = _run_our_rm(qlib, results, tmp_path / "our.out", tmp_path / "our.info", cfg, s.width, s.height)
    assert a[0] == b[0] == N_FRAMES
    assert a[1].tobytes() == b[1].tobytes()
    assert a[2] == b[2] == 5 and a[3].tobytes() == b[3].tobytes()
    assert a[4] == b[4] == 0
    assert a[5] == b[5]
    assert a[6] == b[6]
    ra, rb = (tmp_path / "ref.out").read_bytes(), (tmp_path / "our.out").read_bytes()
    if binary:
        assert len(ra) == len(rb) and ra[:16] == rb[:16] and ra[20:] == rb[20:]
        assert rb[16:20] == b"moto"
    else:
        assert ra == rb
        assert (tmp_path / "ref.info").read_bytes() == (tmp_path / "our.info").read_bytes()
    # positions are ROI-centred, offset, then scaled
    r0 = results[np.lexsort((results["zlutIndex"], results["frame"]))]
    got = b[1]
    np.testing.assert_array_equal(got["pos"][:, 0], ((r0["pos"][:, 0] - s.width * 0.5) + 1.0).astype(np.float32)
                                  * np.float32(0.1))


def _store(lib, rm, frames, beads, w=60, h=60, skip=()):
    res = np.zeros(len(frames) * len(beads), abi.RESULT_DTYPE)
    k = 0
    for f in frames:
        for b in beads:
            if (f, b) in skip:
                continue
            res[k]["frame"], res[k]["zlutIndex"] = f, b
            res[k]["pos"] = (30 + f, 30 + b, f * 0.5)
            k += 1
    res = res[:k]
    lib.QTrkB200RMStoreResults(rm, res.ctypes.data_as(C.c_void_p), k, w, h)


def test_result_manager_edge_cases(qlib, tmp_path):
    cfg = rmm.config(3, 0, write_interval=1, max_frames_in_memory=4, binary_output=True)
    with rmm.ResultManager(str(tmp_path / "a.bin"), "", cfg, lib=qlib) as rm:
        # a bead index outside numBeads and a frame far ahead are lost, not stored
        _store(qlib, rm.handle, [0], [0, 1, 2, 7])
        c = rm.GetFrameCounters()
        assert c["processedFrames"] == 1 and c["lostFrames"] == 1 and c["localizationsDone"] == 3
        _store(qlib, rm.handle, [30000], [0])
        assert rm.GetFrameCounters()["lostFrames"] == 2
        # frames 1..9 complete; at most 4 frames stay in memory, all are written
        _store(qlib, rm.handle, range(1, 10), [0, 1, 2])
        c = rm.GetFrameCounters()
        assert c["processedFrames"] == 10 and c["startFrame"] == 6 and c["lastSaveFrame"] == 10
        assert len(rm.GetResults(5, 2)) == 0  # frame 5 left memory
        r = rm.GetResults(6, 4)  # ROI-centred: x = frame, y = bead
        assert r.shape == (4, 3) and np.allclose(r[:, 1]["pos"][:, 0], np.arange(6, 10))
        assert np.allclose(r["pos"][:, :, 1], [0, 1, 2])
        # a frame with a missing bead waits (and a fifth frame in memory evicts frame 6);
        # RemoveBead shifts the later beads' columns
        _store(qlib, rm.handle, [10], [0, 1, 2], skip={(10, 1)})
        c = rm.GetFrameCounters()
        assert c["processedFrames"] == 10 and c["startFrame"] == 7
        rm.RemoveBead(0)
        r = rm.GetResults(7, 3)
        assert np.allclose(r["pos"][:, :2, 1], [1, 2]) and (r[:, 2]["pos"] == 0).all()
        cfg2 = rm.GetConfig()
        assert cfg2.numBeads == 3 and cfg2.maxFramesInMemory == 4
    data = (tmp_path / "a.bin").read_bytes()
    hdr = np.frombuffer(data[:16], np.int32)
    assert list(hdr) == [3, 3, 0, 16]
    rec = 4 + 8 + 3 * 20
    assert len(data) == 16 + 10 * rec
    frames = [int(np.frombuffer(data[16 + k * rec:20 + k * rec], np.uint32)[0]) for k in range(10)]
    assert frames == list(range(10))
