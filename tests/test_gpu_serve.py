"""Request server (QTrkB200Server*): frames of four instances with different ROI sizes, pixel
types and modes, served alone and interleaved. Each frame's results must be bit-identical
whether it was served alone or batched with others, and equal to what QTrkScheduleFrame
(cputrack/QueuedTracker.cpp:91-111) gives for the same frame on the same instance; the
reference parity of ScheduleFrame itself is covered in test_gpu_parity.py."""
import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200.server import Server
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu


def _lut_from_stack(settings, mode, stack_f32, nbeads):
    """A normalized Z-LUT built by the instance itself (BeginLUT/BuildLUT/FinalizeLUT), copied to nbeads."""
    t = QTrkInstance(settings)
    try:
        t.SetLocalizationMode(mode)
        planes = stack_f32.shape[0]
        t.SetRadialZLUTSize(1, planes)
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        w = settings.width
        for k in range(planes):
            t.BuildLUT(stack_f32[k:k + 1], k, np.array([[w / 2, settings.height / 2]], np.float32))
        t.FinalizeLUT()
        lut = t.GetRadialZLUT()
    finally:
        t.Destroy()
    return np.ascontiguousarray(np.concatenate([lut.reshape(1, planes, -1)] * nbeads))


def _u8_workload(n, seed):
    """40x40 u8 ROIs: 10 + 100 p(r; z) + Poisson clipped to 255; Z-LUT 40 planes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = 40
    cx = 20 + rng.uniform(-2, 2, n)
    cy = 20 + rng.uniform(-2, 2, n)
    z = rng.uniform(5, 35, n)
    rois = np.minimum(rng.poisson(synth.render(w, w, cx, cy, z, 10.0, 100.0)), 255).astype(np.uint8)
    kz = np.arange(40, dtype=np.float64)
    stack = synth.render(w, w, np.full(40, w / 2), np.full(40, w / 2), kz, 10.0, 100.0).astype(np.float32)
    s = synth.settings_roi60(width=40, height=40)
    return s, rois, stack


def _frame_of(rois, gap, seed, outside=True):
    """Place the ROIs on a grid inside a frame; add positions outside the frame (skipped)."""
    n, h, w = rois.shape
    cols = int(np.ceil(np.sqrt(n)))
    rows = (n + cols - 1) // cols
    H, W = rows * (h + gap) + gap, cols * (w + gap) + gap
    rng = np.random.Generator(np.random.PCG64(seed))
    frame = np.zeros((H, W), rois.dtype)
    pos = []
    for i in range(n):
        y, x = gap + (i // cols) * (h + gap), gap + (i % cols) * (w + gap)
        frame[y:y + h, x:x + w] = rois[i]
        pos.append((x, y))
    if outside:
        pos.insert(int(rng.integers(0, n)), (W - w + 1, 0))
        pos.append((-1, 3))
    return frame, np.array(pos, np.int32)


@pytest.fixture(scope="module")
def fleet():
    """Four instances (each with its own LUT) and four frames for each."""
    insts, frames = [], []
    # A: 60x60 f32, QI + Z
    wl = synth.roi60_f32(48, seed=71)
    A = QTrkInstance(wl.settings)
    A.SetLocalizationMode(wl.mode)
    A.SetRadialZLUT(_lut_from_stack(wl.settings, wl.mode, wl.lut_stack[:, 0], 13))
    insts.append(A)
    frames.append([_frame_of(wl.rois[12 * k:12 * k + 12], 3, k) for k in range(4)])
    # B: 100x100 u16, QI + Z
    wl = synth.roi100_u16(120, seed=72)
    B = QTrkInstance(wl.settings)
    B.SetLocalizationMode(wl.mode)
    B.SetRadialZLUT(_lut_from_stack(wl.settings, wl.mode, wl.lut_stack[:, 0], 31))
    insts.append(B)
    frames.append([_frame_of(wl.rois[30 * k:30 * k + 30], 5, 10 + k) for k in range(4)])
    # C: 40x40 u8, QI + Z
    s, rois, stack = _u8_workload(80, 73)
    C_ = QTrkInstance(s)
    C_.SetLocalizationMode(synth.MODE_QI_Z)
    C_.SetRadialZLUT(_lut_from_stack(s, synth.MODE_QI_Z, stack, 21))
    insts.append(C_)
    frames.append([_frame_of(rois[20 * k:20 * k + 20], 2, 20 + k) for k in range(4)])
    # D: 16x16 f32, Gaussian 2D (warp-per-ROI kernel), no LUT
    wl = synth.gauss16_f32(200, seed=74)
    D = QTrkInstance(wl.settings)
    D.SetLocalizationMode(wl.mode)
    insts.append(D)
    frames.append([_frame_of(wl.rois[50 * k:50 * k + 50], 1, 30 + k) for k in range(4)])
    yield insts, frames
    for t in insts:
        t.Destroy()


def _schedule_frame(t, frame, pos, frame_no):
    n = t.ScheduleFrame(frame, pos, frame_no=frame_no)
    r = t.WaitForResults(n)
    return r[np.argsort(r["zlutIndex"], kind="stable")]


def _same(a, b):
    assert len(a) == len(b)
    for f in ("frame", "zlutIndex", "pos", "firstGuess", "error", "imageMean"):
        assert np.array_equal(a[f], b[f]), f


def test_alone_mixed_and_schedule_frame_agree(fleet):
    insts, frames = fleet
    # through ScheduleFrame
    expect = {}
    for i, t in enumerate(insts):
        for k, (frame, pos) in enumerate(frames[i]):
            expect[i, k] = _schedule_frame(t, frame, pos, 100 * i + k)
            n_in = len(pos) - 2
            assert len(expect[i, k]) == n_in
    with Server(0, 1 << 30) as sv:
        ids = [sv.attach(t) for t in insts]
        assert ids == [0, 1, 2, 3]
        # alone: one frame in flight at a time
        alone = {}
        for i in range(4):
            for k, (frame, pos) in enumerate(frames[i]):
                alone[i, k] = sv.wait(sv.submit(i, frame, pos, frame_no=100 * i + k))
        # mixed: every frame submitted at once, interleaved over the instances
        order = [(i, k) for k in range(4) for i in range(4)]
        rid = {(i, k): sv.submit(i, *frames[i][k], frame_no=100 * i + k) for i, k in order}
        mixed = {key: sv.wait(r) for key, r in rid.items()}
        st = sv.stats()
    for key in expect:
        a = alone[key]
        _same(a, expect[key])
        _same(mixed[key], a)
        # result i of a frame carries zlutIndex = i over the ROIs inside the frame
        assert (a["frame"] == 100 * key[0] + key[1]).all()
    assert st["frames"] == 32
    assert st["rois"] == sum(len(v) for v in expect.values()) * 2
    assert 1 <= st["launches"] <= 32
    assert st["graphs"] >= 4
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_one_lane_batches_and_completes(fleet):
    """A budget below one lane still gives one lane; frames that waited (held admission) are
    merged into one launch, each frame's results unchanged."""
    insts, frames = fleet
    t = insts[1]
    expect = [_schedule_frame(t, f, p, k) for k, (f, p) in enumerate(frames[1])]
    with Server(0, 1) as sv:
        sv.attach(t)
        reps = 8
        sv.hold(True)
        rid = [sv.submit(0, *frames[1][k % 4], frame_no=k % 4) for k in range(4 * reps)]
        assert all(sv.poll(r) is None for r in rid)
        sv.hold(False)
        out = [sv.wait(r) for r in rid]
        st = sv.stats()
        # with the lane free, frames that keep arriving are served too
        more = [sv.wait(sv.submit(0, *frames[1][k], frame_no=k)) for k in range(4)]
    assert st["lanes"] == 1
    for k, r in enumerate(out):
        _same(r, expect[k % 4])
    for k, r in enumerate(more):
        _same(r, expect[k])
    assert st["frames"] == 4 * reps
    # 32 frames of ~0.7 MB and 30 ROIs each fit one lane (48 MiB, 8,192 ROIs): one launch
    assert st["launches"] == 1


def test_graph_reuse_and_edge_cases(fleet):
    insts, frames = fleet
    with Server(0, 1) as sv:
        sv.attach(insts[0])
        for _ in range(6):
            sv.wait(sv.submit(0, *frames[0][0]))
        assert sv.stats()["graphs"] == 1  # one bucket, one lane: captured once, replayed
        # a frame whose ROIs all lie outside completes with no results
        f, _ = frames[0][0]
        r = sv.wait(sv.submit(0, f, np.array([[-5, 0], [f.shape[1], 0]], np.int32)))
        assert len(r) == 0
        with pytest.raises(KeyError):
            sv.poll(123456789)
        with pytest.raises(RuntimeError):
            sv.submit(7, f, np.zeros((1, 2), np.int32))  # unknown instance
        with pytest.raises(RuntimeError):
            sv.submit(0, f, np.zeros((9000, 2), np.int32))  # more ROIs than a lane holds
