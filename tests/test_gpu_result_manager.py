"""ResultManager attached to this library's GPU tracker: its fetch thread bins the tracker's
results per frame and bead exactly as the same results stored directly would be."""
import ctypes as C
import time

import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200 import result_manager as rmm
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu

N_BEADS, N_FRAMES = 5, 40


def _schedule(t, rois):
    for f in range(N_FRAMES):
        for b in range(N_BEADS):
            t.ScheduleLocalization(rois[f * N_BEADS + b], frame=f, zlut=b)
    t.Flush()


def test_result_manager_on_gpu_tracker(tmp_path):
    wl = synth.roi60_f32(N_BEADS * N_FRAMES, seed=43)
    cfg = rmm.config(N_BEADS, 1, scaling=(0.065, 0.065, 1.0), offset=(0.5, -0.5, 0.0), write_interval=7)
    with QTrkInstance(wl.settings) as t, rmm.ResultManager(str(tmp_path / "r.txt"), str(tmp_path / "i.txt"), cfg) as rm:
        t.SetLocalizationMode(abi.LT_QI)
        for f in range(N_FRAMES):
            rm.StoreFrameInfo(f, f * 0.002, [float(f)])
        rm.SetTracker(t)
        _schedule(t, wl.rois)
        deadline = time.monotonic() + 60
        while rm.GetFrameCounters()["processedFrames"] < N_FRAMES:
            assert time.monotonic() < deadline
            time.sleep(0.002)
        rm.Flush()
        got = rm.GetResults(0, N_FRAMES)
        c = rm.GetFrameCounters()
        rm.SetTracker(None)
    assert c["localizationsDone"] == N_BEADS * N_FRAMES and c["lostFrames"] == 0 and c["lastSaveFrame"] == N_FRAMES
    with QTrkInstance(wl.settings) as t2:
        t2.SetLocalizationMode(abi.LT_QI)
        _schedule(t2, wl.rois)
        raw = t2.WaitForResults(N_BEADS * N_FRAMES)
    cfg2 = rmm.config(N_BEADS, 1, scaling=(0.065, 0.065, 1.0), offset=(0.5, -0.5, 0.0), write_interval=7)
    with rmm.ResultManager("", "", cfg2) as rm2:
        rm2.StoreResults(raw, wl.settings.width, wl.settings.height)
        want = rm2.GetResults(0, N_FRAMES)
    assert got.tobytes() == want.tobytes()
    lines = (tmp_path / "r.txt").read_text().splitlines()
    assert len(lines) == N_FRAMES and lines[3].split("\t")[0] == "3"
    x = float(lines[3].split("\t")[2])
    assert abs(x - got[3, 0]["pos"][0]) < 1e-6
