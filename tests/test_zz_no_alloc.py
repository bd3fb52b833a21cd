"""QTrkB200LocalizeDeviceNoAlloc: the allocation-free device-resident entry point.

Some callers cannot allocate device memory while they run (real-time acquisition threads that
must not wait on the driver's allocator, processes with a fixed device-memory budget). This
entry point runs the same localization as QTrkB200LocalizeDevice but keeps the tensor-core Z
match's intermediate profiles in a fixed 16 MiB array inside the library instead of memory
allocated by the call. The test calls both entry points through the C ABI on the same device
inputs and requires the same results (tolerance of the other parity tests: 1e-3 px in x/y,
0.01 plane in z; the kernels are the same, so the results are expected to be identical), on
two calls in a row with different inputs (the shared array keeps the previous call's contents),
and checks the size limit. The instance's BF16 copy of the LUT is made by an allocating call, so
the no-alloc call refuses (-4, nothing launched) while there is none of the current LUT's shape:
on a fresh instance, and after QTrkSetRadialZLUT installs a LUT of another shape; new contents of
a LUT of the same shape are refreshed in place. This file is collected last so that a failure here
comes after all other tests have run; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu

TOL_XY = 1e-3
TOL_Z = 0.01


def _results(buf) -> np.ndarray:
    return np.frombuffer(buf.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)


def test_no_alloc_entry_matches_device_entry():
    import torch

    wl = synth.roi100_u16(600, seed=41)
    with QTrkInstance(wl.settings) as t:
        t.SetRadialZLUTSize(1, wl.lut_stack.shape[0])
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(wl.lut_stack.shape[0]):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        t.SetLocalizationMode(wl.mode | abi.LT_B200_ZMatchBF16)
        stream = torch.cuda.current_stream().cuda_stream
        lib = t.lib
        # two different input sets, each through both entry points (the allocating entry runs
        # first and also creates the instance's BF16 LUT); the no-alloc calls then run back to
        # back, so the second reuses the array the first one filled
        sets = [wl.rois[:300], wl.rois[300:]]
        dev = [torch.from_numpy(r.view(np.int16).copy()).cuda() for r in sets]
        ref = []
        for d, r in zip(dev, sets):
            out = torch.zeros(r.shape[0] * 52, dtype=torch.uint8, device="cuda")
            rc = lib.QTrkB200LocalizeDevice(t.handle, C.c_void_p(d.data_ptr()), 200, 20000, abi.QTrkU16, r.shape[0],
                                            None, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
            assert rc == 0, t.GetWarnings()
            ref.append(out)
        got = []
        for d, r in zip(dev, sets):
            out = torch.full((r.shape[0] * 52,), 0xFF, dtype=torch.uint8, device="cuda")
            rc = lib.QTrkB200LocalizeDeviceNoAlloc(t.handle, C.c_void_p(d.data_ptr()), 200, 20000, abi.QTrkU16,
                                                   r.shape[0], None, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
            assert rc == 0, t.GetWarnings()
            got.append(out)
        torch.cuda.synchronize()
        for a, b in zip(ref, got):
            ra, rb = _results(a), _results(b)
            assert np.array_equal(ra["frame"], rb["frame"])
            assert np.abs(ra["pos"][:, :2] - rb["pos"][:, :2]).max() <= TOL_XY
            assert np.abs(ra["pos"][:, 2] - rb["pos"][:, 2]).max() <= TOL_Z
            assert np.abs(ra["firstGuess"] - rb["firstGuess"]).max() <= 1e-4
            assert (rb["pos"][:, 2] != 0).mean() > 0.9   # z was computed by the tensor-core match

        # beyond the fixed array: rejected with an error code, nothing launched
        n_big = 40000
        out = torch.zeros(n_big * 52, dtype=torch.uint8, device="cuda")  # large enough in any case
        rc = lib.QTrkB200LocalizeDeviceNoAlloc(t.handle, C.c_void_p(dev[0].data_ptr()), 200, 0, abi.QTrkU16, n_big,
                                               None, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert rc == -3
        assert "fixed array holds" in t.GetWarnings()


def _call(lib, fn, t, d, n, out, stream):
    return getattr(lib, fn)(t.handle, C.c_void_p(d.data_ptr()), 200, 20000, abi.QTrkU16, n, None,
                            C.c_void_p(out.data_ptr()), C.c_void_p(stream))


def _assert_same(a, b):
    ra, rb = _results(a), _results(b)
    assert np.array_equal(ra["frame"], rb["frame"])
    assert np.abs(ra["pos"][:, :2] - rb["pos"][:, :2]).max() <= TOL_XY
    assert np.abs(ra["pos"][:, 2] - rb["pos"][:, 2]).max() <= TOL_Z


def test_no_alloc_refuses_without_a_bf16_lut_of_the_current_shape():
    import torch

    wl = synth.roi100_u16(256, seed=43)
    n = wl.rois.shape[0]
    with QTrkInstance(wl.settings) as t:
        lib = t.lib
        stream = torch.cuda.current_stream().cuda_stream
        d = torch.from_numpy(wl.rois.view(np.int16).copy()).cuda()
        t.SetRadialZLUTSize(1, wl.lut_stack.shape[0])
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(wl.lut_stack.shape[0]):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        lut1 = t.GetRadialZLUT()  # 1 x 200 x 64
        t.SetLocalizationMode(wl.mode | abi.LT_B200_ZMatchBF16)
        nb = lut1.shape[-1]

        # fresh instance: no BF16 copy yet
        out = torch.zeros(n * 52, dtype=torch.uint8, device="cuda")
        k0 = t.KernelLaunchCount()
        assert _call(lib, "QTrkB200LocalizeDeviceNoAlloc", t, d, n, out, stream) == -4
        assert t.KernelLaunchCount() == k0
        assert "tensor-core LUT" in t.GetWarnings()

        # an allocating call makes the copy for the 1 x 200 x 64 LUT
        ref1 = torch.zeros(n * 52, dtype=torch.uint8, device="cuda")
        assert _call(lib, "QTrkB200LocalizeDevice", t, d, n, ref1, stream) == 0, t.GetWarnings()

        # a larger LUT (4 beads x 300 planes): the old copy is dropped, so the no-alloc call refuses
        # before launching anything rather than refreshing a copy sized for the old shape
        planes2 = 300
        zi = np.linspace(0, lut1.shape[1] - 1, planes2)
        rows = np.stack([np.interp(zi, np.arange(lut1.shape[1]), lut1[0, :, r]) for r in range(nb)], 1)
        lut2 = np.stack([rows * (1.0 + 0.01 * b) for b in range(4)]).astype(np.float32)
        t.SetRadialZLUT(lut2)
        torch.cuda.synchronize()
        k0 = t.KernelLaunchCount()
        got = torch.full((n * 52,), 0xFF, dtype=torch.uint8, device="cuda")
        assert _call(lib, "QTrkB200LocalizeDeviceNoAlloc", t, d, n, got, stream) == -4
        assert t.KernelLaunchCount() == k0
        # one allocating call makes the copy of the new shape; the no-alloc call then succeeds and
        # returns the same results
        ref2 = torch.zeros(n * 52, dtype=torch.uint8, device="cuda")
        assert _call(lib, "QTrkB200LocalizeDevice", t, d, n, ref2, stream) == 0, t.GetWarnings()
        assert _call(lib, "QTrkB200LocalizeDeviceNoAlloc", t, d, n, got, stream) == 0, t.GetWarnings()
        torch.cuda.synchronize()
        _assert_same(ref2, got)
        assert (_results(got)["pos"][:, 2] != 0).mean() > 0.9

        # same shape, new contents (radial weights change the weighted BF16 rows): refreshed in place
        # by the no-alloc call itself, then equal to the allocating call's results
        w = np.linspace(0.5, 1.5, nb).astype(np.float32)
        t.SetRadialWeights(w)
        got2 = torch.full((n * 52,), 0xFF, dtype=torch.uint8, device="cuda")
        assert _call(lib, "QTrkB200LocalizeDeviceNoAlloc", t, d, n, got2, stream) == 0, t.GetWarnings()
        ref3 = torch.zeros(n * 52, dtype=torch.uint8, device="cuda")
        assert _call(lib, "QTrkB200LocalizeDevice", t, d, n, ref3, stream) == 0, t.GetWarnings()
        torch.cuda.synchronize()
        _assert_same(ref3, got2)
        assert not np.array_equal(_results(ref2)["pos"][:, 2], _results(ref3)["pos"][:, 2])
