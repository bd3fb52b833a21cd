"""The adjoint of the Z match (QTrkB200ZLUTCostGradient) and the joint Gauss-Newton refinement
(LT_B200_JointRefine) against the FP64 oracle (oracle_zcost_grad / oracle_joint_refine) and central
finite differences; a torch.autograd.Function built on the C ABI (test harness only) drives a few
LUT gradient steps."""
import ctypes as C

import numpy as np
import pytest

from golden_io import load
from qtrk_b200 import abi, synth
from qtrk_b200.tracker import QTrkInstance

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _device_rois(rois):
    torch = _torch()
    return torch.from_numpy(np.ascontiguousarray(rois, np.float32)).cuda()


def _cost_grad(t, d_rois, xyz, beads=None, glut=None):
    """GPU cost and gradients of (N, H, W) f32 device ROIs at xyz (N, 3)."""
    torch = _torch()
    n, h, w = d_rois.shape
    d_xyz = torch.as_tensor(np.ascontiguousarray(xyz, np.float32)).cuda()
    d_beads = None if beads is None else torch.as_tensor(np.asarray(beads, np.int32)).cuda()
    cost = torch.empty(n, device="cuda")
    grad = torch.empty(n, 3, device="cuda")
    rc = t.lib.QTrkB200ZLUTCostGradient(t.handle, d_rois.data_ptr(), w * 4, h * w * 4, abi.QTrkFloat, n,
                                        d_xyz.data_ptr(), None if d_beads is None else d_beads.data_ptr(),
                                        cost.data_ptr(), grad.data_ptr(), None if glut is None else glut.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == 0, t.GetWarnings()
    torch.cuda.synchronize()
    return cost.cpu().numpy().astype(np.float64), grad.cpu().numpy().astype(np.float64)


def _setup(weights=False):
    g = load("roi60_f32.npz")
    s, lut, mode = g["settings"], np.ascontiguousarray(g["lut"], np.float32), int(g["mode"])
    rois = g["rois"].astype(np.float32)
    t = QTrkInstance(s)
    t.SetRadialZLUT(lut)
    t.SetLocalizationMode(mode)
    w = None
    if weights:
        w = np.linspace(0.6, 1.4, lut.shape[2]).astype(np.float32)
        t.SetRadialWeights(w)
    return g, s, lut, mode, rois, t, w


@pytest.mark.parametrize("weights", [False, True])
def test_cost_gradient_matches_fp64_oracle(port, weights):
    torch = _torch()
    g, s, lut, mode, rois, t, w = _setup(weights)
    try:
        loc = t.Localize(rois)
        rng = np.random.default_rng(3)
        xyz = np.stack([loc["pos"][:, 0], loc["pos"][:, 1], loc["pos"][:, 2]], 1).astype(np.float64)
        xyz += rng.uniform([-0.3, -0.3, -0.7], [0.3, 0.3, 0.7], xyz.shape)
        xyz[:, 2] = np.clip(xyz[:, 2], 0, lut.shape[1] - 1)
        xyz = xyz.astype(np.float32).astype(np.float64)
        glut = torch.zeros(lut.size, device="cuda")
        cost, grad = _cost_grad(t, _device_rois(rois), xyz, glut=glut)
        glut = glut.cpu().numpy().reshape(lut.shape[1:]).astype(np.float64)
    finally:
        t.Destroy()
    cc = port.computed_config(s)
    want_c, want_g, want_l = [], [], np.zeros(lut.shape[1:])
    for i, img in enumerate(rois.astype(np.float64)):
        c, gr, gl = port.zcost_grad(img, img.mean(), xyz[i], lut[0], cc.zlut_angularsteps, s.zlut_minradius,
                                    cc.zlut_maxradius, weights=w, normalize=True, want_lut_grad=True)
        want_c.append(c)
        want_g.append(gr)
        want_l += gl
    want_c, want_g = np.array(want_c), np.array(want_g)
    np.testing.assert_allclose(cost, want_c, rtol=2e-4, atol=1e-6)
    scale = np.abs(want_g).max(1, keepdims=True)
    assert (np.abs(grad - want_g) <= 2e-3 * scale + 1e-5).all(), np.abs(grad - want_g).max()
    np.testing.assert_allclose(glut, want_l, rtol=0, atol=2e-3 * np.abs(want_l).max())


def test_cost_gradient_finite_differences():
    """Central differences with step 1e-3 (x, y in px, z in planes; LUT entries)."""
    torch = _torch()
    g, s, lut, mode, rois, t, w = _setup()
    try:
        loc = t.Localize(rois)
        xyz = np.stack([loc["pos"][:, 0] + 0.2, loc["pos"][:, 1] - 0.15, loc["pos"][:, 2] + 0.3], 1)
        d = _device_rois(rois)
        cost, grad = _cost_grad(t, d, xyz)
        h = 1e-3
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            cp, _ = _cost_grad(t, d, xyz + e)
            cm, _ = _cost_grad(t, d, xyz - e)
            fd = (cp - cm) / (2 * h)
            # bilinear interpolation is piecewise linear: samples crossing a pixel edge inside the
            # step bend the difference quotient, by a few percent at most
            tol = 0.05 * np.abs(grad[:, k]) + 0.02 * np.abs(grad).max(1) + 1e-4
            assert (np.abs(fd - grad[:, k]) <= tol).mean() >= 0.9, (k, np.abs(fd - grad[:, k]).max())
        # LUT: the cost is quadratic in the LUT, so the difference quotient is exact up to rounding
        glut = torch.zeros(lut.size, device="cuda")
        _cost_grad(t, d, xyz[:4], glut=glut)
        glut = glut.cpu().numpy().reshape(lut.shape[1:])
        base = _cost_grad(t, d, xyz[:4])[0].sum()
        iz = int(np.floor(xyz[0, 2]))
        for (pl, b) in [(iz, 3), (iz + 1, 10), (iz, 25)]:
            lp, lm = lut.copy(), lut.copy()
            lp[0, pl, b] += h
            lm[0, pl, b] -= h
            t.SetRadialZLUT(lp)
            cp = _cost_grad(t, d, xyz[:4])[0].sum()
            t.SetRadialZLUT(lm)
            cm = _cost_grad(t, d, xyz[:4])[0].sum()
            fd = (cp - cm) / (float(lp[0, pl, b]) - float(lm[0, pl, b]))
            assert abs(fd - glut[pl, b]) <= 2e-2 * abs(glut[pl, b]) + 2e-3 * np.abs(glut).max(), (pl, b, fd, glut[pl, b])
        t.SetRadialZLUT(lut)
        assert abs(_cost_grad(t, d, xyz[:4])[0].sum() - base) < 1e-6 * max(1.0, base)
    finally:
        t.Destroy()


def test_autograd_function_and_lut_steps():
    """A torch.autograd.Function over the C ABI (harness only): backward gives the kernel's
    gradients, and LUT gradient steps lower the total cost."""
    torch = _torch()
    g, s, lut, mode, rois, t, w = _setup()

    class ZCost(torch.autograd.Function):
        @staticmethod
        def forward(ctx, xyz, lut_t):
            t.SetRadialZLUT(lut_t.detach().cpu().numpy())
            n = xyz.shape[0]
            cost = torch.empty(n, device="cuda")
            grad = torch.empty(n, 3, device="cuda")
            glut = torch.zeros(lut_t.numel(), device="cuda")
            rc = t.lib.QTrkB200ZLUTCostGradient(t.handle, d.data_ptr(), 240, 14400, abi.QTrkFloat, n,
                                                xyz.detach().contiguous().data_ptr(), None, cost.data_ptr(),
                                                grad.data_ptr(), glut.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert rc == 0
            ctx.save_for_backward(grad, glut.view_as(lut_t))
            return cost

        @staticmethod
        def backward(ctx, gout):
            grad, glut = ctx.saved_tensors
            # d(sum_i gout_i cost_i)/dL = sum_i gout_i dcost_i/dL: exact for a uniform gout
            return gout[:, None] * grad, glut * gout.mean()

    try:
        d = _device_rois(rois)
        loc = t.Localize(rois)
        xyz = torch.tensor(np.stack([loc["pos"][:, 0], loc["pos"][:, 1], loc["pos"][:, 2]], 1), dtype=torch.float32,
                           device="cuda", requires_grad=True)
        L = torch.tensor(lut, device="cuda", requires_grad=True)
        total = ZCost.apply(xyz, L).sum()
        total.backward()
        cost, grad = _cost_grad(t, d, xyz.detach().cpu().numpy())
        assert np.allclose(xyz.grad.cpu().numpy(), grad, rtol=1e-6, atol=1e-9)
        history = [float(total.detach())]
        Lv = L.detach().clone()
        for _ in range(5):
            Lr = Lv.clone().requires_grad_(True)
            c = ZCost.apply(xyz.detach(), Lr).sum()
            c.backward()
            Lv = Lv - 0.2 * Lr.grad
            history.append(float(ZCost.apply(xyz.detach(), Lv).sum()))
        assert history[-1] < 0.8 * history[0], history
    finally:
        t.Destroy()


def _crossing_free(xyz, cc, s, h):
    """Per ROI and axis: True when moving that coordinate by +-h moves no profile sample across a
    pixel edge (x, y: every bin's samples; z: no plane boundary), so the cost is smooth there and a
    central difference converges to the derivative."""
    n = cc.zlut_angularsteps
    ang = 2 * float(np.float32(3.141593)) * np.arange(n) / n  # the oracle's FP64 sample positions
    d = np.stack([np.cos(ang), np.sin(ang)], 1)
    nb = cc.zlut_radialsteps
    minr, maxr = float(s.zlut_minradius), float(cc.zlut_maxradius)
    r = minr + (maxr - minr) / nb * np.arange(nb)
    out = np.zeros((len(xyz), 3), bool)
    for i, (x, y, z) in enumerate(xyz):
        for k, c in ((0, x), (1, y)):
            v = c + d[None, :, k] * r[:, None]
            out[i, k] = (np.floor(v - h) == np.floor(v + h)).all()
        out[i, 2] = np.floor(z - h) == np.floor(z + h)
    return out


def test_cost_gradient_tight_central_differences(port):
    """The GPU gradient against FP64 central differences of the FP64 oracle's cost with step 1e-5,
    on every (ROI, axis) where the step moves no sample across a pixel edge (there the cost is
    smooth and the quotient is the derivative to ~1e-9): within 2e-3 of the largest gradient
    component, the tolerance of the oracle-gradient comparison, for all of them. The oracle's
    analytic gradient meets the same differences to 1e-6 relative."""
    g, s, lut, mode, rois, t, w = _setup()
    try:
        loc = t.Localize(rois)
        xyz = np.stack([loc["pos"][:, 0] + 0.2, loc["pos"][:, 1] - 0.15, loc["pos"][:, 2] + 0.3], 1)
        xyz = xyz.astype(np.float32).astype(np.float64)
        _, grad = _cost_grad(t, _device_rois(rois), xyz)
    finally:
        t.Destroy()
    cc = port.computed_config(s)
    h = 1e-5
    smooth = _crossing_free(xyz, cc, s, h)
    assert smooth[:, :2].mean() > 0.5, smooth.mean(0)
    checked = 0
    for i, img in enumerate(rois.astype(np.float64)):
        mean = img.mean()
        _, g64, _ = port.zcost_grad(img, mean, xyz[i], lut[0], cc.zlut_angularsteps, s.zlut_minradius,
                                    cc.zlut_maxradius, normalize=True)
        scale = np.abs(g64).max()
        for k in range(3):
            if not smooth[i, k]:
                continue
            e = np.zeros(3)
            e[k] = h
            cp = port.zcost_grad(img, mean, xyz[i] + e, lut[0], cc.zlut_angularsteps, s.zlut_minradius,
                                 cc.zlut_maxradius, normalize=True)[0]
            cm = port.zcost_grad(img, mean, xyz[i] - e, lut[0], cc.zlut_angularsteps, s.zlut_minradius,
                                 cc.zlut_maxradius, normalize=True)[0]
            fd = (cp - cm) / (2 * h)
            assert abs(g64[k] - fd) <= 1e-6 * scale + 1e-9, (i, k, g64[k], fd)
            assert abs(grad[i, k] - fd) <= 2e-3 * scale + 1e-5, (i, k, grad[i, k], fd)
            checked += 1
    assert checked >= len(rois)


def test_joint_refine_mode_matches_oracle(port):
    g, s, lut, mode, rois, t, w = _setup()
    try:
        plain = t.Localize(rois)
        t.SetLocalizationMode(mode | abi.LT_B200_JointRefine)
        refined = t.Localize(rois)
        launches = t.KernelLaunchCount()
    finally:
        t.Destroy()
    assert launches > 0
    cc = port.computed_config(s)
    want = np.array([port.joint_refine(img.astype(np.float64), float(plain["imageMean"][i]), plain["pos"][i],
                                       lut[0], cc.zlut_angularsteps, s.zlut_minradius, cc.zlut_maxradius,
                                       normalize=True, steps=5)
                     for i, img in enumerate(rois)])
    dxy = np.abs(refined["pos"][:, :2] - want[:, :2]).max(1)
    dz = np.abs(refined["pos"][:, 2] - want[:, 2])
    # the backtracking decisions can differ where FP32 and FP64 costs tie: most ROIs agree closely
    assert ((dxy < 2e-3) & (dz < 1e-2)).mean() >= 0.9, (dxy.max(), dz.max())
    assert np.abs(refined["pos"][:, :2] - plain["pos"][:, :2]).max() < 0.5
    assert not np.array_equal(refined["pos"], plain["pos"])


def test_joint_refine_accuracy_vs_plain_fit():
    """On 2,000 synthetic 60x60 ROIs with known truth: refined z no worse than the 7-point fit."""
    wl = synth.roi60_f32(2000, seed=77)
    with QTrkInstance(wl.settings) as t:
        t.SetRadialZLUTSize(1, wl.lut_stack.shape[0])
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for p in range(wl.lut_stack.shape[0]):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        t.SetLocalizationMode(wl.mode)
        plain = t.Localize(wl.rois)
        t.SetLocalizationMode(wl.mode | abi.LT_B200_JointRefine)
        refined = t.Localize(wl.rois)
    truth = wl.true_xyz
    ok = np.abs(plain["pos"][:, 2] - truth[:, 2]) < 3
    ez_plain = np.median(np.abs(plain["pos"][ok, 2] - truth[ok, 2]))
    ez_ref = np.median(np.abs(refined["pos"][ok, 2] - truth[ok, 2]))
    exy_plain = np.median(np.hypot(*(plain["pos"][ok, :2] - truth[ok, :2]).T))
    exy_ref = np.median(np.hypot(*(refined["pos"][ok, :2] - truth[ok, :2]).T))
    print(f"median |dz| plain {ez_plain:.4f} refined {ez_ref:.4f}; |dxy| plain {exy_plain:.4f} refined {exy_ref:.4f}")
    assert ez_ref <= 1.05 * ez_plain and exy_ref <= 1.2 * exy_plain


def test_gaussian_nll_gradient_matches_oracle_and_differences(port):
    """QTrkB200GaussianNLLGradient against the FP64 oracle (oracle_gauss_nll_grad) and central
    differences of its own NLL."""
    torch = _torch()
    wl = synth.gauss16_f32(64, seed=91)
    rng = np.random.default_rng(4)
    params = np.stack([wl.true_xyz[:, 0] + rng.uniform(-0.3, 0.3, 64), wl.true_xyz[:, 1] + rng.uniform(-0.3, 0.3, 64),
                       wl.extra["photons"] * rng.uniform(0.8, 1.2, 64), np.full(64, 10.0) * rng.uniform(0.8, 1.2, 64),
                       rng.uniform(1.3, 1.7, 64)], 1).astype(np.float32)
    d = _device_rois(wl.rois)

    def run(p):
        dp = torch.as_tensor(np.ascontiguousarray(p, np.float32)).cuda()
        nll = torch.empty(len(p), device="cuda")
        grad = torch.empty(len(p), 5, device="cuda")
        rc = t.lib.QTrkB200GaussianNLLGradient(t.handle, d.data_ptr(), 64, 1024, abi.QTrkFloat, len(p), dp.data_ptr(),
                                               nll.data_ptr(), grad.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        return nll.cpu().numpy().astype(np.float64), grad.cpu().numpy().astype(np.float64)

    with QTrkInstance(wl.settings) as t:
        nll, grad = run(params)
        want = [port.gauss_nll_grad(img.astype(np.float64), params[i].astype(np.float64)) for i, img in enumerate(wl.rois)]
        want_n = np.array([w[0] for w in want])
        want_g = np.array([w[1] for w in want])
        np.testing.assert_allclose(nll, want_n, rtol=2e-5, atol=1e-2)
        scale = np.abs(want_g).max(1, keepdims=True)
        assert (np.abs(grad - want_g) <= 2e-3 * scale + 1e-3).all(), np.abs(grad - want_g).max()
        for k, h in enumerate((1e-3, 1e-3, 1.0, 0.05, 1e-3)):
            e = np.zeros(5, np.float32)
            e[k] = h
            fd = (run(params + e)[0] - run(params - e)[0]) / (2 * h)
            tol = 0.02 * np.abs(grad[:, k]) + 0.01 * np.abs(grad).max(1) * (1 if k != 2 else 0.01) + 0.05
            assert (np.abs(fd - grad[:, k]) <= tol).mean() >= 0.9, (k, np.abs(fd - grad[:, k]).max())
