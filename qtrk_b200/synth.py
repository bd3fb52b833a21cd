"""Seeded synthetic bead images for the benchmark workloads (ROI stacks, frames, calibration stacks).

No public dataset is involved: the reference measures on its own generated images
(cputrack-test/SharedTests.h:343-416 renders ROIs from a LUT and adds Poisson noise).
Here the radial bead profile is the analytic family

    p_z(r) = exp(-r^2 / (2 (4 + 0.1 z)^2)) * cos(2 pi r / (6 + 0.05 z))

rendered at pixel centres (r measured from the bead centre in pixel coordinates, the
convention of the reference's samplers), scaled, clamped at zero and Poisson-sampled
with numpy's PCG64 generator seeded per workload. The Z-LUT is built through the
tracker's own BeginLUT/BuildLUT/FinalizeLUT from noise-free images clamped the same way
(cputrack-test/SharedTests.h:35-65 builds its LUTs the same way).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import abi


def profile(r: np.ndarray, zp: np.ndarray | float) -> np.ndarray:
    s = 4.0 + 0.1 * zp
    per = 6.0 + 0.05 * zp
    return np.exp(-r * r / (2 * s * s)) * np.cos(2 * np.pi * r / per)


def render(w: int, h: int, cx: np.ndarray, cy: np.ndarray, zp: np.ndarray, bg: float, amp: float,
           dtype=np.float64) -> np.ndarray:
    """Noise-free expected pixel values, shape (n, h, w), clamped at 0 (float64 unless dtype says)."""
    ys = np.arange(h, dtype=dtype)[None, :, None]
    xs = np.arange(w, dtype=dtype)[None, None, :]
    cx = np.asarray(cx, dtype)[:, None, None]
    cy = np.asarray(cy, dtype)[:, None, None]
    r = np.sqrt((xs - cx) ** 2 + (ys - cy) ** 2)
    lam = dtype(bg) + dtype(amp) * profile(r, np.asarray(zp, dtype)[:, None, None])
    return np.maximum(lam, dtype(0))


@dataclass
class Workload:
    name: str
    settings: abi.QTrkSettings
    mode: int
    rois: np.ndarray            # (n, h, w) u8/u16/f32
    true_xyz: np.ndarray        # (n, 3): x, y in pixels, z in LUT planes
    lut_stack: np.ndarray | None = None   # (planes, 1, h, w) noise-free images for BuildLUT
    lut_known_pos: np.ndarray | None = None
    extra: dict = field(default_factory=dict)


def settings_roi60(**kw) -> abi.QTrkSettings:
    """60x60 ROIs, QI radius 3-28 px, 64 angular steps per quadrant, 40 radial steps
    (rounded to 32 by QTrkComputedConfig::Update, cputrack/QueuedTracker.cpp:20), Z-LUT
    40 bins over radius 3-28, 4 QI iterations."""
    s = abi.settings(width=60, height=60, qi_iterations=4, qi_minradius=3.0, qi_roi_coverage=28 / 30,
                     qi_radial_coverage=1.6, qi_angular_coverage=64.5 * 4 / (2 * np.pi * 28),
                     zlut_minradius=3.0, zlut_roi_coverage=28 / 30, zlut_radial_coverage=1.6 + 1e-4,
                     zlut_angular_coverage=0.7, cuda_device=-2, numThreads=-1)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def settings_roi100(**kw) -> abi.QTrkSettings:
    """100x100 ROIs, radius 3-47 px: QI 64 radial steps x 51 angular steps per quadrant,
    Z-LUT 64 bins x 206 angles, 4 QI iterations."""
    s = abi.settings(width=100, height=100, qi_iterations=4, qi_minradius=3.0, qi_roi_coverage=0.94,
                     qi_radial_coverage=1.4, qi_angular_coverage=0.7, zlut_minradius=3.0, zlut_roi_coverage=0.94,
                     zlut_radial_coverage=64.5 / 44.0, zlut_angular_coverage=0.7, cuda_device=-2, numThreads=-1)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


MODE_QI_Z = abi.LT_QI | abi.LT_LocalizeZ | abi.LT_NormalizeProfile


def roi60_f32(n: int = 1000, seed: int = 1) -> Workload:
    """1,000 ROIs 60x60 f32: centre (30,30)+U(+-3), z ~ U[5,45] planes, 10 + 100 p_z(r) + Poisson;
    Z-LUT 50 planes, plane k <-> z = k."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = h = 60
    cx = 30 + rng.uniform(-3, 3, n)
    cy = 30 + rng.uniform(-3, 3, n)
    z = rng.uniform(5, 45, n)
    rois = np.empty((n, h, w), np.float32)
    for a in range(0, n, 2048):
        b = min(n, a + 2048)
        lam = render(w, h, cx[a:b], cy[a:b], z[a:b], 10.0, 100.0)
        rois[a:b] = rng.poisson(lam).astype(np.float32)
    planes = 50
    kz = np.arange(planes, dtype=np.float64)
    stack = render(w, h, np.full(planes, w / 2), np.full(planes, h / 2), kz, 10.0, 100.0).astype(np.float32)
    return Workload("roi60-f32", settings_roi60(), MODE_QI_Z, rois, np.stack([cx, cy, z], 1),
                    stack[:, None], np.array([[w / 2, h / 2]], np.float32))


def roi100_u16(n: int = 10000, seed: int = 2) -> Workload:
    """10,000 ROIs 100x100 u16 (12-bit): 200 + 2000 p(r; 0.25 z) + Poisson, clipped to 4095;
    centre (50,50)+U(+-3), z ~ U[10,190] planes; Z-LUT 200 planes x 64 bins, plane k <-> 0.25 k."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = h = 100
    cx = 50 + rng.uniform(-3, 3, n)
    cy = 50 + rng.uniform(-3, 3, n)
    z = rng.uniform(10, 190, n)
    rois = np.empty((n, h, w), np.uint16)
    for a in range(0, n, 1024):
        b = min(n, a + 1024)
        lam = render(w, h, cx[a:b], cy[a:b], 0.25 * z[a:b], 200.0, 2000.0)
        rois[a:b] = np.minimum(rng.poisson(lam), 4095).astype(np.uint16)
    planes = 200
    kz = 0.25 * np.arange(planes, dtype=np.float64)
    stack = render(w, h, np.full(planes, w / 2), np.full(planes, h / 2), kz, 200.0, 2000.0).astype(np.float32)
    return Workload("roi100-u16", settings_roi100(), MODE_QI_Z, rois, np.stack([cx, cy, z], 1),
                    stack[:, None], np.array([[w / 2, h / 2]], np.float32))


def gaussian_spots(n: int, w: int, cx, cy, sigma: float, photons, bg: float) -> np.ndarray:
    """Integrated Gaussian spot (GenerateGaussianSpotImage, cputrack/utils.cpp:393-402) in FP64."""
    from math import sqrt

    from scipy.special import erf  # scipy is present in this image

    xs = np.arange(w, dtype=np.float64)
    k = 1.0 / sqrt(2.0) / sigma
    dx = 0.5 * (erf((xs[None, :] - cx[:, None] + 0.5) * k) - erf((xs[None, :] - cx[:, None] - 0.5) * k))
    dy = 0.5 * (erf((xs[None, :] - cy[:, None] + 0.5) * k) - erf((xs[None, :] - cy[:, None] - 0.5) * k))
    return bg + photons[:, None, None] * dy[:, :, None] * dx[:, None, :]


def gauss16_f32(n: int = 100000, seed: int = 3) -> Workload:
    """100,000 ROIs 16x16 f32: integrated Gaussian sigma 1.5, photons log-U[500,5000],
    background 10 photons/px, Poisson; centre 8 + U(+-2)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = 16
    cx = 8 + rng.uniform(-2, 2, n)
    cy = 8 + rng.uniform(-2, 2, n)
    ph = np.exp(rng.uniform(np.log(500), np.log(5000), n))
    rois = np.empty((n, w, w), np.float32)
    for a in range(0, n, 8192):
        b = min(n, a + 8192)
        rois[a:b] = rng.poisson(gaussian_spots(b - a, w, cx[a:b], cy[a:b], 1.5, ph[a:b], 10.0)).astype(np.float32)
    s = abi.settings(width=16, height=16, gauss2D_sigma=1.5, gauss2D_iterations=8, cuda_device=-2, numThreads=-1,
                     qi_minradius=1, zlut_minradius=1)
    return Workload("gauss16-f32", s, abi.LT_Gaussian2D, rois,
                    np.stack([cx, cy, np.zeros(n)], 1), extra={"photons": ph, "bg": 10.0, "sigma": 1.5})


def calib_stack_80x80(nbeads: int = 256, planes: int = 200, seed: int = 4, noise: bool = True) -> tuple:
    """Calibration stack: nbeads x planes ROIs of 80x80 u16, bead b at 40 + U(+-2) (fixed over z),
    plane k <-> profile parameter 0.25 k; 200 + 2000 p + Poisson, clipped to 4095.
    Returns (settings, stack (planes, nbeads, 80, 80) u16, centres (nbeads, 2))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w = 80
    cx = 40 + rng.uniform(-2, 2, nbeads)
    cy = 40 + rng.uniform(-2, 2, nbeads)
    stack = np.empty((planes, nbeads, w, w), np.uint16)
    for k in range(planes):
        lam = render(w, w, cx, cy, np.full(nbeads, 0.25 * k), 200.0, 2000.0)
        img = rng.poisson(lam) if noise else np.rint(lam)
        stack[k] = np.minimum(img, 4095).astype(np.uint16)
    s = abi.settings(width=80, height=80, qi_iterations=4, qi_minradius=3.0, qi_roi_coverage=0.9,
                     qi_radial_coverage=1.4, qi_angular_coverage=0.7, zlut_minradius=3.0, zlut_roi_coverage=0.9,
                     zlut_radial_coverage=48.5 / 33.0, zlut_angular_coverage=0.7, cuda_device=-2, numThreads=-1)
    return s, stack, np.stack([cx, cy], 1).astype(np.float32)


@dataclass
class ServedCamera:
    """One tracker instance of the serving workload: frames tiled with ROIs, its own LUT stack."""
    name: str
    settings: abi.QTrkSettings
    mode: int
    frames: list                # 2-D frames (u8/u16), ROIs tiled on a grid
    positions: np.ndarray       # (beads, 2) int32 ROI corners, the same in every frame
    lut_stack: np.ndarray       # (planes, 1, w, w) f32 noise-free images for BuildLUT
    lut_known_pos: np.ndarray


def settings_square(w: int, **kw) -> abi.QTrkSettings:
    """w x w ROIs with the radius span of settings_roi100 scaled to the ROI (3 px to 0.47 w)."""
    s = settings_roi100(width=w, height=w)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


SERVING_CAMERAS = ((40, np.uint8, 2000, 100), (64, np.uint16, 1000, 150), (100, np.uint16, 300, 200),
                   (128, np.uint8, 50, 200))


def serving_fleet(n_frames: int = 2, seed: int = 5, cameras=SERVING_CAMERAS) -> list:
    """Serving workload: four instances with ROI sizes 40/64/100/128 px, 2000/1000/300/50 beads per
    frame, u8/u16/u16/u8 pixels, LUTs of 100/150/200/200 planes. Bead image: background + amplitude
    p(r; 0.25 z) + Poisson (u8: 10 + 100 p, u16: 200 + 2000 p clipped to 4095); centres within
    +-2 px of the ROI centre, z uniform over the LUT's planes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    fleet = []
    for w, dt, beads, planes in cameras:
        bg, amp, top = (10.0, 100.0, 255) if dt == np.uint8 else (200.0, 2000.0, 4095)
        cols = int(np.ceil(np.sqrt(beads)))
        rows = (beads + cols - 1) // cols
        ys, xs = np.divmod(np.arange(beads), cols)
        positions = np.ascontiguousarray(np.stack([xs * w, ys * w], 1).astype(np.int32))
        frames = []
        for _ in range(n_frames):
            cx = w / 2 + rng.uniform(-2, 2, beads)
            cy = w / 2 + rng.uniform(-2, 2, beads)
            z = rng.uniform(0.05 * planes, 0.95 * planes, beads)
            lam = render(w, w, cx, cy, 0.25 * z, bg, amp, dtype=np.float32)
            rois = np.minimum(rng.poisson(lam), top).astype(dt)
            frame = np.zeros((rows * w, cols * w), dt)
            for b in range(beads):
                frame[ys[b] * w:(ys[b] + 1) * w, xs[b] * w:(xs[b] + 1) * w] = rois[b]
            frames.append(frame)
        kz = 0.25 * np.arange(planes, dtype=np.float64)
        stack = render(w, w, np.full(planes, w / 2), np.full(planes, w / 2), kz, bg, amp).astype(np.float32)
        fleet.append(ServedCamera(f"{w}x{w}-{np.dtype(dt).name}-{beads}beads", settings_square(w), MODE_QI_Z,
                                  frames, positions, stack[:, None], np.array([[w / 2, w / 2]], np.float32)))
    return fleet


def bead_frame(w: int = 320, h: int = 256, n_beads: int = 12, roi: int = 32, seed: int = 6, noise: float = 2.0):
    """A frame for the bead finder: n_beads bead images (10 + 100 p(r; z), z ~ U[5, 15]) at random
    non-overlapping positions at least one ROI from each other and inside the frame, plus
    Gaussian noise (sigma `noise`). Returns (frame f32, centres (n, 2) float64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = []
    tries = 0
    while len(centres) < n_beads and tries < 10000:
        tries += 1
        c = rng.uniform([roi, roi], [w - roi, h - roi])
        if all(np.hypot(*(c - o)) > 1.5 * roi for o in centres):
            centres.append(c)
    centres = np.array(centres)
    ys = np.arange(h, dtype=np.float64)[:, None]
    xs = np.arange(w, dtype=np.float64)[None, :]
    frame = np.full((h, w), 10.0)
    for (cx, cy), z in zip(centres, rng.uniform(5, 15, len(centres))):
        r = np.sqrt((xs - cx) ** 2 + (ys - cy) ** 2)
        frame += 100.0 * profile(r, z) * (r < roi)
    frame = np.maximum(frame + rng.normal(0, noise, frame.shape), 0)
    return frame.astype(np.float32), centres


def calibration_stack(nbeads: int = 16, planes: int = 60, jitter: float = 0.3, n_test: int = 400, seed: int = 8,
                      w: int = 80):
    """A calibration stack whose stage positions are off: plane k is recorded at z = k + d_k
    (d ~ N(0, jitter) planes), profile parameter 0.25 z; 80x80 u16 ROIs of nbeads beads (centres
    40 + U(+-2)), 200 + 2000 p + Poisson clipped to 4095; plus n_test held-out ROIs of the same beads
    at z ~ U[5, planes - 6]. Returns dict(settings, stack (planes, nbeads, w, w) u16, offsets (planes,),
    centres (nbeads, 2), test (n_test, w, w) u16, test_bead, test_z)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    cx = w / 2 + rng.uniform(-2, 2, nbeads)
    cy = w / 2 + rng.uniform(-2, 2, nbeads)
    off = rng.normal(0, jitter, planes)
    stack = np.empty((planes, nbeads, w, w), np.uint16)
    for k in range(planes):
        lam = render(w, w, cx, cy, np.full(nbeads, 0.25 * (k + off[k])), 200.0, 2000.0, dtype=np.float32)
        stack[k] = np.minimum(rng.poisson(lam), 4095).astype(np.uint16)
    tb = rng.integers(0, nbeads, n_test)
    tz = rng.uniform(5, planes - 6, n_test)
    lam = render(w, w, cx[tb], cy[tb], 0.25 * tz, 200.0, 2000.0, dtype=np.float32)
    test = np.minimum(rng.poisson(lam), 4095).astype(np.uint16)
    s = calib_stack_80x80(1, 1, noise=False)[0]
    return dict(settings=s, stack=stack, offsets=off, centres=np.stack([cx, cy], 1), test=test, test_bead=tb,
                test_z=tz)
