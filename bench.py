"""Benchmark: COM + QI + Z-LUT localization of 100x100 ROIs on B200.

Workload (one step): 10,000 ROIs of 100x100 uint16 (12-bit; background 200, amplitude
2000, Poisson noise; seeded synthetic images in place of camera data), COM, then QI
with 4 iterations (64 radial x 51 angular steps per quadrant, radius 3-47 px), then the
radial profile (64 bins x 206 angles) matched against a 200-plane Z-LUT (plain form:
FP32 profiles, FP64-accumulated scores) and the 7-point quadratic fit.

* value   — ROIs/s with the ROI stack resident in HBM: one QTrkB200LocalizeDevice call
            (one kernel launch) per step, timed with CUDA events on the launching stream.
            The stack (200 MB) is larger than L2 (126 MB), so every step streams from HBM.
* e2e     — ROIs/s through the public C ABI with host buffers: per step QTrkScheduleFrame
            of a pinned 10000x10000 u16 frame holding the 10,000 ROIs (host->device copy
            inside the timed region), QTrkFlush, and QTrkFetchResults of a frame's 10,000
            results (device->host copy inside), with one frame in flight as an acquisition
            loop runs it (frame k+1 is handed over before frame k's results are read; the
            timed region ends after the last frame's results). The one-frame-at-a-time rate
            and the box's plain pinned copy rate of the frame are reported beside it.
* roofline — the localization kernel's algorithmic bytes (20,081 B per ROI: pixels +
            job + result + LUT share) per launch / its mean launch time, against the
            measured HBM copy bandwidth.
* cpu_baseline — the reference's own CPU tracker (oracle/_ref, QueuedCPUTracker with
            all host threads, and with one) on a bounded sample of the same workload.
* methods — the same device-resident steps with the tensor-core Z match (BF16 and TF32
            operands); `chosen` is the fastest form within 1 nm of the plain one.
* serving, workloads — the request server (paced and saturated) and the other workloads
            (Gaussian MLE, BuildLUT, adjoint, LUT refinement), rank 0 at N=1 only.

`--impl reference` times the reference CPU tracker alone and prints its line.
Multi-GPU (torchrun): replicas; every rank localizes its own 10,000 ROIs, no collective
in the data path; time = max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ROIs/s (COM+QI+ZLUT, 100^2 ROI) plain vs chosen at <=1 nm err; p99 frame latency"
UNIT = "ROIs/s"
N_ROIS = 10000
BYTES_PER_ROI = 100 * 100 * 2 + 52 + 24 + (200 * 64 * 4) / N_ROIS  # algorithmic bytes (20,081 B)
PIXEL_NM = 100.0  # stated pixel size for nm error reporting


_STDOUT_FD = None


def claim_stdout() -> None:
    """Send everything the process writes to stdout (the reference's C++ tracker prints its thread
    count there) to stderr, keeping the original stdout for the one bench line."""
    global _STDOUT_FD
    if _STDOUT_FD is None:
        sys.stdout.flush()
        _STDOUT_FD = os.dup(1)
        os.dup2(2, 1)


def emit(line: dict) -> None:
    data = (json.dumps(line) + "\n").encode()
    if _STDOUT_FD is None:
        sys.stdout.write(data.decode())
        sys.stdout.flush()
    else:
        os.write(_STDOUT_FD, data)


def _robust_sigma(e: np.ndarray) -> float:
    e = e[np.isfinite(e)]
    return float(1.4826 * np.median(np.abs(e - np.median(e))))


def _crlb(mu: np.ndarray, dmu: list) -> np.ndarray:
    """Poisson Fisher information I_ij = sum_pixels dmu_i dmu_j / mu of each image (the expression of
    SampleFisherMatrix, cputrack/FisherMatrix.h:48-105) and the diagonal of its inverse (the CRLB)."""
    n = mu.shape[0]
    k = len(dmu)
    inv_mu = np.where(mu > 1e-9, 1.0 / np.maximum(mu, 1e-9), 0.0).reshape(n, -1)
    d = np.stack([x.reshape(n, -1) for x in dmu], 1)  # (n, k, pixels)
    fisher = np.einsum("nip,njp,np->nij", d, d, inv_mu)
    return np.linalg.inv(fisher)[:, range(k), range(k)]


def crlb_radial_workload(true_xyz: np.ndarray, res: np.ndarray, m: int = 1000) -> dict:
    """CRLB of x, y, z for the 100x100 u16 bead images (the generating model: 200 + 2000 p(r; 0.25 z),
    Poisson), derivatives by central differences, against the measured spread of the errors."""
    from qtrk_b200 import synth

    m = min(m, len(true_xyz))
    var = np.zeros((m, 3))
    h = 1e-4
    for a in range(0, m, 100):
        b = min(m, a + 100)
        x, y, z = (true_xyz[a:b, i] for i in range(3))
        f = lambda dx, dy, dz: synth.render(100, 100, x + dx, y + dy, 0.25 * (z + dz), 200.0, 2000.0)
        mu = f(0, 0, 0)
        dmu = [(f(h, 0, 0) - f(-h, 0, 0)) / (2 * h), (f(0, h, 0) - f(0, -h, 0)) / (2 * h),
               (f(0, 0, h) - f(0, 0, -h)) / (2 * h)]
        var[a:b] = _crlb(mu, dmu)
    e = res["pos"][:m].astype(np.float64) - true_xyz[:m]
    sx, sz = _robust_sigma(e[:, 0]), _robust_sigma(e[:, 2])
    cx, cz = float(np.sqrt(np.median(var[:, 0]))), float(np.sqrt(np.median(var[:, 2])))
    return {"rois": m, "model": "Poisson Fisher information of the generating image model at the true position",
            "sqrt_crlb_x_nm": cx * PIXEL_NM, "sqrt_crlb_z_planes": cz,
            "measured_sigma_x_nm": sx * PIXEL_NM, "measured_sigma_z_planes": sz,
            "x_sigma_over_crlb": sx / cx, "z_sigma_over_crlb": sz / cz}


def crlb_gauss_workload(wl, res: np.ndarray, m: int = 5000) -> dict:
    """CRLB of x for the 16x16 Gaussian spots (x, y, I0, bg free) against the MLE's measured spread."""
    from qtrk_b200 import synth

    m = min(m, len(wl.rois))
    ph, bg, sig = wl.extra["photons"][:m], wl.extra["bg"], wl.extra["sigma"]
    x, y = wl.true_xyz[:m, 0], wl.true_xyz[:m, 1]
    h = 1e-4
    f = lambda dx, dy: synth.gaussian_spots(m, 16, x + dx, y + dy, sig, ph, bg)
    mu = f(0, 0)
    dmu = [(f(h, 0) - f(-h, 0)) / (2 * h), (f(0, h) - f(0, -h)) / (2 * h), (mu - bg) / ph[:, None, None],
           np.ones_like(mu)]
    var = _crlb(mu, dmu)
    e = res["pos"][:m, 0].astype(np.float64) - x
    # errors scaled by each ROI's own bound, so the mixture of photon counts does not blur the ratio
    ratio = _robust_sigma(e / np.sqrt(var[:, 0]))
    return {"rois": m, "model": "Poisson Fisher information of the integrated Gaussian, x, y, I0, bg free",
            "median_sqrt_crlb_x_nm": float(np.sqrt(np.median(var[:, 0])) * PIXEL_NM),
            "x_error_over_crlb": ratio}


def host_cpu() -> dict:
    """The host CPU the baseline ran on: model name (from /proc/cpuinfo) and usable threads."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    try:
        nproc = len(os.sched_getaffinity(0))
    except AttributeError:
        nproc = os.cpu_count() or 1
    return {"model": model, "threads_available": nproc}


def workload_config(ws: int) -> dict:
    """The `config` of the bench line, the same for this library's arm and the reference arm."""
    return {"workload": "10,000 ROIs/step of 100x100 u16; COM + QI (4 it, 64 radial x 51 angular per quadrant) + "
                        "Z-LUT 200 planes x 64 bins (206 angles); Z match form = methods.chosen",
            "rois_per_step": N_ROIS, "lut_planes": 200, "l2": "inputs larger than L2 (200 MB per step)",
            "parallelism": f"replicas x{ws}"}


def dist_env():
    from qtrk_b200 import replicas

    e = replicas.env()
    return e.world_size, e.rank, e.local_rank


def issue_limits(profile_json: Path, kernel_ms: float, sm_mhz: float | None) -> dict:
    """What binds a kernel that is not HBM-bound: its warp instructions per launch over the SMs'
    issue capacity in the measured time (148 SMs x 4 schedulers x SM clock), and its shared-memory
    wavefronts over the shared-memory data pipe (one wavefront per SM per clock). The per-launch
    counts come from the ncu capture summarised in profiles/ (the same workload and kernel)."""
    out = {"binding_limit": None, "issue_frac": None, "smem_pipe_frac": None}
    if not profile_json.exists() or not sm_mhz or kernel_ms <= 0:
        return out
    d = json.loads(profile_json.read_text())
    cycles = sm_mhz * 1e6 * kernel_ms / 1e3
    if d.get("warp_instructions_per_launch"):
        out["issue_frac"] = d["warp_instructions_per_launch"] / (148 * 4 * cycles)
    if d.get("smem_wavefronts_per_launch"):
        out["smem_pipe_frac"] = d["smem_wavefronts_per_launch"] / (148 * cycles)
    fr = {"instruction issue": out["issue_frac"] or 0.0, "shared-memory pipe": out["smem_pipe_frac"] or 0.0}
    out["binding_limit"] = max(fr, key=fr.get)
    out["counts_source"] = str(profile_json.relative_to(ROOT))
    return out


def measured_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed regions run."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.active = False
        self.marks: list[tuple[float, float]] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            if self.active:
                self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(n: int, seed: int):
    from qtrk_b200 import synth

    return synth.roi100_u16(n, seed=seed)


def build_lut_on_gpu(wl):
    from qtrk_b200.tracker import QTrkInstance

    with QTrkInstance(wl.settings) as t:
        planes = wl.lut_stack.shape[0]
        t.SetRadialZLUTSize(1, planes)
        t.BeginLUT(True)
        for p in range(planes):
            t.BuildLUT(wl.lut_stack[p], p, known_pos=wl.lut_known_pos)
        t.FinalizeLUT()
        return t.GetRadialZLUT()


def cpu_reference_run(wl, lut, n_sample: int, threads: int = -1):
    """The reference CPU tracker (oracle/_ref) on the first n_sample ROIs; returns (ROIs/s, results, cores)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import RefOracle, cpu_count, ref_available

    if not ref_available():
        return None
    ref = RefOracle()
    s = wl.settings
    s.numThreads = threads
    cores = cpu_count() if threads < 0 else threads
    res, dt = ref.track(s, wl.mode, wl.rois[:n_sample], lut, return_seconds=True)
    s.numThreads = -1
    return n_sample / dt, res, cores


def cpu_port_run(wl, lut, n_sample: int):
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import PortOracle

    port = PortOracle()
    cc = port.computed_config(wl.settings)
    t0 = time.perf_counter()
    p = port.localize(cc, wl.mode, wl.rois[:n_sample], lut)
    return n_sample / (time.perf_counter() - t0), p


def _pinned_copy(a: np.ndarray):
    """(pinned torch tensor, numpy view of it) holding a copy of a."""
    import torch

    tdt = {np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.int16, np.dtype(np.float32): torch.float32}
    t = torch.empty(a.shape, dtype=tdt[a.dtype]).pin_memory()
    out = t.numpy().view(a.dtype)
    out[:] = a
    return t, out


class _Camera:
    """Pre-marshalled QTrkB200ServerSubmitFrame arguments of one instance's frames."""

    def __init__(self, idx, frames, positions, pdt):
        self.idx = idx
        pinned = [_pinned_copy(f) for f in frames]
        self._tensors = [t for t, _ in pinned]  # keeps the pinned allocations alive
        self.frames = [v for _, v in pinned]
        self.positions = positions
        self.pdt = pdt
        self.job = None

    def submit_args(self, k):
        f = self.frames[k % len(self.frames)]
        return (self.idx, f.ctypes.data_as(C.c_void_p), f.strides[0], f.shape[1], f.shape[0],
                self.positions.ctypes.data_as(C.c_void_p), self.positions.shape[0], self.pdt)


def serve_paced(server, lib, cams, fps: float, seconds: float, seed: int) -> dict:
    """Frames arrive as a Poisson process at `fps` per camera for `seconds`; a collector thread
    polls results. Latency percentiles come from the server (submission to results on the host)."""
    from qtrk_b200 import abi

    rng = np.random.Generator(np.random.PCG64(seed))
    events = []
    for c in cams:
        t = rng.exponential(1.0 / fps)
        k = 0
        while t < seconds:
            events.append((t, c, k))
            t += rng.exponential(1.0 / fps)
            k += 1
    events.sort(key=lambda e: e[0])
    job = abi.LocalizationJob()
    outstanding: list[int] = []
    lock = threading.Lock()
    done_flag = [False]
    got = [0, 0]
    bad: list[int] = []

    def collector():
        buf = (abi.LocalizationResult * 8192)()
        while True:
            with lock:
                ids = list(outstanding)
            if not ids and done_flag[0]:
                return
            for rid in ids:
                n = lib.QTrkB200ServerPoll(server, rid, buf, 8192)
                if n == -1:
                    continue
                with lock:
                    outstanding.remove(rid)
                if n < 0:
                    bad.append(rid)
                else:
                    got[0] += 1
                    got[1] += n
            time.sleep(0.0001)

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    late = []
    t0 = time.perf_counter()
    for t, c, k in events:
        while True:
            now = time.perf_counter() - t0
            if now >= t:
                break
            if t - now > 0.0005:
                time.sleep(0.0002)
        late.append(time.perf_counter() - t0 - t)
        job.frame = k
        rid = lib.QTrkB200ServerSubmitFrame(server, *c.submit_args(k), C.byref(job))
        if rid < 0:
            raise RuntimeError("QTrkB200ServerSubmitFrame failed")
        with lock:
            outstanding.append(rid)
    done_flag[0] = True
    th.join(timeout=120)
    if bad or th.is_alive():
        raise RuntimeError(f"serving: {len(bad)} failed requests, collector alive={th.is_alive()}")
    st = abi.QTrkB200ServeStats()
    lib.QTrkB200ServerGetStats(server, C.byref(st))
    return {"frames": st.frames, "rois": st.rois, "launches": st.launches, "graphs": st.graphs,
            "lanes": st.lanes, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "max_ms": st.max_ms,
            "rois_per_s": st.rois / st.elapsed_s if st.elapsed_s > 0 else None,
            "offered_frames_per_s": len(events) / seconds, "submit_late_p99_ms": float(np.percentile(late, 99) * 1e3)}


def serve_saturated(server, lib, cams, rounds: int) -> dict:
    """All frames submitted back to back (no pacing); ROIs/s from first submission to last result."""
    from qtrk_b200 import abi

    job = abi.LocalizationJob()
    ids = []
    for k in range(rounds):
        for c in cams:
            job.frame = k
            ids.append(lib.QTrkB200ServerSubmitFrame(server, *c.submit_args(k), C.byref(job)))
    buf = (abi.LocalizationResult * 8192)()
    deadline = time.monotonic() + 300
    for rid in ids:
        while True:
            n = lib.QTrkB200ServerPoll(server, rid, buf, 8192)
            if n >= 0:
                break
            if n < -1 or time.monotonic() > deadline:
                raise RuntimeError(f"saturated serving: request {rid} -> {n}")
    st = abi.QTrkB200ServeStats()
    lib.QTrkB200ServerGetStats(server, C.byref(st))
    return {"frames": st.frames, "rois": st.rois, "launches": st.launches,
            "rois_per_s": st.rois / st.elapsed_s, "elapsed_s": st.elapsed_s}


def _timed(stream, fn, steps: int, warmup: int) -> float:
    """Mean milliseconds per call of fn() on `stream` (CUDA events, after warm-up)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def gpu_calibration_stack(dev, nbeads: int, planes: int, w: int = 80, seed: int = 4):
    """The calibration stack of the BuildLUT workload rendered on the GPU: bead b at 40 + U(+-2),
    plane k at profile parameter 0.25 k, 200 + 2000 p + Poisson clipped to 4095, u16. Returns
    (device tensor (planes, nbeads, w, w) int16 holding u16 bits, centres)."""
    import torch

    g = torch.Generator(device=dev).manual_seed(seed)
    c = w / 2 + (torch.rand(nbeads, 2, device=dev, generator=g) * 4 - 2)
    ys = torch.arange(w, device=dev, dtype=torch.float32)
    out = torch.empty((planes, nbeads, w, w), dtype=torch.int16, device=dev)
    for k in range(planes):
        zp = 0.25 * k
        r = torch.sqrt((ys[None, None, :] - c[:, 0, None, None]) ** 2 + (ys[None, :, None] - c[:, 1, None, None]) ** 2)
        sg, per = 4.0 + 0.1 * zp, 6.0 + 0.05 * zp
        lam = (200.0 + 2000.0 * torch.exp(-r * r / (2 * sg * sg)) * torch.cos(2 * np.pi * r / per)).clamp_min(0)
        out[k] = torch.poisson(lam, generator=g).clamp_max(4095).to(torch.int16)
    return out, c.cpu().numpy()


def _ref_rate(fn, n: int) -> float:
    """ROIs/s of one timed call of fn() that processes n ROIs on the host (seconds measured inside)."""
    return n / fn()


def reference_cpu(kind: str, threads: int, **kw) -> dict | None:
    """The reference's own CPU tracker (oracle/_ref, QueuedCPUTracker) timed on this host for one of the
    BASELINE workloads: `kind` is "track" (kw: settings, mode, rois, lut) or "buildlut" (kw: settings,
    stack (planes, beads, H, W)). threads = -1 uses every host thread."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import RefOracle, cpu_count, ref_available

    from qtrk_b200 import abi

    if not ref_available():
        return None
    ref = RefOracle()
    st = kw["settings"]
    old = st.numThreads
    st.numThreads = threads
    try:
        if kind == "track":
            rois = kw["rois"]
            _, dt = ref.track(st, kw["mode"], rois, kw.get("lut"), return_seconds=True)
            n = rois.shape[0]
        else:
            stack = kw["stack"]
            t0 = time.perf_counter()
            ref.build_lut(st, stack, abi.BUILDLUT_NORMALIZE)
            dt = time.perf_counter() - t0
            n = stack.shape[0] * stack.shape[1]
    finally:
        st.numThreads = old
    cores = cpu_count() if threads < 0 else threads
    return {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "reference", "rois_timed": int(n),
            "seconds": dt}


def workloads_bench(dev, steps: int, warmup: int) -> dict:
    """The other workloads: the Gaussian MLE (100,000 16x16 f32 ROIs, 4- and 5-parameter forms), BuildLUT
    of a 256-bead x 200-plane 80x80 u16 calibration stack from host memory, the adjoint over that stack,
    and 20 iterations of LUT refinement on it."""
    import torch

    from qtrk_b200 import abi, synth
    from qtrk_b200.tracker import QTrkInstance

    out = {}
    launches = 0
    stream = torch.cuda.current_stream(dev)
    # ---- Gaussian MLE ----
    n = 100000
    wl = synth.gauss16_f32(n, seed=3)
    d_rois = torch.from_numpy(wl.rois).to(dev)
    d_res = torch.empty(n * 52, dtype=torch.uint8, device=dev)
    s = wl.settings
    s.cuda_device = dev.index
    for name, mode in (("gauss_mle_4p", abi.LT_Gaussian2D), ("gauss_mle_5p", abi.LT_Gaussian2D | abi.LT_B200_Gaussian5P)):
        with QTrkInstance(s) as t:
            t.SetLocalizationMode(mode)
            l0 = t.KernelLaunchCount()
            ms = _timed(stream, lambda: t.LocalizeDevice(d_rois.data_ptr(), 64, 1024, abi.QTrkFloat, n, d_res.data_ptr(),
                                                         stream=stream.cuda_stream), steps, warmup)
            launches += t.KernelLaunchCount() - l0
        res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)
        err = np.hypot(res["pos"][:, 0] - wl.true_xyz[:, 0], res["pos"][:, 1] - wl.true_xyz[:, 1])
        out[name] = {"workload": f"{n:,} ROIs 16x16 f32, sigma 1.5, 8 iterations, device-resident",
                     "rois_per_s": n / (ms / 1e3), "ms_per_launch": ms,
                     "median_xy_err_nm_vs_truth": float(np.nanmedian(err) * PIXEL_NM),
                     "non_finite_fraction": float(np.mean(~np.isfinite(err))),
                     "crlb": crlb_gauss_workload(wl, res)}
        if mode == abi.LT_Gaussian2D:  # the reference has the 4-parameter form only (LT_Gaussian2D)
            cb = reference_cpu("track", -1, settings=s, mode=mode, rois=wl.rois)
            if cb is not None:
                cb["host"] = host_cpu()
                cb["sample"] = f"all {n:,} ROIs of the workload, QueuedCPUTracker numThreads=-1"
                one = reference_cpu("track", 1, settings=s, mode=mode, rois=wl.rois[:5000])
                one["sample"] = "first 5,000 ROIs, numThreads=1"
                cb["single_thread"] = one
            out[name]["cpu_baseline"] = cb
    del d_rois, d_res
    # ---- BuildLUT / adjoint / LUT refinement on a 256 x 200 calibration stack ----
    nbeads, planes = 256, 200
    d_stack, _ = gpu_calibration_stack(dev, nbeads, planes)
    host = torch.empty(d_stack.shape, dtype=torch.int16).pin_memory()
    host.copy_(d_stack)
    hs = host.numpy().view(np.uint16)
    cs = synth.calib_stack_80x80(1, 1, noise=False)[0]
    cs.cuda_device = dev.index
    with QTrkInstance(cs) as t:
        t.SetLocalizationMode(synth.MODE_QI_Z)
        t.SetRadialZLUTSize(nbeads, planes)
        l0 = t.KernelLaunchCount()
        times = []
        for _ in range(2):  # the first build also allocates the instance's staging buffers
            t.SetRadialZLUTSize(nbeads, planes)  # a zeroed LUT: BuildLUT adds to the LUT's rows
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            t.BeginLUT(abi.BUILDLUT_NORMALIZE)
            for k in range(planes):
                t.BuildLUT(hs[k], k)
            t.FinalizeLUT()
            lut = t.GetRadialZLUT()  # waits for the LUT
            times.append(time.perf_counter() - t0)
        # the same build through QTrkB200BuildLUTAsync (the stack stays untouched until FinalizeLUT)
        t.SetRadialZLUTSize(nbeads, planes)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t.BeginLUT(abi.BUILDLUT_NORMALIZE)
        for k in range(planes):
            t.BuildLUTAsync(hs[k], k)
        t.FinalizeLUT()
        lut_async = t.GetRadialZLUT()
        t_async = time.perf_counter() - t0
        d_plane = torch.empty_like(d_stack[0])
        copy_ms = _timed(stream, lambda: d_plane.copy_(host[0], non_blocking=True), 20, 3)
        out["buildlut_256x200_80x80_u16"] = {
            "workload": "BeginLUT / 200 x BuildLUT(256 ROIs 80x80 u16 from pinned host memory) / FinalizeLUT, "
                        "second build on the instance",
            "rois_per_s": nbeads * planes / times[1], "seconds": times[1], "first_build_seconds": times[0],
            "async": {"call": "QTrkB200BuildLUTAsync (returns once the plane is queued; the caller keeps the stack "
                              "until FinalizeLUT)", "rois_per_s": nbeads * planes / t_async, "seconds": t_async,
                      "lut_equals_sync_build": bool(np.array_equal(lut_async, lut))},
            "copy_bound_rois_per_s": nbeads / (copy_ms / 1e3), "lut_shape": list(lut.shape)}
        cb = reference_cpu("buildlut", -1, settings=cs, stack=hs[:40])
        if cb is not None:
            cb["host"] = host_cpu()
            cb["sample"] = ("BeginLUT / 40 x BuildLUT(256 ROIs) / FinalizeLUT (planes 0-39 of the stack); the "
                            "reference's BuildLUT spreads each plane's beads over every host thread whatever "
                            "numThreads says (parallel_for, threads.h:252-261)")
        out["buildlut_256x200_80x80_u16"]["cpu_baseline"] = cb
        del d_plane
        flat = d_stack.view(-1, 80, 80)
        xyz = torch.zeros(nbeads * planes, 3, device=dev)
        xyz[:, 0] = 40.0
        xyz[:, 1] = 40.0
        xyz[:, 2] = torch.arange(planes, device=dev, dtype=torch.float32).repeat_interleave(nbeads)
        beads = torch.arange(nbeads, device=dev, dtype=torch.int32).repeat(planes)
        cost = torch.empty(nbeads * planes, device=dev)
        grad = torch.empty(nbeads * planes, 3, device=dev)
        glut = torch.zeros(lut.size, device=dev)

        def adjoint():
            t.lib.QTrkB200ZLUTCostGradient(t.handle, flat.data_ptr(), 160, 12800, abi.QTrkU16, nbeads * planes,
                                           xyz.data_ptr(), beads.data_ptr(), cost.data_ptr(), grad.data_ptr(),
                                           glut.data_ptr(), stream.cuda_stream)

        ms = _timed(stream, adjoint, max(3, steps // 10), warmup)
        out["adjoint_256x200_80x80_u16"] = {"workload": "cost + d/dxyz + d/dLUT of 51,200 ROIs 80x80 u16 (device)",
                                            "rois_per_s": nbeads * planes / (ms / 1e3), "ms_per_launch": ms}
        iters = 20
        hist = np.zeros(iters + 1, np.float32)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t.lib.QTrkB200RefineZLUT(t.handle, flat.data_ptr(), 160, 12800, abi.QTrkU16, nbeads, planes, None, iters,
                                 C.c_float(3.0), None, hist.ctypes.data_as(C.c_void_p))
        ref_s = time.perf_counter() - t0
        out["lut_refine_256x200"] = {"workload": "QTrkB200RefineZLUT, 20 iterations, smoothness 3, 51,200 ROIs",
                                     "seconds": ref_s, "seconds_per_iteration": ref_s / iters,
                                     "objective_first": float(hist[0]), "objective_last": float(hist[-1])}
        launches += t.KernelLaunchCount() - l0
    # ---- config 1: 1,000 ROIs of 60x60 f32, COM + QI + Z-LUT 50 x 40 ----
    wl1 = synth.roi60_f32(1000, seed=1)
    s1 = wl1.settings
    s1.cuda_device = dev.index
    lut1 = build_lut_on_gpu(wl1)
    d1 = torch.from_numpy(wl1.rois).to(dev)
    r1 = torch.empty(1000 * 52, dtype=torch.uint8, device=dev)
    with QTrkInstance(s1) as t:
        t.SetRadialZLUT(lut1)
        t.SetLocalizationMode(wl1.mode)
        l0 = t.KernelLaunchCount()
        ms = _timed(stream, lambda: t.LocalizeDevice(d1.data_ptr(), 240, 14400, abi.QTrkFloat, 1000, r1.data_ptr(),
                                                     stream=stream.cuda_stream), steps, warmup)
        launches += t.KernelLaunchCount() - l0
    res1 = np.frombuffer(r1.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)
    out["roi60_f32_1000"] = {"workload": "1,000 ROIs 60x60 f32, COM + QI (4 it, 32 radial x 64 angular per "
                                         "quadrant) + Z-LUT 50 planes x 40 bins, device-resident, one launch",
                             "rois_per_s": 1000 / (ms / 1e3), "ms_per_launch": ms}
    cb = reference_cpu("track", -1, settings=s1, mode=wl1.mode, rois=wl1.rois, lut=lut1)
    if cb is not None:
        cb["host"] = host_cpu()
        cb["sample"] = "all 1,000 ROIs, QueuedCPUTracker numThreads=-1"
        one = reference_cpu("track", 1, settings=s1, mode=wl1.mode, rois=wl1.rois, lut=lut1)
        one["sample"] = "all 1,000 ROIs, numThreads=1"
        cb["single_thread"] = one
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import RefOracle

        rr = RefOracle().track(s1, wl1.mode, wl1.rois, lut1)
        # as in the parity tests: ROIs whose QI walked > 5 px from the COM (the bead was lost) and z
        # values beyond the LUT (parabola vertex extrapolated past its edge) are ill-conditioned in
        # the reference's own arithmetic and are counted, not compared
        conv = np.hypot(rr["pos"][:, 0] - rr["firstGuess"][:, 0], rr["pos"][:, 1] - rr["firstGuess"][:, 1]) <= 5
        zin = conv & (rr["pos"][:, 2] >= 0) & (rr["pos"][:, 2] <= lut1.shape[1] - 1)
        out["roi60_f32_1000"]["vs_reference_max_dxy_px"] = float(np.abs(res1["pos"][conv, :2] - rr["pos"][conv, :2]).max())
        out["roi60_f32_1000"]["vs_reference_max_dz_planes"] = float(np.abs(res1["pos"][zin, 2] - rr["pos"][zin, 2]).max())
        out["roi60_f32_1000"]["rois_where_qi_lost_the_bead"] = int((~conv).sum())
        out["roi60_f32_1000"]["rois_with_z_past_the_lut"] = int((conv & ~zin).sum())
    out["roi60_f32_1000"]["cpu_baseline"] = cb
    out["gpu_launches"] = int(launches)
    return out


COM_BYTES_PER_ROI = 100 * 100 * 2 + 52  # pixels in, result out (no job records: jobs pointer is null)


def com_only_bench(dev, settings, d_rois, n: int, steps: int, warmup: int, sm_mhz: float | None = None) -> dict:
    """LT_OnlyCOM on the headline stack (n ROIs of 100x100 u16 resident in HBM): the warp-per-ROI
    COM kernel (bulk-copied ROI buffers, shuffle reductions), one launch per step, with its roofline
    against the measured HBM copy rate."""
    import torch

    from qtrk_b200 import abi
    from qtrk_b200.tracker import QTrkInstance

    stream = torch.cuda.current_stream(dev)
    d_res = torch.empty(n * 52, dtype=torch.uint8, device=dev)
    with QTrkInstance(settings) as t:
        t.SetLocalizationMode(abi.LT_OnlyCOM)
        l0 = t.KernelLaunchCount()
        ms = _timed(stream, lambda: t.LocalizeDevice(d_rois.data_ptr(), 200, 20000, abi.QTrkU16, n, d_res.data_ptr(),
                                                     stream=stream.cuda_stream), steps, warmup)
        launches = t.KernelLaunchCount() - l0
    peaks, peak_kind = measured_peaks()
    achieved = COM_BYTES_PER_ROI * n / (ms / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "com_100x100_u16_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("dram_bytes_per_launch")
    roof_extra = issue_limits(tfile, ms, sm_mhz)
    return {"workload": f"LT_OnlyCOM, {n:,} ROIs of 100x100 u16 resident in HBM (200 MB > L2), one launch per step",
            "rois_per_s": n / (ms / 1e3), "ms_per_launch": ms, "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "qtrk::com_warp_kernel<1>", "kernel_ms": ms,
                         "bytes_per_roi": COM_BYTES_PER_ROI, **roof_extra}}


def serving_bench(dev, main_trk, main_rois, seconds: float, fps: float) -> dict:
    """The serving workload (four instances: 40/64/100/128 px, 2000/1000/300/50 beads per frame,
    u8/u16, LUTs of 100-200 planes, Poisson arrivals at `fps` per instance), plus one 100x100 u16
    instance with 1,000 beads per frame at the same rate."""
    from qtrk_b200 import abi, synth
    from qtrk_b200.tracker import QTrkInstance

    lib = main_trk.lib
    budget = 256 << 20
    fleet = synth.serving_fleet(2, seed=5)
    insts, cams = [], []
    launches0 = 0
    for i, cam in enumerate(fleet):
        cam.settings.cuda_device = dev.index
        lut = build_lut_on_gpu(cam)
        t = QTrkInstance(cam.settings)
        t.SetRadialZLUT(np.ascontiguousarray(np.broadcast_to(lut, (len(cam.positions),) + lut.shape[1:])))
        t.SetLocalizationMode(cam.mode)
        insts.append(t)
        cams.append(_Camera(i, cam.frames, cam.positions, abi.NUMPY_PDT[cam.frames[0].dtype]))
    out = {"budget_bytes": budget,
           "mix": {"workload": "4 instances: " + ", ".join(c.name for c in fleet) +
                   f"; Poisson arrivals at {fps:g} frames/s per instance; pinned host frames"}}
    launches0 = sum(t.KernelLaunchCount() for t in insts)
    srv = lib.QTrkB200ServerCreate(dev.index, budget)
    if not srv:
        raise RuntimeError("QTrkB200ServerCreate failed")
    for t in insts:
        lib.QTrkB200ServerAttach(srv, t.handle)
    # warm-up on the same server: graphs for the buckets that paced and saturated runs reach
    serve_paced(srv, lib, cams, fps, 0.5, seed=11)
    serve_saturated(srv, lib, cams, 8)
    lib.QTrkB200ServerResetStats(srv)
    out["mix"].update(serve_paced(srv, lib, cams, fps, seconds, seed=13))
    lib.QTrkB200ServerResetStats(srv)
    out["mix_saturated"] = serve_saturated(srv, lib, cams, 200)
    lib.QTrkB200ServerDestroy(srv)
    launches = sum(t.KernelLaunchCount() for t in insts) - launches0
    for t in insts:
        t.Destroy()

    # one 100x100 u16 instance, 1,000 beads per frame (32 x 32 grid, first 1,000 cells)
    side = 32
    ys, xs = np.divmod(np.arange(1000), side)
    frame = np.zeros((side * 100, side * 100), np.uint16)
    for b in range(1000):
        frame[ys[b] * 100:(ys[b] + 1) * 100, xs[b] * 100:(xs[b] + 1) * 100] = main_rois[b]
    pos = np.ascontiguousarray(np.stack([xs * 100, ys * 100], 1).astype(np.int32))
    cam = _Camera(0, [frame], pos, abi.QTrkU16)
    l1 = main_trk.KernelLaunchCount()
    srv = lib.QTrkB200ServerCreate(dev.index, budget)
    lib.QTrkB200ServerAttach(srv, main_trk.handle)
    serve_paced(srv, lib, [cam], fps, 0.3, seed=14)
    serve_saturated(srv, lib, [cam], 8)
    lib.QTrkB200ServerResetStats(srv)
    single = serve_paced(srv, lib, [cam], fps, seconds, seed=15)
    lib.QTrkB200ServerDestroy(srv)
    single["workload"] = f"1 instance: 100x100 u16, 1,000 beads per frame, Poisson arrivals at {fps:g} frames/s"
    out["single_100x100_u16_1000beads"] = single
    launches += main_trk.KernelLaunchCount() - l1
    out["gpu_launches"] = int(launches)
    out["latency"] = "per frame, from QTrkB200ServerSubmitFrame entry to the frame's results on the host"
    return out


def profile_workload(args) -> int:
    """Small device workloads for ncu captures (a few launches, a few hundred MB at most):
    tensorcore  2,048 ROIs 100x100 u16, COM + QI + Z with the tcgen05 Z match (LUT 200 x 64);
    com         10,000 ROIs 100x100 u16 (200 MB), LT_OnlyCOM (the streaming COM kernel);
    gauss5      100,000 ROIs 16x16 f32, 5-parameter Gaussian MLE;
    adjoint     2,048 ROIs 100x100 u16, QTrkB200ZLUTCostGradient with the LUT gradient;
    beadconv    QTrkFindBeads on a 2048 x 2048 frame with a 100 px sample."""
    import torch

    from qtrk_b200 import abi, synth
    from qtrk_b200.tracker import QTrkInstance, load_library

    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    total = args.warmup + args.steps
    if args.profile_workload == "com":
        n = N_ROIS
        wl = make_workload(n, seed=2)
        d = torch.from_numpy(wl.rois.view(np.int16)).to(dev)
        res = torch.empty(n * 52, dtype=torch.uint8, device=dev)
        with QTrkInstance(wl.settings) as t:
            t.SetLocalizationMode(abi.LT_OnlyCOM)
            ms = _timed(stream, lambda: t.LocalizeDevice(d.data_ptr(), 200, 20000, abi.QTrkU16, n, res.data_ptr(),
                                                         stream=stream.cuda_stream), args.steps, args.warmup)
    elif args.profile_workload in ("tensorcore", "adjoint"):
        n = 2048
        wl = make_workload(n, seed=2)
        lut = build_lut_on_gpu(wl)
        d = torch.from_numpy(wl.rois.view(np.int16)).to(dev)
        with QTrkInstance(wl.settings) as t:
            t.SetRadialZLUT(lut)
            if args.profile_workload == "tensorcore":
                t.SetLocalizationMode(wl.mode | abi.LT_B200_ZMatchBF16)
                res = torch.empty(n * 52, dtype=torch.uint8, device=dev)
                f = lambda: t.LocalizeDevice(d.data_ptr(), 200, 20000, abi.QTrkU16, n, res.data_ptr(),
                                             stream=stream.cuda_stream)
            else:
                t.SetLocalizationMode(wl.mode)
                xyz = torch.from_numpy(wl.true_xyz.astype(np.float32)).to(dev)
                cost, grad = torch.empty(n, device=dev), torch.empty(n, 3, device=dev)
                glut = torch.zeros(lut.size, device=dev)
                f = lambda: t.lib.QTrkB200ZLUTCostGradient(t.handle, d.data_ptr(), 200, 20000, abi.QTrkU16, n,
                                                           xyz.data_ptr(), None, cost.data_ptr(), grad.data_ptr(),
                                                           glut.data_ptr(), stream.cuda_stream)
            ms = _timed(stream, f, args.steps, args.warmup)
    elif args.profile_workload == "gauss5":
        n = 100000
        wl = synth.gauss16_f32(n, seed=3)
        d = torch.from_numpy(wl.rois).to(dev)
        res = torch.empty(n * 52, dtype=torch.uint8, device=dev)
        with QTrkInstance(wl.settings) as t:
            t.SetLocalizationMode(abi.LT_Gaussian2D | abi.LT_B200_Gaussian5P)
            ms = _timed(stream, lambda: t.LocalizeDevice(d.data_ptr(), 64, 1024, abi.QTrkFloat, n, res.data_ptr(),
                                                         stream=stream.cuda_stream), args.steps, args.warmup)
    else:
        lib = load_library()
        frame, centres = synth.bead_frame(2048, 2048, 120, 100, seed=9, noise=2.0)
        img = abi.ImageData(frame.ctypes.data_as(C.POINTER(C.c_float)), 2048, 2048)
        corner = (int(centres[0][0] - 50), int(centres[0][1] - 50))
        t0 = time.perf_counter()
        for _ in range(total):
            cnt = C.c_int()
            p = lib.QTrkFindBeads(C.byref(img), corner[0], corner[1], 100, 1.0, 0.5, C.byref(cnt), None)
            lib.QTrkFreeROIPositions(p)
        ms = (time.perf_counter() - t0) * 1e3 / total
    emit({"profile_workload": args.profile_workload, "ms_per_call": ms, "launches": total})
    return 0


def run_reference_arm(args) -> int:
    """The reference CPU tracker (QueuedCPUTracker, all host threads) on the whole 10,000-ROI step of
    this arm's workload, every step: the line's config is this arm's config unchanged."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    n = N_ROIS
    wl = make_workload(n, seed=2)
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import RefOracle, cpu_count, ref_available

    kind = "reference" if ref_available() else "port"
    if kind == "reference":
        ref = RefOracle()
        lut = ref.build_lut(wl.settings, wl.lut_stack, 4, known_pos=wl.lut_known_pos)
    else:
        from oracle import PortOracle

        port = PortOracle()
        lut = port.build_lut(port.computed_config(wl.settings), wl.lut_stack, 4,
                             known_pos=wl.lut_known_pos).astype(np.float32)
    rates = []
    n_port = 200  # the FP64 port is ~100x slower: a bounded sample per step when the reference is absent
    for step in range(args.warmup + args.steps):
        if kind == "reference":
            r = cpu_reference_run(wl, lut, n)
            rate = r[0]
        else:
            rate = cpu_port_run(wl, lut, n_port)[0]
        if step >= args.warmup:
            rates.append(rate)
    value = float(np.mean(rates))
    cores = cpu_count() if kind == "reference" else 1
    per_step = n if kind == "reference" else n_port
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * per_step / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(ws),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "host": host_cpu(),
                         "sample": (f"all {n:,} ROIs of the step, every step, QueuedCPUTracker with numThreads=-1"
                                    if kind == "reference" else
                                    f"first {n_port} ROIs of the step, FP64 restatement, 1 thread")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--sample", type=int, default=2000, help="ROIs per CPU-baseline step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ncu", action="store_true", help="short run for the profiler (no e2e / baseline)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="timed seconds of each paced serving run")
    ap.add_argument("--fps", type=float, default=500.0, help="frame rate per instance in the serving runs")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="skip the Gaussian / BuildLUT / adjoint workloads")
    ap.add_argument("--profile-workload", choices=["com", "tensorcore", "gauss5", "adjoint", "beadconv"],
                    help="run one small device workload --steps times for a profiler and exit")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    claim_stdout()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.profile_workload:
        return profile_workload(args)

    import torch

    from qtrk_b200 import replicas

    ws, rank, local = dist_env()
    torch.cuda.set_device(local if ws > 1 else 0)
    dev = torch.device("cuda", torch.cuda.current_device())
    replicas.init("nccl", timeout_s=300, device=dev)

    from qtrk_b200 import abi
    from qtrk_b200.tracker import QTrkInstance

    wl = make_workload(N_ROIS, seed=2 + 1000 * rank)
    lut = build_lut_on_gpu(wl)
    s = wl.settings
    s.cuda_device = dev.index
    trk = QTrkInstance(s)
    # One LUT per bead: QTrkScheduleFrame gives ROI i the LUT of bead i (QueuedTracker.cpp:105),
    # so the e2e frame path needs N_ROIS LUT rows; all are copies of the workload's 200x64 LUT. The
    # device-resident path passes no jobs (zlutIndex 0) and reads the first copy.
    if args.ncu:
        trk.SetRadialZLUT(lut)  # profiler runs use the device path only: keep the capture small
    else:
        trk.SetRadialZLUT(np.ascontiguousarray(np.broadcast_to(lut, (N_ROIS,) + lut.shape[1:])))
    trk.SetLocalizationMode(wl.mode)

    barrier = replicas.barrier

    def max_over_ranks(x: float) -> float:
        return replicas.reduce_max(x, device=dev)

    # ---- device-resident path (value) ----
    d_rois = torch.from_numpy(wl.rois.view(np.int16)).to(dev)
    d_res = torch.empty(N_ROIS * 52, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    launches0 = trk.KernelLaunchCount()

    def device_step():
        trk.LocalizeDevice(d_rois.data_ptr(), 200, 20000, abi.QTrkU16, N_ROIS, d_res.data_ptr(),
                           stream=stream.cuda_stream)

    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(dev.index)
    sampler.start()
    time.sleep(0.3)
    sampler.active = True
    barrier()
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        device_step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    dev_ms = ev0.elapsed_time(ev1)
    dev_ms_max = max_over_ranks(dev_ms)
    value = replicas.aggregate_rate(N_ROIS * args.steps, ws, dev_ms_max / 1e3)
    launches_value = trk.KernelLaunchCount() - launches0
    # per-launch duration of the localization kernel (one launch per step on this stream)
    kernel_ms = dev_ms / args.steps

    res_dev = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)

    # ---- the same steps with the tensor-core Z match (BF16 or TF32 cross term, exact re-score) ----
    methods = {"plain_fp32": {"rois_per_s": value, "ms_per_step": dev_ms_max / args.steps,
                              "max_dxy_nm_vs_plain": 0.0, "max_dz_planes_vs_plain": 0.0}}
    launches_tc = 0
    if not args.ncu:
        d_res_tc = torch.empty_like(d_res)
        for name, bit in (("tensor_core_bf16", abi.LT_B200_ZMatchBF16), ("tensor_core_tf32", abi.LT_B200_ZMatchTF32)):
            trk.SetLocalizationMode(wl.mode | bit)
            l0 = trk.KernelLaunchCount()

            def tc_step():
                trk.LocalizeDevice(d_rois.data_ptr(), 200, 20000, abi.QTrkU16, N_ROIS, d_res_tc.data_ptr(),
                                   stream=stream.cuda_stream)

            for _ in range(args.warmup):
                tc_step()
            steps_tc = max(1, min(args.steps, 50))
            barrier()
            torch.cuda.synchronize(dev)
            ev0.record(stream)
            for _ in range(steps_tc):
                tc_step()
            ev1.record(stream)
            torch.cuda.synchronize(dev)
            barrier()
            tc_ms = max_over_ranks(ev0.elapsed_time(ev1))
            launches_tc += trk.KernelLaunchCount() - l0
            res_tc = np.frombuffer(d_res_tc.cpu().numpy().tobytes(), dtype=abi.RESULT_DTYPE)
            methods[name] = {
                "rois_per_s": replicas.aggregate_rate(N_ROIS * steps_tc, ws, tc_ms / 1e3),
                "ms_per_step": tc_ms / steps_tc,
                "max_dxy_nm_vs_plain": float(np.abs(res_tc["pos"][:, :2] - res_dev["pos"][:, :2]).max() * PIXEL_NM),
                "max_dz_planes_vs_plain": float(np.abs(res_tc["pos"][:, 2] - res_dev["pos"][:, 2]).max())}
        trk.SetLocalizationMode(wl.mode)
    ok = {k: m for k, m in methods.items() if m["max_dxy_nm_vs_plain"] <= 1.0}
    chosen = max(ok, key=lambda k: ok[k]["rois_per_s"])
    methods["chosen"] = chosen

    # ---- end-to-end path through the C ABI with a pinned host frame ----
    e2e = None
    launches_e2e = 0
    if not args.ncu:
        side = int(np.sqrt(N_ROIS))
        frame_t = torch.empty((side * 100, side * 100), dtype=torch.int16).pin_memory()
        frame = frame_t.numpy().view(np.uint16)
        frame[:] = wl.rois.reshape(side, side, 100, 100).transpose(0, 2, 1, 3).reshape(side * 100, side * 100)
        ys, xs = np.meshgrid(np.arange(side) * 100, np.arange(side) * 100, indexing="ij")
        positions = np.ascontiguousarray(np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32))
        buf = (abi.LocalizationResult * N_ROIS)()
        job = abi.LocalizationJob()

        def schedule():
            n = trk.lib.QTrkScheduleFrame(trk.handle, frame.ctypes.data_as(C.c_void_p), frame.strides[0],
                                          frame.shape[1], frame.shape[0], positions.ctypes.data_as(C.c_void_p),
                                          N_ROIS, abi.QTrkU16, C.byref(job))
            assert n == N_ROIS
            trk.lib.QTrkFlush(trk.handle)

        def drain():
            """Read one frame's N_ROIS results (results come out in submission order)."""
            got = 0
            deadline = time.monotonic() + 60
            while got < N_ROIS:
                got += trk.lib.QTrkFetchResults(trk.handle, C.byref(buf, got * 52), N_ROIS - got)
                if time.monotonic() > deadline:
                    raise TimeoutError("e2e step did not complete")

        def serial(steps):
            for _ in range(steps):
                schedule()
                drain()

        def pipelined(steps):
            # an acquisition loop with one frame in flight: frame k+1 is handed over (its copy runs
            # while frame k's last band is localized) before frame k's results are read
            schedule()
            for _ in range(steps - 1):
                schedule()
                drain()
            drain()

        def timed_e2e(run):
            run(2)
            barrier()
            l0 = trk.KernelLaunchCount()
            t0 = time.perf_counter()
            run(args.e2e_steps)
            t1 = time.perf_counter()
            barrier()
            return max_over_ranks(t1 - t0), trk.KernelLaunchCount() - l0

        serial_s, serial_launches = timed_e2e(serial)
        e2e_s, launches_e2e = timed_e2e(pipelined)
        launches_e2e += serial_launches
        e2e = {"value": ws * N_ROIS * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(frame.nbytes + N_ROIS * (24 + 8)),
               "d2h_bytes_per_step": int(N_ROIS * 52),
               "path": "per step QTrkScheduleFrame(pinned 10000x10000 u16 frame, one LUT copy per bead) + QTrkFlush + "
                       "QTrkFetchResults of the previous frame's 10,000 results (one frame in flight); the timed "
                       "region ends after the last frame's results are read",
               "one_frame_at_a_time": {"value": ws * N_ROIS * args.e2e_steps / serial_s, "unit": UNIT,
                                       "path": "QTrkScheduleFrame + QTrkFlush + QTrkFetchResults of the same frame"}}
        # the host->device copy rate of this box for the same pinned frame (one plain copy): the
        # e2e path cannot be faster than moving the frame
        d_frame = torch.empty_like(frame_t, device=dev)
        copy_ms = _timed(stream, lambda: d_frame.copy_(frame_t, non_blocking=True), 5, 2)
        e2e["pinned_h2d_copy_gbs"] = frame.nbytes / (copy_ms / 1e3) / 1e9
        e2e["frame_copy_bound_rois_per_s"] = N_ROIS / (copy_ms / 1e3)
        del d_frame
        res_e2e = abi.results_to_numpy(buf, N_ROIS)
        res_e2e = res_e2e[np.argsort(res_e2e["zlutIndex"])]
        assert np.array_equal(res_e2e["pos"], res_dev["pos"]), "e2e and device-resident results differ"
    sampler.active = False
    clocks = sampler.stop()

    # ---- serving: frames of several instances as they arrive (rank 0, N=1) ----
    serving = None
    if rank == 0 and ws == 1 and not args.ncu and not args.no_serving:
        serving = serving_bench(dev, trk, wl.rois, args.serve_seconds, args.fps)
    workloads = None
    if rank == 0 and ws == 1 and not args.ncu and not args.no_workloads:
        workloads = workloads_bench(dev, args.steps, args.warmup)
    if rank == 0 and ws == 1 and not args.ncu:
        workloads = workloads or {"gpu_launches": 0}
        workloads["com_only_100x100_u16"] = com_only_bench(dev, s, d_rois, N_ROIS, args.steps, args.warmup,
                                                            clocks.get("sm_mhz"))
        workloads["gpu_launches"] += workloads["com_only_100x100_u16"]["gpu_launches"]

    # ---- roofline of the localization kernel ----
    peaks, peak_kind = measured_peaks()
    achieved = BYTES_PER_ROI * N_ROIS / (kernel_ms / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "localize_100x100_u16_traffic.json"
    if tfile.exists():
        traffic = json.loads(tfile.read_text()).get("dram_bytes_per_launch")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "qtrk::localize_qi_kernel<true>", "kernel_ms": kernel_ms,
                "bytes_per_roi": BYTES_PER_ROI}
    roofline.update(issue_limits(tfile, kernel_ms, clocks.get("sm_mhz")))

    # ---- accuracy vs truth (stated pixel size) ----
    err_xy = np.hypot(res_dev["pos"][:, 0] - wl.true_xyz[:, 0], res_dev["pos"][:, 1] - wl.true_xyz[:, 1])
    accuracy = {"median_xy_err_nm_vs_truth": float(np.median(err_xy) * PIXEL_NM),
                "median_z_err_planes_vs_truth": float(np.median(np.abs(res_dev["pos"][:, 2] - wl.true_xyz[:, 2]))),
                "pixel_nm": PIXEL_NM}
    if rank == 0 and not args.ncu:
        accuracy["crlb"] = crlb_radial_workload(wl.true_xyz, res_dev)

    # ---- error against the FP64 restatement of the algorithm, same LUT (rank 0) ----
    if rank == 0 and not args.ncu:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import PortOracle, port_available

        if port_available():
            port = PortOracle()
            m = min(2000, N_ROIS)
            fp64 = port.localize(port.computed_config(wl.settings), wl.mode, wl.rois[:m], lut)
            d = res_dev[:m]
            conv = np.hypot(fp64[:, 0] - fp64[:, 3], fp64[:, 1] - fp64[:, 4]) <= 5  # QI kept the bead
            dxy = np.abs(d["pos"][:, :2] - fp64[:, :2]).max(1) * PIXEL_NM
            dz = np.abs(d["pos"][:, 2] - fp64[:, 2])
            # a z past either end of the LUT is the vertex of a parabola fitted to a window clipped at
            # the LUT's edge, extrapolated tens of planes: ill-conditioned in any arithmetic (the
            # reference's own FP32 result differs from the FP64 one by ~0.01 plane there)
            inside = (fp64[:, 2] >= 0) & (fp64[:, 2] <= lut.shape[1] - 1)
            zok = conv & inside
            accuracy["vs_fp64_oracle"] = {
                "rois": m, "max_dxy_nm": float(dxy[conv].max()), "p99_dxy_nm": float(np.percentile(dxy[conv], 99)),
                "max_dz_planes": float(dz[zok].max()), "p99_dz_planes": float(np.percentile(dz[zok], 99)),
                "rois_beyond_z_tolerance": int((dz[zok] > 0.01).sum()),  # includes every Z argmax flip
                "rois_where_qi_lost_the_bead": int((~conv).sum()),
                "rois_with_z_extrapolated_past_the_lut": int((conv & ~inside).sum()),
                "max_dz_planes_extrapolated": float(dz[conv & ~inside].max()) if (conv & ~inside).any() else None}

    # ---- CPU baseline: the reference tracker on the host cores (rank 0, N=1) ----
    cpu_baseline = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.ncu:
        r = cpu_reference_run(wl, lut, args.sample)
        if r is not None:
            rate, ref_res, cores = r
            cpu_baseline = {"value": rate, "unit": UNIT, "cores": cores, "kind": "reference", "host": host_cpu(),
                            "sample": f"first {args.sample} ROIs of the same workload, reference QueuedCPUTracker "
                                      f"(oracle/_ref) with numThreads=-1"}
            one = cpu_reference_run(wl, lut, min(args.sample, 500), threads=1)
            cpu_baseline["single_thread"] = {"value": one[0], "unit": UNIT, "cores": 1,
                                             "sample": f"first {min(args.sample, 500)} ROIs, numThreads=1"}
            d = res_dev[: args.sample]
            dz_ref = np.abs(d["pos"][:, 2] - ref_res["pos"][:, 2])
            dz_ref = dz_ref[(ref_res["pos"][:, 2] >= 0) & (ref_res["pos"][:, 2] <= lut.shape[1] - 1)]  # as above
            accuracy["vs_reference_max_dxy_px"] = float(np.abs(d["pos"][:, :2] - ref_res["pos"][:, :2]).max())
            accuracy["vs_reference_max_dz_planes"] = float(dz_ref.max())
            accuracy["vs_reference_rois_beyond_z_tolerance"] = int((dz_ref > 0.01).sum())
            accuracy["vs_reference_max_dxy_nm"] = accuracy["vs_reference_max_dxy_px"] * PIXEL_NM
        else:
            rate, _ = cpu_port_run(wl, lut, 100)
            cpu_baseline = {"value": rate, "unit": UNIT, "cores": 1, "kind": "port",
                            "sample": "first 100 ROIs, FP64 restatement (oracle/qtrk_oracle.c), 1 thread"}

    line = {
        "metric": METRIC, "value": methods[chosen]["rois_per_s"], "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": methods[chosen]["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded Poisson bead images, 100x100 u16 bead ROIs)",
        "config": workload_config(ws),
        "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu_baseline,
        "gpu_launches": int(launches_value + launches_tc + launches_e2e +
                            (serving["gpu_launches"] if serving else 0) +
                            (workloads["gpu_launches"] if workloads else 0)),
        "clocks": clocks, "accuracy": accuracy, "methods": methods, "serving": serving,
        "p99_frame_latency_ms": serving["single_100x100_u16_1000beads"]["p99_ms"] if serving else None,
        "workloads": workloads,
    }
    trk.Destroy()
    if ws > 1:
        replicas.finalize()
    if rank == 0:
        emit(line)
    return 0


if __name__ == "__main__":
    sys.exit(main())
