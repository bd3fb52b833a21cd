"""bench.py's accuracy helpers on the CPU: the Poisson CRLB against closed forms."""
import numpy as np

import bench
from qtrk_b200 import synth


def test_crlb_of_a_bright_gaussian_spot_is_the_pixelated_width_over_photons():
    """Background-free spot: var(x) -> (sigma^2 + 1/12) / N for a pixelated Gaussian (Mortensen et al.,
    Nat. Methods 7:377, 2010, with b -> 0); x, y, I0, bg all free."""
    n, w, sig, ph = 4, 32, 1.5, 1e5
    x = np.array([16.0, 16.3, 15.7, 16.5])
    y = np.array([16.0, 15.8, 16.2, 16.5])
    f = lambda dx, dy: synth.gaussian_spots(n, w, x + dx, y + dy, sig, np.full(n, ph), 1e-6)
    h = 1e-4
    mu = f(0, 0)
    dmu = [(f(h, 0) - f(-h, 0)) / (2 * h), (f(0, h) - f(0, -h)) / (2 * h), (mu - 1e-6) / ph, np.ones_like(mu)]
    var = bench._crlb(mu, dmu)
    want = (sig ** 2 + 1 / 12) / ph
    np.testing.assert_allclose(var[:, 0], want, rtol=0.03)
    np.testing.assert_allclose(var[:, 1], want, rtol=0.03)


def test_crlb_scales_inversely_with_intensity():
    """Doubling background and amplitude halves the variance (Fisher information is linear in the scale)."""
    x, y, z = np.array([50.2]), np.array([49.7]), np.array([30.0])
    h = 1e-4
    out = []
    for k in (1.0, 2.0):
        f = lambda dx, dy, dz: synth.render(100, 100, x + dx, y + dy, 0.25 * (z + dz), 200.0 * k, 2000.0 * k)
        mu = f(0, 0, 0)
        dmu = [(f(h, 0, 0) - f(-h, 0, 0)) / (2 * h), (f(0, h, 0) - f(0, -h, 0)) / (2 * h),
               (f(0, 0, h) - f(0, 0, -h)) / (2 * h)]
        out.append(bench._crlb(mu, dmu)[0])
    np.testing.assert_allclose(out[1], out[0] / 2, rtol=1e-6)


def test_robust_sigma_of_a_normal_sample():
    e = np.random.Generator(np.random.PCG64(1)).normal(0, 0.3, 200000)
    e[:100] = np.nan
    assert abs(bench._robust_sigma(e) - 0.3) < 0.005


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` runs on the host alone and prints exactly one JSON line with the
    keys the bench contract names (its own e2e, no host-device bytes)."""
    import json
    import subprocess
    import sys
    from pathlib import Path

    import pytest

    root = Path(__file__).resolve().parent.parent
    if not (root / "oracle" / "_ref" / "libqtrk_ref.so").exists() and not (root / "oracle" / "liboracle_port.so").exists():
        pytest.skip("oracle not built")
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
                        "--sample", "100"], capture_output=True, text=True, timeout=600, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["warmup"] >= 3 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_issue_limits_from_the_committed_profile_counts():
    """The bench line's issue and shared-memory fractions: warp instructions over 148 SMs x 4
    schedulers x clock x time, wavefronts over 148 x clock x time, and the larger one named."""
    import json

    for name in ("localize_100x100_u16_traffic.json", "com_100x100_u16_traffic.json"):
        path = bench.ROOT / "profiles" / name
        d = json.loads(path.read_text())
        out = bench.issue_limits(path, 1.0, 2000.0)  # 1 ms at 2 GHz: 2e6 cycles
        assert abs(out["issue_frac"] - d["warp_instructions_per_launch"] / (148 * 4 * 2e6)) < 1e-12
        assert abs(out["smem_pipe_frac"] - d["smem_wavefronts_per_launch"] / (148 * 2e6)) < 1e-12
        want = "instruction issue" if out["issue_frac"] >= out["smem_pipe_frac"] else "shared-memory pipe"
        assert out["binding_limit"] == want
        assert out["counts_source"] == f"profiles/{name}"
    # the fused kernel is bound by its shared-memory gathers, the COM-only kernel by issue
    fused = bench.issue_limits(bench.ROOT / "profiles" / "localize_100x100_u16_traffic.json", 1.003, 1965.0)
    com = bench.issue_limits(bench.ROOT / "profiles" / "com_100x100_u16_traffic.json", 0.0576, 1965.0)
    assert fused["binding_limit"] == "shared-memory pipe" and com["binding_limit"] == "instruction issue"


def test_issue_limits_without_counts_or_clock():
    out = bench.issue_limits(bench.ROOT / "profiles" / "no_such_file.json", 1.0, 2000.0)
    assert out == {"binding_limit": None, "issue_frac": None, "smem_pipe_frac": None}
    out = bench.issue_limits(bench.ROOT / "profiles" / "com_100x100_u16_traffic.json", 1.0, None)
    assert out["issue_frac"] is None
