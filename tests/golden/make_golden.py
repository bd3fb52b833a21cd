"""Generate the golden fixtures in tests/golden/ from the reference CPU tracker.

The reference ships no golden vectors (its tests are print-only programs), so these
fixtures are outputs of the reference itself: its cputrack/ sources compiled by
oracle/build.py into oracle/_ref/libqtrk_ref.so and driven through its own C ABI
(QTrkCreateInstance / QTrkSetRadialZLUT / QTrkBuildLUT / QTrkScheduleLocalization /
QTrkFetchResults) and stage entry points. Inputs are seeded synthetic images from
qtrk_b200.synth, stored with the outputs so the fixtures do not depend on the numpy
version. Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from oracle import RefOracle  # noqa: E402
from qtrk_b200 import abi, synth  # noqa: E402


def settings_dict(s: abi.QTrkSettings) -> str:
    return json.dumps({name: getattr(s, name) for name, _ in abi.QTrkSettings._fields_})


def results_arrays(res: np.ndarray, prefix: str = "") -> dict:
    return {prefix + "pos": res["pos"].copy(), prefix + "com": res["firstGuess"].copy(),
            prefix + "error": res["error"].copy(), prefix + "mean": res["imageMean"].copy(),
            prefix + "frame": res["frame"].copy(), prefix + "zlut": res["zlutIndex"].copy()}


def main() -> None:
    ref = RefOracle()

    # --- config 1 shape: 60x60 float, QI(32 x 64, 4 it) + Z (50 planes x 40 bins) ---
    wl = synth.roi60_f32(24, seed=101)
    lut = ref.build_lut(wl.settings, wl.lut_stack, abi.BUILDLUT_NORMALIZE, known_pos=wl.lut_known_pos)
    res = ref.track(wl.settings, wl.mode, wl.rois, lut)
    res_com = ref.track(wl.settings, abi.LT_OnlyCOM, wl.rois)
    res_qi = ref.track(wl.settings, abi.LT_QI, wl.rois)
    cc = ref.computed_config(wl.settings)
    rw = ref.radial_bin_window(cc.qi_radialsteps)
    img0 = wl.rois[0]
    prof0 = ref.radial_profile(img0, res["pos"][0][:2], cc.zlut_radialsteps, cc.zlut_angularsteps,
                               wl.settings.zlut_minradius, cc.zlut_maxradius, True)
    z0, scores0 = ref.lut_compare(prof0, lut[0])
    np.savez_compressed(
        HERE / "roi60_f32.npz", settings=settings_dict(wl.settings), mode=wl.mode,
        rois=wl.rois.astype(np.uint16), lut=lut, qi_weights=rw, prof0=prof0, scores0=scores0, z0=np.float32(z0),
        **results_arrays(res), **results_arrays(res_com, "com_only_"), **results_arrays(res_qi, "qi_only_"))

    # --- config 2 shape: 100x100 u16, QI(64 x 51) + Z (200 planes x 64 bins) ---
    wl2 = synth.roi100_u16(12, seed=102)
    lut2 = ref.build_lut(wl2.settings, wl2.lut_stack, abi.BUILDLUT_NORMALIZE, known_pos=wl2.lut_known_pos)
    res2 = ref.track(wl2.settings, wl2.mode, wl2.rois, lut2)
    np.savez_compressed(HERE / "roi100_u16.npz", settings=settings_dict(wl2.settings), mode=wl2.mode,
                        rois=wl2.rois, lut=lut2, **results_arrays(res2))

    # --- config 3 shape: 16x16 Gaussian spots, reference 4-parameter MLE (8 iterations) ---
    wl3 = synth.gauss16_f32(32, seed=103)
    res3 = ref.track(wl3.settings, abi.LT_Gaussian2D, wl3.rois)
    np.savez_compressed(HERE / "gauss16_f32.npz", settings=settings_dict(wl3.settings),
                        mode=abi.LT_Gaussian2D, rois=wl3.rois.astype(np.uint16), **results_arrays(res3))

    # --- BuildLUT through COM + QI (no known positions), 3 beads x 12 planes of 80x80 u16 ---
    s4, stack4, _ = synth.calib_stack_80x80(nbeads=3, planes=12, seed=104, noise=False)
    lut4 = ref.build_lut(s4, stack4, abi.BUILDLUT_NORMALIZE, known_pos=None)
    lut4_raw = ref.build_lut(s4, stack4, 0, known_pos=None, finalize=False)
    np.savez_compressed(HERE / "buildlut_80x80_u16.npz", settings=settings_dict(s4), stack=stack4, lut=lut4,
                        lut_unnormalized=lut4_raw)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
