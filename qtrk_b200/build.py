"""Build ``qtrk_b200/libqtrk_b200.so`` in-tree with nvcc for sm_100a.

All CUDA sources are compiled with ``-gencode arch=compute_100a,code=sm_100a`` (the only
target: the library refuses to run on other GPUs) and linked with the static CUDA
runtime, so the shared object needs nothing but the NVIDIA driver at run time.
Only the symbols of ``include/qtrk_c_api.h`` are exported (``-fvisibility=hidden``).

Usage: ``python -m qtrk_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "libqtrk_b200.so"
LV_SRC = PKG / "csrc_lv" / "lv_api.cpp"
LV_LIB = PKG / "libqtrk_b200_lv.so"  # LabVIEW binding over the C ABI of LIB

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2",
    "-I", str(CSRC), "-I", str(INCLUDE),
]


def nvcc() -> str:
    exe = shutil.which("nvcc")
    if exe:
        return exe
    cand = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sources()
    hdr_mtime = max((h.stat().st_mtime for h in headers()), default=0.0)
    stale = []
    for s in srcs:
        obj = OBJ / (s.name + ".o")
        if force or not obj.exists() or obj.stat().st_mtime < max(s.stat().st_mtime, hdr_mtime,
                                                                 Path(__file__).stat().st_mtime):
            stale.append(s)
    if stale:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(stale))) as ex:
            list(ex.map(lambda s: _compile(s, verbose), stale))
    objs = [OBJ / (s.name + ".o") for s in srcs]
    if force or stale or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
               "-Xcompiler", "-fPIC", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        tmp.replace(LIB)
        if verbose:
            print(f"built {LIB}")
    build_lv(force or bool(stale), verbose)
    return LIB


def build_lv(force: bool = False, verbose: bool = False) -> Path:
    """libqtrk_b200_lv.so: the LabVIEW binding, linked against libqtrk_b200.so (found next to it
    through an $ORIGIN run path). NumericArrayResize and MoveBlock stay undefined: the LabVIEW
    process that loads the binding provides them."""
    obj = OBJ / (LV_SRC.name + ".o")
    deps = [LV_SRC, INCLUDE / "qtrk_lv_api.h", INCLUDE / "qtrk_c_api.h", Path(__file__)]
    if force or not obj.exists() or obj.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        _compile(LV_SRC, verbose)
    if force or not LV_LIB.exists() or LV_LIB.stat().st_mtime < max(obj.stat().st_mtime, LIB.stat().st_mtime):
        tmp = LV_LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), str(obj), "-L", str(PKG), "-lqtrk_b200",
               "-Xlinker", "-rpath=$ORIGIN", "-Xcompiler", "-fPIC", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed (LabVIEW binding):\n{r.stdout}\n{r.stderr}")
        tmp.replace(LV_LIB)
    return LV_LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="build libqtrk_b200.so for sm_100a")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    build(a.force, a.verbose)
    return 0


if __name__ == "__main__":
    sys.exit(main())
