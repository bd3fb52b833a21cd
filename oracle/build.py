"""Build the oracle libraries: the FP64 restatement and the reference's own CPU tracker.

TEST INFRASTRUCTURE ONLY. ``oracle/liboracle_port.so`` (from ``oracle/qtrk_oracle.c``)
and ``oracle/_ref/libqtrk_ref.so`` (from the reference's sources) are the parity
checkers and the timed CPU baseline; the product library never links or loads them.

The reference library is built as follows.

Recipe (no reference build system is run):

1. copy the reference's ``cputrack/`` sources (and the one header
   ``cudatrack/simplefft.h`` that ``cputrack/cpu_tracker.cpp:25`` includes) into
   ``oracle/_ref/src``; the reference tree itself is read-only and never modified;
2. apply two portability edits to the *copy*:
   - ``cputrack/std_incl.h:98-101`` declares ``template<typename T>`` inside the class
     template ``vector3<T>``; g++ rejects the shadowing, so the inner parameter is
     renamed;
   - ``cputrack/QueuedCPUTracker.cpp:141`` constructs ``std::exception`` from a string
     (an MSVC extension); it becomes ``std::runtime_error``;
3. compile with the Win32 stand-ins in ``oracle/shim`` first on the include path and a
   forced include, and link the reference's C ABI (``cputrack/qtrk_c_api.cpp``), its
   queued CPU tracker and ``oracle/ref_stage_exports.cpp`` into one shared library.

Usage: ``python oracle/build.py [--reference DIR] [--force]``. The reference checkout is
``--reference DIR``, else the ``QTRK_REFERENCE`` environment variable, else a checkout named
``reference`` beside this repository's root directory. When none of them holds the reference
tree (e.g. on a machine that only runs the tests) the script does nothing and reports whether a
prebuilt library is present.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
LIB = OUT_DIR / "libqtrk_ref.so"
PORT_LIB = HERE / "liboracle_port.so"
# a checkout of the reference placed beside this repository (used when no location is given)
SIBLING_REFERENCE = HERE.parent.parent / "reference"

SOURCES = [
    "cpu_tracker.cpp",
    "QueuedTracker.cpp",
    "QueuedCPUTracker.cpp",
    "utils.cpp",
    "qtrk_c_api.cpp",
    "dllmain.cpp",
    "BeadFinder.cpp",
    "ResultManager.cpp",
]

CXXFLAGS = [
    "-std=c++17",
    "-O2",
    "-fPIC",
    "-fpermissive",
    "-w",
    "-DWIN32",
    "-DQTRK_EXPORTS",
    "-D__cdecl=",
    "-D__declspec(x)=__attribute__((visibility(\"default\")))",
    "-D_isnan=std::isnan",
]


def _patch_copy(src_dir: Path) -> None:
    std_incl = src_dir / "cputrack" / "std_incl.h"
    text = std_incl.read_text()
    patched = re.sub(
        r"template<typename T>\s*\n(\s*)friend vector3 operator/\(T a, vector3<T> b\) \{\s*\n(\s*)return vector3<T>",
        r"template<typename Tdiv>\n\1friend vector3 operator/(Tdiv a, vector3<Tdiv> b) {\n\2return vector3<Tdiv>",
        text,
    )
    if patched == text:
        raise RuntimeError("std_incl.h: expected template shadowing pattern not found")
    std_incl.write_text(patched)

    qcpu = src_dir / "cputrack" / "QueuedCPUTracker.cpp"
    text = qcpu.read_text()
    patched = text.replace("throw std::exception(", "throw std::runtime_error(")
    if patched == text:
        raise RuntimeError("QueuedCPUTracker.cpp: expected std::exception(...) not found")
    qcpu.write_text(patched)


def build_port(force: bool = False, verbose: bool = True) -> Path:
    """Compile the FP64 restatement (plain C, no reference sources involved)."""
    src = HERE / "qtrk_oracle.c"
    if PORT_LIB.exists() and not force and PORT_LIB.stat().st_mtime >= src.stat().st_mtime:
        return PORT_LIB
    tmp = PORT_LIB.with_suffix(".so.tmp")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-o", str(tmp), str(src), "-lm"], check=True)
    tmp.replace(PORT_LIB)
    if verbose:
        print(f"[oracle] built {PORT_LIB}")
    return PORT_LIB


def build(reference: str | None = None, force: bool = False, verbose: bool = True) -> Path | None:
    ref_root = Path(reference or os.environ.get("QTRK_REFERENCE") or SIBLING_REFERENCE)
    cputrack = ref_root / "cputrack"
    if not cputrack.is_dir():
        if verbose:
            state = "present" if LIB.exists() else "absent"
            print(f"[oracle] reference tree not found at {ref_root}; prebuilt {LIB.name} is {state}")
        return LIB if LIB.exists() else None

    inputs = [cputrack / s for s in SOURCES] + [HERE / "ref_stage_exports.cpp", Path(__file__)]
    inputs += sorted((HERE / "shim").iterdir())
    if LIB.exists() and not force:
        newest = max(p.stat().st_mtime for p in inputs)
        if LIB.stat().st_mtime >= newest:
            if verbose:
                print(f"[oracle] {LIB} is up to date")
            return LIB

    src_dir = OUT_DIR / "src"
    if src_dir.exists():
        shutil.rmtree(src_dir)
    (src_dir / "cputrack").mkdir(parents=True)
    (src_dir / "cudatrack").mkdir(parents=True)
    for f in cputrack.iterdir():
        if f.suffix in (".h", ".cpp"):
            shutil.copy2(f, src_dir / "cputrack" / f.name)
    shutil.copy2(ref_root / "cudatrack" / "simplefft.h", src_dir / "cudatrack" / "simplefft.h")
    _patch_copy(src_dir)

    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(HERE / "shim"), "-I", str(src_dir / "cputrack"),
           "-include", str(HERE / "shim" / "force_include.h")]
    objs = []
    units = [src_dir / "cputrack" / s for s in SOURCES]
    units += [HERE / "ref_stage_exports.cpp", HERE / "shim" / "jpeg_stubs.cpp"]
    for unit in units:
        obj = obj_dir / (unit.stem + ".o")
        cmd = ["g++", *CXXFLAGS, *inc, "-c", str(unit), "-o", str(obj)]
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run(["g++", "-shared", "-o", str(tmp), *objs, "-lpthread"], check=True)
    tmp.replace(LIB)
    if verbose:
        print(f"[oracle] built {LIB}")
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=None)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    build_port(args.force)
    lib = build(args.reference, args.force)
    return 0 if lib is not None else 1


if __name__ == "__main__":
    sys.exit(main())
