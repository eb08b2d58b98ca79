"""Build the native parts in-tree: libtbmd.so (CUDA kernels + C ABI, sm_100a) and the drop-in
executable tbmd_main (C++ host, the reference's CLI and CSV contract, linked against libtbmd.so).

    python -m threebodymdalgorithms_b200.build [--force] [--bounds-check]

--bounds-check also builds libtbmd_checked.so, the same library compiled with -DTBMD_BOUNDS_CHECK:
every checked kernel index outside its array is recorded on the device (and replaced by 0, so the
kernel runs on without faulting) and read back with tbmd_bounds_report.  Point TBMD_LIBRARY at it to
run a program or the test suite on the checked build.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libtbmd.so"
LIB_CHECKED = PKG / "libtbmd_checked.so"
MAIN = PKG / "tbmd_main"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                  "-I", str(INCLUDE)]

CU_SOURCES = ["tbmd_kernels.cu", "tbmd_api.cu", "tbmd_probe.cu", "tbmd_noalloc.cu", "tbmd_gen.cu", "tbmd_ranks.cpp"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")
    return r


def build(force: bool = False, verbose: bool = False, bounds_check: bool = False) -> Path:
    deps = [CSRC / s for s in CU_SOURCES] + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    targets = [(LIB, [])] + ([(LIB_CHECKED, ["-DTBMD_BOUNDS_CHECK"])] if bounds_check else [])
    for target, extra in targets:
        if force or _stale(target, deps):
            cmd = [NVCC] + NVFLAGS + extra + ["-shared", "-o", str(target)] + [str(CSRC / s) for s in CU_SOURCES]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    main_deps = [CSRC / "tbmd_main.cpp", INCLUDE / "tbmd.h", LIB]
    if (CSRC / "tbmd_main.cpp").exists() and (force or _stale(MAIN, main_deps)):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-pthread", "-I", str(INCLUDE), str(CSRC / "tbmd_main.cpp"), "-o",
               str(MAIN), "-L", str(PKG), "-ltbmd", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, bounds_check="--bounds-check" in sys.argv)
    print(LIB)
