"""In-tree build of libsphk (sm_100a) and the ``sphere`` executable.

``python -m sphere_b200.build`` compiles:
  sphere_b200/lib/libsphk.so   the CUDA kernels and the C ABI (include/sphk.h)
  sphere_b200/bin/sphere       the drop-in CLI over the DEM class
Both are plain nvcc/g++ invocations; no JIT cache is involved, so the
binaries travel with the source tree.

Compiler flags that carry meaning:
  --fmad=false   no FMA contraction, as the reference (src/CMakeLists.txt:16-22)
  no --use_fast_math: IEEE division and square root
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "libsphk.so"
CLI = PKG / "bin" / "sphere"
SCENEGEN = PKG / "lib" / "libscenegen.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent

KERNEL_SOURCES = ["api.cu", "step.cu", "cells.cu", "walls.cu", "bonds.cu", "noalloc.cu",
                  "adjoint.cu", "darcy.cu", "render.cu"]
HOST_SOURCES = ["host/sphere.cpp", "host/file_io.cpp", "host/main.cpp"]


def _run(cmd, log=None):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write(" ".join(map(str, cmd)) + "\n" + res.stdout + res.stderr + "\n")
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"build step failed: {' '.join(map(str, cmd[:3]))} ...")
    return res


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def build_lib(force=False, verbose_ptxas=False) -> Path:
    srcs = [CSRC / s for s in KERNEL_SOURCES]
    deps = srcs + [CSRC / "sphk_internal.cuh", CSRC / "diff_law.h", CSRC / "diff_step.cuh",
                   ROOT / "include" / "sphk.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    objdir = PKG / "lib" / "obj"
    objdir.mkdir(parents=True, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                    "-I", str(ROOT / "include")]
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    with open(PKG / "lib" / "build.log", "w") as log:
        objs = []
        for s in srcs:
            o = objdir / (s.stem + ".o")
            _run([NVCC, *flags, "-c", str(s), "-o", str(o)], log)
            objs.append(str(o))
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"], log)
    return LIB


def build_cli(force=False) -> Path:
    srcs = [CSRC / s for s in HOST_SOURCES]
    if not all(s.exists() for s in srcs):
        return CLI
    deps = srcs + [CSRC / "host" / "sphere.h", ROOT / "include" / "sphk.h", LIB]
    if not force and not _stale(CLI, deps):
        return CLI
    CLI.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(CSRC / "host"),
           *map(str, srcs), "-o", str(CLI), "-L", str(LIB.parent), "-lsphk",
           "-Wl,-rpath,$ORIGIN/../lib"]
    _run(cmd)
    return CLI


def build_scenegen(force=False) -> Path:
    src = CSRC / "host" / "scenegen.c"
    if not force and not _stale(SCENEGEN, [src]):
        return SCENEGEN
    SCENEGEN.parent.mkdir(parents=True, exist_ok=True)
    _run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", str(src), "-o", str(SCENEGEN), "-lm"])
    return SCENEGEN


def build(force=False, verbose_ptxas=False):
    build_lib(force=force, verbose_ptxas=verbose_ptxas)
    build_cli(force=force)
    build_scenegen(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
