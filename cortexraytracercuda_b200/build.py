"""Builds the in-tree shared library librtc_b200.so (sm_100a kernels + host C ABI).

    python -m cortexraytracercuda_b200.build [--force] [--verbose]

Compat-mode kernels are compiled with --fmad=false (reference float semantics), clean-mode kernels
with FMA contraction; host sources with -ffp-contract=off.  Objects go to ``_build/`` beside this
file, the library next to the package (``cortexraytracercuda_b200/librtc_b200.so``).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "librtc_b200.so"
INCLUDE = PKG.parent / "include"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(CSRC), "-I", str(INCLUDE)] + ARCH
CXX = os.environ.get("CXX", "g++")
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
             "-I", str(CSRC), "-I", str(INCLUDE), "-I", os.path.join(CUDA_HOME, "include")]

# (source, object name, compiler, extra flags).  The compat sources are built once per reference
# build flavour: RTC_FLAVOR=1 reproduces a g++ build of the reference (no FMA contraction),
# RTC_FLAVOR=0 its nvcc build (FMA contraction on, nvcc's default).
SOURCES = [
    ("render_compat.cu", "render_compat_host", "nvcc", ["--fmad=false", "-DRTC_FLAVOR=1"]),
    ("render_compat.cu", "render_compat_dev", "nvcc", ["--fmad=true", "-DRTC_FLAVOR=0"]),
    ("wavefront_compat.cu", "wavefront_compat_host", "nvcc", ["--fmad=false", "-DRTC_FLAVOR=1"]),
    ("wavefront_compat.cu", "wavefront_compat_dev", "nvcc", ["--fmad=true", "-DRTC_FLAVOR=0"]),
    ("render_clean.cu", "render_clean", "nvcc", ["--fmad=true"]),
    ("wavefront_clean.cu", "wavefront_clean", "nvcc", ["--fmad=true"]),
    # the same kernels with the xprim BVH walk (RTC_XP=1), for scenes with transformed primitives or boxes
    ("render_compat.cu", "render_compat_host_x", "nvcc", ["--fmad=false", "-DRTC_FLAVOR=1", "-DRTC_XP=1"]),
    ("render_compat.cu", "render_compat_dev_x", "nvcc", ["--fmad=true", "-DRTC_FLAVOR=0", "-DRTC_XP=1"]),
    ("wavefront_compat.cu", "wavefront_compat_host_x", "nvcc", ["--fmad=false", "-DRTC_FLAVOR=1", "-DRTC_XP=1"]),
    ("wavefront_compat.cu", "wavefront_compat_dev_x", "nvcc", ["--fmad=true", "-DRTC_FLAVOR=0", "-DRTC_XP=1"]),
    ("render_clean.cu", "render_clean_x", "nvcc", ["--fmad=true", "-DRTC_XP=1"]),
    ("wavefront_clean.cu", "wavefront_clean_x", "nvcc", ["--fmad=true", "-DRTC_XP=1"]),
    ("render_noalloc.cu", "render_noalloc", "nvcc", []),
    ("rtc_api.cpp", "rtc_api", "cxx", []),
    ("rtc_engine.cpp", "rtc_engine", "cxx", []),
    ("rtc_batch.cpp", "rtc_batch", "cxx", []),
    ("rtc_server.cpp", "rtc_server", "cxx", []),
    ("rtc_obj.cpp", "rtc_obj", "cxx", []),
    ("rtc_scene_file.cpp", "rtc_scene_file", "cxx", []),
    ("bvh_device.cu", "bvh_device", "nvcc", []),
    ("bvh_build.cpp", "bvh_build", "cxx", []),
]
HEADERS = ["rtc_dev.h", "rtc_math.cuh", "rtc_trace.cuh", "rtc_path.cuh", "rtc_wavefront.cuh", "rtc_kernels.h",
           "bvh_build.h", "rtc_internal.h", "rtc_objects.h", "rtc_engine.h"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(str(c) for c in cmd)}")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False, defines=(), out: Path | None = None,
          objdir: Path | None = None) -> Path:
    """Compiles every translation unit (in parallel) and links the library.  `defines` (NAME=VALUE)
    are passed to every compile; with `out`/`objdir` a variant library is built elsewhere."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_dir = Path(objdir) if objdir else BUILD
    lib = Path(out) if out else LIB
    build_dir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(parents=True, exist_ok=True)
    dflags = [f"-D{d}" for d in defines]
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "rtc.h"]
    objs = []
    cmds = []
    for src, obj, comp, extra in SOURCES:
        s = CSRC / src
        o = build_dir / (obj + ".o")
        objs.append(o)
        if not force and not _newer(o, [s] + headers + [Path(__file__)]):
            continue
        if comp == "nvcc":
            cmd = [NVCC] + NVCC_COMMON + extra + dflags + (["-Xptxas", "-v"] if ptxas_verbose else []) + ["-c", str(s), "-o", str(o)]
        else:
            cmd = [CXX] + CXX_FLAGS + extra + dflags + ["-c", str(s), "-o", str(o)]
        cmds.append(cmd)
    # independent translation units compile in parallel
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(_run, cmd, verbose or ptxas_verbose) for cmd in cmds]:
            f.result()
    if force or _newer(lib, objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [NVCC, "-shared"] + ARCH + ["-o", str(tmp)] + [str(o) for o in objs] + ["-cudart", "static", "-lpthread"]
        _run(cmd, verbose)
        os.replace(tmp, lib)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill report")
    ap.add_argument("--define", action="append", default=[], help="NAME=VALUE for every compile (CUDA and host)")
    ap.add_argument("--out", default=None, help="library path (a variant build)")
    ap.add_argument("--objdir", default=None, help="object directory (a variant build)")
    a = ap.parse_args()
    p = build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas, defines=a.define,
              out=Path(a.out) if a.out else None, objdir=Path(a.objdir) if a.objdir else None)
    print(p)


if __name__ == "__main__":
    main()
