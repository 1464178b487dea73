"""Build libcsg.so (sm_100a) and the csg command-line driver in-tree.

The library's translation units compile in parallel into _build/ (the
resident kernel once per lattice side, from pt_instances.cu) and link into
libcsg.so beside this file.

Usage: python spin-glass_b200/build.py [--force]
"""
from __future__ import annotations

import concurrent.futures
import os
import pathlib
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libcsg.so"
CLI = PKG / "csg"
PEAK = PKG / "libcsg_peak.so"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler",
          "-ffp-contract=off", "-fmad=false", f"-I{ROOT / 'include'}", f"-I{CSRC}"]

OBJ = PKG / "_build"
LIB_SOURCES = [CSRC / "csg_engine.cu", CSRC / "stream_sweep.cu", CSRC / "batch.cpp",
               CSRC / "server.cpp", CSRC / "obs_noalloc.cu", CSRC / "analysis_kernels.cu"]
RESIDENT_L = [4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 24]  # lattice sides of the resident kernel
HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "csg.h"]
LIB_DEPS = LIB_SOURCES + [CSRC / "pt_instances.cu"] + HEADERS


def _units():
    """(object file, nvcc arguments) of every translation unit of the library."""
    out = [(OBJ / (src.stem + ".o"), [str(src)]) for src in LIB_SOURCES]
    for L in RESIDENT_L:
        out.append((OBJ / f"pt_L{L}.o", [f"-DCSG_PT_L={L}", str(CSRC / "pt_instances.cu")]))
    return out
CLI_SOURCES = [CSRC / "csg_main.cpp"]


def _stale(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build_lib(force: bool = False) -> pathlib.Path:
    if not (force or _stale(LIB, LIB_DEPS)):
        return LIB
    OBJ.mkdir(exist_ok=True)
    units = _units()

    def compile_unit(unit):
        obj, args = unit
        srcs = [pathlib.Path(a) for a in args if not a.startswith("-")]
        if force or _stale(obj, srcs + HEADERS):
            subprocess.run([NVCC, *ARCH, *COMMON, "-c", "-o", str(obj), *args], check=True)

    workers = max(1, min(len(units), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        for f in [pool.submit(compile_unit, u) for u in units]:
            f.result()
    subprocess.run([NVCC, *ARCH, "-shared", "-o", str(LIB), *[str(o) for o, _ in units]],
                   check=True)
    return LIB


def build_cli(force: bool = False) -> pathlib.Path | None:
    if not all(s.exists() for s in CLI_SOURCES):
        return None
    deps = CLI_SOURCES + [LIB, ROOT / "include" / "csg.h"]
    if force or _stale(CLI, deps):
        cmd = ["g++", "-O2", "-std=c++17", f"-I{ROOT / 'include'}", "-o", str(CLI),
               *map(str, CLI_SOURCES), f"-L{PKG}", "-lcsg", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
    return CLI


def build_peak(force: bool = False) -> pathlib.Path:
    src = CSRC / "int_peak.cu"
    if force or _stale(PEAK, [src]):
        cmd = [NVCC, *ARCH, "-O3", "-Xcompiler", "-fPIC", "-shared", "-o", str(PEAK), str(src)]
        subprocess.run(cmd, check=True)
    return PEAK


def build(force: bool = False) -> None:
    build_lib(force)
    build_cli(force)
    build_peak(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
