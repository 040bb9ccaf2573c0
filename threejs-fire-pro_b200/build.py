"""Build the CUDA library `lib/libfirepro.so` for sm_100a, in tree.

Each source compiles to an object under `_build/` when it (or a header) is newer than its
object; the shared library links them. nvcc cross-compiles: no GPU is needed to build.
`--debug` (build(debug=True)) builds the bounds-checked library `lib/libfirepro_debug.so`
instead (FP_BOUNDS, objects under `_build/debug/`): its kernels check every index they read out
of a table and record the first bad one (fp_sim_read_bounds).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "lib" / "libfirepro.so"
DEBUG_LIB = HERE / "lib" / "libfirepro_debug.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-ccbin", "g++"]
# The multigrid runs the same cell operations in several kernels (per brick, per tile, the
# fused coarse cycle, chosen by a simulation's tile capacity). Without multiply-add
# contraction each operation rounds the same in all of them, so the pressure of a simulation
# does not depend on which kernels ran it.
FILE_FLAGS = {"fp_mg.cu": ["-fmad=false"],
              # The mesh voxelizer decides bits with FP64 edge tests as the reference's JavaScript
              # does: no contraction on the device or the host.
              "fp_mesh.cu": ["-fmad=false", "-Xcompiler", "-ffp-contract=off"]}


def _sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def build(verbose: bool = False, ptxas_info: bool = False, debug: bool = False) -> Path:
    out_dir, lib, defines = (BUILD / "debug", DEBUG_LIB, ["-DFP_BOUNDS"]) if debug else (BUILD, LIB, [])
    out_dir.mkdir(parents=True, exist_ok=True)
    lib.parent.mkdir(exist_ok=True)
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0)
    objects, commands = [], []
    for src in _sources():
        obj = out_dir / (src.name + ".o")
        objects.append(obj)
        if obj.exists() and obj.stat().st_mtime > max(src.stat().st_mtime, newest_header) and not ptxas_info:
            continue
        cmd = [NVCC, *ARCH, *FLAGS, *defines, *FILE_FLAGS.get(src.name, []), "-I", str(INCLUDE), "-c", str(src), "-o",
               str(obj)]
        if ptxas_info and src.suffix == ".cu":
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        commands.append(cmd)
    # The sources compile independently: one nvcc per source at a time, as many as there are cores.
    with ThreadPoolExecutor(max_workers=max(1, min(len(commands), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(subprocess.run, cmd, check=True) for cmd in commands]:
            f.result()
    if not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objects):
        cmd = [NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objects), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv, debug="--debug" in sys.argv)
