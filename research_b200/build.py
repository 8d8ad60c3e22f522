"""Builds the sm_100a CUDA library (libocean.so) and the `spgemm` driver in-tree.

The library is compiled with nvcc for `arch=compute_100a,code=sm_100a`; the
outputs land next to this file so they travel with the source tree.
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
INCLUDE = ROOT / "include"
LIB = PKG / "libocean.so"
CLI = PKG / "bin" / "spgemm"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]

LIB_SOURCES = ["kernels_core.cu", "segmentation.cu", "mlp.cu", "batch.cu", "ocean_api.cu", "ocean_noalloc.cu"]
HEADERS = ["ocean_internal.cuh", "kernels.h", "config.h", "mlp.h", "tc05.cuh", "mlp_weights.inc", "batch.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError(f"build failed: {' '.join(cmd[:4])} ...")


def build_library(force: bool = False, verbose_ptxas: bool = False) -> Path:
    srcs = [CSRC / s for s in LIB_SOURCES]
    deps = srcs + [CSRC / h for h in HEADERS] + [INCLUDE / "ocean.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for s in srcs:
        o = objdir / (s.stem + ".o")
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(s), "-o", str(o)]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
        objs.append(str(o))
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


def build_cli(force: bool = False) -> Path:
    src = CSRC / "spgemm_main.cpp"
    deps = [src, INCLUDE / "ocean.h", INCLUDE / "ocean_spgemm.hpp", CSRC / "config.h", LIB]
    if not src.exists():
        return CLI
    if not force and not _stale(CLI, deps):
        return CLI
    CLI.parent.mkdir(exist_ok=True)
    _run(["/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++", "-O2", "-std=c++17", "-I", str(INCLUDE),
          "-I", str(CSRC), "-I", "/usr/local/cuda/include", str(src),
          "-o", str(CLI), "-L", str(PKG), "-locean", "-Wl,-rpath,$ORIGIN/..",
          "-L", "/usr/local/cuda/lib64", "-lcudart"])
    return CLI


def build_all(force: bool = False) -> None:
    build_library(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(LIB)
