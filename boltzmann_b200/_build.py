"""Build recipe: compiles the CUDA backend (``liblbm_cuda.so``) and the Python extension
(``boltzmann``) in-tree, for sm_100a only.

    python -m boltzmann_b200._build [--force]
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "liblbm_cuda.so"
EXT = PKG / ("boltzmann" + sysconfig.get_config_var("EXT_SUFFIX"))

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    *ARCH,
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    f"-I{INCLUDE}",
]

CUDA_SOURCES = ["aa_d2q9.cu", "aa_d3q27.cu", "fields.cu", "capi.cu", "noalloc.cu", "ensemble.cu", "closure.cu"]
HEADERS = ["aa_step.cuh", "aa_tma.cuh", "aa_pair.cuh", "aa_launch.cuh", "lattice.cuh",
           "storage.cuh", "sim.h"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _newer(target: Path, deps: list[Path]) -> bool:
    return target.exists() and all(d.stat().st_mtime <= target.stat().st_mtime for d in deps)


def build_cuda(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "lbm_cuda.h", INCLUDE / "lbm_closure.h"]
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        objs.append(obj)
        if force or not _newer(obj, [CSRC / src, *headers]):
            jobs.append([NVCC, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or not _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", *map(str, objs), "-o", str(LIB)])
    return LIB


def build_extension(force: bool = False) -> Path:
    import pybind11

    src = CSRC / "pymodule.cpp"
    deps = [src, INCLUDE / "lbm_cuda.h", INCLUDE / "lbm_closure.h", LIB]
    if not force and _newer(EXT, deps):
        return EXT
    py_inc = sysconfig.get_paths()["include"]
    _run(
        [
            "g++",
            "-std=c++17",
            "-O2",
            "-shared",
            "-fPIC",
            "-fvisibility=hidden",
            f"-I{py_inc}",
            f"-I{pybind11.get_include()}",
            f"-I{INCLUDE}",
            str(src),
            "-o",
            str(EXT),
            f"-L{PKG}",
            "-llbm_cuda",
            "-Wl,-rpath,$ORIGIN",
        ]
    )
    return EXT


def build_all(force: bool = False) -> None:
    build_cuda(force)
    build_extension(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
