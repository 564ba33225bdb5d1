"""TEST INFRASTRUCTURE: build recipe for the two CPU checkers.

* ``oracle/liblbm_oracle.so`` -- the C restatement in ``lbm_oracle.c`` (always built).
* ``oracle/_ref/liblbm_ref.so`` -- the reference's own kernels (``src/lib.cl`` of
  djbarker/boltzmann, unmodified, plus the D3Q27 TRT kernel its generator writes) compiled as
  C++ behind ``ref_shim.h`` with the host loop of ``ref_driver.cpp``. Built only where the
  reference tree exists (``BOLTZMANN_REFERENCE``, else a ``reference`` directory beside this
  repository's root); elsewhere the prebuilt library is used as it is.

Both are checkers for the CUDA product and its CPU baseline; nothing in the product imports them.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
ORACLE_SO = HERE / "liblbm_oracle.so"
REF_SO = REF_DIR / "liblbm_ref.so"

# Portable across the x86-64 hosts this image runs on; no FMA contraction so that the C
# arithmetic is the plain IEEE single/double sequence the sources spell out.
CFLAGS = ["-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off"]


def reference_root() -> Path:
    """The reference checkout: $BOLTZMANN_REFERENCE, else ``../reference`` from the repo root."""
    env = os.environ.get("BOLTZMANN_REFERENCE")
    return Path(env) if env else HERE.parent.parent / "reference"


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    src = HERE / "lbm_oracle.c"
    deps = [src, HERE / "lbm_oracle_impl.h"]
    if force or _stale(ORACLE_SO, deps):
        _run(["gcc", "-std=c11", *CFLAGS, str(src), "-o", str(ORACLE_SO), "-lm"])
    return ORACLE_SO


def build_ref(force: bool = False) -> Path | None:
    """Compile the reference kernels; returns None where the reference tree is absent."""
    root = reference_root()
    lib_cl = root / "src" / "lib.cl"
    if not lib_cl.exists():
        return REF_SO if REF_SO.exists() else None
    gen = REF_DIR / "gen"
    deps = [lib_cl, HERE / "ref_driver.cpp", HERE / "ref_shim.h", HERE / "gen_ref_kernels.py"]
    if not (force or _stale(REF_SO, deps)):
        return REF_SO
    REF_DIR.mkdir(exist_ok=True)
    _run([sys.executable, str(HERE / "gen_ref_kernels.py"), str(root), str(gen)])
    _run(
        [
            "g++",
            "-std=c++17",
            *CFLAGS,
            "-Wno-unknown-pragmas",
            f"-I{HERE}",
            f"-I{root / 'src'}",
            f"-I{gen}",
            str(HERE / "ref_driver.cpp"),
            "-o",
            str(REF_SO),
        ]
    )
    return REF_SO


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_ref(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
