"""TEST INFRASTRUCTURE (the checker, never the product).

Runs the reference's own sympy kernel generator (python/boltzmann/kernel_gen.py:250-462 of
djbarker/boltzmann) to produce the D3Q27 TRT update kernel, which the reference can generate but
never registers (src/opencl.rs:123-129). The output is written under oracle/_ref/gen/ and is
never committed.

kernel_gen imports boltzmann.core, which imports the compiled extension boltzmann.boltzmann
(python/boltzmann/core.py:31). That extension cannot be built here (no Rust toolchain), so a
stand-in module exposing ``Omega`` is registered first; kernel_gen only needs ``CellFlags``.

Usage: python gen_ref_kernels.py <reference_root> <out_dir>
"""

from __future__ import annotations

import re
import sys
import types
from pathlib import Path


def _stub_extension() -> None:
    ext = types.ModuleType("boltzmann.boltzmann")

    class Omega:  # only referenced inside bgk()/trt(), never called by kernel_gen
        pass

    ext.Omega = Omega
    import boltzmann  # the reference's python package (on sys.path)

    sys.modules["boltzmann.boltzmann"] = ext
    boltzmann.boltzmann = ext


def generate(reference_root: Path, out_dir: Path) -> None:
    sys.path.insert(0, str(reference_root / "python"))
    _stub_extension()
    import boltzmann.kernel_gen as kg  # noqa: E402  (reference generator)

    out_dir.mkdir(parents=True, exist_ok=True)
    src = kg.gen_kernel_AA_v1(kg.D3Q27, "fluid", "trt")
    (out_dir / "update_d3q27_trt.cl").write_text(src + "\n")

    # Self-check of the generator: its D2Q9 TRT must equal lib.cl's update_d2q9_trt up to
    # whitespace (the reference's own kernel was produced this way).
    gen_d2q9 = kg.gen_kernel_AA_v1(kg.D2Q9, "fluid", "trt")
    lib = (reference_root / "src" / "lib.cl").read_text()
    start = lib.index("kernel void update_d2q9_trt")
    in_lib = lib[start:]
    squash = lambda s: re.sub(r"\s+", "", s)  # noqa: E731
    if squash(gen_d2q9) != squash(in_lib):
        raise SystemExit("kernel_gen D2Q9 TRT differs from lib.cl update_d2q9_trt")


if __name__ == "__main__":
    generate(Path(sys.argv[1]), Path(sys.argv[2]))
