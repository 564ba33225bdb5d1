"""TEST INFRASTRUCTURE (the checker, never the product).

Runs the reference's own sympy kernel generator (python/boltzmann/kernel_gen.py:250-462 of
djbarker/boltzmann) to produce the update kernels the reference can generate but never registers
(src/opencl.rs:123-129): D3Q27 TRT for the fluid, D2Q5 and D3Q7 TRT for tracers. The output is
written under oracle/_ref/gen/ and is never committed.

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
    for model, kind, name in ((kg.D3Q27, "fluid", "update_d3q27_trt"),
                              (kg.D2Q5, "scalar", "update_d2q5_trt"),
                              (kg.D3Q7, "scalar", "update_d3q7_trt")):
        (out_dir / f"{name}.cl").write_text(kg.gen_kernel_AA_v1(model, kind, "trt") + "\n")

    # Self-checks of the generator against the kernels lib.cl registers (the reference's own
    # kernels were produced this way): each generated kernel must equal, up to whitespace, the
    # text of lib.cl from that kernel's first line on.
    lib = (reference_root / "src" / "lib.cl").read_text()
    squash = lambda s: re.sub(r"\s+", "", s)  # noqa: E731
    for model, kind, omega, name in ((kg.D2Q9, "fluid", "trt", "update_d2q9_trt"),
                                     (kg.D2Q5, "scalar", "bgk", "update_d2q5_bgk"),
                                     (kg.D3Q7, "scalar", "bgk", "update_d3q7_bgk")):
        gen = kg.gen_kernel_AA_v1(model, kind, omega)
        in_lib = lib[lib.index("kernel void " + name):]
        if not squash(in_lib).startswith(squash(gen)):
            raise SystemExit(f"kernel_gen output differs from lib.cl {name}")


if __name__ == "__main__":
    generate(Path(sys.argv[1]), Path(sys.argv[2]))
