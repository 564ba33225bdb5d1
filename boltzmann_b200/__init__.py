"""boltzmann_b200: the lattice-Boltzmann hot path of djbarker/boltzmann on NVIDIA B200.

``boltzmann_b200.boltzmann`` is the compiled extension with the reference's classes
(``Simulation``, ``Fluid``, ``Scalar``, ``Cells``, ``Omega``); ``boltzmann_b200.core`` re-exports
them with the helpers ``bgk``, ``trt`` and ``CellFlags``, as ``boltzmann.core`` does.

The extension and its CUDA backend (``liblbm_cuda.so``) are built in-tree by
``python -m boltzmann_b200._build``; importing the package without them raises ImportError --
there is no CPU fallback.
"""

from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIBRARY = _PKG / "liblbm_cuda.so"

__all__ = ["LIBRARY"]
