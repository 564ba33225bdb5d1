"""Generates tests/golden/postproc.npz from the reference's own post-processing functions
(python/boltzmann/utils/postproc.py: calc_curl, calc_vmag) on seeded velocity fields.

Run from the repository root where the reference tree exists:
    python tests/golden/make_postproc_golden.py
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.build import reference_root  # noqa: E402

REFERENCE_PYTHON = reference_root() / "python"
OUT = Path(__file__).resolve().parent / "postproc.npz"


def main() -> None:
    sys.path.insert(0, str(REFERENCE_PYTHON))
    from boltzmann.utils.postproc import calc_curl, calc_vmag

    rng = np.random.default_rng(7)
    v2 = rng.normal(0, 0.05, (37, 23, 2)).astype(np.float32)
    v3 = rng.normal(0, 0.05, (9, 7, 6, 3)).astype(np.float32)
    np.savez_compressed(
        OUT,
        vel2d=v2,
        curl2d=calc_curl(v2),
        vmag2d=calc_vmag(v2),
        vel3d=v3,
        curl3d=calc_curl(v3),
        vmag3d=calc_vmag(v3),
    )
    print("wrote", OUT)


if __name__ == "__main__":
    main()
