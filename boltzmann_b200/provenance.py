"""Digests of the kernel sources behind a measurement.

A profile summary under ``profiles/`` records the digest of the sources its kernel was built
from (``kernel_sources: <digest>``); ``bench.py`` prints the digest of the sources it runs and
uses a summary's DRAM traffic only when the two agree, so a figure from an older build of a
kernel is never reported beside a newer kernel's timing.
"""

from __future__ import annotations

import hashlib
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"

# The files each kernel family is compiled from (its own translation units and headers).
GROUPS = {
    "stencil": ["aa_step.cuh", "aa_tma.cuh", "aa_pair.cuh", "aa_launch.cuh", "lattice.cuh",
                "storage.cuh", "aa_d2q9.cu", "aa_d3q27.cu"],
    "ensemble": ["ensemble.cu", "aa_step.cuh", "aa_tma.cuh", "aa_pair.cuh", "lattice.cuh",
                 "storage.cuh"],
    "closure": ["closure.cu"],
}


def digest(group: str) -> str:
    """First 16 hex digits of the SHA-256 over the group's files (name and bytes, in order)."""
    h = hashlib.sha256()
    for name in GROUPS[group]:
        h.update(name.encode())
        h.update(b"\0")
        h.update((CSRC / name).read_bytes())
        h.update(b"\0")
    return h.hexdigest()[:16]
