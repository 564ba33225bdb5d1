"""Loads the golden fixtures written by tests/golden/make_golden.py and replays their specs."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def names() -> list[str]:
    """The stencil fixtures (files with a case spec; postproc.npz holds other vectors)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if "spec" in np.load(p).files)


def load(name: str) -> tuple[dict, dict[str, np.ndarray], list[dict[str, np.ndarray]]]:
    z = np.load(GOLDEN / f"{name}.npz")
    spec = json.loads(str(z["spec"]))
    inputs = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    outs = []
    for i in range(len(spec["calls"])):
        p = f"out{i}_"
        outs.append({k[len(p):]: z[k] for k in z.files if k.startswith(p)})
    return spec, inputs, outs


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """Norm-wise relative error ||a - b|| / ||b|| in float64."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
