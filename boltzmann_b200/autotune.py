"""Autotuner for the ensemble's launch shape: the kernel (row-staged, or tiles of a given width)
and its CTAs per SM.

Candidates are timed on the ensemble itself with CUDA events on its stream (a few AA step pairs
each, after one warm-up pair); the populations are saved before and restored after, so tuning
leaves the state unchanged. The winner is cached in a JSON file keyed by lattice, collision,
storage and a size class of the ensemble (total cells and median domain width, both rounded to
powers of two), so later ensembles of the same class skip the search. Cache file:
``$BOLTZMANN_B200_TUNE_CACHE`` or ``~/.cache/boltzmann_b200/autotune.json``.
"""

from __future__ import annotations

import json
import math
import os
from pathlib import Path

import numpy as np

TILES = (32, 64, 128, 256, 512)  # tile kernel widths
BLOCKS = (0, 2, 4, 8)
ROW_BLOCKS = (0, 1, 2)  # CTAs per SM of the row-staged kernel (tile 0; 0 = as many as fit)
ROW_MAX = 512  # longest row the row-staged kernel takes
KERNELS = "rows+tiles"  # part of the cache key: entries made before the row kernel are ignored


def cache_path() -> Path:
    env = os.environ.get("BOLTZMANN_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "boltzmann_b200" / "autotune.json"


def size_class(ens) -> str:
    widths = sorted(b for _, b in ens.counts)
    median = widths[len(widths) // 2]
    return f"cells2^{round(math.log2(max(ens.n, 1)))}-width2^{round(math.log2(median))}"


def key(ens, storage: str) -> str:
    coll = "trt" if ens.collision else "bgk"
    rows = "rows" if max(b for _, b in ens.counts) <= ROW_MAX else "tiles-only"
    return f"D2Q9/{coll}/{storage}/{size_class(ens)}/{KERNELS}/{rows}"


def _load() -> dict:
    p = cache_path()
    if p.exists():
        try:
            return json.loads(p.read_text())
        except (OSError, ValueError):
            return {}
    return {}


def _store(entries: dict) -> None:
    p = cache_path()
    p.parent.mkdir(parents=True, exist_ok=True)
    tmp = p.with_suffix(f".{os.getpid()}.tmp")  # ranks of one job may store at the same time
    tmp.write_text(json.dumps(entries, indent=1, sort_keys=True))
    os.replace(tmp, p)


def time_shape(ens, tile: int, blocks: int, pairs: int = 4) -> float:
    """Device milliseconds per AA step pair for one shape (persistent launches)."""
    import torch

    ens.set_shape(tile, blocks)
    stream = torch.cuda.ExternalStream(ens.stream())
    ens.iterate(2, mode="persistent", read_back=False)  # warm-up
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    ens.iterate(2 * pairs, mode="persistent", read_back=False)
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop) / pairs


def tune(ens, storage: str = "f32", use_cache: bool = True, pairs: int = 4) -> dict:
    """Picks and applies the fastest (tile, blocks_per_sm); returns the record with timings."""
    k = key(ens, storage)
    entries = _load() if use_cache else {}
    if use_cache and k in entries:
        rec = entries[k]
        ens.set_shape(rec["tile"], rec["blocks_per_sm"])
        return dict(rec, cached=True)
    if ens.iteration == 0:
        ens.iterate(0)  # upload + equilibrate so the timings run on real data
    saved = ens.populations()
    saved_iteration = ens.iteration
    timings = {}
    shapes = [(0, b) for b in ROW_BLOCKS] if max(b for _, b in ens.counts) <= ROW_MAX else []
    shapes += [(t, b) for t in TILES for b in BLOCKS]
    for tile, blocks in shapes:
        timings[f"{tile}x{blocks}"] = time_shape(ens, tile, blocks, pairs)
    best = min(timings, key=timings.get)
    tile, blocks = (int(v) for v in best.split("x"))
    ens.set_shape(tile, blocks)
    ens.set_populations(saved)
    ens.iteration = saved_iteration
    rec = {"tile": tile, "blocks_per_sm": blocks, "ms_per_pair": timings[best],
           "timings_ms_per_pair": timings}
    if use_cache:
        entries[k] = rec
        _store(entries)
    return dict(rec, cached=False)
