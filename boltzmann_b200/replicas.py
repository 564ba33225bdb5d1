"""One process per GPU for the hot path, with no collective on the data path.

The reference runs one simulation on one device and its steps have no exchange, so more GPUs
serve more work, never the same step faster:

* a single simulation (the channel, the Taylor-Green box) runs as independent replicas, one per
  rank (weak scaling);
* a batched ensemble shards its independent domains across ranks by cell count
  (``shard_by_cells``), each rank advancing only its own domains (the total work is fixed).

The only collectives are on the host side of measurement: a barrier around timed regions and the
maximum (or sum) of per-rank numbers. ``Group`` wraps ``torch.distributed`` for that: NCCL on
GPUs, gloo on CPU (tests), with a short timeout so that ranks waiting on a lost peer end with an
error instead of hanging.
"""

from __future__ import annotations

import datetime
import os


class Group:
    """Rank information and the few host-side collectives the benchmark needs."""

    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self._dist = None
        self._device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist
            self._device = "cuda" if backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """The largest value over ranks (device times: the slowest rank sets the job time)."""
        return x if self._dist is None else self._reduce(x, self._dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return x if self._dist is None else self._reduce(x, self._dist.ReduceOp.SUM)

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def shard_by_cells(counts, world: int) -> list[list[int]]:
    """Domain indices per rank: largest domain first to the rank with the fewest cells so far
    (ties to the lower rank), each shard in ascending domain order. Deterministic, so every rank
    computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world must be at least 1")
    sizes = [int(a) * int(b) for a, b in counts]
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += sizes[i]
    return [sorted(s) for s in shards]
