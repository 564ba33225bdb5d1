"""The multi-process plumbing of the hot path (boltzmann_b200/replicas.py) on CPU: two gloo ranks
agree on the maximum and sum of per-rank numbers and on the ensemble's domain partition, and the
partition covers every domain once and balances cells."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from boltzmann_b200.replicas import Group, shard_by_cells


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    g = Group(backend="gloo", timeout_s=30)
    g.barrier()
    counts = [(64 + 7 * i, 64 + 5 * i) for i in range(23)]
    mine = shard_by_cells(counts, world)[g.rank]
    cells = sum(a * b for a, b in (counts[i] for i in mine))
    out.put((g.rank, g.max(float(rank + 1) * 1.5), g.sum(float(cells)), tuple(mine)))
    g.close()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    counts = [(64 + 7 * i, 64 + 5 * i) for i in range(23)]
    total = sum(a * b for a, b in counts)
    assert all(r[1] == 1.5 * world for r in results)  # max over ranks
    assert all(r[2] == total for r in results)        # every cell on exactly one rank
    shards = [set(r[3]) for r in results]
    assert set.union(*shards) == set(range(23)) and sum(len(s) for s in shards) == 23


def test_single_process_group_is_a_no_op(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    g = Group()
    assert (g.rank, g.world) == (0, 1) and g.max(3.0) == 3.0 and g.sum(2.0) == 2.0
    g.barrier()
    g.close()


def test_shard_by_cells_balances():
    import numpy as np

    rng = np.random.default_rng(0)
    sides = rng.integers(64, 513, 512)
    counts = [(int(s), int(s)) for s in sides]
    for world in (1, 2, 4, 8):
        shards = shard_by_cells(counts, world)
        assert sorted(i for s in shards for i in s) == list(range(512))
        loads = [sum(counts[i][0] * counts[i][1] for i in s) for s in shards]
        # greedy largest-first: within the largest domain of the mean
        assert max(loads) - min(loads) <= max(a * b for a, b in counts)
    assert shard_by_cells([(2, 2)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        shard_by_cells(counts, 0)
