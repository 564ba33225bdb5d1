"""The run loop of a simulation, with device-side hooks.

A drop-in for ``run_sim`` of the reference (python/boltzmann/simulation.py:174-271) and its
helpers (``IterInfo`` 30-82, the checkpoint gaters 85-171): the same generator protocol -- yield
the current output index once before stepping (the resumed one after a restart), then after
every batch of ``meta.interval`` steps (rounded to an even count), checkpoint through a
temporary file moved into place when the gater allows -- and the same errors. What runs
differently, on the device:

* the non-finite check reads the kernels' status flag (set by the step that ends each batch when
  a density or velocity component is not finite) instead of scanning the host copy of the
  velocity with ``np.isfinite``;
* MLUP/s come from CUDA events recorded on the simulation's stream around the steps, not from
  the host clock around ``iterate`` (which also holds the read-back);
* the steps run with the GIL released (the reference's ``iterate`` holds it).

The host mirrors (``sim.fluid``, tracer values) are refreshed after every batch, as the
reference's ``iterate`` does, before the caller's code runs at the ``yield``.
"""

from __future__ import annotations

import datetime
import logging
import os
import re
from abc import ABC, abstractmethod
from dataclasses import dataclass, field
from pathlib import Path
from typing import Generator

logger = logging.getLogger("boltzmann_b200")


@dataclass
class IterInfo:
    """Output interval (LBM steps per output) and output count."""

    interval: int
    count: int

    @staticmethod
    def make(*, dt: float, dt_output: float | None = None, t_max: float | None = None,
             count: int | None = None) -> "IterInfo":
        """From ``dt`` and exactly two of ``dt_output``, ``t_max``, ``count``: the interval is
        dt_output / dt, the count t_max / dt_output (python/boltzmann/simulation.py:44-82)."""
        given = (dt_output is not None, t_max is not None, count is not None)
        if given == (False, True, True):
            dt_output = t_max / count
        elif given == (True, False, True):
            t_max = count * dt_output
        elif given == (True, True, False):
            count = int(t_max / dt_output + 1e-8)
        else:
            raise ValueError(
                f"Must specify dt and exactly two other arguments! [{dt_output=}, {t_max=}, {count=}]"
            )
        return IterInfo(int(dt_output / dt), count)


class CheckpointGater(ABC):
    """Tells ``run_sim`` when to write a checkpoint."""

    @abstractmethod
    def allow(self) -> bool: ...


@dataclass
class NoCheckpoints(CheckpointGater):
    def allow(self) -> bool:
        return False


@dataclass
class EveryN(CheckpointGater):
    """True on call ``interval - 1`` and then on every ``interval``-th call after it, as the
    reference's gater counts (so from ``interval`` 3 on, never on the first call)."""

    interval: int
    _curr: int = field(default=1)

    def __post_init__(self):
        assert self.interval > 0, "Checkpoint Interval must be positive!"

    def allow(self) -> bool:
        self._curr = (self._curr + 1) % self.interval
        return self._curr == 0


@dataclass
class EveryT(CheckpointGater):
    """True when more than ``interval`` has passed since the last True (or since creation)."""

    interval: datetime.timedelta
    _last: datetime.datetime = field(default_factory=datetime.datetime.now)

    def allow(self) -> bool:
        now = datetime.datetime.now()
        if now - self._last > self.interval:
            self._last = now
            return True
        return False


def parse_checkpoints(s: str) -> CheckpointGater:
    """``"off"``, ``"<N>"`` (every N outputs) or ``"<N>m"`` (every N minutes)."""
    if s == "off":
        return NoCheckpoints()
    if (m := re.match(r"^(\d+)$", s)) is not None:
        return EveryN(int(m.group(1)))
    if (m := re.match(r"^(\d+)m$", s)) is not None:
        return EveryT(datetime.timedelta(minutes=int(m.group(1))))
    raise ValueError(f"Unable to parse checkpoint interval! [{s!r}]")


def _device_steps(sim, iters: int) -> float:
    """Runs iters steps on the simulation's stream; returns their device time in seconds."""
    import torch

    stream = torch.cuda.ExternalStream(sim._stream())
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    sim._iterate_device(iters)
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop) / 1e3


def run_sim(sim, meta, output_dir: Path | str,
            checkpoints: CheckpointGater | None = None) -> Generator[int, None, None]:
    """Generator over output indices; see the module docstring."""
    output_dir = Path(output_dir)
    if output_dir.exists():
        assert output_dir.is_dir(), f"Base path must be a directory! [{output_dir=}]"
    else:
        output_dir.mkdir()
    checkpoints = checkpoints or EveryN(5)
    batch_iters = 2 * int(meta.interval / 2 + 0.5)  # even: the AA pattern

    cells = int(sim.cells.count)
    logger.info("device %s, %s MB, %d iters / output, %.1fM cells (%s)",
                " ".join(sim.device_info.split()), f"{sim.size_bytes // 1_000_000:,d}",
                batch_iters, cells / 1e6, " x ".join(str(int(c)) for c in sim.cells.counts))

    max_i = meta.count
    sim_i = sim.iteration // batch_iters
    if sim.iteration > 0:
        logger.info("Resuming from step %d", sim_i)
    yield sim_i

    start_all = datetime.datetime.now()
    for i in range(sim_i + 1, max_i):
        seconds = _device_steps(sim, batch_iters)
        if sim._nonfinite():
            raise ValueError("Non-finite value detected!")
        sim._read_back()
        mlups = cells * batch_iters / (1e6 * seconds) if seconds > 0 else float("inf")

        t_out = datetime.datetime.now()
        yield i
        if checkpoints.allow():
            sim.write_checkpoint(str(output_dir / "checkpoint.mpk.tmp"))
            os.replace(output_dir / "checkpoint.mpk.tmp", output_dir / "checkpoint.mpk")
            logger.info("Checkpoint written.")
        out_s = (datetime.datetime.now() - t_out).total_seconds()

        elapsed = datetime.datetime.now() - start_all
        eta = datetime.datetime.now() + (max_i - i) * elapsed / (i - sim_i)
        logger.info("Batch %d: %s %6.0f MLUP/s (device), sim %.3fs, out %.1fs, eta %s", i,
                    str(elapsed).split(".")[0], mlups, seconds, out_s, f"{eta:%H:%M:%S}")
