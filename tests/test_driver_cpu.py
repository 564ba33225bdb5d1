"""CPU checks of the run loop's helpers (boltzmann_b200/driver.py) against the behaviour of the
reference's python/boltzmann/simulation.py:30-171, and of the generator protocol of run_sim on a
stand-in simulation (python/boltzmann/simulation.py:174-271)."""

from __future__ import annotations

import datetime

import pytest

from boltzmann_b200 import driver


def test_iter_info_make():
    assert driver.IterInfo.make(dt=0.5, dt_output=2.0, count=7) == driver.IterInfo(4, 7)
    assert driver.IterInfo.make(dt=0.5, dt_output=2.0, t_max=10.0) == driver.IterInfo(4, 5)
    assert driver.IterInfo.make(dt=0.5, t_max=10.0, count=5) == driver.IterInfo(4, 5)
    with pytest.raises(ValueError, match="exactly two other"):
        driver.IterInfo.make(dt=0.5, dt_output=2.0, t_max=10.0, count=5)
    with pytest.raises(ValueError):
        driver.IterInfo.make(dt=0.5, count=5)


def test_gaters():
    g = driver.EveryN(3)
    assert [g.allow() for _ in range(7)] == [False, True, False, False, True, False, False]
    g = driver.EveryN(5)
    assert [g.allow() for _ in range(9)] == [False, False, False, True, False, False, False, False, True]
    assert not driver.NoCheckpoints().allow()
    t = driver.EveryT(datetime.timedelta(minutes=10))
    assert not t.allow()
    t._last -= datetime.timedelta(minutes=11)
    assert t.allow() and not t.allow()
    assert isinstance(driver.parse_checkpoints("off"), driver.NoCheckpoints)
    assert driver.parse_checkpoints("7").interval == 7
    assert driver.parse_checkpoints("3m").interval == datetime.timedelta(minutes=3)
    with pytest.raises(ValueError, match="Unable to parse"):
        driver.parse_checkpoints("3h")


class _Cells:
    count = 12
    counts = [4, 3]


class FakeSim:
    """Records the calls run_sim makes; `bad_after` batches in, the status flag reports NaN."""

    device_info = "Fake   Device"
    size_bytes = 10_000_000
    cells = _Cells()

    def __init__(self, iteration=0, bad_after=None):
        self.iteration = iteration
        self.calls = []
        self.bad_after = bad_after
        self.batches = 0

    def _iterate_device(self, n):
        self.calls.append(("steps", n))
        self.iteration += n
        self.batches += 1

    def _nonfinite(self):
        return self.bad_after is not None and self.batches >= self.bad_after

    def _read_back(self):
        self.calls.append(("read_back",))

    def write_checkpoint(self, path):
        self.calls.append(("checkpoint",))
        open(path, "w").write("x")


@pytest.fixture
def no_cuda(monkeypatch):
    def steps(sim, n):
        sim._iterate_device(n)
        return 1e-3

    monkeypatch.setattr(driver, "_device_steps", steps)


def test_run_sim_protocol(tmp_path, no_cuda):
    sim = FakeSim()
    out = list(driver.run_sim(sim, driver.IterInfo(interval=5, count=5), tmp_path / "o",
                              driver.EveryN(2)))
    assert out == [0, 1, 2, 3, 4]
    # interval 5 rounds to 6 (even); every batch is read back before the caller runs
    assert [c for c in sim.calls if c[0] == "steps"] == [("steps", 6)] * 4
    assert sim.calls.count(("read_back",)) == 4
    assert sim.calls.count(("checkpoint",)) == 2
    assert (tmp_path / "o" / "checkpoint.mpk").exists()
    assert not (tmp_path / "o" / "checkpoint.mpk.tmp").exists()


def test_run_sim_resumes_and_detects_nonfinite(tmp_path, no_cuda):
    sim = FakeSim(iteration=12)
    assert list(driver.run_sim(sim, driver.IterInfo(4, 5), tmp_path, driver.NoCheckpoints())) == [3, 4]
    bad = FakeSim(bad_after=2)
    gen = driver.run_sim(bad, driver.IterInfo(2, 10), tmp_path, driver.NoCheckpoints())
    assert next(gen) == 0 and next(gen) == 1
    with pytest.raises(ValueError, match="Non-finite value detected!"):
        next(gen)
