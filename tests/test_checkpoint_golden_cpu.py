"""Checkpoint bytes: boltzmann_b200.checkpoint.encode against tests/golden/checkpoint_d2q9_2x2.mpk,
the bytes the reference's write_checkpoint (src/simulation.rs:448-462) produces for a 2 x 2 D2Q9
simulation with one tracer, gravity and a coupling, assembled by hand from the MessagePack
specification and the rmp-serde / ndarray serde conventions by
tests/golden/make_checkpoint_golden.py (independently of the encoder under test). No GPU needed:
the encoder reads a simulation's host mirrors, here a stand-in holding the same arrays."""

from __future__ import annotations

import types
from pathlib import Path

import numpy as np

from tests.golden import make_checkpoint_golden as gold

GOLDEN = Path(__file__).resolve().parent / "golden" / "checkpoint_d2q9_2x2.mpk"


class _Omega:
    def __init__(self, w: float) -> None:
        self.kind, self._0, self._1 = "BGK", w, None


class _StandIn:
    """The attributes boltzmann_b200.checkpoint.encode reads from a Simulation."""

    def __init__(self) -> None:
        self.cells = types.SimpleNamespace(counts=list(gold.COUNTS),
                                           flags=np.asarray(gold.FLAGS, np.int32))
        self.fluid = types.SimpleNamespace(rho=np.asarray(gold.rho_values(), np.float32),
                                           vel=np.asarray(gold.vel_values(), np.float32))
        self._acc_allocated = True
        self._q = 9
        self._omega = _Omega(gold.OMEGA)
        self._gravity = np.asarray(gold.GRAVITY, np.float32)
        self.iteration = gold.ITERATION
        self._dye = types.SimpleNamespace(val=np.asarray(gold.c_values(), np.float32))

    def _populations(self):
        return np.asarray(gold.f_values(), np.float32)

    def _tracer_names(self):
        return ["dye"]

    def _tracer_populations(self, name):
        return np.asarray(gold.g_values(), np.float32)

    def get_tracer(self, name):
        return self._dye

    def _tracer_q(self, name):
        return 5

    def _tracer_omega(self, name):
        return _Omega(gold.TRACER_OMEGA)

    def _couplings(self):
        name, alpha, c0, g = gold.COUPLING
        return [(name, alpha, c0, np.asarray(g, np.float32))]


def test_golden_file_is_what_the_generator_writes():
    assert GOLDEN.read_bytes() == gold.build()


def test_encoder_reproduces_the_golden_bytes():
    from boltzmann_b200 import checkpoint

    got = checkpoint.encode(_StandIn())
    want = GOLDEN.read_bytes()
    if got != want:
        n = min(len(got), len(want))
        i = next((k for k in range(n) if got[k] != want[k]), n)
        raise AssertionError(f"first difference at byte {i}: {got[max(0, i - 8):i + 8].hex()} vs "
                             f"{want[max(0, i - 8):i + 8].hex()} (lengths {len(got)}, {len(want)})")


def test_golden_parses_back_to_the_arrays():
    from boltzmann_b200 import checkpoint

    r = checkpoint._Reader(GOLDEN.read_bytes())
    assert r.array_header() == 6
    assert r.array_header() == 2 and r.array_header() == 1
    np.testing.assert_array_equal(r.ndarray(np.int32), np.asarray(gold.FLAGS, np.int32))
    np.testing.assert_array_equal(r.ndarray(np.uint64), gold.COUNTS)
    assert r.array_header() == 6 and r.array_header() == 1
    np.testing.assert_array_equal(r.ndarray(np.float32), np.asarray(gold.f_values(), np.float32))
