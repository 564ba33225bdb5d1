"""lbm_iterate's CUDA-graph replay: the step pairs of a call before its last one go out as
captured graphs of 8 to 16 pairs while that many are left, each captured once per simulation
state and replayed. The
results must be the bits of the same steps launched one pair per call (no graph), the library's
launch counters must count the replayed launches, and a setter that changes what a step launches
must drop the captured graphs."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from tests.capi import _lib
from tests.golden.make_golden import seeded_inputs
from tests.test_gpu_parity import TMA_CASES, _capi_from_spec

pytestmark = pytest.mark.gpu


def _counts(sim) -> tuple[int, int]:
    d, s = C.c_int64(), C.c_int64()
    assert _lib.lbm_launch_counts(sim.h, C.byref(d), C.byref(s)) == 0
    return d.value, s.value


def _state(sim, index) -> list[np.ndarray]:
    out = [sim.populations(), sim.rho.copy(), sim.vel.copy()]
    for t in index.values():
        out += [sim.vals[t].copy(), sim.tracer_populations(t)]
    return out


def _pair(name, path, storage="f32"):
    spec = TMA_CASES[name]
    inputs = seeded_inputs(spec, seed=23)
    a, ia = _capi_from_spec(spec, inputs, storage=storage, path=path)
    b, ib = _capi_from_spec(spec, inputs, storage=storage, path=path)
    return a, ia, b, ib


@pytest.mark.parametrize("path", ["staged", "direct"])
@pytest.mark.parametrize("name,storage", [("d2q9_trt_tracer_coupling", "f32"),
                                          ("d2q9_trt_tracer_coupling", "f16"),
                                          ("d3q27_single_row", "f32")])
def test_graph_replay_matches_single_calls(name, storage, path):
    a, ia, b, ib = _pair(name, path, storage)
    a.iterate(2)  # upload + equilibrate, no graph
    b.iterate(2)
    a.iterate(40)  # 1 pair directly, a graph of 16 pairs, 3 pairs directly
    for _ in range(20):
        b.iterate(2)
    for x, y in zip(_state(a, ia), _state(b, ib)):
        np.testing.assert_array_equal(x, y)
    assert _counts(a) == _counts(b)
    assert sum(_counts(a)) == 42
    a.iterate(76)  # the graph of 16 pairs replayed twice, 6 pairs directly
    a.iterate(22)  # a new graph of 10 pairs
    for _ in range(38 + 11):
        b.iterate(2)
    for x, y in zip(_state(a, ia), _state(b, ib)):
        np.testing.assert_array_equal(x, y)
    assert _counts(a) == _counts(b)


def test_graph_dropped_when_gravity_changes():
    a, ia, b, ib = _pair("d2q9_bgk_gravity_long_rows", "staged")
    for sim in (a, b):
        sim.iterate(2)
    a.iterate(40)
    for _ in range(20):
        b.iterate(2)
    for sim in (a, b):
        sim.set_gravity([2e-4, -1e-3])
    a.iterate(40)  # a graph captured with the old gravity must not be replayed
    for _ in range(20):
        b.iterate(2)
    # (a replay of a graph captured with the old gravity would make a differ from b)
    for x, y in zip(_state(a, ia), _state(b, ib)):
        np.testing.assert_array_equal(x, y)
