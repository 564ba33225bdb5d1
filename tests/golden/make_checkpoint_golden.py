"""Writes tests/golden/checkpoint_d2q9_2x2.mpk: the checkpoint bytes the reference's
``Simulation::write_checkpoint`` (src/simulation.rs:448-462) produces for a tiny simulation,
assembled here by hand from the MessagePack specification and the serde conventions of the crates
the reference serialises with, independently of boltzmann_b200/checkpoint.py:

  - rmp-serde 1.3 ``Serializer::new`` (its default configuration): a struct is an array of its
    fields in declaration order; ``Option::None`` is nil and ``Some(v)`` is v itself; an
    externally tagged enum variant is a one-entry map {name: value} (a tuple variant's value an
    array); integers take their shortest encoding; f32 is float 32 (0xca);
  - ndarray 0.16 serde: an array is the struct [v = 1, dim, data] (dim one entry per axis, data
    the elements in standard order);
  - the reference's structs (src/simulation.rs:23-29, 93-104, 130-140; src/fields.rs:54-65,
    142-148; src/velocities.rs:15-18; src/opencl.rs:183-192, whose device buffer is skipped):
      Simulation = [cells, fluid, tracers, gravity, iteration, couplings]
      Cells      = [flags: Data, counts: Array1<usize>]
      Fluid      = [f: Data, rho: Data, vel: Data, acc: Option<Data>, model, omega]
      Scalar     = [g: Data, C: Data, model, omega]
      Data       = [host ndarray]
      VelocitySet = [ws: Array1<f32>, qs: Array2<i32>]
      BoussinesqCoupling = [tracer, alpha, c0, gravity: Data]

The case: D2Q9 BGK (omega 1.25) on 2 x 2 cells with flags [[1, 0], [0, 6]], one D2Q5 BGK tracer
"dye" (omega 1.5), gravity (0, -0.5) and one coupling to "dye" (alpha 0.25, c0 0, g (0, -1)),
after 4 iterations; every value is exact in float32. Run from the repository root:
    python tests/golden/make_checkpoint_golden.py
"""

from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "checkpoint_d2q9_2x2.mpk"

COUNTS = [2, 2]
FLAGS = [[1, 0], [0, 6]]
OMEGA, TRACER_OMEGA = 1.25, 1.5
GRAVITY = [0.0, -0.5]
ITERATION = 4
COUPLING = ("dye", 0.25, 0.0, [0.0, -1.0])


def f_values():
    """Populations [2, 2, 9]: cell c, slot i -> (16 + 4 c + i) / 64."""
    return [[[(16 + 4 * (2 * x + y) + i) / 64 for i in range(9)] for y in range(2)]
            for x in range(2)]


def rho_values():
    return [[1.0, 1.0625], [0.9375, 1.125]]


def vel_values():
    return [[[0.0, 0.0], [0.03125, -0.015625]], [[0.0078125, 0.0], [0.046875, 0.0]]]


def g_values():
    return [[[(1 + 2 * (2 * x + y) + i) / 32 for i in range(5)] for y in range(2)]
            for x in range(2)]


def c_values():
    return [[0.0, 1.0], [0.5, 0.25]]


# D2Q9 and D2Q5 of src/velocities.rs:66-107 (weights as f32 of the exact rationals).
D2Q9_QS = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)]
D2Q9_WS = [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4
D2Q5_QS = [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)]
D2Q5_WS = [1 / 3] + [1 / 6] * 4


# ---- MessagePack by hand -------------------------------------------------------------------

def arr(n: int) -> bytes:
    assert n < 16
    return bytes([0x90 | n])


def fmap(n: int) -> bytes:
    assert n < 16
    return bytes([0x80 | n])


def fstr(s: str) -> bytes:
    b = s.encode()
    assert len(b) < 32
    return bytes([0xA0 | len(b)]) + b


def uint(v: int) -> bytes:
    assert 0 <= v < 128
    return bytes([v])


def sint(v: int) -> bytes:
    if 0 <= v < 128:
        return bytes([v])
    assert -32 <= v < 0
    return bytes([0x100 + v])


def f32(v: float) -> bytes:
    assert float(np.float32(v)) == v or v in (4 / 9, 1 / 9, 1 / 36, 1 / 3, 1 / 6)
    return b"\xca" + struct.pack(">f", v)


def ndarray(shape, flat, elem) -> bytes:
    out = arr(3) + uint(1) + arr(len(shape)) + b"".join(uint(s) for s in shape)
    n = len(flat)
    out += arr(n) if n < 16 else b"\xdc" + struct.pack(">H", n)
    return out + b"".join(elem(v) for v in flat)


def flat(nested):
    return np.asarray(nested, np.float64).reshape(-1).tolist()


def model(ws, qs) -> bytes:
    return arr(2) + ndarray([len(ws)], ws, f32) + ndarray([len(qs), 2],
                                                         [c for q in qs for c in q], sint)


def build() -> bytes:
    out = arr(6)
    # cells = [Data(flags), counts]
    out += arr(2) + arr(1) + ndarray([2, 2], [v for row in FLAGS for v in row], sint)
    out += ndarray([2], COUNTS, uint)
    # fluid = [Data(f), Data(rho), Data(vel), Some(Data(acc)) = zeros, model, omega]
    out += arr(6)
    out += arr(1) + ndarray([2, 2, 9], flat(f_values()), f32)
    out += arr(1) + ndarray([2, 2], flat(rho_values()), f32)
    out += arr(1) + ndarray([2, 2, 2], flat(vel_values()), f32)
    out += arr(1) + ndarray([2, 2, 2], [0.0] * 8, f32)  # acc: allocated, never read back
    out += model(D2Q9_WS, D2Q9_QS)
    out += fmap(1) + fstr("BGK") + f32(OMEGA)
    # tracers = {"dye": [Data(g), Data(C), model, omega]}
    out += fmap(1) + fstr("dye") + arr(4)
    out += arr(1) + ndarray([2, 2, 5], flat(g_values()), f32)
    out += arr(1) + ndarray([2, 2], flat(c_values()), f32)
    out += model(D2Q5_WS, D2Q5_QS)
    out += fmap(1) + fstr("BGK") + f32(TRACER_OMEGA)
    # gravity = Some(Data(g)), iteration, couplings
    out += arr(1) + ndarray([2], GRAVITY, f32)
    out += uint(ITERATION)
    name, alpha, c0, g = COUPLING
    out += arr(1) + arr(4) + fstr(name) + f32(alpha) + f32(c0) + arr(1) + ndarray([2], g, f32)
    return out


def main() -> None:
    OUT.write_bytes(build())
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
