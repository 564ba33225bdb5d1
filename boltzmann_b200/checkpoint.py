"""Checkpoints in the reference's MessagePack layout (src/simulation.rs:448-479).

The reference serialises its whole ``Simulation`` with rmp-serde 1.3 (structs as positional
arrays) and ndarray 0.16 serde (an array is ``[version=1, dim, data]``), skipping device buffers
(src/opencl.rs:182-192):

    Simulation = [cells, fluid, tracers, gravity, iteration, couplings]
    cells      = [[flags], counts]                    flags i32 ndarray, counts usize ndarray
    fluid      = [[f], [rho], [vel], acc, model, omega]
    acc        = nil | [[acc]]
    model      = [ws, qs]                             f32 [q] and i32 [q, d] ndarrays
    omega      = {"BGK": w} | {"TRT": [w_pos, w_neg]}
    tracers    = {name: [[g], [C], model, omega]}
    gravity    = nil | [g]
    couplings  = [[tracer, alpha, c0, [g]], ...]

Populations are stored in the host layout [*counts, q], float32 elements as MessagePack
float32 (0xca), integers in their shortest encoding. Big arrays are encoded and decoded with
numpy. The byte layout follows those crates' documented conventions; no reference-written file
was available to compare bytes with, so only the round trip is pinned by tests.
"""

from __future__ import annotations

import os
import struct

import numpy as np

# Velocity-set tables of src/velocities.rs:66-191 (weights as f32 of the exact rationals).
_SETS = {
    (1, 3): ([(0,), (1,), (-1,)], [4 / 6, 1 / 6, 1 / 6]),
    (2, 9): (
        [(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)],
        [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4,
    ),
    (2, 5): ([(0, 0), (1, 0), (-1, 0), (0, 1), (0, -1)], [1 / 3] + [1 / 6] * 4),
    (3, 7): (
        [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)],
        [1 / 20] + [19 / 120] * 6,
    ),
}


def _d3q27():
    axis = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    edges = [(1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (0, 1, 1),
             (0, -1, -1), (1, 0, -1), (-1, 0, 1), (0, 1, -1), (0, -1, 1)]  # fmt: skip
    corners = [(1, 1, 1), (-1, -1, -1), (1, -1, 1), (-1, 1, -1), (1, 1, -1), (-1, -1, 1),
               (1, -1, -1), (-1, 1, 1)]  # fmt: skip
    ws = [8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8
    return axis + edges + corners, ws


_SETS[(3, 27)] = _d3q27()


def velocity_set(d: int, q: int) -> tuple[np.ndarray, np.ndarray]:
    qs, ws = _SETS[(d, q)]
    return np.asarray(ws, np.float32), np.asarray(qs, np.int32).reshape(q, d)


# ---------------------------------------------------------------------------------------------
# MessagePack writer


class _Writer:
    def __init__(self) -> None:
        self.parts: list[bytes] = []

    def raw(self, b: bytes) -> None:
        self.parts.append(b)

    def nil(self) -> None:
        self.raw(b"\xc0")

    def array_header(self, n: int) -> None:
        if n < 16:
            self.raw(bytes([0x90 | n]))
        elif n < 1 << 16:
            self.raw(b"\xdc" + struct.pack(">H", n))
        else:
            self.raw(b"\xdd" + struct.pack(">I", n))

    def map_header(self, n: int) -> None:
        if n < 16:
            self.raw(bytes([0x80 | n]))
        elif n < 1 << 16:
            self.raw(b"\xde" + struct.pack(">H", n))
        else:
            self.raw(b"\xdf" + struct.pack(">I", n))

    def string(self, s: str) -> None:
        b = s.encode()
        n = len(b)
        if n < 32:
            self.raw(bytes([0xA0 | n]) + b)
        elif n < 256:
            self.raw(b"\xd9" + bytes([n]) + b)
        elif n < 1 << 16:
            self.raw(b"\xda" + struct.pack(">H", n) + b)
        else:
            self.raw(b"\xdb" + struct.pack(">I", n) + b)

    def integer(self, v: int) -> None:
        self.raw(_int_bytes(int(v)))

    def f32(self, v: float) -> None:
        self.raw(b"\xca" + struct.pack(">f", v))

    def ndarray(self, a: np.ndarray) -> None:
        """ndarray serde: [1, dim, data]."""
        self.array_header(3)
        self.integer(1)
        self.array_header(a.ndim)
        for s in a.shape:
            self.integer(s)
        flat = np.ascontiguousarray(a).reshape(-1)
        self.array_header(flat.size)
        if flat.dtype == np.float32:
            rec = np.empty(flat.size, dtype=[("t", "u1"), ("v", ">f4")])
            rec["t"] = 0xCA
            rec["v"] = flat
            self.raw(rec.tobytes())
        elif flat.dtype.kind in "iu":
            if flat.size and flat.min() >= 0 and flat.max() < 128:
                self.raw(flat.astype(np.uint8).tobytes())
            else:
                self.raw(b"".join(_int_bytes(int(x)) for x in flat))
        else:
            raise TypeError(f"unsupported dtype {flat.dtype}")


def _int_bytes(v: int) -> bytes:
    if 0 <= v < 128:
        return bytes([v])
    if -32 <= v < 0:
        return struct.pack("b", v)
    if v >= 0:
        for code, fmt, lim in ((0xCC, ">B", 1 << 8), (0xCD, ">H", 1 << 16), (0xCE, ">I", 1 << 32)):
            if v < lim:
                return bytes([code]) + struct.pack(fmt, v)
        return b"\xcf" + struct.pack(">Q", v)
    for code, fmt, lim in ((0xD0, ">b", 1 << 7), (0xD1, ">h", 1 << 15), (0xD2, ">i", 1 << 31)):
        if v >= -lim:
            return bytes([code]) + struct.pack(fmt, v)
    return b"\xd3" + struct.pack(">q", v)


# ---------------------------------------------------------------------------------------------
# MessagePack reader (the subset the layout above uses)


class _Reader:
    def __init__(self, buf: bytes) -> None:
        self.b = memoryview(buf)
        self.p = 0

    def byte(self) -> int:
        v = self.b[self.p]
        self.p += 1
        return v

    def take(self, n: int) -> bytes:
        v = bytes(self.b[self.p : self.p + n])
        self.p += n
        return v

    def peek(self) -> int:
        return self.b[self.p]

    def array_header(self) -> int:
        t = self.byte()
        if 0x90 <= t <= 0x9F:
            return t & 0x0F
        if t == 0xDC:
            return struct.unpack(">H", self.take(2))[0]
        if t == 0xDD:
            return struct.unpack(">I", self.take(4))[0]
        raise ValueError(f"expected an array at byte {self.p - 1}")

    def map_header(self) -> int:
        t = self.byte()
        if 0x80 <= t <= 0x8F:
            return t & 0x0F
        if t == 0xDE:
            return struct.unpack(">H", self.take(2))[0]
        if t == 0xDF:
            return struct.unpack(">I", self.take(4))[0]
        raise ValueError(f"expected a map at byte {self.p - 1}")

    def is_nil(self) -> bool:
        if self.peek() == 0xC0:
            self.p += 1
            return True
        return False

    def string(self) -> str:
        t = self.byte()
        if 0xA0 <= t <= 0xBF:
            n = t & 0x1F
        elif t == 0xD9:
            n = self.byte()
        elif t == 0xDA:
            n = struct.unpack(">H", self.take(2))[0]
        elif t == 0xDB:
            n = struct.unpack(">I", self.take(4))[0]
        else:
            raise ValueError(f"expected a string at byte {self.p - 1}")
        return self.take(n).decode()

    def number(self):
        t = self.byte()
        if t < 0x80:
            return t
        if t >= 0xE0:
            return t - 0x100
        table = {
            0xCC: ">B", 0xCD: ">H", 0xCE: ">I", 0xCF: ">Q",
            0xD0: ">b", 0xD1: ">h", 0xD2: ">i", 0xD3: ">q",
            0xCA: ">f", 0xCB: ">d",
        }  # fmt: skip
        fmt = table.get(t)
        if fmt is None:
            raise ValueError(f"expected a number at byte {self.p - 1}")
        return struct.unpack(fmt, self.take(struct.calcsize(fmt)))[0]

    def ndarray(self, dtype) -> np.ndarray:
        if self.array_header() != 3:
            raise ValueError("ndarray must be [v, dim, data]")
        if self.number() != 1:
            raise ValueError("unsupported ndarray serialisation version")
        shape = tuple(int(self.number()) for _ in range(self.array_header()))
        n = self.array_header()
        if np.dtype(dtype) == np.float32:
            raw = np.frombuffer(self.b, dtype=[("t", "u1"), ("v", ">f4")], count=n, offset=self.p)
            if n and not (raw["t"] == 0xCA).all():
                raise ValueError("float32 array elements must be MessagePack float32")
            self.p += 5 * n
            data = raw["v"].astype(np.float32)
        else:
            head = np.frombuffer(self.b, dtype=np.uint8, count=n, offset=self.p)
            if (head < 0x80).all():
                data = head.astype(dtype)
                self.p += n
            else:
                data = np.array([self.number() for _ in range(n)], dtype=dtype)
        return data.reshape(shape)


# ---------------------------------------------------------------------------------------------


def _write_omega(w: _Writer, om) -> None:
    w.map_header(1)
    if om.kind == "BGK":
        w.string("BGK")
        w.f32(om._0)
    else:
        w.string("TRT")
        w.array_header(2)
        w.f32(om._0)
        w.f32(om._1)


def _read_omega(r: _Reader, Omega):
    if r.map_header() != 1:
        raise ValueError("Omega must be a one-entry map")
    kind = r.string()
    if kind == "BGK":
        return Omega.BGK(r.number())
    if r.array_header() != 2:
        raise ValueError("Omega.TRT needs two values")
    return Omega.TRT(r.number(), r.number())


def _write_model(w: _Writer, d: int, q: int) -> None:
    ws, qs = velocity_set(d, q)
    w.array_header(2)
    w.ndarray(ws)
    w.ndarray(qs)


def _read_model(r: _Reader) -> tuple[int, int]:
    if r.array_header() != 2:
        raise ValueError("model must be [ws, qs]")
    r.ndarray(np.float32)
    qs = r.ndarray(np.int32)
    return qs.shape[1], qs.shape[0]


def encode(sim) -> bytes:
    """Serialises a ``boltzmann_b200.boltzmann.Simulation``."""
    w = _Writer()
    counts = [int(c) for c in sim.cells.counts]
    d = len(counts)
    w.array_header(6)
    # cells
    w.array_header(2)
    w.array_header(1)
    w.ndarray(np.asarray(sim.cells.flags, np.int32))
    w.ndarray(np.asarray(counts, np.uint64))
    # fluid
    w.array_header(6)
    for arr in (sim._populations(), sim.fluid.rho, sim.fluid.vel):
        w.array_header(1)
        w.ndarray(np.asarray(arr, np.float32))
    if sim._acc_allocated:
        # The reference never reads acc back to its host array: it serialises zeros.
        w.array_header(1)
        w.ndarray(np.zeros(counts + [d], np.float32))
    else:
        w.nil()
    _write_model(w, d, sim._q)
    _write_omega(w, sim._omega)
    # tracers
    names = sim._tracer_names()
    w.map_header(len(names))
    for name in names:
        w.string(name)
        w.array_header(4)
        w.array_header(1)
        w.ndarray(np.asarray(sim._tracer_populations(name), np.float32))
        w.array_header(1)
        w.ndarray(np.asarray(sim.get_tracer(name).val, np.float32))
        _write_model(w, d, sim._tracer_q(name))
        _write_omega(w, sim._tracer_omega(name))
    # gravity
    g = sim._gravity
    if g is None:
        w.nil()
    else:
        w.array_header(1)
        w.ndarray(np.asarray(g, np.float32))
    w.integer(int(sim.iteration))
    couplings = sim._couplings()
    w.array_header(len(couplings))
    for tracer, alpha, c0, gc in couplings:
        w.array_header(4)
        w.string(tracer)
        w.f32(alpha)
        w.f32(c0)
        w.array_header(1)
        w.ndarray(np.asarray(gc, np.float32))
    return b"".join(w.parts)


def decode(buf: bytes, storage: str = "f32"):
    """Rebuilds a Simulation from checkpoint bytes and uploads it (src/simulation.rs:464-479)."""
    from boltzmann_b200.boltzmann import Omega, Simulation

    r = _Reader(buf)
    if r.array_header() != 6:
        raise ValueError("not a boltzmann checkpoint")
    if r.array_header() != 2 or r.array_header() != 1:
        raise ValueError("bad cells record")
    flags = r.ndarray(np.int32)
    counts = [int(c) for c in r.ndarray(np.uint64)]
    if r.array_header() != 6:
        raise ValueError("bad fluid record")
    fields = []
    for _ in range(3):
        if r.array_header() != 1:
            raise ValueError("bad fluid field")
        fields.append(r.ndarray(np.float32))
    f, rho, vel = fields
    acc_allocated = not r.is_nil()
    if acc_allocated:
        if r.array_header() != 1:
            raise ValueError("bad acc field")
        r.ndarray(np.float32)
    _, q = _read_model(r)
    omega = _read_omega(r, Omega)
    tracers = []
    for _ in range(r.map_header()):
        name = r.string()
        if r.array_header() != 4 or r.array_header() != 1:
            raise ValueError("bad tracer record")
        g = r.ndarray(np.float32)
        if r.array_header() != 1:
            raise ValueError("bad tracer record")
        val = r.ndarray(np.float32)
        _, tq = _read_model(r)
        tracers.append((name, g, val, tq, _read_omega(r, Omega)))
    gravity = None
    if not r.is_nil():
        if r.array_header() != 1:
            raise ValueError("bad gravity record")
        gravity = r.ndarray(np.float32)
    iteration = int(r.number())
    couplings = []
    for _ in range(r.array_header()):
        if r.array_header() != 4:
            raise ValueError("bad coupling record")
        tracer = r.string()
        alpha = float(r.number())
        c0 = float(r.number())
        if r.array_header() != 1:
            raise ValueError("bad coupling record")
        couplings.append((tracer, alpha, c0, r.ndarray(np.float32)))

    sim = Simulation("gpu", counts, omega, q=q, storage=storage)
    sim.cells.flags[...] = flags.reshape(counts)
    sim.fluid.rho[...] = rho.reshape(counts)
    sim.fluid.vel[...] = vel.reshape(counts + [len(counts)])
    tracer_g = {}
    for name, g, val, tq, tom in tracers:
        sim.add_tracer(name, tom, tq).val[...] = val.reshape(counts)
        tracer_g[name] = g
    if gravity is not None:
        sim.set_gravity(gravity)
    for tracer, alpha, c0, gc in couplings:
        sim.add_boussinesq_coupling(sim.get_tracer(tracer), alpha, c0, gc)
    sim._restore(f, tracer_g, iteration, acc_allocated)
    return sim


def write_checkpoint(sim, path: str) -> None:
    """``Simulation.write_checkpoint`` (src/simulation.rs:448-462)."""
    data = encode(sim)
    with open(path, "wb") as fh:
        fh.write(data)


def load_checkpoint(path: str, storage: str = "f32"):
    """``Simulation.load_checkpoint`` (src/simulation.rs:464-479)."""
    with open(os.fspath(path), "rb") as fh:
        return decode(fh.read(), storage)
