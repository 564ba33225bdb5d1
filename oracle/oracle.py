"""TEST INFRASTRUCTURE: Python front end of the CPU checkers.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this module. It drives

* ``backend="port"``: the C restatement ``oracle/liblbm_oracle.so`` (FP32 or FP64), or
* ``backend="reference"``: the reference's own ``src/lib.cl`` kernels compiled as C++
  (``oracle/_ref/liblbm_ref.so``, FP32 only),

with the host-side semantics of the reference's ``Simulation`` (src/simulation.rs):

* fields live in the reference's host layouts (f ``[*counts, q]``, rho ``counts``,
  vel ``[*counts, d]``, flags i32);
* the first ``iterate`` call equilibrates f and every tracer's g from rho/vel/C in FP32
  (src/simulation.rs:283-286, src/fields.rs:106-114, 185-193, src/velocities.rs:43-52);
* the acceleration buffer is allocated (zeros) on the first call that has gravity or a coupling
  and persists (src/simulation.rs:288-295);
* ``iterate(n)`` rejects odd n (src/simulation.rs:279-281).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIBS: dict[str, C.CDLL] = {}

BGK, TRT = 0, 1
DEFAULT_Q = {1: 3, 2: 9, 3: 27}
DEFAULT_TRACER_Q = {1: 3, 2: 5, 3: 7}


def _lib(name: str) -> C.CDLL:
    if name not in _LIBS:
        path = HERE / "liblbm_oracle.so" if name == "port" else HERE / "_ref" / "liblbm_ref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (run oracle/build.py)")
        _LIBS[name] = C.CDLL(str(path))
    return _LIBS[name]


def reference_available() -> bool:
    return (HERE / "_ref" / "liblbm_ref.so").exists()


def _ptr(a: np.ndarray | None) -> C.c_void_p:
    return C.c_void_p(0 if a is None else a.ctypes.data)


@dataclass
class Omega:
    """Collision parameters, as the reference's ``Omega`` enum (src/fields.rs:37-41)."""

    kind: int  # BGK or TRT
    pos: float
    neg: float = 0.0

    @staticmethod
    def bgk(tau: float) -> "Omega":
        return Omega(BGK, np.float32(1.0 / tau))

    @staticmethod
    def trt(tau_pos: float, tau_neg: float | None = None, magic: float = 0.25) -> "Omega":
        # python/boltzmann/core.py:50-62
        tau_neg = tau_neg or (magic / (tau_pos - 0.5) + 0.5)
        return Omega(TRT, np.float32(1.0 / tau_pos), np.float32(1.0 / tau_neg))


@dataclass
class Tracer:
    q: int
    omega: Omega
    val: np.ndarray
    g: np.ndarray


@dataclass
class Coupling:
    tracer: str
    alpha: float
    c0: float
    gravity: np.ndarray


def equilibrate(d: int, q: int, rho: np.ndarray, vel: np.ndarray) -> np.ndarray:
    """Equilibrium populations [*shape, q] (src/velocities.rs:43-52), FP32 or FP64."""
    f64 = rho.dtype == np.float64
    dt = np.float64 if f64 else np.float32
    rho = np.ascontiguousarray(rho, dtype=dt)
    vel = np.ascontiguousarray(vel, dtype=dt)
    out = np.empty(rho.shape + (q,), dtype=dt)
    fn = _lib("port").lbm_oracle_equilibrate_f64 if f64 else _lib("port").lbm_oracle_equilibrate_f32
    rc = fn(C.c_int(d), C.c_int(q), C.c_int64(rho.size), _ptr(rho), _ptr(vel), _ptr(out))
    if rc != 0:
        raise ValueError(f"Unknown model: D{d}Q{q}")
    return out


def velocity_set(d: int, q: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(c [q, d] int, w [q] float64, opp [q] int) of the oracle's table."""
    c = np.zeros((q, d), np.int32)
    wn = np.zeros(q, np.int32)
    wd = np.zeros(q, np.int32)
    opp = np.zeros(q, np.int32)
    rc = _lib("port").lbm_oracle_velocity_set(d, q, _ptr(c), _ptr(wn), _ptr(wd), _ptr(opp))
    if rc != 0:
        raise ValueError(f"Unknown model: D{d}Q{q}")
    return c, wn / wd, opp


class OracleSimulation:
    """CPU stand-in for the reference's ``Simulation`` used to check the CUDA path."""

    def __init__(
        self,
        counts,
        omega: Omega,
        q: int | None = None,
        backend: str = "port",
        precision: str = "f32",
        nthreads: int = 0,
    ) -> None:
        if backend == "reference" and precision != "f32":
            raise ValueError("the reference kernels are FP32 only")
        self.counts = [int(c) for c in counts]
        self.d = len(self.counts)
        self.q = q or DEFAULT_Q[self.d]
        velocity_set(self.d, self.q)  # src/velocities.rs:62: unknown model fails at construction
        self.backend = backend
        self.precision = precision
        self.nthreads = nthreads
        self.dt = np.float64 if precision == "f64" else np.float32
        self.omega = omega
        self.flags = np.zeros(self.counts, np.int32)
        self.rho = np.ones(self.counts, self.dt)
        self.vel = np.zeros(self.counts + [self.d], self.dt)
        self.f = np.zeros(self.counts + [self.q], self.dt)
        self.acc: np.ndarray | None = None
        self.gravity: np.ndarray | None = None
        self.couplings: list[Coupling] = []
        self.tracers: dict[str, Tracer] = {}
        self.iteration = 0

    # -- configuration (src/simulation.rs:194-236, src/lib.rs:254-333) --
    def add_tracer(self, name: str, omega: Omega, q: int | None = None) -> Tracer:
        if name not in self.tracers:
            tq = q or DEFAULT_TRACER_Q[self.d]
            self.tracers[name] = Tracer(
                tq,
                omega,
                np.zeros(self.counts, self.dt),
                np.zeros(self.counts + [tq], self.dt),
            )
        return self.tracers[name]

    def set_gravity(self, g) -> None:
        self.gravity = np.asarray(g, self.dt).copy()

    def add_boussinesq_coupling(self, tracer: str, alpha: float, c0: float, g) -> None:
        assert tracer in self.tracers
        self.couplings.append(Coupling(tracer, alpha, c0, np.asarray(g, self.dt).copy()))

    def equilibrate(self) -> None:
        self.f = equilibrate(self.d, self.q, self.rho, self.vel)
        for t in self.tracers.values():
            t.g = equilibrate(self.d, t.q, t.val, self.vel)

    # -- the step loop --
    def iterate(self, iters: int) -> None:
        if iters % 2 != 0:
            raise ValueError("iters must be even")
        if self.iteration == 0:
            self.equilibrate()
        n = int(np.prod(self.counts))
        if (self.gravity is not None or self.couplings) and self.acc is None:
            self.acc = np.zeros((n, self.d), self.dt)

        names = list(self.tracers)
        tr = [self.tracers[k] for k in names]
        ntr = len(tr)
        dt = self.dt
        ct = C.c_double if dt == np.float64 else C.c_float
        arr_i = lambda xs: np.ascontiguousarray(np.asarray(xs, np.int32).reshape(-1))  # noqa: E731
        arr_r = lambda xs: np.ascontiguousarray(np.asarray(xs, dt).reshape(-1))  # noqa: E731
        c_tracer = arr_i([names.index(c.tracer) for c in self.couplings] or [0])
        c_alpha = arr_r([c.alpha for c in self.couplings] or [0])
        c_c0 = arr_r([c.c0 for c in self.couplings] or [0])
        c_g = arr_r([c.gravity for c in self.couplings] or [np.zeros(self.d)])
        t_q = arr_i([t.q for t in tr] or [0])
        t_col = arr_i([t.omega.kind for t in tr] or [0])
        t_om = arr_r([t.omega.pos for t in tr] or [0])
        t_om_neg = arr_r([t.omega.neg for t in tr] or [0])
        t_g = (C.c_void_p * max(ntr, 1))(*[t.g.ctypes.data for t in tr])
        t_C = (C.c_void_p * max(ntr, 1))(*[t.val.ctypes.data for t in tr])
        counts = np.asarray(self.counts, np.int64)
        for a in [self.flags, self.rho, self.vel, self.f] + [t.g for t in tr] + [t.val for t in tr]:
            assert a.flags.c_contiguous
        self.flags = np.ascontiguousarray(self.flags, np.int32)

        if self.backend == "reference":
            fn = _lib("reference").lbm_ref_iterate
        elif dt == np.float64:
            fn = _lib("port").lbm_oracle_iterate_f64
        else:
            fn = _lib("port").lbm_oracle_iterate_f32
        grav = None if self.gravity is None else np.ascontiguousarray(self.gravity, dt)
        rc = fn(
            C.c_int(self.d),
            _ptr(counts),
            _ptr(self.flags),
            C.c_int(self.q),
            C.c_int(self.omega.kind),
            ct(self.omega.pos),
            ct(self.omega.neg),
            _ptr(self.f),
            _ptr(self.rho),
            _ptr(self.vel),
            _ptr(self.acc),
            C.c_int(self.acc is not None),
            _ptr(grav),
            C.c_int(len(self.couplings)),
            _ptr(c_tracer),
            _ptr(c_alpha),
            _ptr(c_c0),
            _ptr(c_g),
            C.c_int(ntr),
            _ptr(t_q),
            _ptr(t_col),
            _ptr(t_om),
            _ptr(t_om_neg),
            t_g,
            t_C,
            C.c_int64(iters),
            C.c_int(self.nthreads),
        )
        if rc != 0:
            lib = _lib(self.backend)
            err_fn = lib.lbm_ref_last_error if self.backend == "reference" else lib.lbm_oracle_last_error
            err_fn.restype = C.c_char_p
            raise RuntimeError(err_fn().decode())
        self.iteration += iters


def default_threads() -> int:
    return len(os.sched_getaffinity(0))
