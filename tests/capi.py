"""ctypes harness over the C ABI (include/lbm_cuda.h), used by the GPU parity tests to drive the
CUDA library directly, the way a foreign host layer (pyo3, cgo, ...) would."""

from __future__ import annotations

import ctypes as C

import numpy as np

from boltzmann_b200 import LIBRARY

_lib = C.CDLL(str(LIBRARY))
_lib.lbm_last_error.restype = C.c_char_p
_P = C.c_void_p

STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3}


def _ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"lbm error {rc}: {_lib.lbm_last_error().decode()}")


class CApiSim:
    """One lbm_sim handle plus host arrays, with the reference's iterate semantics."""

    def __init__(self, counts, kind: int, om_pos: float, om_neg: float = 0.0, q=None, storage="f32",
                 path: str = "auto"):
        self.counts = [int(c) for c in counts]
        self.d = len(self.counts)
        self.q = q or {2: 9, 3: 27}[self.d]
        self.h = C.c_void_p()
        arr = (C.c_int64 * self.d)(*self.counts)
        check(
            _lib.lbm_create(self.d, arr, self.q, kind, C.c_float(om_pos), C.c_float(om_neg),
                            STORAGE[storage], C.byref(self.h))
        )
        if path != "auto":
            self.set_kernel_path(path)
        self.flags = np.zeros(self.counts, np.int32)
        self.rho = np.ones(self.counts, np.float32)
        self.vel = np.zeros(self.counts + [self.d], np.float32)
        self.vals: list[np.ndarray] = []
        self.tq: list[int] = []
        self.iteration = 0

    def __del__(self):
        if getattr(self, "h", None):
            _lib.lbm_destroy(self.h)
            self.h = None

    def add_tracer(self, om: float, q=None, kind: int = 0, om_neg: float = 0.0) -> int:
        """kind 0: BGK with om; 1: TRT with (om, om_neg)."""
        idx = C.c_int()
        tq = q or {2: 5, 3: 7}[self.d]
        check(_lib.lbm_add_tracer(self.h, tq, kind, C.c_float(om), C.c_float(om_neg),
                                  C.byref(idx)))
        self.vals.append(np.zeros(self.counts, np.float32))
        self.tq.append(tq)
        return idx.value

    def set_tracer_storage(self, storage: str) -> int:
        """lbm_set_tracer_storage; returns the status (0 on success)."""
        return _lib.lbm_set_tracer_storage(self.h, STORAGE[storage])

    def set_gravity(self, g) -> None:
        g = np.ascontiguousarray(g, np.float32)
        check(_lib.lbm_set_gravity(self.h, _ptr(g)))

    def add_coupling(self, tracer: int, alpha: float, c0: float, g) -> None:
        g = np.ascontiguousarray(g, np.float32)
        check(_lib.lbm_add_coupling(self.h, tracer, C.c_float(alpha), C.c_float(c0), _ptr(g)))

    def iterate(self, n: int) -> None:
        if self.iteration == 0:
            check(_lib.lbm_upload_flags(self.h, _ptr(self.flags)))
            check(_lib.lbm_upload_fluid(self.h, _ptr(self.rho), _ptr(self.vel)))
            for t, v in enumerate(self.vals):
                check(_lib.lbm_upload_tracer(self.h, t, _ptr(v)))
            check(_lib.lbm_equilibrate(self.h))
        check(_lib.lbm_iterate(self.h, C.c_int64(n)))
        check(_lib.lbm_download_fluid(self.h, _ptr(self.rho), _ptr(self.vel)))
        for t, v in enumerate(self.vals):
            check(_lib.lbm_download_tracer(self.h, t, _ptr(v)))
        self.iteration += n

    def fluid_f64(self) -> tuple[np.ndarray, np.ndarray]:
        rho = np.empty(self.counts, np.float64)
        vel = np.empty(self.counts + [self.d], np.float64)
        check(_lib.lbm_download_fluid_f64(self.h, _ptr(rho), _ptr(vel)))
        return rho, vel

    def populations(self) -> np.ndarray:
        f = np.empty(self.counts + [self.q], np.float32)
        check(_lib.lbm_download_f(self.h, _ptr(f)))
        return f

    def tracer_populations(self, t: int) -> np.ndarray:
        g = np.empty(self.counts + [self.tq[t]], np.float32)
        check(_lib.lbm_download_g(self.h, t, _ptr(g)))
        return g

    def upload_populations(self, f: np.ndarray) -> None:
        check(_lib.lbm_upload_f(self.h, _ptr(np.ascontiguousarray(f, np.float32))))

    def conservation(self) -> np.ndarray:
        out = np.zeros(1 + self.d + len(self.vals), np.float64)
        check(_lib.lbm_conservation(self.h, _ptr(out), C.c_int(out.size)))
        return out

    def nonfinite(self) -> bool:
        v = C.c_int()
        check(_lib.lbm_nonfinite(self.h, C.byref(v)))
        return bool(v.value)

    def set_kernel_path(self, path: str) -> None:
        check(_lib.lbm_set_kernel_path(self.h, {"auto": 0, "direct": 1, "staged": 2}[path]))

    def raw_iterate(self, n: int) -> int:
        return _lib.lbm_iterate(self.h, C.c_int64(n))

    @staticmethod
    def last_error() -> str:
        return _lib.lbm_last_error().decode()
