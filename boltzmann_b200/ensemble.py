"""Batched ensembles of independent 2D D2Q9 domains on one GPU (parameter sweeps).

No counterpart in the reference, which runs one domain per ``Simulation``: here all domains live
in one population array and advance with one launch per step (or a replayed CUDA graph of such
launches). Host arrays follow the reference's per-domain layout, concatenated in domain order;
``Ensemble.domain(i)`` gives per-domain views.

    ens = Ensemble([(L1, L1), (L2, L2), ...], tau=[...])
    ens.flags[...] = ...; ens.vel[...] = ...
    ens.iterate(1000, mode="graph")
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from boltzmann_b200 import LIBRARY

_lib = C.CDLL(str(LIBRARY))
_lib.lbm_last_error.restype = C.c_char_p

MODES = {"persistent": 0, "graph": 1, "per_domain": 2}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2}


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_lib.lbm_last_error().decode())


def _ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


class Ensemble:
    """Independent D2Q9 domains advanced together. ``omega`` per domain: BGK rates
    (``tau`` is the convenience form 1/omega)."""

    def __init__(self, counts, tau=None, omega=None, omega_neg=None, storage: str = "f32"):
        self.counts = [(int(a), int(b)) for a, b in counts]
        if omega is None:
            omega = [1.0 / t for t in tau]
        self.collision = 0 if omega_neg is None else 1
        om = np.asarray(omega, np.float32)
        om_neg = None if omega_neg is None else np.asarray(omega_neg, np.float32)
        arr = np.asarray(self.counts, np.int64).reshape(-1)
        self.h = C.c_void_p()
        _check(
            _lib.lbm_ensemble_create(
                len(self.counts), _ptr(arr), self.collision, _ptr(om),
                None if om_neg is None else _ptr(om_neg), STORAGE[storage], C.byref(self.h),
            )
        )
        n = C.c_int64()
        _check(_lib.lbm_ensemble_cells(self.h, C.byref(n)))
        self.n = n.value
        self.flags = np.zeros(self.n, np.int32)
        self.rho = np.ones(self.n, np.float32)
        self.vel = np.zeros((self.n, 2), np.float32)
        self.iteration = 0
        # The library's default: the row-staged kernel (tile 0) when every row has at most 512
        # cells, else tiles of 256 cells; CTAs per SM as many as fit.
        self.shape = (0 if max(b for _, b in self.counts) <= 512 else 256, 0)

    def __del__(self):
        if getattr(self, "h", None):
            _lib.lbm_ensemble_destroy(self.h)
            self.h = None

    def domain(self, i: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(flags, rho, vel) views of domain i in its own [nx, ny] shape."""
        start = sum(a * b for a, b in self.counts[:i])
        a, b = self.counts[i]
        sl = slice(start, start + a * b)
        return (self.flags[sl].reshape(a, b), self.rho[sl].reshape(a, b),
                self.vel[sl].reshape(a, b, 2))

    def set_shape(self, tile_cells: int, blocks_per_sm: int = 0) -> None:
        _check(_lib.lbm_ensemble_set_shape(self.h, tile_cells, blocks_per_sm))
        self.shape = (tile_cells, blocks_per_sm)

    def upload(self) -> None:
        _check(_lib.lbm_ensemble_upload(self.h, _ptr(self.flags), _ptr(self.rho), _ptr(self.vel)))

    def iterate(self, iters: int, mode: str = "graph", read_back: bool = True) -> None:
        """As Simulation.iterate: the first call uploads and equilibrates, every call reads
        rho and vel back (unless read_back is False)."""
        if iters % 2:
            raise ValueError("iters must be even")
        if self.iteration == 0:
            self.upload()
            _check(_lib.lbm_ensemble_equilibrate(self.h))
        _check(_lib.lbm_ensemble_iterate(self.h, C.c_int64(iters), MODES[mode]))
        if read_back:
            _check(_lib.lbm_ensemble_download(self.h, _ptr(self.rho), _ptr(self.vel)))
        self.iteration += iters

    def synchronize(self) -> None:
        _check(_lib.lbm_ensemble_synchronize(self.h))

    def stream(self) -> int:
        p = C.c_void_p()
        _check(_lib.lbm_ensemble_stream(self.h, C.byref(p)))
        return p.value or 0

    def populations(self) -> np.ndarray:
        f = np.empty((self.n, 9), np.float32)
        _check(_lib.lbm_ensemble_download_f(self.h, _ptr(f)))
        return f

    def set_populations(self, f: np.ndarray) -> None:
        _check(_lib.lbm_ensemble_upload_f(self.h, _ptr(np.ascontiguousarray(f, np.float32))))
