"""The bounded waits of the tensor-memory-accelerated kernels give up cleanly.

The TMA-staged AA kernel and the fused closure kernel never wait without a bound: a wait that runs
out records a status bit, the kernel still drains the copies or tensor-core products it issued
(with the default bound) and returns. These tests make the pipeline waits run out on purpose --
the spin limit set to 0 polls, a wait that gives up at once -- and check that the failure is
reported on the host, once, and that the simulation and the closure work again afterwards. Nothing
here faults or hangs a GPU: every wait still ends, and no copy outlives its kernel.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LBM_ERR_CUDA, LBM_ERR_STATE = 3, 4


def _staged_sim(seed: int, storage: str = "f32"):
    from tests.capi import CApiSim

    counts = [4, 4, 256]  # one-tile rows: even steps by four-row tensor copies, odd by boxes
    rng = np.random.default_rng(seed)
    sim = CApiSim(counts, 0, 1 / 0.55, storage=storage, path="staged")
    sim.rho[...] = (1 + rng.uniform(-0.01, 0.01, counts)).astype(np.float32)
    sim.vel[...] = rng.uniform(-0.05, 0.05, counts + [3]).astype(np.float32)
    return sim


def _counts(sim):
    from tests.capi import _lib

    direct, staged = C.c_int64(), C.c_int64()
    assert _lib.lbm_launch_counts(sim.h, C.byref(direct), C.byref(staged)) == 0
    return direct.value, staged.value


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_staged_kernel_wait_timeout_is_reported_once_and_recoverable(storage):
    from tests.capi import _lib, check

    sim = _staged_sim(3, storage)
    sim.iterate(2)
    f_start = sim.populations()

    # Every pipeline wait gives up at once: the steps are enqueued, the kernels return early and
    # the next synchronising call reports it.
    check(_lib.lbm_set_spin_limit(sim.h, C.c_int64(0)))
    assert sim.raw_iterate(4) == 0
    assert _lib.lbm_synchronize(sim.h) == LBM_ERR_CUDA
    assert "status bit 1" in sim.last_error()
    assert _lib.lbm_synchronize(sim.h) == 0  # reported once
    assert _counts(sim) == (0, 6)  # the staged kernel ran (and gave up) in each of those steps

    # Default limit again: restore the populations and continue; the result equals a run of the
    # same steps that never timed out (with the same download/upload round trip), bit for bit.
    check(_lib.lbm_set_spin_limit(sim.h, C.c_int64(-1)))
    sim.upload_populations(f_start)
    sim.iterate(4)
    ref = _staged_sim(3, storage)
    ref.iterate(2)
    ref.upload_populations(ref.populations())
    ref.iterate(4)
    np.testing.assert_array_equal(sim.rho, ref.rho)
    np.testing.assert_array_equal(sim.vel, ref.vel)
    assert np.isfinite(sim.rho).all()


def test_staged_kernel_with_a_generous_limit_runs_normally():
    from tests.capi import _lib, check

    sim = _staged_sim(4)
    check(_lib.lbm_set_spin_limit(sim.h, C.c_int64(1 << 20)))
    sim.iterate(4)
    ref = _staged_sim(4)
    ref.iterate(4)
    np.testing.assert_array_equal(sim.rho, ref.rho)
    assert _lib.lbm_synchronize(sim.h) == 0


def test_closure_wait_timeout_is_reported_and_recoverable():
    import torch

    from boltzmann_b200 import closure as cl
    from oracle import closure_oracle as co

    nx, ny = 30, 70
    rng = np.random.default_rng(5)
    rho = torch.tensor((1 + 0.01 * rng.normal(size=(nx, ny))).astype(np.float32), device="cuda")
    vel = torch.tensor((0.05 * rng.normal(size=(nx, ny, 2))).astype(np.float32), device="cuda")
    flags = torch.zeros((nx, ny), dtype=torch.int32, device="cuda")
    norm = np.array([0.0, 0.01, 0.0, 0.0, 80.0, 15.0, 20.0, 30.0], np.float32)
    net = cl.Net(co.init_params(4), norm, gain=0.02, max_dtau=0.05)
    good = torch.full((nx * ny,), float("nan"), device="cuda")
    cl.relaxation(net, rho, vel, flags, nx, ny, 0.51, good, 0)
    torch.cuda.synchronize()
    cl.status()

    try:
        assert cl._lib.lbm_closure_set_spin_limit(0) == 0
        out = torch.full((nx * ny,), float("nan"), device="cuda")
        cl.relaxation(net, rho, vel, flags, nx, ny, 0.51, out, 0)
        torch.cuda.synchronize()
        assert cl._lib.lbm_closure_status() == LBM_ERR_STATE
        assert b"gave up waiting" in cl._lib.lbm_last_error()
        assert cl._lib.lbm_closure_status() == 0  # cleared by the query
    finally:
        assert cl._lib.lbm_closure_set_spin_limit(-1) == 0

    again = torch.full((nx * ny,), float("nan"), device="cuda")
    cl.relaxation(net, rho, vel, flags, nx, ny, 0.51, again, 0)
    torch.cuda.synchronize()
    cl.status()
    assert torch.equal(again, good)
