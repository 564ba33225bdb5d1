"""lbm_population_sums_noalloc against lbm_conservation.

The allocation-free entry point serves callers that cannot allocate device memory (a solver
embedded in another framework's memory arena, or running under an allocator that forbids extra
cudaMalloc calls): they pass populations they already own and an output buffer, and the library
uses only a fixed scratch array of its own. Here the caller's buffers come from torch, and the
result must equal the sums of the existing, allocating entry point over the same populations.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_CELLS = 2048 * 65536


def _sums_without_allocation(lib, d, q, f_dev, n, out_dev, stream):
    return lib.lbm_population_sums_noalloc(
        C.c_int(d), C.c_int(q), C.c_int(0), C.c_void_p(f_dev), C.c_int64(n), C.c_void_p(out_dev),
        C.c_void_p(stream),
    )


def _case(counts, seed):
    from tests.capi import CApiSim

    rng = np.random.default_rng(seed)
    sim = CApiSim(counts, 0, 1 / 0.6)
    sim.rho[...] = (1 + rng.uniform(-0.02, 0.02, sim.rho.shape)).astype(np.float32)
    sim.vel[...] = rng.uniform(-0.05, 0.05, sim.vel.shape).astype(np.float32)
    sim.iterate(10)
    return sim


def test_noalloc_sums_match_existing_entry_point():
    import torch

    from tests.capi import _lib

    stream = torch.cuda.current_stream().cuda_stream
    # Several calls in a row, alternating shapes, so stale scratch from one call would show up
    # in the next.
    for counts, seed in (([40, 300], 1), ([12, 10, 20], 2), ([40, 300], 3)):
        sim = _case(counts, seed)
        d, q = len(counts), sim.q
        n = int(np.prod(counts))
        existing = sim.conservation()[: 1 + d]
        soa = np.ascontiguousarray(sim.populations().reshape(n, q).T)  # [q][n]
        f = torch.from_numpy(soa).cuda()
        out = torch.full((1 + d,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _sums_without_allocation(_lib, d, q, f.data_ptr(), n, out.data_ptr(), stream)
        assert rc == 0, _lib.lbm_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # FP64 sums of the same FP32 values, added in a different order.
        np.testing.assert_allclose(got, existing, rtol=0, atol=1e-12 * existing[0])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from tests.capi import _lib

    f = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _sums_without_allocation(_lib, 2, 9, f.data_ptr(), MAX_CELLS + 1, out.data_ptr(), 0)
    assert rc == 1
    assert b"exceeds the maximum" in _lib.lbm_last_error()
