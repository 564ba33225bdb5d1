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


def _encoded(storage, v32, w32):
    """The device encoding of float populations v32 [q][n]: float, the 16-bit offsets v - w
    (as the library stores them), or double."""
    import torch

    if storage == "f32":
        return torch.from_numpy(v32)
    if storage == "f64":
        return torch.from_numpy(v32.astype(np.float64))
    dev = torch.from_numpy(v32 - w32[:, None])  # exact: v and w are within a factor of 2
    return dev.to(torch.float16 if storage == "f16" else torch.bfloat16)


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64"])
@pytest.mark.parametrize("counts", [[300, 500], [40, 40, 60]])
def test_noalloc_sums_every_storage_kind_over_several_partials(storage, counts):
    """150,000 and 96,000 cells: three and two per-block partials in the scratch array. The
    populations are uploaded to a simulation of the same storage kind, whose own conservation
    sums (the existing entry point) are the reference; the caller's array is the same values in
    that storage's encoding. Deviations are kept at least 5% of each weight, so the 16-bit
    encodings made here and on the device agree bit for bit."""
    import torch

    from oracle.oracle import velocity_set
    from tests.capi import STORAGE, CApiSim, _lib

    d = len(counts)
    n = int(np.prod(counts))
    c, wn, _ = velocity_set(d, {2: 9, 3: 27}[d])
    q = len(wn)
    w32 = (np.rint(wn * 216 * 216).astype(np.float32) / np.float32(216 * 216)).astype(np.float32)
    rng = np.random.default_rng(11 + d)
    frac = rng.uniform(0.05, 0.3, (q, n)) * rng.choice([-1.0, 1.0], (q, n))
    v32 = (w32[:, None] * (1.0 + frac)).astype(np.float32)  # [q][n]

    sim = CApiSim(counts, 0, 1 / 0.6, storage=storage)
    sim.upload_populations(np.ascontiguousarray(v32.T.reshape(counts + [q])))
    existing = sim.conservation()[: 1 + d]

    f = _encoded(storage, v32, w32).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row on the shared scratch
        out = torch.full((1 + d,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _lib.lbm_population_sums_noalloc(
            C.c_int(d), C.c_int(q), C.c_int(STORAGE[storage]), C.c_void_p(f.data_ptr()),
            C.c_int64(n), C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert rc == 0, _lib.lbm_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, existing, rtol=0, atol=1e-12 * existing[0])
    # and against the host's FP64 sums of the decoded values
    if storage in ("f16", "bf16"):
        decoded = f.float().cpu().numpy() + w32[:, None]
    else:
        decoded = f.cpu().numpy()
    decoded = decoded.astype(np.float64)
    host = [decoded.sum()] + [(c[:, k, None] * decoded).sum() for k in range(d)]
    np.testing.assert_allclose(got, host, rtol=0, atol=1e-12 * host[0])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from tests.capi import _lib

    f = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _sums_without_allocation(_lib, 2, 9, f.data_ptr(), MAX_CELLS + 1, out.data_ptr(), 0)
    assert rc == 1
    assert b"exceeds the maximum" in _lib.lbm_last_error()
