"""CPU checks of the closure oracle (oracle/closure_oracle.py): its post-processing against the
reference's own functions (tests/golden/postproc.npz, made by postproc.calc_curl / calc_vmag),
its backward pass against finite differences of its forward pass, and its BF16 rounding."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import closure_oracle as co

GOLDEN = Path(__file__).resolve().parent / "golden" / "postproc.npz"


def test_postproc_matches_reference_golden():
    g = np.load(GOLDEN)
    np.testing.assert_array_equal(co.curl2d(g["vel2d"]), g["curl2d"])
    np.testing.assert_array_equal(co.curl3d(g["vel3d"]), g["curl3d"])
    np.testing.assert_array_equal(co.vmag(g["vel2d"]), g["vmag2d"])
    np.testing.assert_array_equal(co.vmag(g["vel3d"]), g["vmag3d"])


def test_bf16_rounding():
    vals = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.1415927, 1e-3, 0.0], np.float32)
    r = co.bf16(vals)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1). 1 + 1.5 * 2^-8 rounds up.
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125) and r[3] == np.float32(1.0078125)
    assert abs(r[4] + 3.140625) < 1e-7
    assert (co.bf16(r) == r).all()  # idempotent
    assert (r.view(np.uint32) & 0xFFFF == 0).all()


def _case(seed, B=2, nx=6, ny=5):
    rng = np.random.default_rng(seed)
    params = co.init_params(seed).astype(np.float64)
    x = rng.normal(size=(B, nx, ny, 4))
    flags = np.zeros((nx, ny), np.int32)
    flags[0, :] = 1
    flags[-1, 2] = 6
    target = rng.normal(size=(B, nx, ny))
    return params, x, flags, target


def _objective(params, x, flags, target):
    y = co.forward(params, x, exact=True)["y"]
    return co.loss(y, target, flags)[0]


def test_backward_matches_finite_differences():
    params, x, flags, target = _case(3)
    acts = co.forward(params, x, exact=True)
    _, dy = co.loss(acts["y"], target, flags)
    grad = co.backward(params, x, acts, dy, exact=True)
    rng = np.random.default_rng(4)
    # every bias, and a sample of each weight block
    idx = list(range(co.OFF["b1"], co.OFF["w2"])) + list(range(co.OFF["b2"], co.OFF["w3"])) + [co.OFF["b3"]]
    for lo, hi in ((co.OFF["w1"], co.OFF["b1"]), (co.OFF["w2"], co.OFF["b2"]), (co.OFF["w3"], co.OFF["b3"])):
        idx += list(rng.choice(np.arange(lo, hi), 40, replace=False))
    h = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        fd = (_objective(p1, x, flags, target) - _objective(p2, x, flags, target)) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_rounded_backward_close_to_exact():
    """The BF16 roundings the kernels apply move the gradient by well under a percent."""
    params, x, flags, target = _case(5, B=2, nx=12, ny=9)
    xr = co.bf16(x.astype(np.float32)).astype(np.float64)
    ea = co.forward(params, xr, exact=True)
    ra = co.forward(params, xr)
    _, dye = co.loss(ea["y"], target, flags)
    _, dyr = co.loss(ra["y"], target, flags)
    ge = co.backward(params, xr, ea, dye, exact=True)
    gr = co.backward(params, xr, ra, dyr)
    assert np.linalg.norm(gr - ge) / np.linalg.norm(ge) < 2e-2


def test_features_and_coarsen():
    rng = np.random.default_rng(1)
    nx, ny = 8, 12
    rho = (1 + 0.01 * rng.normal(size=(nx, ny))).astype(np.float32)
    vel = (0.05 * rng.normal(size=(nx, ny, 2))).astype(np.float32)
    flags = np.zeros((nx, ny), np.int32)
    flags[3, 4] = 1
    norm = np.array([0, 0, 0, 0, 100, 20, 20, 50], np.float32)
    x = co.features(rho, vel, flags, norm)
    assert x.shape == (1, nx, ny, 4) and (x[0, 3, 4] == 0).all()
    v = vel.copy()
    v[3, 4] = 0
    want = co.bf16(co.curl2d(v) * np.float32(50))
    want[3, 4] = 0
    np.testing.assert_array_equal(x[0, ..., 3], want)
    r, u, c, s = co.coarsen(rho, vel, rho, 4)
    assert r.shape == (2, 3) and u.shape == (2, 3, 2) and s.shape == (2, 3)
    blk = vel[:4, :4].reshape(-1, 2).astype(np.float64)
    k = 0.5 * ((blk - blk.mean(0)) ** 2).sum(1).mean()
    assert abs(s[0, 0] - np.sqrt(k)) < 1e-12
