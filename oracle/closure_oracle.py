"""CPU oracle for the learned closure and the on-device post-processing (test infrastructure).

Only the tests, ``__graft_entry__.smoke()`` and the CPU leg of ``bench.py`` use this module, as
the checker of the CUDA kernels in ``boltzmann_b200/csrc/closure.cu``; the product never calls it.

* ``curl2d`` / ``curl3d`` / ``vmag`` restate python/boltzmann/utils/postproc.py:12-82
  (``calc_vmag``, ``calc_curl``: ``np.gradient`` derivatives, d(u_x)/dy - d(u_y)/dx in 2D).
  Pinned by ``tests/golden/postproc.npz``, made by the reference's own functions.
* ``forward`` / ``backward`` restate the network (4 -> 32 -> 32 -> 1 channels, 3x3 convolutions,
  zero padding, GELU in its tanh form) in float64 numpy, with the BF16 roundings the CUDA kernels
  apply (weights, activations, pre-activation gradients; round to nearest even). With ``exact=True`` the
  roundings are skipped, and the tests pin ``backward`` against finite differences of
  ``forward`` -- the reference has no closure, so that is what pins the gradients.

Parameter layout (flat float vector of 10721): w1 [32][9][4], b1 [32], w2 [32][9][32], b2 [32],
w3 [9][32], b3 [1]; tap = 3 (dx + 1) + (dy + 1), x the slow axis.
"""

from __future__ import annotations

import numpy as np

C = 32
OFF = {"w1": 0, "b1": 1152, "w2": 1184, "b2": 10400, "w3": 10432, "b3": 10720}
NPARAMS = 10721
TAPS = [(tap // 3 - 1, tap % 3 - 1) for tap in range(9)]


def bf16(a: np.ndarray) -> np.ndarray:
    """Rounds float32 values to BF16 (nearest, ties to even), returned as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def unpack(params: np.ndarray) -> dict[str, np.ndarray]:
    p = np.asarray(params, np.float64)
    return {
        "w1": p[OFF["w1"] : OFF["b1"]].reshape(C, 9, 4),
        "b1": p[OFF["b1"] : OFF["w2"]],
        "w2": p[OFF["w2"] : OFF["b2"]].reshape(C, 9, C),
        "b2": p[OFF["b2"] : OFF["w3"]],
        "w3": p[OFF["w3"] : OFF["b3"]].reshape(9, C),
        "b3": p[OFF["b3"] :],
    }


def pack(parts: dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([np.ravel(parts[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3")])


# ---- post-processing (python/boltzmann/utils/postproc.py) ----------------------------------


def _np_gradient_f32(f: np.ndarray, axis: int) -> np.ndarray:
    """np.gradient along one axis at unit spacing, in float32 (postproc.py:64)."""
    f = np.moveaxis(np.asarray(f, np.float32), axis, 0)
    out = np.empty_like(f)
    out[1:-1] = (f[2:] - f[:-2]) * np.float32(0.5)
    out[0] = f[1] - f[0]
    out[-1] = f[-1] - f[-2]
    return np.moveaxis(out, 0, axis)


def curl2d(vel: np.ndarray) -> np.ndarray:
    """postproc.calc_curl for [nx, ny, 2] (postproc.py:66-67)."""
    return _np_gradient_f32(vel[..., 0], 1) - _np_gradient_f32(vel[..., 1], 0)


def curl3d(vel: np.ndarray) -> np.ndarray:
    """postproc.calc_curl for [nx, ny, nz, 3] (postproc.py:69-77)."""
    d = [[_np_gradient_f32(vel[..., c], a) for c in range(3)] for a in range(3)]  # d[axis][comp]
    return np.stack((d[2][1] - d[1][2], d[0][2] - d[2][0], d[1][0] - d[0][1]), axis=-1)


def vmag(vel: np.ndarray) -> np.ndarray:
    """postproc.calc_vmag (postproc.py:25)."""
    v = np.asarray(vel, np.float32)
    s = v[..., 0] * v[..., 0]
    for c in range(1, v.shape[-1]):
        s = s + v[..., c] * v[..., c]
    return np.sqrt(s)


# ---- features, coarsening ------------------------------------------------------------------


def features(rho: np.ndarray, vel: np.ndarray, flags: np.ndarray, norm: np.ndarray) -> np.ndarray:
    """[B, nx, ny, 4] BF16-rounded inputs: ((rho-1, u_x, u_y, curl u) - mean) * inv_std, zero on
    walls; the curl takes the velocity on wall cells as 0."""
    rho = np.asarray(rho, np.float32).reshape((-1,) + flags.shape)
    vel = np.asarray(vel, np.float32).reshape((-1,) + flags.shape + (2,))
    wall = (flags & 1) != 0
    norm = np.asarray(norm, np.float32)
    out = np.zeros(rho.shape + (4,), np.float32)
    for b in range(rho.shape[0]):
        v = vel[b].copy()
        v[wall] = 0.0
        curl = curl2d(v)
        vals = [rho[b] - np.float32(1.0), vel[b][..., 0], vel[b][..., 1], curl]
        for c in range(4):
            out[b, ..., c] = bf16((vals[c] - norm[c]) * norm[4 + c])
        out[b][wall] = 0.0
    return out


def coarsen(rho, vel, c, f: int):
    """Block means of a fine state and sqrt of the subgrid kinetic energy per coarse cell."""
    nx, ny = rho.shape
    blk = lambda a: a.reshape(nx // f, f, ny // f, f, *a.shape[2:]).astype(np.float64)
    r = blk(rho).mean(axis=(1, 3))
    v = blk(vel).mean(axis=(1, 3))
    dv = blk(vel) - v[:, None, :, None, :]
    k = 0.5 * (dv**2).sum(-1).mean(axis=(1, 3))
    cc = None if c is None else blk(c).mean(axis=(1, 3))
    return r, v, cc, np.sqrt(k)


# ---- network -------------------------------------------------------------------------------


_C = np.sqrt(2.0 / np.pi)


def gelu(z):
    """GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(_C * (z + 0.044715 * z**3)))


def gelu_grad(z):
    t = np.tanh(_C * (z + 0.044715 * z**3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3 * 0.044715 * z**2)


def _pad(a):
    return np.pad(a, ((0, 0), (1, 1), (1, 1), (0, 0)))


def _conv(inp, w, bias=None):
    """out[b, p, co] = sum_{tap, ci} w[co, tap, ci] inp[b, p + tap, ci] (zero padding)."""
    B, nx, ny, _ = inp.shape
    p = _pad(np.asarray(inp, np.float64))
    out = np.zeros((B, nx, ny, w.shape[0]))
    for tap, (dx, dy) in enumerate(TAPS):
        out += p[:, 1 + dx : 1 + dx + nx, 1 + dy : 1 + dy + ny, :] @ w[:, tap, :].T
    if bias is not None:
        out += bias
    return out


def _conv_t(g, w):
    """Adjoint of _conv: out[b, q, ci] = sum_{tap, co} w[co, tap, ci] g[b, q - tap, co]."""
    B, nx, ny, _ = g.shape
    p = _pad(np.asarray(g, np.float64))
    out = np.zeros((B, nx, ny, w.shape[2]))
    for tap, (dx, dy) in enumerate(TAPS):
        out += p[:, 1 - dx : 1 - dx + nx, 1 - dy : 1 - dy + ny, :] @ w[:, tap, :]
    return out


def _wgrad(g, inp):
    """dW[co, tap, ci] = sum_p g[p, co] inp[p + tap, ci]."""
    B, nx, ny, _ = g.shape
    p = _pad(np.asarray(inp, np.float64))
    gg = np.asarray(g, np.float64).reshape(-1, g.shape[-1])
    out = np.zeros((g.shape[-1], 9, inp.shape[-1]))
    for tap, (dx, dy) in enumerate(TAPS):
        sh = p[:, 1 + dx : 1 + dx + nx, 1 + dy : 1 + dy + ny, :].reshape(-1, inp.shape[-1])
        out[:, tap, :] = gg.T @ sh
    return out


def _round(a, exact):
    return np.asarray(a, np.float64) if exact else bf16(np.asarray(a, np.float32)).astype(np.float64)


def forward(params, x, exact: bool = False) -> dict[str, np.ndarray]:
    """x [B, nx, ny, 4] -> activations (z1, a1, z2, a2) and output y [B, nx, ny]."""
    P = unpack(params)
    w = {k: _round(P[k], exact) for k in ("w1", "w2", "w3")}
    x = np.asarray(x, np.float64)
    z1 = _conv(x, w["w1"], P["b1"])
    a1 = _round(gelu(z1), exact)
    z2 = _conv(a1, w["w2"], P["b2"])
    a2 = _round(gelu(z2), exact)
    y = _conv(a2, w["w3"][None], P["b3"])[..., 0]
    return {"z1": z1, "a1": a1, "z2": z2, "a2": a2, "y": y}


def loss(y, target, flags):
    """Masked MSE over cells that are neither walls nor fixed, and its gradient."""
    m = ((np.asarray(flags) & 7) == 0)[None].astype(np.float64)
    d = (np.asarray(y, np.float64) - np.asarray(target, np.float64)) * m
    count = m.sum() * np.asarray(y).shape[0]
    return float((d**2).sum() / count), 2.0 * d / count


def backward(params, x, acts, dy, exact: bool = False) -> np.ndarray:
    """Gradient of the loss (given dL/dy) with respect to the flat parameter vector."""
    P = unpack(params)
    w = {k: _round(P[k], exact) for k in ("w1", "w2", "w3")}
    dy4 = np.asarray(dy, np.float64)[..., None]
    g = {}
    g["w3"] = _wgrad(dy4, acts["a2"])[0]
    g["b3"] = np.array([dy4.sum()])
    dz2 = _round(_conv_t(dy4, w["w3"][None]) * gelu_grad(acts["z2"]), exact)
    g["b2"] = dz2.reshape(-1, C).sum(0)
    g["w2"] = _wgrad(dz2, acts["a1"])
    dz1 = _round(_conv_t(dz2, w["w2"]) * gelu_grad(acts["z1"]), exact)
    g["b1"] = dz1.reshape(-1, C).sum(0)
    g["w1"] = _wgrad(dz1, x)
    return pack(g)


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases, as torch's Conv2d default."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape, fan in (("w1", (C, 9, 4), 36), ("w2", (C, 9, C), 288), ("w3", (9, C), 288)):
        bound = 1.0 / np.sqrt(fan)
        parts[name] = rng.uniform(-bound, bound, shape)
        bname = "b" + name[1]
        parts[bname] = rng.uniform(-bound, bound, C if name != "w3" else 1)
    return pack(parts).astype(np.float32)
