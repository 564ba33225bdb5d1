"""Seeded synthetic set-ups of the benchmark configurations, as plain numpy arrays.

Each builder returns a :class:`Setup`; :func:`apply` loads it into any object with the
reference's ``Simulation`` API (the CUDA one here, or a CPU checker), so the GPU run and its
comparison run start from identical host arrays.

* ``kelvin_helmholtz``: D2Q9 BGK, fully periodic shear layer (256x256, tau 0.55).
* ``cylinder_channel``: D2Q9 TRT channel with bounce-back walls, a bounce-back cylinder, fixed
  inflow/outflow columns and a Boussinesq-coupled D2Q5 tracer (4096x2048, Re 10,000 on the
  cylinder diameter).
* ``taylor_green_3d``: D3Q27 periodic Taylor-Green vortex (256^3, Re 1600).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

WALL, FIXED_FLUID, FIXED_SCALAR = 1, 6, 8


@dataclass
class Setup:
    name: str
    counts: list[int]
    collision: str  # "bgk" or "trt"
    tau: float  # BGK tau, or TRT tau+
    flags: np.ndarray
    rho: np.ndarray
    vel: np.ndarray
    tracers: list[tuple[str, float, np.ndarray]] = field(default_factory=list)  # name, tau, C
    gravity: list[float] | None = None
    couplings: list[tuple[str, float, float, list[float]]] = field(default_factory=list)
    params: dict = field(default_factory=dict)
    tau_neg: float | None = None  # TRT tau-; None = from the magic parameter 1/4

    @property
    def cells(self) -> int:
        return int(np.prod(self.counts))


def kelvin_helmholtz(nx: int = 256, ny: int = 256, tau: float = 0.55, seed: int = 0) -> Setup:
    """u_x = 0.05 tanh((y - ny/4)/4) below ny/2 and 0.05 tanh((3ny/4 - y)/4) above,
    u_y = 1e-3 sin(2 pi x / nx) + U(-1e-4, 1e-4); rho = 1."""
    rng = np.random.default_rng(seed)
    y = np.arange(ny, dtype=np.float64)[None, :]
    x = np.arange(nx, dtype=np.float64)[:, None]
    ux = np.where(y < ny / 2, 0.05 * np.tanh((y - ny / 4) / 4), 0.05 * np.tanh((3 * ny / 4 - y) / 4))
    ux = np.broadcast_to(ux, (nx, ny))
    uy = 1e-3 * np.sin(2 * np.pi * x / nx) + rng.uniform(-1e-4, 1e-4, (nx, ny))
    vel = np.stack([ux, uy], axis=-1).astype(np.float32)
    return Setup(
        "kelvin_helmholtz",
        [nx, ny],
        "bgk",
        tau,
        np.zeros((nx, ny), np.int32),
        np.ones((nx, ny), np.float32),
        vel,
        params={"u0": 0.05},
    )


def cylinder_channel(
    nx: int = 4096,
    ny: int = 2048,
    radius: float = 64.0,
    u_in: float = 0.05,
    re: float = 10_000.0,
    diffusivity: float = 1e-3,
    buoyancy: float = 1e-5,
    seed: int = 0,
) -> Setup:
    """Channel flow past a cylinder with a buoyant tracer.

    TRT with tau- = 0.52, as the reference's vortex-street example sets it
    (python/examples/vortex_street/vortex_street.py: ``trt(tau_ns, 0.52)``): with the magic
    parameter 1/4 (tau- ~ 130 at tau+ = 0.50192) this set-up diverges within ~200 steps on the
    reference's own kernels.

    Bounce-back rows at y = 0 and y = ny-1, a bounce-back disc of ``radius`` at (nx/4, ny/2),
    fixed-velocity (and fixed-tracer) columns at x = 0 and x = nx-1 holding u = (u_in, 0).
    nu = u_in * 2 radius / re, tau+ = 3 nu + 1/2. The D2Q5 tracer has
    tau = 3 D + 1/2 and starts as a seeded random 0/1 band across the middle third of the
    channel height; it couples back with acc = g * alpha * C, alpha g = buoyancy * (0, -1).
    """
    rng = np.random.default_rng(seed)
    nu = u_in * 2 * radius / re
    tau = 3 * nu + 0.5
    flags = np.zeros((nx, ny), np.int32)
    flags[:, 0] = WALL
    flags[:, -1] = WALL
    x = np.arange(nx)[:, None]
    y = np.arange(ny)[None, :]
    cx, cy = nx // 4, ny // 2
    flags[(x - cx) ** 2 + (y - cy) ** 2 <= radius**2] = WALL
    flags[0, 1:-1] = FIXED_FLUID | FIXED_SCALAR
    flags[-1, 1:-1] = FIXED_FLUID | FIXED_SCALAR
    vel = np.zeros((nx, ny, 2), np.float32)
    vel[..., 0] = u_in
    vel[flags == WALL] = 0.0
    rho = np.ones((nx, ny), np.float32)
    band = np.zeros((nx, ny), np.float32)
    lo, hi = ny // 3, 2 * ny // 3
    band[:, lo:hi] = (rng.uniform(size=(nx, hi - lo)) < 0.5).astype(np.float32)
    band[0, :] = 0.0
    band[-1, :] = 0.0
    tau_g = 3 * diffusivity + 0.5
    return Setup(
        "cylinder_channel",
        [nx, ny],
        "trt",
        tau,
        flags,
        rho,
        vel,
        tracers=[("tracer", tau_g, band)],
        couplings=[("tracer", 1.0, 0.0, [0.0, -buoyancy])],
        params={"radius": radius, "u_in": u_in, "re": re, "nu": nu, "diffusivity": diffusivity},
        tau_neg=0.52,
    )


def taylor_green_3d(n: int = 256, u0: float = 0.05, re: float = 1600.0,
                    nz: int | None = None) -> Setup:
    """u = u0 (sin kx cos ky cos kz, -cos kx sin ky cos kz, 0), k = 2 pi / n, with the pressure
    field in rho = 1 + 3 p, p = u0^2/16 (cos 2kx + cos 2ky)(cos 2kz + 2);
    nu = u0 (n / 2 pi) / re, tau = 3 nu + 1/2. ``nz`` (profiling cases only) stretches the box
    along z to n x n x nz, with k_z = 2 pi / nz."""
    nz = nz or n
    k, kz = 2 * math.pi / n, 2 * math.pi / nz
    c = np.arange(n, dtype=np.float64)
    X, Y, Z = np.meshgrid(c, c, np.arange(nz, dtype=np.float64), indexing="ij")
    vel = np.empty((n, n, nz, 3), np.float32)
    vel[..., 0] = u0 * np.sin(k * X) * np.cos(k * Y) * np.cos(kz * Z)
    vel[..., 1] = -u0 * np.cos(k * X) * np.sin(k * Y) * np.cos(kz * Z)
    vel[..., 2] = 0.0
    p = u0**2 / 16 * (np.cos(2 * k * X) + np.cos(2 * k * Y)) * (np.cos(2 * kz * Z) + 2)
    rho = (1.0 + 3.0 * p).astype(np.float32)
    nu = u0 * (n / (2 * math.pi)) / re
    return Setup(
        "taylor_green_3d",
        [n, n, nz],
        "bgk",
        3 * nu + 0.5,
        np.zeros((n, n, nz), np.int32),
        rho,
        vel,
        params={"u0": u0, "re": re, "nu": nu},
    )


def apply(sim, setup: Setup, omega_for, tracer_handle=None) -> None:
    """Loads ``setup`` into a Simulation-like object.

    ``omega_for(kind, tau)`` builds the collision parameters of that object's API.
    ``tracer_handle(sim, name, omega)`` adds a tracer and returns (handle, val array);
    by default the reference API ``sim.add_tracer(name, omega).val`` is used.
    """
    flags = sim.cells.flags if hasattr(sim, "cells") else sim.flags
    rho = sim.fluid.rho if hasattr(sim, "fluid") else sim.rho
    vel = sim.fluid.vel if hasattr(sim, "fluid") else sim.vel
    flags[...] = setup.flags
    rho[...] = setup.rho
    vel[...] = setup.vel
    handles = {}
    for name, tau_t, val in setup.tracers:
        if tracer_handle is None:
            h = sim.add_tracer(name, omega_for("bgk", tau_t))
            h.val[...] = val
        else:
            h, arr = tracer_handle(sim, name, omega_for("bgk", tau_t))
            arr[...] = val
        handles[name] = h
    if setup.gravity is not None:
        sim.set_gravity(np.asarray(setup.gravity, np.float32))
    for name, alpha, c0, g in setup.couplings:
        sim.add_boussinesq_coupling(handles[name], alpha, c0, np.asarray(g, np.float32))


@dataclass
class EnsembleSetup:
    """Independent 2D domains for an ensemble run: per-domain counts and rates, plus the
    concatenated host arrays (each domain in the reference's row-major order)."""

    name: str
    counts: list[tuple[int, int]]
    tau: list[float]
    flags: np.ndarray
    rho: np.ndarray
    vel: np.ndarray
    params: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return int(sum(a * b for a, b in self.counts))

    def domain_slices(self) -> list[slice]:
        out, start = [], 0
        for a, b in self.counts:
            out.append(slice(start, start + a * b))
            start += a * b
        return out

    def subset(self, indices) -> "EnsembleSetup":
        """The listed domains only (in the given order), e.g. one rank's shard."""
        sl = self.domain_slices()
        pick = lambda a: (np.concatenate([a[sl[i]] for i in indices]) if len(indices)
                          else a[:0].copy())
        params = {k: ([v[i] for i in indices] if isinstance(v, list) and len(v) == len(self.counts)
                      else v) for k, v in self.params.items()}
        return EnsembleSetup(self.name, [self.counts[i] for i in indices],
                             [self.tau[i] for i in indices], pick(self.flags), pick(self.rho),
                             pick(self.vel), params)


def lid_driven_cavities(
    count: int = 512,
    lo: int = 64,
    hi: int = 512,
    u_lid: float = 0.05,
    re_range: tuple[float, float] = (100.0, 5000.0),
    seed: int = 0,
) -> EnsembleSetup:
    """``count`` square lid-driven cavities: side L ~ U{lo..hi}, Re ~ log-uniform on re_range,
    tau = 1/2 + 3 u_lid L / Re (BGK). Walls on the left, right and bottom edges; the top row
    (y = L-1, inner cells) is FIXED_FLUID with u = (u_lid, 0); rho = 1, fluid at rest."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=count)
    res = np.exp(rng.uniform(np.log(re_range[0]), np.log(re_range[1]), size=count))
    counts, taus, flags, rho, vel = [], [], [], [], []
    for L, re in zip(sides.tolist(), res.tolist()):
        fl = np.zeros((L, L), np.int32)
        fl[0, :] = WALL
        fl[-1, :] = WALL
        fl[:, 0] = WALL
        fl[1:-1, -1] = FIXED_FLUID
        v = np.zeros((L, L, 2), np.float32)
        v[1:-1, -1, 0] = u_lid
        counts.append((L, L))
        taus.append(0.5 + 3.0 * u_lid * L / re)
        flags.append(fl.reshape(-1))
        rho.append(np.ones(L * L, np.float32))
        vel.append(v.reshape(-1, 2))
    return EnsembleSetup(
        "lid_driven_cavities",
        counts,
        taus,
        np.concatenate(flags),
        np.concatenate(rho),
        np.concatenate(vel),
        params={"u_lid": u_lid, "re": res.tolist(), "sides": sides.tolist()},
    )
