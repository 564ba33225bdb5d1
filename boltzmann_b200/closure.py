"""Learned subgrid closure for coarse 2D runs (D2Q9), trained on box-filtered fine runs.

No counterpart in the reference. A small CNN (3x3 convolutions, 4 -> 32 -> 32 -> 1 channels,
GELU in its tanh form; BF16 weights and activations, FP32 accumulation; ``csrc/closure.cu``) reads the coarse
state -- (rho - 1, u_x, u_y, curl u) per cell -- and predicts the subgrid velocity scale
sqrt(k_sgs), where k_sgs is the kinetic energy below the coarse grid that a 4x4 box filter of a
fine run removes. Every ``every`` steps the coarse run turns the prediction into a per-cell
relaxation time tau = tau0 + min(max_dtau, gain * max(y, 0)) -- an eddy viscosity
nu_t = C_k * sqrt(k_sgs) * dx with gain = 3 C_k s (s the target scale) -- handed to the stencil
through ``lbm_set_omega_field``.

Training data come from the plain method itself: seeded fine runs of the cylinder channel, box
filtered onto the coarse lattice on the device. The network is trained by the project's own
forward/backward kernels and an Adam kernel. ``evaluate`` judges a trained closure a posteriori
on a held-out seed: coarse runs started from the filtered fine state, with and without the
closure, against the filtered fine run at several horizons. A closure whose mean relative
velocity error exceeds ``bound`` (or that is worse than plain coarse at the last horizon it
survives) is rejected, and ``run_closed_or_fine`` then falls back to the plain fine run.

PyTorch only holds device memory here (buffers, batches); every arithmetic step on the path is a
kernel of this project.
"""

from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import dataclass, field

import numpy as np

from boltzmann_b200 import LIBRARY

_lib = C.CDLL(str(LIBRARY))
_lib.lbm_last_error.restype = C.c_char_p
_lib.lbm_closure_workspace_bytes.restype = C.c_int64
_lib.lbm_closure_workspace_bytes.argtypes = [C.c_int64, C.c_int64, C.c_int64]

_P, _I64, _F, _I = C.c_void_p, C.c_int64, C.c_float, C.c_int
_SIGS = {
    "lbm_postproc_curl2d": [_P, _I64, _I64, _P, _P],
    "lbm_postproc_curl3d": [_P, _I64, _I64, _I64, _P, _P],
    "lbm_postproc_vmag": [_P, _I64, _I, _P, _P],
    "lbm_closure_features": [_P, _P, _P, _I64, _I64, _I64, _P, _P, _P],
    "lbm_closure_forward": [_P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P],
    "lbm_closure_loss": [_P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _P],
    "lbm_closure_backward": [_P, _P, _P, _P, _P, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P],
    "lbm_closure_adam": [_P, _P, _P, _P, _P, _F, _F, _F, _F, _I64, _P],
    "lbm_closure_sync_bf16": [_P, _P, _P],
    "lbm_closure_omega": [_P, _P, _I64, _I64, _F, _F, _F, _P, _P],
    "lbm_closure_coarsen": [_P, _P, _P, _I64, _I64, _I, _P, _P, _P, _P, _P],
    "lbm_closure_relaxation": [_P, _P, _P, _P, _P, _I64, _I64, _P, _F, _F, _F, _P, _P],
    "lbm_closure_status": [],
    "lbm_closure_set_spin_limit": [_I64],
    "lbm_closure_set_layer2_kernel": [_I],
}
for _name, _args in _SIGS.items():
    getattr(_lib, _name).argtypes = _args
    getattr(_lib, _name).restype = C.c_int

NPARAMS = 10721
LAYER2_KERNELS = {"tcgen05": 0, "warp_mma": 1}


def set_layer2_kernel(kind: str) -> None:
    """Selects the kernel of layer 2 in training (forward and the transposed conv): "tcgen05"
    (default) or "warp_mma"; process-wide."""
    _check(_lib.lbm_closure_set_layer2_kernel(LAYER2_KERNELS[kind]))
CHANNELS = 32


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(_lib.lbm_last_error().decode())


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the closure runs on the CUDA device; no GPU is available")
    return torch


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(torch) -> int:
    return torch.cuda.current_stream().cuda_stream


# ---- on-device post-processing (python/boltzmann/utils/postproc.py) --------------------------


def curl(vel, stream: int | None = None):
    """postproc.calc_curl on a device tensor [nx, ny, 2] (-> [nx, ny]) or [nx, ny, nz, 3]."""
    torch = _torch()
    vel = vel.contiguous().float()
    s = _stream(torch) if stream is None else stream
    if vel.dim() == 3 and vel.shape[-1] == 2:
        out = torch.empty(vel.shape[:2], device=vel.device)
        _check(_lib.lbm_postproc_curl2d(_ptr(vel), vel.shape[0], vel.shape[1], _ptr(out), s))
    elif vel.dim() == 4 and vel.shape[-1] == 3:
        out = torch.empty_like(vel)
        _check(_lib.lbm_postproc_curl3d(_ptr(vel), *vel.shape[:3], _ptr(out), s))
    else:
        raise ValueError(f"Invalid array dimensionality! {tuple(vel.shape)}")
    return out


def vmag(vel, stream: int | None = None):
    """postproc.calc_vmag on a device tensor [..., dim]."""
    torch = _torch()
    vel = vel.contiguous().float()
    out = torch.empty(vel.shape[:-1], device=vel.device)
    s = _stream(torch) if stream is None else stream
    _check(_lib.lbm_postproc_vmag(_ptr(vel), out.numel(), vel.shape[-1], _ptr(out), s))
    return out


# ---- the network -----------------------------------------------------------------------------


class Net:
    """Parameters (FP32 master + BF16 mirror on the device), feature normalisation, and the
    output-to-relaxation mapping (``gain``, ``max_dtau``)."""

    def __init__(self, params: np.ndarray, norm: np.ndarray, target_scale: float = 1.0,
                 gain: float = 0.0, max_dtau: float = 0.05, meta: dict | None = None):
        torch = _torch()
        params = np.asarray(params, np.float32).reshape(-1)
        if params.size != NPARAMS:
            raise ValueError(f"expected {NPARAMS} parameters, got {params.size}")
        self.params = torch.tensor(params, device="cuda")
        self.bf16 = torch.empty(NPARAMS + 7, dtype=torch.int16, device="cuda")  # 16-B multiple
        self.norm = np.asarray(norm, np.float32).reshape(8)
        self.target_scale = float(target_scale)
        self.gain = float(gain)
        self.max_dtau = float(max_dtau)
        self.meta = dict(meta or {})
        self.sync()

    def sync(self, stream: int | None = None) -> None:
        torch = _torch()
        s = _stream(torch) if stream is None else stream
        _check(_lib.lbm_closure_sync_bf16(_ptr(self.params), _ptr(self.bf16), s))

    def save(self, path) -> None:
        np.savez(path, params=self.params.cpu().numpy(), norm=self.norm,
                 target_scale=self.target_scale, gain=self.gain, max_dtau=self.max_dtau,
                 meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path) -> "Net":
        d = np.load(path)
        return cls(d["params"], d["norm"], float(d["target_scale"]), float(d["gain"]),
                   float(d["max_dtau"]), json.loads(str(d["meta"])))


class Buffers:
    """Device buffers for one (nx, ny, batch) shape; ``train`` adds what a backward pass needs."""

    def __init__(self, nx: int, ny: int, batch: int, train: bool):
        torch = _torch()
        n = nx * ny * batch
        self.shape = (nx, ny, batch)
        self.x = torch.empty(n * 4, dtype=torch.int16, device="cuda")
        self.a1 = torch.empty(n * CHANNELS, dtype=torch.int16, device="cuda")
        self.a2 = torch.empty(n * CHANNELS, dtype=torch.int16, device="cuda")
        self.y = torch.empty(n, device="cuda")
        self.z1 = self.z2 = self.dy = self.grad = self.ws = self.loss = None
        if train:
            self.z1 = torch.empty(n * CHANNELS, device="cuda")
            self.z2 = torch.empty(n * CHANNELS, device="cuda")
            self.dy = torch.empty(n, device="cuda")
            self.grad = torch.empty(NPARAMS, device="cuda")
            wsb = _lib.lbm_closure_workspace_bytes(nx, ny, batch)
            if wsb < 0:
                raise ValueError("bad closure shape")
            self.ws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
            self.loss = torch.zeros(1, dtype=torch.float64, device="cuda")


def features(rho, vel, flags, norm, bufs: Buffers, stream: int) -> None:
    """Coarse state(s) (device pointers or tensors) -> bufs.x."""
    nx, ny, batch = bufs.shape
    rp = rho if isinstance(rho, int) else _ptr(rho)
    vp = vel if isinstance(vel, int) else _ptr(vel)
    nm = np.ascontiguousarray(norm, np.float32)
    _check(_lib.lbm_closure_features(rp, vp, _ptr(flags), nx, ny, batch,
                                     nm.ctypes.data_as(C.c_void_p), _ptr(bufs.x), stream))


def forward(net: Net, bufs: Buffers, stream: int, x=None) -> None:
    nx, ny, batch = bufs.shape
    xs = bufs.x if x is None else x
    _check(_lib.lbm_closure_forward(_ptr(net.params), _ptr(net.bf16), _ptr(xs), nx, ny, batch,
                                    _ptr(bufs.z1), _ptr(bufs.a1), _ptr(bufs.z2), _ptr(bufs.a2),
                                    _ptr(bufs.y), stream))


def loss_and_grad(net: Net, bufs: Buffers, target, flags, stream: int, x=None) -> None:
    """Loss of bufs.y against target, then the gradient into bufs.grad."""
    nx, ny, batch = bufs.shape
    xs = bufs.x if x is None else x
    _check(_lib.lbm_closure_loss(_ptr(bufs.y), _ptr(target), _ptr(flags), nx, ny, batch,
                                 _ptr(bufs.dy), _ptr(bufs.loss), _ptr(bufs.ws), stream))
    _check(_lib.lbm_closure_backward(_ptr(net.params), _ptr(net.bf16), _ptr(xs), _ptr(bufs.z1),
                                     _ptr(bufs.a1), _ptr(bufs.z2), _ptr(bufs.a2), _ptr(bufs.dy),
                                     nx, ny, batch, _ptr(bufs.grad), _ptr(bufs.ws), stream))


def relaxation(net: Net, rho, vel, flags, nx: int, ny: int, tau0: float, omega, stream: int) -> None:
    """The relaxation field omega [nx, ny] of a coarse state (device pointers or tensors) in one
    kernel: features, network and the tau mapping fused (``lbm_closure_relaxation``)."""
    rp = rho if isinstance(rho, int) else _ptr(rho)
    vp = vel if isinstance(vel, int) else _ptr(vel)
    nm = np.ascontiguousarray(net.norm, np.float32)
    _check(_lib.lbm_closure_relaxation(_ptr(net.params), _ptr(net.bf16), rp, vp, _ptr(flags), nx,
                                       ny, nm.ctypes.data_as(C.c_void_p), tau0, net.gain,
                                       net.max_dtau, _ptr(omega), stream))


def status() -> None:
    """Raises if a fused relaxation kernel gave up waiting on its tensor cores (synchronous)."""
    _check(_lib.lbm_closure_status())


def relaxation_layered(net: Net, rho, vel, flags, bufs: Buffers, tau0: float, omega,
                       stream: int) -> None:
    """The same field through the layer-by-layer kernels (features, forward, omega)."""
    nx, ny, _ = bufs.shape
    features(rho, vel, flags, net.norm, bufs, stream)
    forward(net, bufs, stream)
    _check(_lib.lbm_closure_omega(_ptr(bufs.y), _ptr(flags), nx, ny, tau0, net.gain, net.max_dtau,
                                  _ptr(omega), stream))


class Adam:
    def __init__(self, net: Net, lr: float = 2e-3, betas=(0.9, 0.999), eps: float = 1e-8):
        torch = _torch()
        self.net, self.lr, self.betas, self.eps = net, lr, betas, eps
        self.m = torch.zeros(NPARAMS, device="cuda")
        self.v = torch.zeros(NPARAMS, device="cuda")
        self.step_count = 0

    def step(self, grad, stream: int, lr: float | None = None) -> None:
        self.step_count += 1
        _check(_lib.lbm_closure_adam(_ptr(self.net.params), _ptr(self.net.bf16), _ptr(grad),
                                     _ptr(self.m), _ptr(self.v), self.lr if lr is None else lr,
                                     self.betas[0], self.betas[1], self.eps, self.step_count,
                                     stream))


# ---- data from fine runs ---------------------------------------------------------------------


@dataclass
class Config:
    """Sizes of the closure experiment (the coarse 1024x512 analogue of the 4096x2048 cylinder
    channel, radius 64 -> 16, Re 10,000), in fine steps unless stated."""

    fine: tuple[int, int] = (4096, 2048)
    factor: int = 4
    radius: float = 64.0
    re: float = 10_000.0
    u_in: float = 0.05
    diffusivity: float = 1e-3
    buoyancy: float = 1e-5
    train_seeds: tuple[int, ...] = (1, 2)
    calib_seed: int = 2
    test_seed: int = 3
    # The fine channel goes non-finite for most seeds after 6,000-16,000 steps (in FP64 too, so
    # the set-up, not the precision): data and judging stay inside the first 5,000 fine steps.
    spinup: int = 1_000
    snapshots: int = 40  # per training seed
    snapshot_every: int = 100
    batch: int = 8
    iters: int = 400
    lr: float = 2e-3
    every: int = 10  # coarse steps between closure applications
    horizons: tuple[int, ...] = (100, 200, 300, 400, 500, 600, 700, 800, 900, 1000)  # coarse steps
    gains_ck: tuple[float, ...] = (0.00625, 0.0125, 0.025, 0.05, 0.1)  # C_k candidates
    max_dtau: float = 0.05
    bound: float = 0.05  # mean relative velocity L2 error a closure must stay below
    net_seed: int = 0

    @property
    def coarse(self) -> tuple[int, int]:
        return (self.fine[0] // self.factor, self.fine[1] // self.factor)


def fine_setup(cfg: Config, seed: int):
    from boltzmann_b200 import workloads

    return workloads.cylinder_channel(nx=cfg.fine[0], ny=cfg.fine[1], radius=cfg.radius,
                                      u_in=cfg.u_in, re=cfg.re, diffusivity=cfg.diffusivity,
                                      buoyancy=cfg.buoyancy, seed=seed)


def coarse_setup(cfg: Config):
    """The same channel on the coarse lattice: lengths / f, so nu / f, D / f, g * f (velocity
    kept, time step f times longer)."""
    from boltzmann_b200 import workloads

    f = cfg.factor
    return workloads.cylinder_channel(nx=cfg.coarse[0], ny=cfg.coarse[1], radius=cfg.radius / f,
                                      u_in=cfg.u_in, re=cfg.re, diffusivity=cfg.diffusivity / f,
                                      buoyancy=cfg.buoyancy * f, seed=0)


def build_sim(setup):
    from boltzmann_b200 import workloads
    from boltzmann_b200.core import Simulation, bgk, trt

    def om(kind, tau, tau_neg=None):
        return bgk(tau) if kind == "bgk" else trt(tau, tau_neg)

    sim = Simulation("gpu", setup.counts, om(setup.collision, setup.tau, setup.tau_neg))
    workloads.apply(sim, setup, lambda k, t: om(k, t))
    return sim


class FineRun:
    """A fine run on the device, read out as box-filtered coarse states."""

    def __init__(self, cfg: Config, seed: int):
        torch = _torch()
        self.cfg = cfg
        self.setup = fine_setup(cfg, seed)
        self.sim = build_sim(self.setup)
        self.stream = self.sim._stream()
        self.steps = 0
        nxc, nyc = cfg.coarse
        self.c_dev = None
        self._tmp = torch.empty(nxc * nyc * 4, device="cuda")

    def advance(self, steps: int) -> float:
        """Fine steps on the device; returns their device time in seconds."""
        torch = _torch()
        ext = torch.cuda.ExternalStream(self.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        self.sim._iterate_device(steps)
        e1.record(ext)
        e1.synchronize()
        self.steps += steps
        return e0.elapsed_time(e1) / 1e3

    def coarse_state(self, rho_c, vel_c, sgs=None, c_c=None, tracer_dev=None) -> None:
        """Box-filter the current fine state into the given device tensors (on the run's
        stream; synchronised before returning)."""
        nx, ny = self.cfg.fine
        rp, vp = self.sim._fluid_device()
        _check(_lib.lbm_closure_coarsen(rp, vp, tracer_dev, nx, ny, self.cfg.factor, _ptr(rho_c),
                                        _ptr(vel_c), _ptr(c_c), _ptr(sgs), self.stream))
        self.sim._synchronize()


def clean_coarse_state(rho, vel, flags_t, u_in: float) -> None:
    """Filtered states on the coarse lattice's own cell flags: walls at rest (rho 1, u 0), fixed
    cells at the inflow value, as a coarse run holds them."""
    wall = (flags_t & 1) != 0
    fixed = (flags_t & 6) != 0
    rho[..., wall] = 1.0
    vel[..., wall, :] = 0.0
    rho[..., fixed] = 1.0
    vel[..., fixed, 0] = u_in
    vel[..., fixed, 1] = 0.0


@dataclass
class Dataset:
    rho: object  # [S, nx, ny]
    vel: object  # [S, nx, ny, 2]
    sgs: object  # [S, nx, ny]
    fine_seconds: float = 0.0


def generate(cfg: Config, seeds=None) -> Dataset:
    """Filtered snapshots of seeded fine runs (device tensors)."""
    torch = _torch()
    seeds = cfg.train_seeds if seeds is None else seeds
    nxc, nyc = cfg.coarse
    S = cfg.snapshots * len(seeds)
    rho = torch.empty((S, nxc, nyc), device="cuda")
    vel = torch.empty((S, nxc, nyc, 2), device="cuda")
    sgs = torch.empty((S, nxc, nyc), device="cuda")
    flags_t = torch.tensor(coarse_setup(cfg).flags, device="cuda")
    seconds = 0.0
    k = 0
    for seed in seeds:
        run = FineRun(cfg, seed)
        seconds += run.advance(cfg.spinup)
        for _ in range(cfg.snapshots):
            seconds += run.advance(cfg.snapshot_every)
            run.coarse_state(rho[k], vel[k], sgs[k])
            k += 1
        del run
    clean_coarse_state(rho, vel, flags_t, cfg.u_in)
    sgs[:, (flags_t & 7) != 0] = 0.0
    return Dataset(rho, vel, sgs, seconds)


def normalisation(data: Dataset, flags: np.ndarray) -> tuple[np.ndarray, float]:
    """Per-channel mean and inverse standard deviation of the inputs over fluid cells, and the
    target scale (RMS of sqrt(k_sgs) over fluid cells)."""
    torch = _torch()
    S, nx, ny = data.rho.shape
    flags_t = torch.tensor(np.asarray(flags, np.int32), device="cuda")
    bufs = Buffers(nx, ny, S, train=False)
    unit = np.array([0, 0, 0, 0, 1, 1, 1, 1], np.float32)
    features(data.rho, data.vel, flags_t, unit, bufs, _stream(torch))
    x = bufs.x.view(torch.bfloat16).float().view(S, nx, ny, 4)
    fluid = (flags_t & 7) == 0
    v = x[:, fluid, :]  # [S, cells, 4]
    mean = v.mean(dim=(0, 1))
    std = v.std(dim=(0, 1)).clamp_min(1e-12)
    scale = float(data.sgs[:, fluid].pow(2).mean().sqrt())
    norm = np.concatenate([mean.cpu().numpy(), (1.0 / std).cpu().numpy()]).astype(np.float32)
    return norm, max(scale, 1e-12)


# ---- training --------------------------------------------------------------------------------


@dataclass
class TrainReport:
    losses: list = field(default_factory=list)  # (iteration, loss)
    seconds: float = 0.0  # device time of the training iterations
    iters: int = 0


def train(cfg: Config, data: Dataset, net: Net | None = None, log_every: int = 20) -> tuple[Net, TrainReport]:
    """Adam on the masked MSE between the network output and sqrt(k_sgs) / scale."""
    torch = _torch()
    S, nx, ny = data.rho.shape
    flags = coarse_setup(cfg).flags
    flags_t = torch.tensor(flags, device="cuda")
    stream = _stream(torch)
    norm, scale = normalisation(data, flags)
    if net is None:
        net = Net(init_params(cfg.net_seed), norm, scale, max_dtau=cfg.max_dtau)
    else:
        net.norm, net.target_scale = norm, scale
    all_x = Buffers(nx, ny, S, train=False)
    features(data.rho, data.vel, flags_t, net.norm, all_x, stream)
    xs = all_x.x.view(S, nx * ny * 4)
    target = (data.sgs / scale).contiguous().view(S, nx * ny)
    bufs = Buffers(nx, ny, cfg.batch, train=True)
    opt = Adam(net, lr=cfg.lr)
    gen = torch.Generator(device="cpu").manual_seed(cfg.net_seed)
    report = TrainReport()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for it in range(cfg.iters):
        idx = torch.randperm(S, generator=gen)[: cfg.batch].cuda()
        xb = xs.index_select(0, idx).reshape(-1)
        tb = target.index_select(0, idx).reshape(-1)
        forward(net, bufs, stream, x=xb)
        loss_and_grad(net, bufs, tb, flags_t, stream, x=xb)
        lr = cfg.lr * 0.5 * (1 + math.cos(math.pi * it / cfg.iters))  # cosine decay
        opt.step(bufs.grad, stream, lr=lr)
        if it % log_every == 0 or it == cfg.iters - 1:
            report.losses.append((it, float(bufs.loss.item())))
    e1.record()
    e1.synchronize()
    report.seconds = e0.elapsed_time(e1) / 1e3
    report.iters = cfg.iters
    return net, report


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases (fan_in = 9 x channels in)."""
    rng = np.random.default_rng(seed)
    out = []
    for shape, fan, nb in (((CHANNELS, 9, 4), 36, CHANNELS), ((CHANNELS, 9, CHANNELS), 288, CHANNELS),
                           ((9, CHANNELS), 288, 1)):
        bound = 1.0 / math.sqrt(fan)
        out.append(rng.uniform(-bound, bound, shape).ravel())
        out.append(rng.uniform(-bound, bound, nb))
    return np.concatenate(out).astype(np.float32)


# ---- closed coarse runs ----------------------------------------------------------------------


class ClosedRun:
    """A coarse Simulation whose relaxation field the closure refreshes every ``every`` steps
    (all on the simulation's stream). ``net=None`` runs the plain method."""

    def __init__(self, sim, flags: np.ndarray, net: Net | None, every: int, tau0: float):
        torch = _torch()
        self.sim, self.net, self.every, self.tau0 = sim, net, every, tau0
        self.nx, self.ny = flags.shape
        self.stream = sim._stream()
        self.flags = torch.tensor(np.asarray(flags, np.int32), device="cuda")
        self.steps = 0
        if net is not None:
            self.omega = torch.full((self.nx * self.ny,), 1.0 / tau0, device="cuda")
            torch.cuda.synchronize()
            sim._set_omega_field(self.omega.data_ptr())

    def apply(self) -> None:
        """Refresh the relaxation field from the current state (one fused kernel)."""
        rp, vp = self.sim._fluid_device()
        relaxation(self.net, rp, vp, self.flags, self.nx, self.ny, self.tau0, self.omega,
                   self.stream)

    def advance(self, steps: int) -> None:
        if steps % self.every != 0:
            raise ValueError("steps must be a multiple of the closure interval")
        if self.net is None:
            self.sim._iterate_device(steps)
        else:
            n = self.net
            self.sim._iterate_closure(steps, self.every, _ptr(n.params), _ptr(n.bf16),
                                      _ptr(self.flags), n.norm, self.tau0, n.gain, n.max_dtau,
                                      _ptr(self.omega))
        self.steps += steps

    def close(self) -> None:
        if self.net is not None:
            self.sim._set_omega_field(0)


def start_coarse(cfg: Config, rho, vel, c=None):
    """A coarse Simulation initialised from a filtered fine state (host arrays)."""
    setup = coarse_setup(cfg)
    sim = build_sim(setup)
    sim.fluid.rho[...] = rho
    sim.fluid.vel[...] = vel
    if c is not None:
        sim.get_tracer("tracer").val[...] = c
    return sim, setup


def rel_error(vel_c, ref, fluid) -> float:
    d = (vel_c - ref)[fluid]
    den = float(ref[fluid].pow(2).sum().sqrt())
    err = float(d.pow(2).sum().sqrt()) / den
    return err if math.isfinite(err) else float("inf")


@dataclass
class Trajectory:
    errors: list
    seconds: float  # device time of the coarse run (steps + closure)

    @property
    def mean(self) -> float:
        return float(np.mean(self.errors)) if all(map(math.isfinite, self.errors)) else float("inf")


class Reference:
    """The held-out fine run: its filtered state at t0 and at every horizon, and the device time
    the plain fine method took to get there."""

    def __init__(self, cfg: Config, seed: int):
        torch = _torch()
        nxc, nyc = cfg.coarse
        run = FineRun(cfg, seed)
        run.advance(cfg.spinup)
        self.rho0 = torch.empty((nxc, nyc), device="cuda")
        self.vel0 = torch.empty((nxc, nyc, 2), device="cuda")
        self.c0 = torch.empty((nxc, nyc), device="cuda")
        run.sim._read_back()
        tracer = torch.tensor(run.sim.get_tracer("tracer").val, device="cuda")
        run.coarse_state(self.rho0, self.vel0, c_c=self.c0, tracer_dev=tracer.data_ptr())
        flags_t = torch.tensor(coarse_setup(cfg).flags, device="cuda")
        clean_coarse_state(self.rho0, self.vel0, flags_t, cfg.u_in)
        self.c0[(flags_t & 6) != 0] = 0.0
        self.vel = {}
        self.fine_seconds = 0.0
        done = 0
        for h in cfg.horizons:
            self.fine_seconds += run.advance(cfg.factor * (h - done))
            done = h
            v = torch.empty((nxc, nyc, 2), device="cuda")
            r = torch.empty((nxc, nyc), device="cuda")
            run.coarse_state(r, v)
            self.vel[h] = v
        self.fine_steps = cfg.factor * cfg.horizons[-1]
        self.fluid = (flags_t & 7) == 0


def coarse_trajectory(cfg: Config, ref: Reference, net: Net | None,
                      uniform_dtau: float | None = None) -> Trajectory:
    """The coarse run from ref's filtered start: plain (net None), with the closure, or with a
    spatially uniform relaxation-time correction ``uniform_dtau`` on every fluid cell (the
    ablation of the network's spatial field: tau = tau0 + uniform_dtau, constant in time)."""
    torch = _torch()
    sim, setup = start_coarse(cfg, ref.rho0.cpu().numpy(), ref.vel0.cpu().numpy(),
                              ref.c0.cpu().numpy())
    run = ClosedRun(sim, setup.flags, net, cfg.every, setup.tau)
    uniform = None
    if uniform_dtau is not None:
        if net is not None:
            raise ValueError("a uniform correction replaces the network")
        fluid = torch.tensor((np.asarray(setup.flags) & 7) == 0, device="cuda").reshape(-1)
        uniform = torch.full((fluid.numel(),), 1.0 / setup.tau, device="cuda")
        uniform[fluid] = 1.0 / (setup.tau + uniform_dtau)
        torch.cuda.synchronize()
        sim._set_omega_field(uniform.data_ptr())
    ext = torch.cuda.ExternalStream(run.stream)
    errors, seconds, done = [], 0.0, 0
    for h in cfg.horizons:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        run.advance(h - done)
        e1.record(ext)
        e1.synchronize()
        seconds += e0.elapsed_time(e1) / 1e3
        done = h
        sim._read_back()
        vel = torch.tensor(sim.fluid.vel, device="cuda")
        errors.append(rel_error(vel, ref.vel[h], ref.fluid))
        if not math.isfinite(errors[-1]):
            errors += [float("inf")] * (len(cfg.horizons) - len(errors))
            break
    run.close()
    if uniform is not None:
        sim._set_omega_field(0)
    return Trajectory(errors, seconds)


def field_mean(cfg: Config, net: Net, ref: Reference) -> float:
    """Mean relaxation-time correction tau - tau0 the network installs over the fluid cells,
    averaged over every application of the closed coarse run from ref's start."""
    torch = _torch()
    sim, setup = start_coarse(cfg, ref.rho0.cpu().numpy(), ref.vel0.cpu().numpy(),
                              ref.c0.cpu().numpy())
    run = ClosedRun(sim, setup.flags, net, cfg.every, setup.tau)
    fluid = torch.tensor((np.asarray(setup.flags) & 7) == 0, device="cuda").reshape(-1)
    ext = torch.cuda.ExternalStream(run.stream)
    total, count = 0.0, 0
    for _ in range(cfg.horizons[-1] // cfg.every):
        with torch.cuda.stream(ext):
            run.apply()
            total += float((1.0 / run.omega[fluid] - setup.tau).mean())
        count += 1
        sim._iterate_device(cfg.every)
    sim._synchronize()
    run.close()
    return total / count


# Uniform corrections tried for the calibrated constant, besides multiples of the network field's
# mean: from 6% to 60x the coarse set-up's own tau0 - 1/2 (4.8e-4), i.e. a constant eddy
# viscosity up to well past what the coarse run needs to stay finite, with steps of about 1.2x
# around the smallest values that keep it finite (more dissipation only adds error there).
UNIFORM_DTAU = (3e-5, 1e-4, 1.2e-4, 1.4e-4, 1.7e-4, 2e-4, 2.4e-4, 3e-4, 4e-4, 6e-4, 1e-3, 3e-3,
                1e-2, 3e-2)


def ablation(cfg: Config, net: Net, calib: Reference, test: Reference,
             factors=(0.25, 0.5, 1.0, 2.0, 4.0), absolute=UNIFORM_DTAU) -> dict:
    """What the network's spatial field adds over a spatially uniform correction. Judged on the
    test seed, like the closure: (a) the uniform correction equal to the mean of the network's
    own field there; (b) the best uniform correction among factors x that mean and the absolute
    values, picked on the calibration seed. Mean relative velocity L2 errors against the filtered
    fine run."""
    mean_dtau = field_mean(cfg, net, test)
    candidates = sorted({f * mean_dtau for f in factors} | set(absolute))
    calibration = {d: coarse_trajectory(cfg, calib, None, d).mean for d in candidates}
    best = min(calibration, key=lambda d: calibration[d])
    a = coarse_trajectory(cfg, test, None, mean_dtau)
    b = coarse_trajectory(cfg, test, None, best)
    closed = coarse_trajectory(cfg, test, net)
    return {
        "field_mean_dtau": mean_dtau,
        "calibration_mean_errors": {f"{d:.3g}": e for d, e in calibration.items()},
        "calibrated_dtau": best,
        "uniform_mean": {"dtau": mean_dtau, "errors": a.errors, "mean": a.mean},
        "uniform_calibrated": {"dtau": best, "errors": b.errors, "mean": b.mean},
        "closure": {"errors": closed.errors, "mean": closed.mean},
    }


def calibrate(cfg: Config, net: Net, ref: Reference) -> dict:
    """Picks C_k (gain = 3 C_k scale) with the lowest mean error on a training seed."""
    results = {}
    for ck in cfg.gains_ck:
        net.gain = 3.0 * ck * net.target_scale
        results[ck] = coarse_trajectory(cfg, ref, net).mean
    best = min(results, key=lambda k: results[k])
    net.gain = 3.0 * best * net.target_scale
    net.meta["c_k"] = best
    return {"c_k": best, "mean_errors": results}


@dataclass
class Verdict:
    accepted: bool
    bound: float
    plain: Trajectory
    closed: Trajectory
    fine_seconds: float
    fine_steps: int
    horizons: tuple

    def summary(self) -> dict:
        d = {
            "accepted": self.accepted,
            "bound": self.bound,
            "horizons_coarse_steps": list(self.horizons),
            "plain_coarse_errors": self.plain.errors,
            "closure_errors": self.closed.errors,
            "plain_coarse_mean": self.plain.mean,
            "closure_mean": self.closed.mean,
            "closure_seconds": self.closed.seconds,
            "plain_coarse_seconds": self.plain.seconds,
            "fine_seconds": self.fine_seconds,
            "fine_steps": self.fine_steps,
            "time_ratio_fine_over_closure": self.fine_seconds / max(self.closed.seconds, 1e-12),
        }
        return d


def judge(cfg: Config, net: Net, ref: Reference) -> Verdict:
    """A posteriori test on a held-out fine run. Accepted when the closure's mean relative error
    is finite and at most ``cfg.bound``, and at the last horizon plain coarse survives the closure
    is no worse than it."""
    plain = coarse_trajectory(cfg, ref, None)
    closed = coarse_trajectory(cfg, ref, net)
    ok = math.isfinite(closed.mean) and closed.mean <= cfg.bound
    finite_plain = [i for i, e in enumerate(plain.errors) if math.isfinite(e)]
    if ok and finite_plain:
        last = finite_plain[-1]
        ok = closed.errors[last] <= plain.errors[last] * (1 + 1e-9) or last < len(plain.errors) - 1
    return Verdict(ok, cfg.bound, plain, closed, ref.fine_seconds, ref.fine_steps, cfg.horizons)


def run_closed_or_fine(cfg: Config, verdict: Verdict, net: Net, ref: Reference):
    """What a user gets: the coarse+closure velocity at the last horizon when the closure was
    accepted, else the plain fine run's (box-filtered) velocity -- the fallback."""
    if verdict.accepted:
        sim, setup = start_coarse(cfg, ref.rho0.cpu().numpy(), ref.vel0.cpu().numpy(),
                                  ref.c0.cpu().numpy())
        run = ClosedRun(sim, setup.flags, net, cfg.every, setup.tau)
        run.advance(cfg.horizons[-1])
        sim._read_back()
        run.close()
        return "closure", np.array(sim.fluid.vel)
    return "fine", ref.vel[cfg.horizons[-1]].cpu().numpy()
