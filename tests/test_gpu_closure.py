"""The closure and post-processing kernels (csrc/closure.cu) against the CPU oracle
(oracle/closure_oracle.py): post-processing bit-exact against the reference's own outputs,
features bit-exact, each layer of the forward pass and the full gradient within the BF16/FP32
tolerances below, deterministic reductions, training that lowers the loss, and the per-cell
relaxation field of the stencil."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import closure_oracle as co

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "postproc.npz"


@pytest.fixture(scope="module")
def torch():
    import torch

    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def cl():
    from boltzmann_b200 import closure

    return closure


def _bf16_tensor_to_np(t):
    return (t.cpu().numpy().view(np.uint16).astype(np.uint32) << 16).view(np.float32)


def test_postproc_matches_reference(torch, cl):
    g = np.load(GOLDEN)
    v2 = torch.tensor(g["vel2d"], device="cuda")
    v3 = torch.tensor(g["vel3d"], device="cuda")
    np.testing.assert_array_equal(cl.curl(v2).cpu().numpy(), g["curl2d"])
    np.testing.assert_array_equal(cl.curl(v3).cpu().numpy(), g["curl3d"])
    np.testing.assert_array_equal(cl.vmag(v2).cpu().numpy(), g["vmag2d"])
    np.testing.assert_array_equal(cl.vmag(v3).cpu().numpy(), g["vmag3d"])


def _inputs(seed, B, nx, ny):
    rng = np.random.default_rng(seed)
    rho = (1 + 0.01 * rng.normal(size=(B, nx, ny))).astype(np.float32)
    vel = (0.05 * rng.normal(size=(B, nx, ny, 2))).astype(np.float32)
    flags = np.zeros((nx, ny), np.int32)
    flags[0, :] = 1
    flags[nx // 2, 3 : ny // 2] = 1
    flags[-1, 1:-1] = 6
    norm = np.array([0.0, 0.01, 0.0, 0.0, 80.0, 15.0, 20.0, 30.0], np.float32)
    return rho, vel, flags, norm


# nx = 10 leaves a partial tile along x (tiles are 4 rows), ny = 70 one along y (64 columns).
SHAPES = [(2, 10, 70), (1, 8, 64), (3, 5, 9)]


@pytest.mark.parametrize("B,nx,ny", SHAPES)
def test_features_bit_exact(torch, cl, B, nx, ny):
    rho, vel, flags, norm = _inputs(1, B, nx, ny)
    bufs = cl.Buffers(nx, ny, B, train=False)
    cl.features(torch.tensor(rho, device="cuda"), torch.tensor(vel, device="cuda"),
                torch.tensor(flags, device="cuda"), norm, bufs, 0)
    torch.cuda.synchronize()
    got = _bf16_tensor_to_np(bufs.x).reshape(B, nx, ny, 4)
    want = co.features(rho, vel, flags, norm)
    np.testing.assert_array_equal(got, want)


def _forward(torch, cl, B, nx, ny, seed=2):
    rho, vel, flags, norm = _inputs(seed, B, nx, ny)
    params = co.init_params(seed)
    net = cl.Net(params, norm)
    bufs = cl.Buffers(nx, ny, B, train=True)
    flags_t = torch.tensor(flags, device="cuda")
    cl.features(torch.tensor(rho, device="cuda"), torch.tensor(vel, device="cuda"), flags_t,
                norm, bufs, 0)
    cl.forward(net, bufs, 0)
    torch.cuda.synchronize()
    C = co.C
    acts = {
        "z1": bufs.z1.cpu().numpy().reshape(B, nx, ny, C).astype(np.float64),
        "a1": _bf16_tensor_to_np(bufs.a1).reshape(B, nx, ny, C).astype(np.float64),
        "z2": bufs.z2.cpu().numpy().reshape(B, nx, ny, C).astype(np.float64),
        "a2": _bf16_tensor_to_np(bufs.a2).reshape(B, nx, ny, C).astype(np.float64),
        "y": bufs.y.cpu().numpy().reshape(B, nx, ny).astype(np.float64),
    }
    x = _bf16_tensor_to_np(bufs.x).reshape(B, nx, ny, 4).astype(np.float64)
    return net, bufs, flags, flags_t, params, x, acts


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.fixture(params=["tcgen05", "warp_mma"])
def layer2(request, cl):
    """Runs a test with each kernel of layer 2 (training forward and transposed conv)."""
    cl.set_layer2_kernel(request.param)
    yield request.param
    cl.set_layer2_kernel("tcgen05")


@pytest.mark.parametrize("B,nx,ny", SHAPES)
def test_forward_layers_match_oracle(torch, cl, B, nx, ny, layer2):
    """Each layer from the GPU's own (BF16) input: FP32 accumulation of BF16 products against a
    float64 sum of the same products; BF16 outputs may differ by one unit where the FP32 value
    sits on a rounding boundary."""
    net, bufs, flags, _, params, x, g = _forward(torch, cl, B, nx, ny)
    P = co.unpack(params)
    w1, w2, w3 = (co.bf16(P[k].astype(np.float32)).astype(np.float64) for k in ("w1", "w2", "w3"))
    z1 = co._conv(x, w1, P["b1"])
    assert np.abs(g["z1"] - z1).max() <= 2e-6 * max(1.0, np.abs(z1).max())
    a1 = co.bf16(co.gelu(g["z1"]).astype(np.float32))
    assert np.mean(a1 != g["a1"]) < 1e-3
    assert np.abs(a1 - g["a1"]).max() <= 2.0**-7 * np.abs(a1).max()
    z2 = co._conv(g["a1"], w2, P["b2"])
    assert np.abs(g["z2"] - z2).max() <= 1e-5 * max(1.0, np.abs(z2).max())
    a2 = co.bf16(co.gelu(g["z2"]).astype(np.float32))
    assert np.mean(a2 != g["a2"]) < 1e-3
    y = co._conv(g["a2"], w3[None], P["b3"])[..., 0]
    assert np.abs(g["y"] - y).max() <= 1e-5 * max(1.0, np.abs(y).max())
    # and end to end against the oracle's own forward pass
    ref = co.forward(params, x)
    assert _rel(g["y"], ref["y"]) < 5e-3


@pytest.mark.parametrize("B,nx,ny", SHAPES + [(2, 30, 130)])
def test_loss_and_gradient_match_oracle(torch, cl, B, nx, ny, layer2):
    net, bufs, flags, flags_t, params, x, g = _forward(torch, cl, B, nx, ny, seed=3)
    rng = np.random.default_rng(9)
    target = rng.normal(size=(B, nx, ny)).astype(np.float32)
    tt = torch.tensor(target, device="cuda").reshape(-1)
    cl.loss_and_grad(net, bufs, tt, flags_t, 0)
    torch.cuda.synchronize()
    loss_ref, dy_ref = co.loss(g["y"], target, flags)
    assert abs(bufs.loss.item() - loss_ref) <= 1e-6 * loss_ref
    dy = bufs.dy.cpu().numpy().reshape(B, nx, ny).astype(np.float64)
    assert np.abs(dy - dy_ref).max() <= 1e-6 * np.abs(dy_ref).max()
    grad = bufs.grad.cpu().numpy().astype(np.float64)
    want = co.backward(params, x, g, dy)
    for name, lo, hi in (("w1", 0, 1152), ("b1", 1152, 1184), ("w2", 1184, 10400),
                         ("b2", 10400, 10432), ("w3", 10432, 10720), ("b3", 10720, 10721)):
        # FP32 tile sums vs float64, plus rare one-unit BF16 flips of the gradients inside
        assert _rel(grad[lo:hi], want[lo:hi]) < 5e-3, name
    # deterministic: the same call again gives the same bits
    first = bufs.grad.clone()
    cl.loss_and_grad(net, bufs, tt, flags_t, 0)
    torch.cuda.synchronize()
    assert torch.equal(first, bufs.grad)


def test_adam_matches_formula(torch, cl):
    rng = np.random.default_rng(4)
    p0 = rng.normal(size=cl.NPARAMS).astype(np.float32)
    net = cl.Net(p0, np.zeros(8, np.float32))
    opt = cl.Adam(net, lr=1e-2)
    m = np.zeros(cl.NPARAMS)
    v = np.zeros(cl.NPARAMS)
    p = p0.astype(np.float64)
    for step in range(1, 4):
        gnp = rng.normal(size=cl.NPARAMS).astype(np.float32)
        opt.step(torch.tensor(gnp, device="cuda"), 0)
        m = 0.9 * m + 0.1 * gnp
        v = 0.999 * v + 0.001 * gnp.astype(np.float64) ** 2
        p = p - 1e-2 * (m / (1 - 0.9**step)) / (np.sqrt(v / (1 - 0.999**step)) + 1e-8)
    torch.cuda.synchronize()
    got = net.params.cpu().numpy()
    assert np.abs(got - p).max() < 1e-5
    np.testing.assert_array_equal(_bf16_tensor_to_np(net.bf16)[: cl.NPARAMS], co.bf16(got))


def test_training_lowers_the_loss(torch, cl):
    """Fit the network to a smooth function of its inputs on a small batch."""
    B, nx, ny = 4, 16, 64
    rho, vel, flags, norm = _inputs(5, B, nx, ny)
    flags[:] = 0
    flags_t = torch.tensor(flags, device="cuda")
    net = cl.Net(co.init_params(1), norm)
    bufs = cl.Buffers(nx, ny, B, train=True)
    cl.features(torch.tensor(rho, device="cuda"), torch.tensor(vel, device="cuda"), flags_t,
                norm, bufs, 0)
    target = torch.tensor(np.sqrt(vel[..., 0] ** 2 + vel[..., 1] ** 2) * 20, device="cuda").reshape(-1)
    opt = cl.Adam(net, lr=3e-3)
    losses = []
    for it in range(150):
        cl.forward(net, bufs, 0)
        cl.loss_and_grad(net, bufs, target, flags_t, 0)
        opt.step(bufs.grad, 0)
        if it % 50 == 0 or it == 149:
            losses.append(bufs.loss.item())
    assert losses[-1] < 0.2 * losses[0], losses


def test_coarsen_matches_oracle(torch, cl):
    rng = np.random.default_rng(6)
    nx, ny, f = 16, 24, 4
    rho = (1 + 0.01 * rng.normal(size=(nx, ny))).astype(np.float32)
    vel = (0.05 * rng.normal(size=(nx, ny, 2))).astype(np.float32)
    c = rng.uniform(size=(nx, ny)).astype(np.float32)
    inputs = [torch.tensor(a, device="cuda") for a in (rho, vel, c)]  # kept alive for the call
    rc, vc, cc, sg = (torch.empty((nx // f, ny // f) + s, device="cuda") for s in ((), (2,), (), ()))
    cl._check(cl._lib.lbm_closure_coarsen(*(t.data_ptr() for t in inputs), nx, ny, f,
                                          rc.data_ptr(), vc.data_ptr(), cc.data_ptr(),
                                          sg.data_ptr(), 0))
    torch.cuda.synchronize()
    r, v, c2, s = co.coarsen(rho, vel, c, f)
    for got, want in ((rc, r), (vc, v), (cc, c2), (sg, s)):
        assert np.abs(got.cpu().numpy() - want).max() <= 1e-6 * max(1e-3, np.abs(want).max())


def _sim(tau, counts=(48, 40)):
    from boltzmann_b200.core import Simulation, bgk

    rng = np.random.default_rng(0)
    sim = Simulation("gpu", list(counts), bgk(tau))
    sim.cells.flags[0, :] = 1
    sim.cells.flags[-1, :] = 1
    sim.fluid.vel[...] = rng.uniform(-0.03, 0.03, sim.fluid.vel.shape).astype(np.float32)
    sim.fluid.vel[sim.cells.flags == 1] = 0
    return sim


def test_uniform_omega_field_equals_that_rate(torch):
    """A field holding 1/tau' everywhere gives exactly the run of a simulation built with tau'."""
    a, b = _sim(0.8), _sim(0.6)
    field = torch.full((48 * 40,), np.float32(1.0 / np.float32(0.6)), device="cuda")
    torch.cuda.synchronize()
    a._set_omega_field(field.data_ptr())
    a.iterate(20)
    b.iterate(20)
    np.testing.assert_array_equal(a.fluid.vel, b.fluid.vel)
    np.testing.assert_array_equal(a.fluid.rho, b.fluid.rho)
    a._set_omega_field(0)


def test_omega_field_is_local(torch):
    """A field that differs from the uniform rate only in the right half leaves the left half
    unchanged for as many steps as information needs to cross the gap."""
    a, b = _sim(0.7), _sim(0.7)
    om = np.full((48, 40), 1.0 / 0.7, np.float32)
    om[30:] = 1.0 / 0.9
    field = torch.tensor(om.reshape(-1), device="cuda")
    torch.cuda.synchronize()
    a._set_omega_field(field.data_ptr())
    a.iterate(10)
    b.iterate(10)
    np.testing.assert_array_equal(a.fluid.vel[:19], b.fluid.vel[:19])
    assert not np.array_equal(a.fluid.vel[30:], b.fluid.vel[30:])
    a._set_omega_field(0)


# Partial tiles in both directions (tiles are 14 x 64 output cells), an exact tile, a tiny domain,
# and the full coarse lattice of the closure experiment.
FUSED_SHAPES = [(30, 70), (14, 64), (5, 9), (1024, 512)]


@pytest.mark.parametrize("nx,ny", FUSED_SHAPES)
def test_fused_relaxation_matches_layered_kernels(torch, cl, nx, ny):
    """lbm_closure_relaxation (features, three layers and the tau mapping in one kernel, halos
    recomputed per tile, layer 2 on tcgen05) against the layer-by-layer kernels on the same state.
    Every layer sums in a different order there (FP32 FMAs, warp MMAs), so BF16 activations may
    differ by one unit on rounding boundaries; the relaxation rates agree to 1e-4 relative."""
    rho, vel, flags, norm = _inputs(11, 1, nx, ny)
    net = cl.Net(co.init_params(4), norm, gain=0.02, max_dtau=0.05)
    flags_t = torch.tensor(flags, device="cuda")
    r = torch.tensor(rho[0], device="cuda")
    v = torch.tensor(vel[0], device="cuda")
    fused = torch.full((nx * ny,), float("nan"), device="cuda")
    layered = torch.full((nx * ny,), float("nan"), device="cuda")
    bufs = cl.Buffers(nx, ny, 1, train=False)
    for _ in range(2):  # two calls in a row: no state carried between them
        cl.relaxation(net, r, v, flags_t, nx, ny, 0.51, fused, 0)
    cl.relaxation_layered(net, r, v, flags_t, bufs, 0.51, layered, 0)
    torch.cuda.synchronize()
    cl.status()
    a, b = fused.cpu().numpy(), layered.cpu().numpy()
    assert np.isfinite(a).all()
    assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()
    assert np.mean(a == b) > 0.9
    fixed_or_wall = (flags.reshape(-1) & 7) != 0
    assert (a[fixed_or_wall] == np.float32(1.0) / np.float32(0.51)).all()
    # the network's output really varies the rate inside the fluid
    assert np.ptp(a[~fixed_or_wall]) > 1e-3


def test_layer2_kernels_agree(torch, cl):
    """The tcgen05 and the warp-MMA kernels of layer 2 compute the same products in a different
    summation order: z2 within FP32 accumulation noise, the BF16 activations and every gradient
    block nearly identical."""
    B, nx, ny = 2, 40, 150  # several 14 x 64 and 4 x 64 tiles, partial ones at both edges
    runs = {}
    for kind in ("warp_mma", "tcgen05"):
        cl.set_layer2_kernel(kind)
        net, bufs, flags, flags_t, params, x, g = _forward(torch, cl, B, nx, ny, seed=5)
        rng = np.random.default_rng(4)
        tt = torch.tensor(rng.normal(size=(B, nx, ny)).astype(np.float32), device="cuda")
        cl.loss_and_grad(net, bufs, tt.reshape(-1), flags_t, 0)
        torch.cuda.synchronize()
        runs[kind] = (g, bufs.grad.cpu().numpy().astype(np.float64))
    cl.set_layer2_kernel("tcgen05")
    (ga, grad_a), (gb, grad_b) = runs["warp_mma"], runs["tcgen05"]
    assert np.abs(ga["z2"] - gb["z2"]).max() <= 1e-5 * max(1.0, np.abs(ga["z2"]).max())
    assert np.mean(ga["a2"] != gb["a2"]) < 1e-3
    assert _rel(gb["y"], ga["y"]) < 1e-3
    for lo, hi in ((0, 1152), (1152, 1184), (1184, 10400), (10400, 10432), (10432, 10721)):
        assert _rel(grad_b[lo:hi], grad_a[lo:hi]) < 5e-3, (lo, hi)
