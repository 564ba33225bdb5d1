"""What the trained closure gains over the coarse method without it, on the full-size closure
experiment: coarse 1024x512 cylinder channel (radius 16, Re 10,000) against the 4x4 box filter of
the 4096x2048 plain run. Data, training (the project's forward/backward/Adam kernels),
calibration and the a posteriori judgement all run here; every step is deterministic."""

from __future__ import annotations

import dataclasses
import math

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from boltzmann_b200 import closure as cl

    cfg = cl.Config()
    data = cl.generate(cfg)
    net, rep = cl.train(cfg, data)
    del data
    calref = cl.Reference(cfg, cfg.calib_seed)
    cal = cl.calibrate(cfg, net, calref)
    ref = cl.Reference(cfg, cfg.test_seed)
    return cl, cfg, net, rep, cal, ref, calref


def test_training_converges(trained):
    cl, cfg, net, rep, cal, ref, calref = trained
    assert rep.losses[-1][1] < 0.2 * rep.losses[0][1], rep.losses


def test_closure_beats_plain_coarse_and_is_accepted(trained):
    cl, cfg, net, rep, cal, ref, calref = trained
    v = cl.judge(cfg, net, ref)
    s = v.summary()
    # accepted: finite over every horizon, mean relative velocity L2 error within the bound
    assert v.accepted, s
    assert all(math.isfinite(e) for e in v.closed.errors)
    assert v.closed.mean <= cfg.bound
    # the gain: without the closure the coarse run is worse at the last horizon (here it does not
    # survive it at all)
    assert v.plain.errors[-1] > v.closed.errors[-1], s
    # and it costs far less GPU time than the fine run over the same physical time
    assert s["time_ratio_fine_over_closure"] >= 5.0, s
    kind, vel = cl.run_closed_or_fine(cfg, v, net, ref)
    assert kind == "closure" and vel.shape == (cfg.coarse[0], cfg.coarse[1], 2)


def test_rejected_closure_falls_back_to_fine(trained):
    cl, cfg, net, rep, cal, ref, calref = trained
    strict = dataclasses.replace(cfg, bound=1e-4)
    v = cl.judge(strict, net, ref)
    assert not v.accepted
    kind, vel = cl.run_closed_or_fine(strict, v, net, ref)
    assert kind == "fine"
    assert (vel == ref.vel[cfg.horizons[-1]].cpu().numpy()).all()


def test_network_field_beats_uniform_corrections(trained):
    """The ablation of the network's spatial field: the same coarse runs with a relaxation-time
    correction that is uniform over the fluid cells. (a) The uniform correction equal to the mean
    of the network's own field does not keep the coarse run finite: the network's dissipation is
    concentrated where the coarse grid needs it. (b) The best uniform correction, calibrated on the
    calibration seed over a grid up to 60x the coarse run's own viscosity, is beaten by the
    network at every horizon of the held-out seed (measured: mean 0.0362 against 0.0365; 0.0418
    against 0.0430 at the last horizon)."""
    cl, cfg, net, rep, cal, ref, calref = trained
    ab = cl.ablation(cfg, net, calref, ref)
    closure = ab["closure"]
    assert all(math.isfinite(e) for e in closure["errors"]), ab
    assert not math.isfinite(ab["uniform_mean"]["mean"]), ab
    best = ab["uniform_calibrated"]
    assert math.isfinite(best["mean"]), ab
    assert closure["mean"] < best["mean"], ab
    assert all(c <= u for c, u in zip(closure["errors"], best["errors"])), ab
