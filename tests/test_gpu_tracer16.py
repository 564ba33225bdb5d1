"""16-bit tracer populations (lbm_set_tracer_storage): the fused tracer of a 16-bit fluid stored in
the same 16-bit kind, as values (not offsets from the weights; the tracer spans 0 .. 1).

Against the same run with float tracer populations the tracer and the fluid agree to the 16-bit
rounding (~1e-3); the TMA-staged and direct kernels give the same bits; the tracer mass is
conserved to the rounding; and the API refuses what the kernels do not take."""

from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import Omega as OOmega
from tests.golden_cases import rel_err

pytestmark = pytest.mark.gpu


def _channel(counts, storage, tracer_storage=None, path="auto", seed=0):
    from tests.capi import CApiSim, check

    om = OOmega.trt(0.52, 0.6)
    sim = CApiSim(counts, om.kind, float(om.pos), float(om.neg), storage=storage, path=path)
    if tracer_storage:
        check(sim.set_tracer_storage(tracer_storage))
    rng = np.random.default_rng(seed)
    d = len(counts)
    sim.flags[(slice(None),) * (d - 1) + (0,)] = 1  # a wall plane at the first z
    sim.vel[...] = rng.uniform(-0.03, 0.03, sim.vel.shape).astype(np.float32)
    sim.vel[..., 0] += 0.04
    t = sim.add_tracer(float(OOmega.bgk(0.503).pos))
    band = (rng.uniform(size=counts) < 0.5).astype(np.float32)
    sim.vals[t][...] = band
    g = [0.0] * d
    g[-1] = -1e-5
    sim.add_coupling(t, 1.0, 0.0, g)
    return sim, t


@pytest.mark.parametrize("counts,storage", [([64, 512], "f16"), ([64, 512], "bf16"),
                                            ([8, 8, 256], "f16")])
def test_tracer16_close_to_float_tracer(counts, storage):
    a, ta = _channel(counts, storage)
    b, tb = _channel(counts, storage, tracer_storage=storage)
    for _ in range(3):
        a.iterate(40)
        b.iterate(40)
    tol = 5e-3 if storage == "f16" else 3e-2
    assert rel_err(b.vals[tb], a.vals[ta]) < tol
    assert rel_err(b.vel, a.vel) < tol
    assert np.isfinite(b.vals[tb]).all()


@pytest.mark.parametrize("counts", [[16, 512], [4, 6, 256]])
def test_tracer16_staged_and_direct_agree_bitwise(counts):
    runs = {}
    for path in ("direct", "staged"):
        sim, t = _channel(counts, "f16", tracer_storage="f16", path=path, seed=3)
        sim.iterate(20)
        runs[path] = (sim.rho.copy(), sim.vel.copy(), sim.vals[t].copy(), sim.tracer_populations(t))
    for x, y in zip(runs["direct"], runs["staged"]):
        np.testing.assert_array_equal(x, y)


def test_tracer16_mass_and_populations():
    sim, t = _channel([32, 512], "f16", tracer_storage="f16", seed=5)
    sim.iterate(2)
    m0 = sim.conservation()[3]
    sim.iterate(200)
    m1 = sim.conservation()[3]
    # walls and fixed cells aside, the tracer mass changes only by the 16-bit rounding
    assert abs(m1 - m0) <= 2e-3 * abs(m0)
    g = sim.tracer_populations(t)  # decoded to float, the checkpoint layout
    assert np.isfinite(g).all() and g.shape == (32, 512, 5)
    fluid = sim.flags == 0  # wall cells keep their first value and hold bounced populations
    np.testing.assert_allclose(g.sum(axis=-1)[fluid], sim.vals[t][fluid], rtol=0, atol=2e-3)


def test_tracer16_api_refusals():
    from tests.capi import CApiSim

    sim = CApiSim([16, 64], 0, 1.5, storage="f16")
    assert sim.set_tracer_storage("bf16") == 2  # not the fluid's kind: unsupported
    assert sim.set_tracer_storage("f16") == 0
    sim.add_tracer(1.6)
    with pytest.raises(RuntimeError, match="one tracer"):
        sim.add_tracer(1.6)
    assert sim.set_tracer_storage("f32") == 4  # after the first tracer: state error
    f32 = CApiSim([16, 64], 0, 1.5, storage="f32")
    assert f32.set_tracer_storage("f16") == 2
