"""run_sim of boltzmann_b200.driver on real simulations: the generator protocol, checkpoints that
resume bit for bit, and the device-side non-finite check (a NaN planted in the host density
before the first step)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(tau=0.6, n=(48, 32), seed=0):
    from boltzmann_b200.core import Simulation, bgk

    rng = np.random.default_rng(seed)
    sim = Simulation("gpu", list(n), bgk(tau))
    sim.cells.flags[:, 0] = 1
    sim.cells.flags[:, -1] = 1
    sim.fluid.vel[...] = rng.uniform(-0.02, 0.02, sim.fluid.vel.shape).astype(np.float32)
    sim.fluid.vel[sim.cells.flags == 1] = 0
    return sim


def test_run_sim_steps_checkpoints_and_resumes(tmp_path):
    from boltzmann_b200 import driver
    from boltzmann_b200.core import Simulation

    sim = _sim()
    seen = []
    for i in driver.run_sim(sim, driver.IterInfo(interval=10, count=6), tmp_path, driver.EveryN(4)):
        seen.append((i, sim.iteration, float(sim.fluid.vel[10, 10, 0])))
    assert [s[0] for s in seen] == [0, 1, 2, 3, 4, 5]
    assert [s[1] for s in seen] == [0, 10, 20, 30, 40, 50]
    ck = tmp_path / "checkpoint.mpk"
    assert ck.exists()  # EveryN(4) allows on its third call: after output 3 (step 30)

    # A straight run to the same step gives the same state.
    ref = _sim()
    ref.iterate(50)
    np.testing.assert_array_equal(ref.fluid.vel, sim.fluid.vel)

    # Resume from the checkpoint and finish the run.
    res = Simulation.load_checkpoint("gpu", str(ck))
    assert res.iteration == 30
    out = list(driver.run_sim(res, driver.IterInfo(10, 6), tmp_path / "r", driver.NoCheckpoints()))
    assert out == [3, 4, 5]
    np.testing.assert_array_equal(res.fluid.vel, sim.fluid.vel)


def test_run_sim_raises_on_nonfinite(tmp_path):
    from boltzmann_b200 import driver

    sim = _sim()
    sim.fluid.rho[20, 10] = np.nan  # the equilibrium of this cell is NaN from the first step on
    gen = driver.run_sim(sim, driver.IterInfo(4, 5), tmp_path, driver.NoCheckpoints())
    assert next(gen) == 0
    with pytest.raises(ValueError, match="Non-finite value detected!"):
        next(gen)
