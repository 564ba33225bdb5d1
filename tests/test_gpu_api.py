"""The reference's Python API on the CUDA backend.

The first four tests are the hot-path tests of the reference's own suite
(python/tests/test_core.py:57-127), with "cpu" meaning "the CUDA device" as everywhere here,
imported as the reference's scripts import them: ``boltzmann.core`` through the aliases of
``boltzmann_b200.alias``. (The reference's module itself runs unchanged through the same aliases
in ``tests/test_reference_suite_cpu.py`` wherever the reference checkout exists.)
"""

from __future__ import annotations

import tempfile

import numpy as np
import pytest

from boltzmann_b200 import alias

alias.install()
from boltzmann.core import PanicException, Simulation, bgk, trt  # noqa: E402
from tests import golden_cases  # noqa: E402
from tests.golden_cases import rel_err  # noqa: E402

pytestmark = pytest.mark.gpu


def test_simulation_1():
    sim = Simulation("cpu", [100, 100], bgk(0.51))
    assert sim.fluid.vel.shape == (100, 100, 2)
    assert sim.fluid.rho.shape == (100, 100)
    assert sim.cells.flags.shape == (100, 100)
    assert abs(sim.fluid.vel.min() - 0) < 1e-8
    assert abs(sim.fluid.vel.max() - 0) < 1e-8
    assert abs(sim.fluid.rho.max() - 1) < 1e-8
    sim.iterate(10)
    assert abs(sim.fluid.vel.mean() - 0) < 1e-4
    assert abs(sim.fluid.rho.mean() - 1) < 1e-4


def test_simulation_2():
    sim = Simulation("cpu", [100, 100], bgk(0.51))
    tracer = sim.add_tracer("tracer", bgk(0.51))
    tracer.val[10:20, 30:40] = 1.0
    sim.iterate(10)
    assert abs(tracer.val.sum() - 10**2) < 1e-4


def test_simulation_3():
    sim = Simulation("cpu", [100, 100], bgk(1.0))
    sim.set_gravity(np.array([0, 0.1], dtype=np.float32))
    sim.iterate(10)
    assert abs(sim.fluid.vel[..., 1].mean() - 0.1 * 10) < 1e-4


def test_simulation_serde():
    with tempfile.TemporaryDirectory() as tmpdirname:
        path = tmpdirname + "/checkpoint.mpk"
        sim1 = Simulation("cpu", [100, 100], bgk(0.51))
        trc1 = sim1.add_tracer("tracer", bgk(0.51))
        trc1.val[10:20, 30:40] = 1.0
        sim1.add_boussinesq_coupling(trc1, 0.1, 0, np.array([0, 1], np.float32))
        sim1.iterate(10)
        sim1.write_checkpoint(path)
        sim2 = Simulation.load_checkpoint("cpu", path)
        trc2 = sim2.get_tracer("tracer")
        assert np.allclose(sim1.fluid.rho, sim2.fluid.rho)
        assert np.allclose(sim1.fluid.vel, sim2.fluid.vel)
        assert np.allclose(trc1.val, trc2.val)


def test_checkpoint_resume_is_exact():
    """A loaded checkpoint continues bit-identically (f in standard order after even steps)."""
    with tempfile.TemporaryDirectory() as d:
        a = Simulation("gpu", [40, 30], trt(0.6))
        t = a.add_tracer("c", bgk(0.7))
        t.val[5:15, 5:15] = 1.0
        a.cells.flags[:, 0] = 1
        a.cells.flags[:, -1] = 1
        a.add_boussinesq_coupling(t, 0.5, 0.0, np.array([0.0, -1e-3], np.float32))
        a.iterate(20)
        a.write_checkpoint(d + "/c.mpk")
        b = Simulation.load_checkpoint("gpu", d + "/c.mpk")
        assert b.iteration == 20
        assert a.size_bytes == b.size_bytes
        a.iterate(20)
        b.iterate(20)
        np.testing.assert_array_equal(a.fluid.rho, b.fluid.rho)
        np.testing.assert_array_equal(a.fluid.vel, b.fluid.vel)
        np.testing.assert_array_equal(a.get_tracer("c").val, b.get_tracer("c").val)


def test_api_errors():
    sim = Simulation("gpu", [8, 8], bgk(0.6))
    with pytest.raises(PanicException, match="even"):
        sim.iterate(3)
    with pytest.raises(PanicException, match="Unknown model"):
        Simulation("gpu", [8, 8], bgk(0.6), q=27)
    with pytest.raises(PanicException, match="Invalid number of dimensions"):
        Simulation("gpu", [2, 2, 2, 2], bgk(0.6))
    one_d = Simulation("gpu", [8], bgk(0.6))
    with pytest.raises(PanicException, match="Kernel not found"):
        one_d.iterate(2)


def test_api_shapes_and_sizes():
    sim = Simulation("GPU", [6, 5, 4], bgk(0.6))
    assert sim.fluid.vel.shape == (6, 5, 4, 3)
    assert list(sim.cells.counts) == [6, 5, 4] and sim.cells.count == 120
    t = sim.add_tracer("a", bgk(0.8))
    assert sim.add_tracer("a", bgk(0.9)).val.shape == (6, 5, 4)  # idempotent over the name
    n = 120
    assert sim.fluid.size_bytes == 4 * (n * 27 + n + 3 * n)
    assert t.size_bytes == 4 * (n * 7 + n)
    assert sim.size_bytes == sim.fluid.size_bytes + 4 * n + t.size_bytes
    sim.set_gravity(np.array([0, 0, 1e-4], np.float32))
    sim.iterate(2)
    assert sim.fluid.size_bytes == 4 * (n * 27 + n + 3 * n + 3 * n)  # acc allocated
    assert "GPU" in sim.device_info
    assert sim.iteration == 2


def test_host_edits_after_first_iterate_are_overwritten():
    """After iteration 0 the host arrays are outputs: edits are not uploaded (src/simulation.rs
    283-286) and the read-back overwrites them."""
    sim = Simulation("gpu", [16, 16], bgk(0.6))
    sim.iterate(2)
    before = sim.fluid.rho.copy()
    sim.fluid.rho[...] = 5.0
    sim.iterate(2)
    assert np.abs(sim.fluid.rho - before).max() < 1e-3


@pytest.mark.parametrize("name", golden_cases.names())
def test_golden_through_python_api(name):
    from tests.golden.make_golden import CASES  # noqa: F401  (spec format)

    spec, inputs, outs = golden_cases.load(name)

    def om(s):
        return bgk(s[1]) if s[0] == "bgk" else trt(s[1])

    sim = Simulation("gpu", spec["counts"], om(spec["omega"]))
    sim.cells.flags[...] = inputs["flags"]
    sim.fluid.rho[...] = inputs["rho"]
    sim.fluid.vel[...] = inputs["vel"]
    handles = {}
    for tname, tom in spec.get("tracers", []):
        handles[tname] = sim.add_tracer(tname, om(tom))
        handles[tname].val[...] = inputs[f"val_{tname}"]
    if spec.get("gravity") is not None:
        sim.set_gravity(np.asarray(spec["gravity"], np.float32))
    for tname, alpha, c0, g in spec.get("couplings", []):
        sim.add_boussinesq_coupling(handles[tname], alpha, c0, np.asarray(g, np.float32))
    for n, ref in zip(spec["calls"], outs):
        sim.iterate(n)
        assert rel_err(sim.fluid.rho, ref["rho"]) < 1e-5
        assert rel_err(sim.fluid.vel, ref["vel"]) < 1e-5
        for tname, h in handles.items():
            assert rel_err(h.val, ref[f"val_{tname}"]) < 1e-5
