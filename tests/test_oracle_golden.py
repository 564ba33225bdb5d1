"""The CPU oracle (C restatement) against the golden fixtures made by the reference's kernels."""

import numpy as np
import pytest

from oracle import build as oracle_build
from oracle.oracle import OracleSimulation, velocity_set
from tests import golden_cases
from tests.golden.make_golden import omega_of

oracle_build.build_oracle()

# After at most 10 steps the restatement differs from the reference's kernels only by the
# rounding order of float moments (a few ulp): 1e-6 norm-wise relative is the pin.
TOL = 1e-6


def _run_port(spec, inputs):
    sim = OracleSimulation(spec["counts"], omega_of(spec["omega"]), backend="port")
    sim.flags[...] = inputs["flags"]
    sim.rho[...] = inputs["rho"]
    sim.vel[...] = inputs["vel"]
    for name, om in spec.get("tracers", []):
        sim.add_tracer(name, omega_of(om)).val[...] = inputs[f"val_{name}"]
    if spec.get("gravity") is not None:
        sim.set_gravity(spec["gravity"])
    for name, alpha, c0, g in spec.get("couplings", []):
        sim.add_boussinesq_coupling(name, alpha, c0, g)
    for n in spec["calls"]:
        sim.iterate(n)
        yield sim


@pytest.mark.parametrize("name", golden_cases.names())
def test_oracle_matches_reference_kernels(name):
    spec, inputs, outs = golden_cases.load(name)
    for sim, ref in zip(_run_port(spec, inputs), outs):
        assert golden_cases.rel_err(sim.rho, ref["rho"]) < TOL
        assert golden_cases.rel_err(sim.vel, ref["vel"]) < 10 * TOL
        assert golden_cases.rel_err(sim.f, ref["f"]) < TOL
        for tname in sim.tracers:
            assert golden_cases.rel_err(sim.tracers[tname].val, ref[f"val_{tname}"]) < TOL
            assert golden_cases.rel_err(sim.tracers[tname].g, ref[f"g_{tname}"]) < TOL


def test_golden_walls_hold_populations():
    """Wall cells are never updated (src/lib.cl:210-213): their rho/vel stay at the inputs."""
    spec, inputs, outs = golden_cases.load("d2q9_bgk_walls_fixed")
    wall = (inputs["flags"] & 1) == 1
    assert wall.any()
    np.testing.assert_array_equal(outs[-1]["rho"][wall], inputs["rho"][wall])
    np.testing.assert_array_equal(outs[-1]["vel"][wall], inputs["vel"][wall])


def test_golden_fixed_cells_keep_rho_vel():
    """FIXED_FLUID_VELOCITY (2) and FIXED_FLUID_DENSITY (4) both pin rho and vel (c & 6)."""
    spec, inputs, outs = golden_cases.load("d2q9_bgk_walls_fixed")
    fixed = ((inputs["flags"] & 6) != 0) & ((inputs["flags"] & 1) == 0)
    assert fixed.any()
    np.testing.assert_array_equal(outs[-1]["rho"][fixed], inputs["rho"][fixed])
    np.testing.assert_array_equal(outs[-1]["vel"][fixed], inputs["vel"][fixed])


@pytest.mark.parametrize("d,q", [(1, 3), (2, 9), (2, 5), (3, 7), (3, 27)])
def test_velocity_sets(d, q):
    """Tables of src/velocities.rs:66-191: weights sum to 1, opposite pairs, zero first moment."""
    c, w, opp = velocity_set(d, q)
    assert abs(w.sum() - 1.0) < 1e-15
    np.testing.assert_array_equal(c[opp], -c)
    np.testing.assert_allclose((w[:, None] * c).sum(0), 0, atol=1e-15)
    assert (c[0] == 0).all()


@pytest.mark.parametrize("name", golden_cases.names())
def test_fixtures_regenerate_from_their_seeds(name):
    """Each fixture's inputs come from its case's seed (its position in CASES), and, where the
    reference's kernels are built, its outputs are exactly what they produce: the committed
    vectors are the reference's, not a snapshot of this implementation."""
    from oracle.oracle import reference_available
    from tests.golden.make_golden import CASES, run_oracle, seeded_inputs

    spec, inputs, outs = golden_cases.load(name)
    assert CASES[name] == spec
    seed = list(CASES).index(name)
    regen = seeded_inputs(spec, seed=seed)
    assert sorted(regen) == sorted(inputs)
    for key, value in regen.items():
        np.testing.assert_array_equal(value, inputs[key])
    if not reference_available():
        pytest.skip("reference kernels not built here")
    for got, want in zip(run_oracle(spec, inputs, backend="reference"), outs):
        assert sorted(got) == sorted(want)
        for key in want:
            np.testing.assert_array_equal(got[key], want[key])
