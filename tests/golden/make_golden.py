"""Generates the golden fixtures in this folder from the reference's own kernels.

The reference (djbarker/boltzmann) ships no golden vectors, so these are made by running its
``src/lib.cl`` kernels, compiled unmodified as C++ (``oracle/_ref``; see ``oracle/build.py``),
under the host semantics of its ``Simulation`` (``oracle/oracle.py``). Each fixture stores the
case spec, the seeded inputs and the outputs after every ``iterate`` call, so later checks need
neither the reference tree nor the RNG.

Run from the repository root where the reference tree exists:
    python tests/golden/make_golden.py [case ...]
Cases take their seeds from their position in CASES, so new cases go at the end.
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import build as oracle_build  # noqa: E402
from oracle.oracle import Omega, OracleSimulation  # noqa: E402

OUT = Path(__file__).resolve().parent

# name -> spec. omega: ["bgk", tau] or ["trt", tau_pos]; calls: iterate() arguments in order.
CASES: dict[str, dict] = {
    "d2q9_bgk_periodic": dict(counts=[17, 13], omega=["bgk", 0.55], calls=[2, 8]),
    "d2q9_bgk_walls_fixed": dict(counts=[17, 13], omega=["bgk", 0.55], walls=True, calls=[10]),
    "d2q9_trt_walls_gravity": dict(
        counts=[19, 11], omega=["trt", 0.6], walls=True, gravity=[1e-3, -2e-3], calls=[4, 6]
    ),
    "d2q9_trt_tracer_coupling": dict(
        counts=[16, 12],
        omega=["trt", 0.56],
        walls=True,
        tracers=[["t0", ["bgk", 0.6]]],
        couplings=[["t0", 0.1, 0.5, [0.0, -0.01]]],
        calls=[10],
    ),
    "d2q9_bgk_two_tracers_two_couplings": dict(
        counts=[15, 14],
        omega=["bgk", 0.7],
        walls=True,
        gravity=[0.0, 1e-3],
        tracers=[["a", ["bgk", 0.55]], ["b", ["bgk", 0.8]]],
        couplings=[["a", 0.2, 0.0, [0.0, -0.01]], ["b", 0.05, 0.5, [0.01, 0.0]]],
        calls=[2, 4],
    ),
    "d3q27_bgk_periodic": dict(counts=[6, 5, 7], omega=["bgk", 0.6], calls=[4]),
    "d3q27_bgk_walls_gravity": dict(
        counts=[7, 5, 6], omega=["bgk", 0.55], walls=True, gravity=[1e-3, 0.0, -1e-3], calls=[2, 2]
    ),
    "d3q27_trt_tracer_coupling": dict(
        counts=[6, 5, 7],
        omega=["trt", 0.58],
        walls=True,
        tracers=[["t0", ["bgk", 0.65]]],
        couplings=[["t0", 0.1, 0.5, [0.0, 0.0, -0.01]]],
        calls=[4],
    ),
    # TRT tracers: the D2Q5 / D3Q7 TRT kernels the reference's generator writes
    # (python/boltzmann/kernel_gen.py:250-462) but src/opencl.rs never registers.
    "d2q9_trt_trt_tracer": dict(
        counts=[16, 12],
        omega=["trt", 0.57],
        walls=True,
        tracers=[["t0", ["trt", 0.62]]],
        couplings=[["t0", 0.1, 0.5, [0.0, -0.01]]],
        calls=[4, 6],
    ),
    "d3q27_bgk_trt_tracer": dict(
        counts=[6, 5, 7],
        omega=["bgk", 0.6],
        walls=True,
        tracers=[["t0", ["trt", 0.66]]],
        calls=[4],
    ),
}


def omega_of(spec) -> Omega:
    kind, tau = spec
    return Omega.bgk(tau) if kind == "bgk" else Omega.trt(tau)


def seeded_inputs(spec: dict, seed: int) -> dict[str, np.ndarray]:
    """Smooth-ish random state with every flag kind the kernels distinguish."""
    rng = np.random.default_rng(seed)
    counts = spec["counts"]
    d = len(counts)
    out = {
        "rho": (1.0 + rng.uniform(-0.01, 0.01, counts)).astype(np.float32),
        "vel": rng.uniform(-0.05, 0.05, counts + [d]).astype(np.float32),
        "flags": np.zeros(counts, np.int32),
    }
    if spec.get("walls"):
        u = rng.uniform(size=counts)
        flags = np.zeros(counts, np.int32)
        flags[u < 0.08] = 1  # WALL
        flags[(u >= 0.08) & (u < 0.11)] = 2  # FIXED_FLUID_VELOCITY
        flags[(u >= 0.11) & (u < 0.13)] = 4  # FIXED_FLUID_DENSITY
        flags[(u >= 0.13) & (u < 0.16)] = 6  # FIXED_FLUID
        if spec.get("tracers"):
            flags[rng.uniform(size=counts) < 0.06] |= 8  # FIXED_SCALAR_VALUE
        out["flags"] = flags
    for name, _ in spec.get("tracers", []):
        out[f"val_{name}"] = (rng.uniform(size=counts) < 0.5).astype(np.float32)
    return out


def run_oracle(spec: dict, inputs: dict, backend: str) -> list[dict[str, np.ndarray]]:
    sim = OracleSimulation(spec["counts"], omega_of(spec["omega"]), backend=backend)
    sim.flags[...] = inputs["flags"]
    sim.rho[...] = inputs["rho"]
    sim.vel[...] = inputs["vel"]
    for name, om in spec.get("tracers", []):
        t = sim.add_tracer(name, omega_of(om))
        t.val[...] = inputs[f"val_{name}"]
    if spec.get("gravity") is not None:
        sim.set_gravity(spec["gravity"])
    for name, alpha, c0, g in spec.get("couplings", []):
        sim.add_boussinesq_coupling(name, alpha, c0, g)
    outs = []
    for n in spec["calls"]:
        sim.iterate(n)
        o = {"rho": sim.rho.copy(), "vel": sim.vel.copy(), "f": sim.f.copy()}
        for name, t in sim.tracers.items():
            o[f"val_{name}"] = t.val.copy()
            o[f"g_{name}"] = t.g.copy()
        outs.append(o)
    return outs


def main(only: list[str]) -> None:
    if oracle_build.build_ref() is None:
        raise SystemExit("the reference tree is needed to generate golden fixtures")
    oracle_build.build_oracle()
    for k, (name, spec) in enumerate(CASES.items()):
        if only and name not in only:
            continue
        inputs = seeded_inputs(spec, seed=k)
        outs = run_oracle(spec, inputs, backend="reference")
        arrays = {f"in_{key}": v for key, v in inputs.items()}
        for i, o in enumerate(outs):
            arrays.update({f"out{i}_{key}": v for key, v in o.items()})
        np.savez_compressed(OUT / f"{name}.npz", spec=np.array(json.dumps(spec)), **arrays)
        print(f"wrote {name}.npz")


if __name__ == "__main__":
    main(sys.argv[1:])  # case names; none: every case
