"""Benchmark of the lattice-Boltzmann hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload taylor_green_3d|cylinder_channel|kelvin_helmholtz|
                                cavity_ensemble|closure|closure_forward]
                    [--storage f32|f16|bf16|f64]

One bench step is one AA step pair (two LBM time steps: the even and the odd kernel), the
smallest unit after which the populations are back in the reference's standard layout.
The metric is MLUPS = cells x LBM steps / s, counting every cell (walls included) as the
reference's run_sim does (python/boltzmann/simulation.py:245-246).

Default workload: the D3Q27 BGK Taylor-Green vortex on 256^3 (u0 0.05, Re 1600), FP32 -- the
largest single-GPU configuration, seeded synthetic inputs of that set-up. Its populations
(1.81 GB) exceed the 126 MB L2, so no flush is needed between steps. Every line states the
velocity L2 error of the benched run against an FP64 run of the same set-up and step count.

``--impl reference`` times the reference's own kernels (src/lib.cl compiled as C++, the CPU
checker in oracle/_ref) on all host cores for the same workload, on a bounded number of steps.
Multi-GPU (torchrun): every rank runs an independent replica (the path has no exchange step);
value is the aggregate over ranks, timed as the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}


def measured_peaks() -> tuple[dict, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return PEAKS_FALLBACK, "fallback"


def make_setup(workload: str, size: int | None = None):
    """The workload's set-up; ``size`` (profiling captures only) shrinks the Taylor-Green box to
    size x size x 256 cells (rows stay one 256-cell tile, as at full size, so the same kernel
    runs) or the channel to 2 size x size."""
    from boltzmann_b200 import workloads

    if workload in ("cylinder_channel", "closure"):
        # closure: the reference's way to that accuracy is the plain fine channel itself
        if size:
            return workloads.cylinder_channel(2 * size, size, radius=size / 32)
        return workloads.cylinder_channel()
    if workload == "kelvin_helmholtz":
        return workloads.kelvin_helmholtz()
    if workload == "taylor_green_3d":
        return workloads.taylor_green_3d(size, nz=256) if size else workloads.taylor_green_3d()
    raise SystemExit(f"unknown workload {workload}")


def algorithmic_bytes_per_cell(setup, storage: str, tracer_storage: str | None = None) -> float:
    """Population bytes read + written per cell update (+ the coupled tracer value, read and
    written every step). Flags and the end-of-call rho/vel writes are not counted."""
    q = 9 if len(setup.counts) == 2 else 27
    qt = 5 if len(setup.counts) == 2 else 7
    pop = {"f32": 4, "f16": 2, "bf16": 2, "f64": 8}[storage]
    real = 8 if storage == "f64" else 4
    tpop = {"f16": 2, "bf16": 2}.get(tracer_storage or "", real)
    b = 2 * q * pop + len(setup.tracers) * 2 * qt * tpop
    if setup.couplings:
        b += 2 * real
    return float(b)


def profiled_traffic(kernel_tag: str, group: str) -> tuple[float | None, str]:
    """DRAM bytes per cell update from the committed ncu summary of this kernel, and where the
    figure comes from. The summary records the digest of the kernel sources it was captured
    from; a figure whose digest differs from the sources being run is not used."""
    from boltzmann_b200 import provenance

    current = provenance.digest(group)
    for p in sorted((ROOT / "profiles").glob(f"*{kernel_tag}*.md")):
        text = p.read_text()
        m = re.search(r"dram_bytes_per_cell_update:\s*([0-9.]+)", text)
        if not m:
            continue
        d = re.search(r"kernel_sources:\s*([0-9a-f]{16})", text)
        if d is None or d.group(1) != current:
            return None, (f"profiles/{p.name} was captured from other kernel sources "
                          f"({d.group(1) if d else 'no digest'}, running {current}); not used")
        return float(m.group(1)), f"ncu dram__bytes_read+write per launch, profiles/{p.name}"
    return None, "no ncu summary for this kernel"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = (
        "timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int) -> None:
        self.device = device
        self.proc = None
        self.path = None
        self.window: tuple[float, float] | None = None

    def mark(self, t0: float, t1: float) -> None:
        """The timed region's wall-clock window (time.time()); samples inside it are preferred."""
        self.window = (t0, t1)

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL,
            )
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        if self.path is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                t = time.mktime(time.strptime(parts[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                t += float("0." + parts[0].split(".")[1]) if "." in parts[0] else 0.0
                rows.append((t, float(parts[2]), float(parts[3]),
                             {n for n, v in zip(names, parts[6:10]) if v.lower() == "active"}))
            except (ValueError, IndexError):
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        where = "all samples (sampler ran around the timed region)"
        if self.window is not None:
            t0, t1 = self.window
            inside = [r for r in rows if t0 - 0.025 <= r[0] <= t1 + 0.025]
            if inside:
                rows, where = inside, "samples inside the timed region (20 ms polling)"
            else:  # a region shorter than the polling interval: the samples nearest to it
                mid = 0.5 * (t0 + t1)
                rows = sorted(rows, key=lambda r: abs(r[0] - mid))[:3]
                where = "the 3 samples nearest the timed region (shorter than the polling)"
        return {
            "sm_mhz": statistics.median(r[1] for r in rows),
            "sm_max_mhz": max(r[2] for r in rows),
            "reasons": sorted(set().union(*(r[3] for r in rows))),
            "samples": len(rows),
            "which": where,
        }


def omega_for(kind: str, tau: float, tau_neg: float | None = None):
    from boltzmann_b200.core import bgk, trt

    return bgk(tau) if kind == "bgk" else trt(tau, tau_neg)


def build_sim(setup, storage: str, tracer_storage: str | None = None):
    from boltzmann_b200 import workloads
    from boltzmann_b200.core import Simulation

    sim = Simulation("gpu", setup.counts, omega_for(setup.collision, setup.tau, setup.tau_neg),
                     storage=storage, tracer_storage=tracer_storage)
    workloads.apply(sim, setup, omega_for)
    return sim


def cpu_reference_rate(setup, budget_s: float, max_pairs: int | None = None) -> dict:
    """MLUPS of the reference kernels compiled as C++ (oracle/_ref), all host threads."""
    from boltzmann_b200 import workloads
    from oracle import build as oracle_build
    from oracle.oracle import Omega, OracleSimulation, default_threads, reference_available

    oracle_build.build_ref()
    kind = "reference" if reference_available() else "port"
    threads = default_threads()

    def om(k, tau, tau_neg=None):
        return Omega.bgk(tau) if k == "bgk" else Omega.trt(tau, tau_neg)

    sim = OracleSimulation(setup.counts, om(setup.collision, setup.tau, setup.tau_neg),
                           backend=kind, nthreads=threads)

    def tracer_handle(s, name, o):
        return name, s.add_tracer(name, o).val

    workloads.apply(sim, setup, om, tracer_handle)
    t0 = time.perf_counter()
    sim.iterate(2)  # first pair: equilibrate + one AA pair (untimed warm-up)
    first = time.perf_counter() - t0
    pairs = max(1, int(budget_s / max(first, 1e-3)))
    if max_pairs is not None:
        pairs = min(pairs, max_pairs)
    t0 = time.perf_counter()
    sim.iterate(2 * pairs)
    dt = time.perf_counter() - t0
    mlups = setup.cells * 2 * pairs / dt / 1e6
    return {
        "value": mlups,
        "unit": "MLUPS",
        "cores": threads,
        "kind": kind,
        "sample": f"{setup.name} {'x'.join(map(str, setup.counts))}, {2 * pairs} LBM steps "
        f"(full domain) after one untimed step pair; {threads} OpenMP threads",
        "pairs": pairs,
        "seconds": dt,
    }


def dist_env() -> tuple[int, int, int]:
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def run_reference(args) -> None:
    rank, world, _ = dist_env()
    if rank != 0:
        return
    setup = make_setup(args.workload, args.size)
    # Bounded: the whole arm stays within a few minutes.
    base = cpu_reference_rate(setup, budget_s=min(60.0, 2.0 * max(args.steps, 1)),
                              max_pairs=args.steps)
    line = {
        "impl": "reference",
        "metric": "MLUPS",
        "value": base["value"],
        "unit": "MLUPS",
        "n_gpus": args.gpus,
        "steps": base["pairs"],
        "warmup": 1,
        "ms_per_step": 1e3 * base["seconds"] / base["pairs"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config_block(setup, "f32", world),
        "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": base["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


WORKLOAD_TITLES = {
    "taylor_green_3d": "D3Q27 BGK Taylor-Green vortex, u0 0.05, Re 1600",
    "cylinder_channel": "D2Q9 TRT channel with cylinder + D2Q5 tracer + Boussinesq",
    "kelvin_helmholtz": "D2Q9 BGK Kelvin-Helmholtz shear layer",
}


def config_block(setup, storage: str, world: int) -> dict:
    from boltzmann_b200 import provenance

    return {
        "workload": f"{setup.name} {'x'.join(map(str, setup.counts))} "
        f"({WORKLOAD_TITLES.get(setup.name, setup.name)})",
        "lattice": "D2Q9" if len(setup.counts) == 2 else "D3Q27",
        "collision": setup.collision,
        "storage": storage,
        "cells": setup.cells,
        "lbm_steps_per_bench_step": 2,
        "l2": "inputs larger than L2 (populations > 126 MB); no flush",
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "kernel_sources": provenance.digest("stencil"),
    }


def velocity_l2_vs_f64(setup, vel, lbm_steps: int, tracer=None) -> dict:
    """Relative velocity L2 error ||u - u64|| / ||u64|| of a run's final field against an FP64 run
    of the same set-up on the GPU for the same number of steps (outside any timed region); with a
    tracer, its value's error as well."""
    sim = build_sim(setup, "f64")
    sim.iterate(lbm_steps)
    _, vel64 = sim._fluid_f64()
    c64 = None
    if tracer is not None:
        c64 = np.array(sim.get_tracer(setup.tracers[0][0]).val, np.float64)
    del sim
    rel = lambda a, b: float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel())
                             / np.linalg.norm(b.ravel()))
    out = {"value": rel(vel, vel64), "lbm_steps": lbm_steps, "field": "velocity",
           "norm": "relative L2 over all cells", "against": "FP64 run on the GPU (same set-up)"}
    if tracer is not None:
        out["tracer"] = rel(tracer, c64)
    return out


def run_ours(args) -> None:
    import torch

    from boltzmann_b200.replicas import Group

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = Group()  # replicas: no data-path collective; barrier + max of device times only
    barrier, max_over_ranks = group.barrier, group.max

    setup = make_setup(args.workload, args.size)
    K, W = args.steps, max(args.warmup, 3)

    # Device-timed run: inputs resident in HBM, only the AA kernels in the timed region.
    sim = build_sim(setup, args.storage, args.tracer_storage)
    sim.iterate(2 * W)  # upload, equilibrate, warm-up steps
    # One untimed call of the timed length: the library captures the CUDA graphs a call of that
    # many steps replays once per simulation state, and that one-time capture stays out of the
    # timed region.
    sim._iterate_device(2 * K)
    stream = torch.cuda.ExternalStream(sim._stream())
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    sim._synchronize()
    before = sim._launch_counts()
    with ClockSampler(local) as clocks:
        t_wall0 = time.time()
        start.record(stream)
        sim._iterate_device(2 * K)
        stop.record(stream)
        stop.synchronize()
        clocks.mark(t_wall0, time.time())
    after = sim._launch_counts()
    barrier()
    torch.cuda.synchronize()
    elapsed_ms = max_over_ranks(start.elapsed_time(stop))
    sim.iterate(2)  # read back; checks the state is still finite
    finite = bool(np.isfinite(sim.fluid.rho).all())
    final_vel = np.array(sim.fluid.vel, copy=True)
    final_c = (np.array(sim.get_tracer(setup.tracers[0][0]).val, copy=True)
               if setup.tracers else None)
    total_steps = sim.iteration
    del sim
    # The kernels the library launched in the timed region, from its own counters.
    direct, staged = after[0] - before[0], after[1] - before[1]
    launches = direct + staged
    kernel = ("aa_tma_kernel" if staged == launches else
              "aa_step_kernel" if direct == launches else
              f"aa_tma_kernel x{staged} + aa_step_kernel x{direct}")

    l2 = None
    if args.storage != "f64" and not args.no_l2:
        l2 = velocity_l2_vs_f64(setup, final_vel, total_steps, final_c)

    lbm_steps = 2 * K
    value = world * setup.cells * lbm_steps / (elapsed_ms * 1e-3) / 1e6
    launch_ms = elapsed_ms / lbm_steps
    bpc = algorithmic_bytes_per_cell(setup, args.storage, args.tracer_storage)
    peaks, peak_kind = measured_peaks()
    achieved = bpc * setup.cells / (launch_ms * 1e-3) / 1e9
    tag = {"cylinder_channel": "d2q9_trt_tracer", "kelvin_helmholtz": "d2q9_bgk",
           "taylor_green_3d": "d3q27_bgk"}[args.workload]
    if args.tracer_storage in ("f16", "bf16") and setup.tracers:
        tag += "16"
    tag += f"_{args.storage}"
    traffic_pc, traffic_src = profiled_traffic(f"{kernel}_{tag}", "stencil")

    # End to end through the public API with host buffers: a fresh Simulation from host arrays;
    # one iterate(2K) call uploads flags/rho/vel/C, equilibrates, steps and reads rho/vel/C back.
    n = setup.cells
    d = len(setup.counts)
    nt = len(setup.tracers)
    h2d = n * (1 + d) * 4 + n * 4 + nt * n * 4  # flags (sent as i32), rho, vel, tracer C
    d2h = n * (1 + d) * 4 + nt * n * 4
    e2e_value, e2e_runs = None, []
    if not args.no_e2e:
        # Three fresh simulations, each timed over its one iterate call; the median is reported.
        for _ in range(3):
            sim2 = build_sim(setup, args.storage, args.tracer_storage)
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            sim2.iterate(lbm_steps)
            e2e_s = max_over_ranks(time.perf_counter() - t0)
            e2e_runs.append(world * n * lbm_steps / e2e_s / 1e6)
            del sim2
        e2e_value = statistics.median(e2e_runs)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(setup, budget_s=args.cpu_seconds)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": "MLUPS",
            "value": value,
            "unit": "MLUPS",
            "n_gpus": world,
            "steps": K,
            "warmup": W,
            "ms_per_step": elapsed_ms / K,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"f32": "f32", "f16": "f16-offset storage, f32 compute",
                      "bf16": "bf16-offset storage, f32 compute", "f64": "f64"}[args.storage],
            "data": "synthetic",
            "config": dict(config_block(setup, args.storage, world),
                           tracer_storage=args.tracer_storage or
                           ("f64" if args.storage == "f64" else "f32")),
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": peaks["hbm_gbs"],
                "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"],
                "traffic": None if traffic_pc is None else traffic_pc * setup.cells,
                "traffic_source": traffic_src,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_cell_update": bpc,
                "kernel": f"{kernel} ({tag})",
                "frac_of_nominal_8tbs": achieved / 8000.0,
            },
            "cpu_baseline": cpu,
            "e2e": None if e2e_value is None else {
                "value": e2e_value,
                "unit": "MLUPS",
                "h2d_bytes_per_step": h2d / K,
                "d2h_bytes_per_step": d2h / K,
                "how": f"fresh Simulation from host arrays, one iterate({lbm_steps}) call "
                "(upload + equilibrate + steps + read-back), host wall clock; median of 3 runs",
                "runs": e2e_runs,
            },
            "gpu_launches": launches,
            "launches_by_kernel": {"aa_tma_kernel": staged, "aa_step_kernel": direct},
            "clocks": clocks.summary(),
            "finite": finite,
            "l2_vs_f64": l2,
        }
        print(json.dumps(line), flush=True)
    group.close()


def cpu_ensemble_rate(setup, budget_s: float) -> dict:
    """Reference kernels (oracle/_ref) on the host: the first domains of the ensemble, one after
    another, each for a few steps (the reference has no batched mode)."""
    from oracle import build as oracle_build
    from oracle.oracle import Omega, OracleSimulation, default_threads, reference_available

    oracle_build.build_ref()
    kind = "reference" if reference_available() else "port"
    threads = default_threads()
    cells = steps_done = 0
    t_total = 0.0
    for i, (counts, tau) in enumerate(zip(setup.counts, setup.tau)):
        sl = setup.domain_slices()[i]
        sim = OracleSimulation(list(counts), Omega.bgk(tau), backend=kind, nthreads=threads)
        sim.flags[...] = setup.flags[sl].reshape(counts)
        sim.vel[...] = setup.vel[sl].reshape(tuple(counts) + (2,))
        sim.iterate(2)
        t0 = time.perf_counter()
        sim.iterate(10)
        t_total += time.perf_counter() - t0
        cells += counts[0] * counts[1] * 10
        steps_done += 1
        if t_total > budget_s:
            break
    return {
        "value": cells / t_total / 1e6,
        "unit": "MLUPS",
        "cores": threads,
        "kind": kind,
        "sample": f"first {steps_done} of {len(setup.counts)} cavities, 10 LBM steps each, one "
        f"domain at a time; {threads} OpenMP threads",
    }


def run_ensemble(args) -> None:
    """The cavity ensemble: 512 lid-driven cavities advanced in one persistent launch per step,
    replayed from a CUDA graph, autotuned tile shape; per-domain launches timed for comparison."""
    import torch

    from boltzmann_b200 import autotune, workloads
    from boltzmann_b200.ensemble import Ensemble

    from boltzmann_b200.replicas import Group, shard_by_cells

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    group = Group()
    full = workloads.lid_driven_cavities(count=args.size or 512)
    # The domains are independent: under torchrun each rank advances its own share (by cells).
    setup = full if world == 1 else full.subset(shard_by_cells(full.counts, world)[rank])
    K, W = args.steps, max(args.warmup, 3)

    def fresh():
        ens = Ensemble(setup.counts, tau=setup.tau, storage=args.storage)
        ens.flags[...] = setup.flags
        ens.rho[...] = setup.rho
        ens.vel[...] = setup.vel
        return ens

    ens = fresh()
    ens.iterate(2 * W, mode="persistent")
    if args.shape:
        tile, blocks = (int(v) for v in args.shape.split(","))
        ens.set_shape(tile, blocks)
        tuned = {"tile": tile, "blocks_per_sm": blocks, "cached": False, "fixed": True}
    else:
        tuned = autotune.tune(ens, args.storage, use_cache=True, pairs=2)
    stream = torch.cuda.ExternalStream(ens.stream())

    def timed(mode: str, pairs: int) -> float:
        # Warm-up with the timed pair count: graph mode captures its graphs (chunks of 50 pairs
        # and the remainder) on first use, and that capture must not fall in the timed region.
        ens.iterate(2 * pairs, mode=mode, read_back=False)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ens.synchronize()
        group.barrier()
        start.record(stream)
        ens.iterate(2 * pairs, mode=mode, read_back=False)
        stop.record(stream)
        stop.synchronize()
        group.barrier()
        return group.max(start.elapsed_time(stop))

    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        graph_ms = timed("graph", K)
    persistent_ms = timed("persistent", K)
    pd_pairs = max(2, min(K, 20))
    per_domain_ms = timed("per_domain", pd_pairs)
    ens.iterate(2, read_back=True)
    finite_domains = int(group.sum(sum(
        bool(np.isfinite(ens.rho[sl]).all()) for sl in setup.domain_slices()
    )))
    del ens

    e2 = fresh()
    torch.cuda.synchronize()
    group.barrier()
    t0 = time.perf_counter()
    e2.iterate(2 * K, mode="graph")
    e2e_s = group.max(time.perf_counter() - t0)
    del e2

    n = full.cells
    value = n * 2 * K / (graph_ms * 1e-3) / 1e6
    bpc = {"f32": 72.0, "f16": 36.0, "bf16": 36.0}[args.storage]
    peaks, peak_kind = measured_peaks()
    achieved = bpc * n * 2 * K / (graph_ms * 1e-3) / 1e9 / world  # per GPU
    ens_kernel = "ensemble_rows_kernel" if tuned["tile"] == 0 else "ensemble_step_kernel"
    # DRAM bytes per cell update (ncu) of the kernel the tuned shape runs
    ens_traffic, ens_traffic_src = profiled_traffic(ens_kernel, "ensemble")
    cpu = None if (args.no_cpu_baseline or world > 1) else cpu_ensemble_rate(setup, args.cpu_seconds)
    line = {
        "metric": "MLUPS",
        "value": value,
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": graph_ms / K,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": args.storage,
        "data": "synthetic",
        "config": {
            "workload": f"lid_driven_cavities x{len(full.counts)} (sides 64..512, Re 100..5000)",
            "ensemble_cells": setup.cells,
            "parallelism": "single GPU" if world == 1 else
            f"{world} ranks, domains sharded by cell count (no collective)",
            "lattice": "D2Q9",
            "collision": "bgk",
            "storage": args.storage,
            "cells": n,
            "lbm_steps_per_bench_step": 2,
            "mode": "one persistent launch per step, replayed from a CUDA graph",
            "kernel_sources": __import__("boltzmann_b200.provenance").provenance.digest("ensemble"),
            "tile_cells": tuned["tile"],
            "blocks_per_sm": tuned["blocks_per_sm"],
            "autotune": "fixed by --shape" if tuned.get("fixed") else
            ("cached" if tuned.get("cached") else "searched"),
            "autotune_ms_per_pair": tuned.get("timings_ms_per_pair"),
            "l2": "inputs larger than L2; no flush",
        },
        "roofline": {
            "bound": "hbm",
            "achieved": achieved,
            "peak": peaks["hbm_gbs"],
            "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"],
            "traffic": None if ens_traffic is None else ens_traffic * setup.cells,  # a launch
            "traffic_source": ens_traffic_src,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "algorithmic_bytes_per_cell_update": bpc,
            "kernel": ens_kernel,
        },
        "comparison": {
            "persistent_no_graph_mlups": n * 2 * K / (persistent_ms * 1e-3) / 1e6,
            "per_domain_launches_mlups": n * 2 * pd_pairs / (per_domain_ms * 1e-3) / 1e6,
            "speedup_vs_per_domain": (n * 2 * K / graph_ms) / (n * 2 * pd_pairs / per_domain_ms),
            "per_domain_launches_per_step": len(setup.counts),  # on each rank
        },
        "cpu_baseline": cpu,
        "e2e": {
            "value": n * 2 * K / e2e_s / 1e6,
            "unit": "MLUPS",
            "h2d_bytes_per_step": n * (4 + 4 + 8) / K,
            "d2h_bytes_per_step": n * (4 + 8) / K,
            "how": "fresh ensemble from host arrays, one iterate(2K) call in graph mode",
        },
        "gpu_launches": 2 * K,
        "clocks": clocks.summary(),
        "finite_domains": finite_domains,
        "note": "cavities with side < Re/24 violate the BGK stability bound "
        "(python/boltzmann/core.py:106) and diverge; throughput is unaffected",
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    group.close()


def run_closure(args) -> None:
    """The learned closure on the coarse 1024x512 analogue of the 4096x2048 cylinder channel:
    data from seeded fine runs, training by the project's kernels, calibration on a training
    seed, a posteriori judgement on a held-out seed. The value is the GPU-time ratio of the plain
    fine run to the coarse+closure run over the same physical time, quoted at the closure's
    accepted error (its mean relative velocity L2 error against the filtered fine run)."""
    import torch

    from boltzmann_b200 import closure as cl

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    cfg = cl.Config()
    t0 = time.perf_counter()
    data = cl.generate(cfg)
    net, rep = cl.train(cfg, data)
    S = data.rho.shape[0]
    del data
    calref = cl.Reference(cfg, cfg.calib_seed)
    cal = cl.calibrate(cfg, net, calref)
    ref = cl.Reference(cfg, cfg.test_seed)
    with ClockSampler(local) as clocks:
        verdict = cl.judge(cfg, net, ref)
    summary = verdict.summary()
    ablation = cl.ablation(cfg, net, calref, ref)  # the network field against uniform ones
    t1 = time.perf_counter()
    kind, _ = cl.run_closed_or_fine(cfg, verdict, net, ref)
    e2e_s = time.perf_counter() - t1
    pipeline_s = time.perf_counter() - t0

    nx, ny = cfg.coarse
    # One closure application alone: the fused inference kernel on the coarse state.
    setup_c = cl.coarse_setup(cfg)
    flags_c = torch.tensor(setup_c.flags, device="cuda")
    omega_c = torch.empty(nx * ny, device="cuda")
    stream0 = torch.cuda.current_stream().cuda_stream
    for _ in range(5):
        cl.relaxation(net, ref.rho0, ref.vel0, flags_c, nx, ny, setup_c.tau, omega_c, stream0)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(50):
        cl.relaxation(net, ref.rho0, ref.vel0, flags_c, nx, ny, setup_c.tau, omega_c, stream0)
    ev1.record()
    ev1.synchronize()
    fused_s = ev0.elapsed_time(ev1) / 1e3 / 50

    # Tensor-core roofline of the network's forward pass on a batch of coarse states.
    B = 8
    bufs = cl.Buffers(nx, ny, B, train=False)
    bufs.x.zero_()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(max(args.warmup, 3)):
        cl.forward(net, bufs, stream)
    reps = 20
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(reps):
        cl.forward(net, bufs, stream)
    ev1.record()
    ev1.synchronize()
    fwd_s = ev0.elapsed_time(ev1) / 1e3 / reps
    flops = 21_312.0 * nx * ny * B  # 2 x (36 x 32 + 288 x 32 + 288) per cell
    peaks, peak_kind = measured_peaks()
    peak_tf = peaks.get("bf16_tflops", 1590.0)
    achieved_tf = flops / fwd_s / 1e12

    coarse_steps = cfg.horizons[-1]
    line = {
        "metric": "plain fine GPU time / coarse+closure GPU time, same physical time, at the "
        "closure's accepted error",
        "value": summary["time_ratio_fine_over_closure"],
        "unit": "x",
        "n_gpus": world,
        "steps": coarse_steps,
        "warmup": max(args.warmup, 3),
        "ms_per_step": summary["closure_seconds"] * 1e3 / coarse_steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16 network (fp32 accumulate), f32 stencil",
        "data": "synthetic",
        "config": {
            "workload": f"closure: cylinder channel {cfg.coarse[0]}x{cfg.coarse[1]} (r "
            f"{cfg.radius / cfg.factor:g}, Re {cfg.re:g}) vs {cfg.fine[0]}x{cfg.fine[1]}",
            "network": "3x3 conv 4->32->32->1, GELU, BF16 weights, FP32 accumulation",
            "target": "sqrt(k_sgs) of 4x4 box-filtered fine runs",
            "every": cfg.every,
            "train_seeds": list(cfg.train_seeds),
            "test_seed": cfg.test_seed,
            "snapshots": S,
            "fine_steps_judged": verdict.fine_steps,
            "kernel_sources": __import__("boltzmann_b200.provenance").provenance.digest("closure"),
            "l2": "stencil inputs larger than L2 at the fine size; no flush",
        },
        "closure": summary,
        "calibration": cal,
        "ablation_uniform_correction": ablation,
        "fused_relaxation": {
            "us_per_application": fused_s * 1e6,
            "tflops": 21_312.0 * nx * ny / fused_s / 1e12,
            "kernel": "closure_fused_kernel (features + 3 layers + tau mapping, 14x64 tiles)",
        },
        "training": {"iters": rep.iters, "device_seconds": rep.seconds,
                     "loss_first": rep.losses[0][1], "loss_last": rep.losses[-1][1]},
        "roofline": {
            "bound": "tensor",
            "achieved": achieved_tf,
            "peak": peak_tf,
            "unit": "TFLOP/s",
            "frac": achieved_tf / peak_tf,
            "traffic": None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json bf16_tflops)",
            "kernel": "closure forward (conv1 + conv32 mma.sync + conv3), batch 8 x 1024x512",
            "flops_per_cell": 21_312,
            "forward_ms": fwd_s * 1e3,
        },
        "cpu_baseline": None,
        "e2e": {
            "value": summary["fine_seconds"] / e2e_s,
            "unit": "x",
            "h2d_bytes_per_step": nx * ny * 16 / coarse_steps,
            "d2h_bytes_per_step": nx * ny * 12 / coarse_steps,
            "how": f"run_closed_or_fine ({kind}) from host arrays, host wall clock, against the "
            "fine run's device time",
        },
        "gpu_launches": coarse_steps + 5 * (coarse_steps // cfg.every),
        "clocks": clocks.summary(),
        "pipeline_seconds": pipeline_s,
    }
    if not args.no_cpu_baseline:
        cpu = cpu_reference_rate(cl.fine_setup(cfg, cfg.test_seed), args.cpu_seconds)
        cpu["seconds_for_judged_fine_steps"] = (
            cfg.fine[0] * cfg.fine[1] * verdict.fine_steps / (cpu["value"] * 1e6))
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_closure_forward(args) -> None:
    """Kernel-level line for the closure network: K forward passes over a batch of 8 coarse
    1024x512 states (random weights and inputs), device-timed, against the BF16 tensor peak."""
    import torch

    from boltzmann_b200 import closure as cl

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    nx, ny, B = 1024, 512, 8
    rng = np.random.default_rng(0)
    params = rng.uniform(-0.06, 0.06, cl.NPARAMS).astype(np.float32)
    net = cl.Net(params, np.array([0, 0, 0, 0, 1, 1, 1, 1], np.float32))
    bufs = cl.Buffers(nx, ny, B, train=False)
    x = torch.tensor(rng.normal(size=nx * ny * B * 4).astype(np.float32), device="cuda")
    bufs.x.copy_(x.to(torch.bfloat16).view(torch.int16))
    stream = torch.cuda.current_stream().cuda_stream
    K, W = args.steps, max(args.warmup, 3)
    for _ in range(W):
        cl.forward(net, bufs, stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e0.record()
        for _ in range(K):
            cl.forward(net, bufs, stream)
        e1.record()
        e1.synchronize()
    ms = e0.elapsed_time(e1) / K
    flops = 21_312.0 * nx * ny * B
    peaks, peak_kind = measured_peaks()
    peak = peaks.get("bf16_tflops", 1590.0)
    achieved = flops / (ms * 1e-3) / 1e12

    # One training step on the same batch: forward keeping the activations, loss, backward.
    tb = cl.Buffers(nx, ny, B, train=True)
    tb.x.copy_(bufs.x)
    flags0 = torch.zeros((nx, ny), dtype=torch.int32, device="cuda")
    target = torch.tensor(rng.normal(size=nx * ny * B).astype(np.float32), device="cuda")
    for _ in range(W):
        cl.forward(net, tb, stream)
        cl.loss_and_grad(net, tb, target, flags0, stream)
    e0.record()
    for _ in range(K):
        cl.forward(net, tb, stream)
        cl.loss_and_grad(net, tb, target, flags0, stream)
    e1.record()
    e1.synchronize()
    train_ms = e0.elapsed_time(e1) / K
    del tb

    # The inference kernel: features + network + relaxation rates of one 1024x512 state, fused.
    rho = torch.tensor((1 + 0.01 * rng.normal(size=(nx, ny))).astype(np.float32), device="cuda")
    vel = torch.tensor((0.05 * rng.normal(size=(nx, ny, 2))).astype(np.float32), device="cuda")
    flags = torch.zeros((nx, ny), dtype=torch.int32, device="cuda")
    omega = torch.empty(nx * ny, device="cuda")
    for _ in range(W):
        cl.relaxation(net, rho, vel, flags, nx, ny, 0.51, omega, stream)
    e0.record()
    for _ in range(K):
        cl.relaxation(net, rho, vel, flags, nx, ny, 0.51, omega, stream)
    e1.record()
    e1.synchronize()
    fused_ms = e0.elapsed_time(e1) / K
    fused_tf = 21_312.0 * nx * ny / (fused_ms * 1e-3) / 1e12
    line = {
        "metric": "closure forward TFLOP/s",
        "value": achieved * world,
        "unit": "TFLOP/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16 (fp32 accumulate)",
        "data": "synthetic",
        "config": {"workload": "closure network forward, batch 8 x 1024x512, 3x3 conv "
                               "4->32->32->1", "flops_per_cell": 21_312,
                   "l2": "activations 2 x 268 MB per pass exceed L2; no flush",
                   "kernel_sources": __import__("boltzmann_b200.provenance").provenance.digest(
                       "closure")},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json bf16_tflops)",
                     "kernel": "conv1_fwd + conv32_tc_kernel (tcgen05, TMEM) + conv3_fwd"},
        "fused_relaxation": {"ms": fused_ms, "tflops": fused_tf, "frac": fused_tf / peak,
                             "cells": nx * ny,
                             "kernel": "closure_fused_kernel (features + 3 layers + tau)"},
        "training_step": {"ms": train_ms, "flops": 3 * flops,
                          "tflops": 3 * flops / (train_ms * 1e-3) / 1e12,
                          "what": "forward with activations kept + loss + backward (batch 8)"},
        "cpu_baseline": None,
        "e2e": None,
        "gpu_launches": 4 * K,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawTextHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="taylor_green_3d",
                    choices=["cylinder_channel", "kelvin_helmholtz", "taylor_green_3d",
                             "cavity_ensemble", "closure", "closure_forward"])
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16", "f64"])
    ap.add_argument("--tracer-storage", default=None, choices=["f16", "bf16"],
                    help="store the fused tracer's populations in the fluid's 16-bit kind")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-l2", action="store_true",
                    help="skip the FP64 comparison run (profiling runs only)")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end run (profiling runs only)")
    ap.add_argument("--size", type=int, default=None,
                    help="smaller case for profiling captures: Taylor-Green size x size x 256, "
                    "channel 2 size x size, ensemble the first `size` cavities")
    ap.add_argument("--shape", default=None,
                    help="ensemble only: fixed launch shape 'tile,blocks_per_sm' instead of the "
                    "autotuner's (tile 0: the row-staged kernel)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "cavity_ensemble":
        run_ensemble(args)
    elif args.workload == "closure":
        run_closure(args)
    elif args.workload == "closure_forward":
        run_closure_forward(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
