#!/usr/bin/env python
"""GP iterations/s of the adaptive + neumann + course_eplace_v1 global placer on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]

Workload: the mid design -- 210k movable cells, 400 fixed macros, 1,200 boundary
terminals, 220k nets (~850k pins), rows sized for 70 % utilisation, target
density 0.9, 512 x 512 bins -- seeded synthetic data with the design law of the
benchmark, random initial placement from seed 2026.  A step is one adaptive
controller iteration (1-16 objective evaluations).  The early stop is off, so
exactly W + K iterations run.  The L2 cache (126 MB; the working set is ~100 MB)
is flushed by a 256 MiB device write between timed steps, outside the timing.

Output: one JSON line on rank 0.  `value` is device-timed iterations/s with the
design resident on the device; `e2e` is the same metric through the public API
with host buffers (GlobalPlacer.run: host setup, upload, the run with its early
stop, download).  `--impl reference` times the reference's own CPU path (and,
beside it, the reference CUDA backend rebuilt for sm_100a) on the same workload.
With N > 1 each rank runs an independent replica on its own GPU (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "GP iterations/s at 210k cells vs plain GPU form; p50/p99 solve latency @≤0.10 ovfl"
WORKLOAD = "mid_210k"
PEAKS_FILE = REPO / "MEASURED_PEAKS.json"
PROFILE_TRAFFIC = REPO / "profiles" / "traffic_mid_210k.md"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
# The kernel behind each timed family (families of one kernel are summed for the roofline).
KERNEL_OF_FAMILY = {"dct_forward": "tcGemmKernel", "dct_inverse": "tcGemmKernel",
                    "field_forward": "fieldKernel", "field_gradient": "fieldKernel", "field_inverse": "fieldKernel",
                    "wirelength": "wirelengthKernel", "scatter": "scatterKernel",
                    "metrics": "metricsSplitKernel", "gather": "gatherKernel", "reduce": "reduceKernel",
                    "vector": "velocityKernel", "dct_split": "splitSourceKernel", "rudy": "rudy kernels"}
# Iteration budget of the end-to-end runs (early stop on): large enough that the run stops on its
# own once the design overflow is <= 0.10 (the reference's default budget of 280 iterations ends
# this design at overflow 0.13).
E2E_BUDGET = 1000


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--seed", type=int, default=2026)
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--rudy", action="store_true",
                   help="routability term on (hinge L2, capacity 1.2 x the activation mean demand), as the "
                        "precision configuration runs it")
    p.add_argument("--form", choices=["plain", "batched", "serving", "detailed", "bookshelf"], default="plain",
                   help="plain: the one-design metric; batched: many small instances at once; "
                        "serving: an open-loop stream of jobs; detailed: window-reorder detailed placement "
                        "of the workload packed legally, against the reference CUDA backend; bookshelf: "
                        "reading the workload as BookShelf files (host only), against the reference reader")
    p.add_argument("--instances", type=int, default=256, help="batched form: instance count")
    p.add_argument("--jobs", type=int, default=240, help="serving form: job count")
    p.add_argument("--workers", type=int, default=64, help="batched / serving forms: worker threads (the most "
                                                                   "placements running at once)")
    return p.parse_args()


def load_peaks() -> tuple[dict, str]:
    if PEAKS_FILE.is_file():
        try:
            return json.loads(PEAKS_FILE.read_text()), "measured"
        except json.JSONDecodeError:
            pass
    return dict(FALLBACK_PEAKS), "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"mpgp_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def samples(self) -> int:
        try:
            return sum(1 for line in self.path.read_text().splitlines() if line.count(",") >= 8)
        except OSError:
            return 0

    def hold(self, load, minimum: int = 3, limit_s: float = 3.0) -> None:
        """Keeps the GPU busy with `load` until `minimum` samples exist (the timed steps are far
        shorter than nvidia-smi's sampling interval), at most `limit_s` seconds."""
        if self.proc is None:
            return
        deadline = time.perf_counter() + limit_s
        while self.samples() < minimum and time.perf_counter() < deadline:
            load()

    def summary(self) -> dict:
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        clocks, max_clock, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                clocks.append(float(parts[1]))
                max_clock = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(clocks) if clocks else None, "sm_max_mhz": max_clock,
                "reasons": sorted(reasons), "samples": len(clocks),
                "sampled": "nvidia-smi every 200 ms from the first timed step until a few samples exist "
                           "(the steps, then the 256 MiB flush write as load)"}


def algorithmic_units(design, particles: int, bins_x: int, bins_y: int) -> dict:
    """Per-launch algorithmic bytes (HBM-bound families) or FLOPs (DCT) of each kernel family.

    Bytes per unit are the compulsory bytes of each pass (each array counted once per pass): wirelength
    20 B/pin + 8 B/net + 8 B/particle; scatter 20 B/particle + 24 B/bin; metrics
    36 B/bin; gather + update 80 B/particle.  A DCT launch is one (forward) or
    two (inverse) M x N x K contractions at 2 flops per multiply-add (the transform's
    own work, not the three tensor-core products of the split); a banded field launch
    is the two forward contractions, and with a gradient the two inverse ones along y (an
    inverse launch only those two);
    the source split reads 4 B and writes two 2-byte planes per bin.
    """
    pins, nets, bins = design.pin_count, design.net_count, bins_x * bins_y
    m, n = bins_y, bins_x
    return {
        "wirelength": ("hbm", 20 * pins + 8 * nets + 8 * particles),
        "scatter": ("hbm", 20 * particles + 24 * bins),
        "metrics": ("hbm", 36 * bins),
        "gather": ("hbm", 80 * particles),
        "dct_forward": ("tensor", 2.0 * m * n * (n + m) / 2.0),
        "dct_inverse": ("tensor", 2 * 2.0 * m * n * (n + m) / 2.0),
        # The banded solve: Q = S Cx^T and rho_hat = Cy Q, then M1 and M2 (two m x n x m) with a gradient.
        "field_forward": ("tensor", 2.0 * m * n * (n + m)),
        "field_gradient": ("tensor", 2.0 * m * n * (n + m) + 2 * 2.0 * m * n * m),
        "field_inverse": ("tensor", 2 * 2.0 * m * n * m),
        "reduce": ("hbm", 8 * 64),
        "vector": ("hbm", 48 * particles),
        "dct_split": ("hbm", 4 * bins + 4 * bins),
        "rudy": ("hbm", 20 * pins + 12 * nets),
    }


def read_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if present."""
    if not PROFILE_TRAFFIC.is_file():
        return None
    for line in PROFILE_TRAFFIC.read_text().splitlines():
        m = re.match(rf"\|\s*{re.escape(kernel)}\s*\|\s*([0-9.eE+]+)\s*\|", line)
        if m:
            return float(m.group(1))
    return None


def flush_l2(buffer, stream_ptr):
    import torch

    with torch.cuda.stream(torch.cuda.ExternalStream(stream_ptr)):
        buffer.add_(1)


def reference_cpu_sample(design, bins: int, warmup: int, steps: int, variant: str = "cpu", device: int = 0):
    """Per-iteration time of the reference path: (T(warmup + steps) - T(warmup)) / steps,
    each T being the reference's own GlobalPlacementResult.elapsed_seconds."""
    from oracle.ref import ReferenceLibrary, default_options

    ref = ReferenceLibrary(variant)
    common = dict(bins_x=bins, bins_y=bins, target_density=0.9, feasible_refinement_iterations=10 ** 9,
                  compute_backend=0 if variant == "cpu" else 1, cuda_device=device)
    if variant != "cpu":
        # The first CUDA run pays for context creation; keep it out of both samples.
        ref.global_place(design, default_options(iterations=1, **common))
    _, _, short, _ = ref.global_place(design, default_options(iterations=max(1, warmup), **common))
    _, _, long, _ = ref.global_place(design, default_options(iterations=max(1, warmup) + steps, **common))
    seconds = max(long.elapsed_seconds - short.elapsed_seconds, 1e-9)
    return {"iterations": steps, "seconds": seconds, "value": steps / seconds,
            "setup_and_warmup_seconds": short.elapsed_seconds,
            "completed": long.completed_iterations, "hpwl_after": long.hpwl_after}


def rudy_options(args) -> dict:
    """The routability options of the precision configuration (none unless --rudy)."""
    if not getattr(args, "rudy", False):
        return {}
    return {"rudy_penalty_model": 1, "rudy_capacity_factor": 1.2}


def workload_text(args, design, bins: int) -> str:
    import myplacement_b200 as mp

    spec = mp.design.WORKLOADS[args.workload]
    macros, terminals = spec.get("macros", 0), spec.get("terminals", 0)
    text = (f"{args.workload}: {design.module_count - macros - terminals} cells, {macros} fixed macros, "
            f"{terminals} terminals, {design.net_count} nets, {design.pin_count} pins, {bins}x{bins} bins, "
            "target density 0.9")
    if getattr(args, "rudy", False):
        text += ", RUDY hinge L2 at capacity 1.2 x mean demand"
    return text


def make_workload(name: str, seed: int, placer=None):
    """The seeded synthetic design with its random initial placement (randomPlacement,
    InitialPlacer.cpp:102-121).  `placer` draws the placement; the reference arm passes
    the reference's own, so that it loads nothing of this engine."""
    import myplacement_b200 as mp

    design, bins = mp.workload(name)
    x, y = (placer or mp.random_placement)(design, seed)
    return design.copy_with_positions(x, y), bins


def bench_config(args, design, bins: int, world: int) -> dict:
    """The `config` object both arms print (the same workload, step and timing rules)."""
    return {"workload": workload_text(args, design, bins), "step": "one adaptive controller iteration",
            "early_stop": "off in the timed run (fixed iteration count)",
            "l2": "flushed between timed steps (256 MiB device write, outside the timing)",
            "parallelism": f"replicas x{world}", "seed": args.seed}


def native_libraries() -> list[str]:
    """The shared objects of this repository mapped into the process (from /proc/self/maps)."""
    found = set()
    try:
        for line in Path("/proc/self/maps").read_text().splitlines():
            path = line.split()[-1] if line.split() else ""
            if path.endswith(".so") and str(REPO) in path:
                found.add(str(Path(path).relative_to(REPO)))
    except OSError:
        pass
    return sorted(found)


def run_mine(args) -> None:
    import torch

    import myplacement_b200 as mp
    from myplacement_b200 import replicas

    rank, world, local = replicas.world()
    torch.cuda.set_device(local)
    replicas.init()
    design, bins = make_workload(args.workload, replicas.replica_seed(args.seed, rank))
    iterations = args.warmup + args.steps
    options = mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9, cuda_device=local,
                                 iterations=max(280, iterations), feasible_refinement_iterations=10 ** 9,
                                 **rudy_options(args))
    session = mp.Session(design, options)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    stream_ptr = session.stream
    # The last warm-up steps time every kernel family (shares, dominant family);
    # the timed steps time only the dominant family, since every event pair costs
    # host time inside the step.
    profiled_warmup = min(2, args.warmup)
    for i in range(args.warmup):
        if i == args.warmup - profiled_warmup:
            session.set_profiling(True)
        session.step(1)
    torch.cuda.synchronize()
    warm_stats = session.kernel_stats()
    session.reset_kernel_stats()
    # The dominant kernel: families that launch the same kernel are summed (the field
    # contractions' forward and inverse launches are one kernel, tcGemmKernel).
    groups = {}
    for name, (n, ms) in warm_stats.items():
        if n > 0:
            groups.setdefault(KERNEL_OF_FAMILY.get(name, name), []).append(name)
    dominant = max(groups, key=lambda g: sum(warm_stats[f][1] for f in groups[g])) if groups else "tcGemmKernel"
    families = groups.get(dominant, ["dct_forward", "dct_inverse"])
    session.set_profiling(families)
    launches_before = session.kernel_launches
    step_ms = []
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    ext = torch.cuda.ExternalStream(stream_ptr)
    replicas.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush_l2(flush, stream_ptr)
            start.record(ext)
            session.step(1)
            end.record(ext)
            end.synchronize()
            step_ms.append(start.elapsed_time(end))
        wall_timed = time.perf_counter() - wall0

        def load():
            flush_l2(flush, stream_ptr)
            torch.cuda.synchronize()

        # The clocks right after the timed steps, under the flush write's load, until
        # nvidia-smi has a few samples.
        clocks.hold(load)
    torch.cuda.synchronize()
    replicas.barrier()
    wall = wall_timed
    launches = session.kernel_launches - launches_before
    stats = session.kernel_stats()
    session.set_profiling(False)
    total_ms = float(sum(step_ms))
    max_ms = replicas.reduce_max(total_ms)
    total_steps = replicas.reduce_sum(args.steps)
    value = total_steps / (max_ms / 1e3)
    clock_info = clocks.summary()
    result = session.finish()
    session.close()
    del flush

    particles = int(mp.host_setup(design, options)["particle_count"]) if rank == 0 else 0
    roofline = roofline_hbm = None
    if rank == 0:
        peaks, peak_kind = load_peaks()
        units = algorithmic_units(design, particles, bins, bins)

        def rate(family_names, source):
            launches_f = sum(source[f][0] for f in family_names)
            seconds = sum(source[f][1] for f in family_names) / 1e3
            amount = sum(units[f][1] * source[f][0] for f in family_names)  # algorithmic bytes or FLOPs
            bound = units[family_names[0]][0]
            traffic = [read_traffic(f) for f in family_names]
            per_launch = (sum(t * source[f][0] for t, f in zip(traffic, family_names)) / launches_f
                          if launches_f and all(t is not None for t in traffic) else None)
            if bound == "hbm":
                achieved, peak, unit = amount / seconds / 1e9, peaks.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"]), "GB/s"
            else:
                achieved = amount / seconds / 1e12
                peak = peaks.get("bf16_tflops_sustained", FALLBACK_PEAKS["bf16_tflops_sustained"])
                unit = "TFLOP/s"
            return {"bound": bound, "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak,
                    "traffic": per_launch, "peak_source": peak_kind, "launches": launches_f,
                    "avg_launch_us": seconds / max(launches_f, 1) * 1e6,
                    "algorithmic_per_launch": amount / max(launches_f, 1)}

        roofline = {"kernel": dominant, "families": families, **rate(families, stats),
                    "timed": f"CUDA events around every {'/'.join(families)} launch of the timed steps",
                    "kernel_share_warmup": {k: round(v[1] / max(sum(s[1] for s in warm_stats.values()), 1e-12), 4)
                                            for k, v in warm_stats.items() if v[0] > 0},
                    "kernel_us_per_step_warmup": {k: round(v[1] * 1e3 / profiled_warmup, 1)
                                                  for k, v in warm_stats.items() if v[0] > 0}}
        # For context: the busiest HBM-bound kernel, from the profiled warm-up steps.
        hbm = [g for g in groups if units[groups[g][0]][0] == "hbm"]
        if hbm:
            top = max(hbm, key=lambda g: sum(warm_stats[f][1] for f in groups[g]))
            roofline_hbm = {"kernel": top, "families": groups[top], **rate(groups[top], warm_stats),
                            "timed": "CUDA events around every launch of the last two warm-up steps"}

    e2e = None
    if not args.no_e2e:
        e2e_options = mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9, cuda_device=local,
                                         iterations=E2E_BUDGET, **rudy_options(args))
        # Three whole runs through the public API; the median one is reported (a single
        # run of ~0.15 s is at the mercy of the shared host).
        runs = []
        for _ in range(3):
            replicas.barrier()
            t0 = time.perf_counter()
            s2 = mp.Session(design, e2e_options)
            while not s2.step(64)[1]:
                pass
            placed = s2.finish()
            t1 = time.perf_counter()
            h2d, d2h = s2.transfer_bytes()
            s2.close()
            runs.append((replicas.reduce_max(t1 - t0), placed, h2d, d2h))
        e2e_time, placed, h2d, d2h = sorted(runs, key=lambda r: r[0])[1]
        it = placed.completed_iterations
        e2e_iters = replicas.reduce_sum(it)
        e2e = {"value": e2e_iters / e2e_time, "unit": "iterations/s",
               "h2d_bytes_per_step": int(h2d / max(it, 1)), "d2h_bytes_per_step": int(d2h / max(it, 1)),
               "api": f"Session create/step/finish (= GlobalPlacer.run) on host arrays, {E2E_BUDGET}-iteration "
                      "budget with the early stop on (the run ends once overflow <= 0.10); median of three runs",
               "completed_iterations": it, "seconds": e2e_time, "seconds_of_runs": [r[0] for r in runs],
               "hpwl_after": placed.hpwl_after, "overflow_after": placed.overflow_after}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            sample = reference_cpu_sample(design, bins, warmup=1, steps=3)
            cpu = {"value": sample["value"], "unit": "iterations/s", "cores": 1, "kind": "reference",
                   "sample": f"reference CPU path (oracle/_ref/libref_cpu.so, single thread as in the reference) "
                             f"on this workload: iterations 2-4, (T(4) - T(1)) / 3 = {sample['seconds']:.2f} s"}
        except Exception as error:  # the oracle library is absent
            cpu = {"value": None, "unit": "iterations/s", "cores": 1, "kind": "reference",
                   "sample": f"unavailable: {error}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(args, design, bins, world),
            "details": {"particles": particles,
                        "arithmetic": "f32 kernels, int64 fixed-point density, f64 reductions and controller",
                        "wall_seconds_timed_region": wall},
            "roofline": roofline, "roofline_hbm": roofline_hbm, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clock_info,
            "quality": {"hpwl_after": result.hpwl_after, "overflow_after": result.overflow_after,
                        "iterations": result.completed_iterations},
            "native_libraries": native_libraries(),
        }
        if result.completed_iterations > 0 and result.evaluations > 0:
            # An iteration holds one or more objective evaluations (candidates,
            # backtracks, the accepted point's gradient).
            per_iteration = result.evaluations / result.completed_iterations
            line["evaluations"] = {"per_iteration": per_iteration, "per_s": value * per_iteration,
                                   "us_per_evaluation": 1e6 / (value * per_iteration),
                                   "counted_over": "the whole run (initial evaluations, warm-up and timed steps)"}
        print(json.dumps(line), flush=True)
    replicas.shutdown()


def reference_quality(design, bins: int, device: int) -> dict:
    """One whole run of the reference CUDA backend (rebuilt for sm_100a) with the reference's
    default options and the e2e run's iteration budget (early stop on): the quality the engine's
    e2e run is compared with."""
    from oracle.ref import ReferenceLibrary, default_options

    lib = ReferenceLibrary("cuda")
    options = default_options(bins_x=bins, bins_y=bins, target_density=0.9, compute_backend=1, cuda_device=device,
                              iterations=E2E_BUDGET)
    _, _, result, _ = lib.global_place(design, options)
    return {"hpwl_after": result.hpwl_after, "overflow_after": result.overflow_after,
            "completed_iterations": result.completed_iterations,
            "best_checkpoint_iteration": result.best_checkpoint_iteration,
            "seconds": result.elapsed_seconds,
            "backend_used": "cuda" if result.compute_backend_used == 1 else "cpu",
            "what": f"reference CUDA backend rebuilt for sm_100a, default options with the e2e run's "
                    f"{E2E_BUDGET}-iteration budget (early stop on), same design and initial placement"}


def run_reference(args) -> None:
    """The reference's own CPU path (oracle/_ref/libref_cpu.so, built from the reference sources) on the
    same workload; the inputs are generated without this engine's library (the reference's randomPlacement)."""
    from myplacement_b200 import replicas
    from oracle.ref import ReferenceLibrary

    rank, world, local = replicas.world()
    if rank != 0:
        return  # the reference CPU path runs on rank 0 only
    design, bins = make_workload(args.workload, args.seed, placer=ReferenceLibrary("cpu").random_placement)
    try:
        cpu = reference_cpu_sample(design, bins, warmup=args.warmup, steps=args.steps)
    except Exception as error:
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path failed: {error}"}))
        return
    cuda = None
    try:
        sample = reference_cpu_sample(design, bins, warmup=args.warmup, steps=args.steps, variant="cuda",
                                      device=local)
        cuda = {"value": sample["value"], "unit": "iterations/s",
                "what": "the reference CUDA backend (src/placement/cuda/CudaPlacementBackend.cu) rebuilt for "
                        "sm_100a, driven by the reference controller, same workload and step definition",
                "seconds": sample["seconds"], "iterations": sample["iterations"]}
    except Exception as error:
        cuda = {"value": None, "unavailable": str(error)}
    quality = None
    if not args.no_e2e:
        try:
            quality = reference_quality(design, bins, local)
        except Exception as error:
            quality = {"unavailable": str(error)}
    value = cpu["value"]
    line = {
        "metric": METRIC, "value": value, "unit": "iterations/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": bench_config(args, design, bins, world),
        "timing": "(T(W + K) - T(W)) / K from the reference's own elapsed_seconds",
        "cpu_baseline": {"value": value, "unit": "iterations/s", "cores": 1, "kind": "reference",
                         "sample": f"reference CPU path (single-threaded, as the reference runs it), iterations "
                                   f"{args.warmup + 1}-{args.warmup + args.steps}"},
        "e2e": {"value": value, "unit": "iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda_backend": cuda,
        "reference_quality": quality,
        "native_libraries": native_libraries(),
    }
    print(json.dumps(line), flush=True)


def batched_instances(count: int, seed: int):
    """Instances of the batched form: cells log-normal (median 4k) clipped to 1k-20k, the small
    design's structure, bins the power of two nearest sqrt(cells) (32..256), early stop on."""
    import numpy as np

    import myplacement_b200 as mp
    from myplacement_b200.design import small_instance

    rng = np.random.default_rng(seed)
    sigma = math.log(20_000 / 4_000) / 2.5
    cells = np.clip(np.round(np.exp(rng.normal(math.log(4_000), sigma, count))), 1_000, 20_000).astype(int)
    jobs = []
    for k, c in enumerate(cells):
        design, bins = small_instance(int(c), seed + k)
        bins = max(32, min(256, bins))
        x, y = mp.random_placement(design, seed + k)
        jobs.append((design.copy_with_positions(x, y),
                     mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9)))
    return jobs


def run_batched(args) -> None:
    """Aggregate iterations/s of many independent instances: one at a time (plain) against the server,
    batched (every round of the running instances' evaluations in one launch per kernel family) and,
    for comparison, concurrent (every instance launching its own kernels).  Each server mode runs
    three times; the line reports the median and the spread, and whether every instance's result is
    bit-identical to its plain run."""
    import numpy as np

    import myplacement_b200 as mp

    jobs = batched_instances(args.instances, args.seed)
    placer = mp.GlobalPlacer()
    placer.run(*jobs[0])  # context and module load outside the timing
    t0 = time.perf_counter()
    plain = [placer.run(d, o) for d, o in jobs]
    plain_seconds = time.perf_counter() - t0
    plain_rate = sum(r.completed_iterations for r in plain) / plain_seconds

    def server_runs(batched: bool, repeats: int):
        rates, last = [], None
        for _ in range(repeats):
            t0 = time.perf_counter()
            placed, job_stats, server_stats = mp.batch_place([d for d, _ in jobs], [o for _, o in jobs],
                                                             workers=args.workers, batched=batched)
            seconds = time.perf_counter() - t0
            rates.append(sum(r.completed_iterations for r in placed) / seconds)
            last = (placed, server_stats, seconds)
        return rates, last

    batched_rates, (placed, server_stats, batched_seconds) = server_runs(True, 3)
    concurrent_rates, _ = server_runs(False, 1)
    iterations = sum(r.completed_iterations for r in placed)
    same = all(np.array_equal(a.module_x, b.module_x) and np.array_equal(a.module_y, b.module_y) and
               a.hpwl_after == b.hpwl_after and a.completed_iterations == b.completed_iterations
               for a, b in zip(placed, plain))
    value = statistics.median(batched_rates)
    line = {
        "form": "batched", "metric": "aggregate GP iterations/s, independent instances on one GPU",
        "value": value, "unit": "iterations/s", "n_gpus": 1, "higher_is_better": True,
        "runs": batched_rates, "spread": [min(batched_rates), max(batched_rates)],
        "plain_one_at_a_time": plain_rate, "speedup_vs_plain": value / plain_rate,
        "concurrent_without_batching": concurrent_rates[0],
        "instances": len(jobs), "workers": args.workers, "iterations": iterations,
        "seconds": batched_seconds, "plain_seconds": plain_seconds,
        "results_identical_to_plain": bool(same),
        "overflow_le_0.10": sum(r.overflow_after <= 0.10 for r in placed),
        "hpwl_total": sum(r.hpwl_after for r in placed), "hpwl_total_plain": sum(r.hpwl_after for r in plain),
        "peak_running": server_stats["peak_running"], "batch_rounds": server_stats["batch_rounds"],
        "evaluations_per_round": server_stats["batch_evaluations"] / max(1, server_stats["batch_rounds"]),
        "round_busy_us": 1e6 * server_stats["batch_busy_seconds"] / max(1, server_stats["batch_rounds"]),
        "round_device_us": 1e6 * server_stats["batch_device_seconds"] / max(1, server_stats["batch_rounds"]),
        "round_us": 1e6 * batched_seconds / max(1, server_stats["batch_rounds"]),
        "host_cpus": os.cpu_count(),
        "gpu_launches": server_stats["batch_launches"],
        "data": "synthetic: cells log-normal median 4k in 1k-20k, small-design net law, bins 32^2-256^2, "
                "early stop on (280-iteration budget)",
    }
    print(json.dumps(line))


def run_serving(args) -> None:
    """Jobs of 2k-210k cells (log-uniform, mid-design structure scaled), each run to overflow <= 0.10
    (1000-iteration budget, early stop on): the plain capacity (one job at a time), the served
    capacity (all at once) and an open-loop Poisson stream at 70 % of the served capacity."""
    import numpy as np

    import myplacement_b200 as mp

    rng = np.random.default_rng(args.seed)
    pool = []
    for k, cells in enumerate(np.exp(rng.uniform(math.log(2_000), math.log(210_000), 24))):
        design, bins = mp.workload("mid_210k", seed=args.seed + k, scale=float(cells) / 210_000)
        pool.append((design, max(32, bins)))

    def job(i: int):
        design, bins = pool[i % len(pool)]
        x, y = mp.random_placement(design, args.seed + 1000 + i)
        return design.copy_with_positions(x, y), mp.default_options(bins_x=bins, bins_y=bins, target_density=0.9,
                                                                    iterations=1000)

    # Plain: the first three rounds of the pool, one job at a time.
    placer = mp.GlobalPlacer()
    placer.run(*job(0))
    first = [job(i) for i in range(3 * len(pool))]
    t0 = time.perf_counter()
    plain = [placer.run(d, o) for d, o in first]
    plain_capacity = len(first) / (time.perf_counter() - t0)
    plain_iterations = sum(r.completed_iterations for r in plain)

    jobs = [job(i) for i in range(args.jobs)]
    with mp.PlacementServer(device=0, workers=args.workers) as server:
        # Served capacity: the same jobs, all submitted at once.
        t0 = time.perf_counter()
        ids = [server.submit(d, o) for d, o in first]
        served = []
        for i in ids:
            server.wait(i)
            served.append(server.take(i, history=False)[0])
        capacity = len(first) / (time.perf_counter() - t0)
        same = all(a.hpwl_after == b.hpwl_after for a, b in zip(served, plain))
        rate = 0.7 * capacity
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(jobs)))
        t0 = time.perf_counter()
        submitted = []
        for (design, options), at in zip(jobs, arrivals):
            delay = at - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            submitted.append(server.submit(design, options))
        latencies, overflow_ok, iterations = [], 0, 0
        for i in submitted:
            server.wait(i)
            placed, stats = server.take(i, history=False)
            latencies.append(stats["latency_seconds"])
            overflow_ok += placed.overflow_after <= 0.10
            iterations += placed.completed_iterations
        seconds = time.perf_counter() - t0
        server_stats = server.stats()
    line = {
        "form": "serving", "metric": "jobs/s and p50/p99 latency, open-loop Poisson arrivals at 70% capacity",
        "value": len(jobs) / seconds, "unit": "jobs/s", "n_gpus": 1, "higher_is_better": True,
        "p50_latency_s": float(np.percentile(latencies, 50)), "p99_latency_s": float(np.percentile(latencies, 99)),
        "served_capacity_jobs_per_s": capacity, "plain_capacity_jobs_per_s": plain_capacity,
        "capacity_speedup_vs_plain": capacity / plain_capacity,
        "plain_iterations_per_s": plain_iterations * plain_capacity / len(first),
        "served_results_identical_to_plain": same,
        "arrival_rate_jobs_per_s": rate, "jobs": len(jobs), "workers": args.workers,
        "aggregate_iterations_per_s": iterations / seconds,
        "overflow_le_0.10": overflow_ok, "peak_running": server_stats["peak_running"],
        "data": "synthetic: 24 mid-design-structured designs, cells log-uniform 2k-210k, each job its own "
                "random initial placement; 1000-iteration budget, early stop on",
    }
    print(json.dumps(line))


def run_detailed(args) -> None:
    """Detailed placement (two passes of the four-cell window reorder) of the workload's cells packed
    legally in shuffled order: seconds for this engine and for the reference CUDA backend rebuilt for
    sm_100a (oracle/_ref/libref_cuda.so through DetailedPlacer::run) on the same device, and whether the
    two placements are bit-identical."""
    import numpy as np

    import myplacement_b200 as mp
    from myplacement_b200.design import packed_placement
    from oracle.ref import ReferenceLibrary

    design, _ = mp.workload(args.workload, seed=args.seed)
    placed = packed_placement(design, 7)
    options = mp.default_detailed_options(passes=2)
    runs = []
    for _ in range(3):
        out, result = mp.DetailedPlacer().run(placed, options)
        runs.append(result["elapsed_seconds"])
    reference = ReferenceLibrary("cuda")
    ref_runs = []
    for _ in range(2):
        x, y, orientation, theirs, used = reference.detailed_place(placed, options, 1)
        ref_runs.append(theirs["elapsed_seconds"])
    same = (np.array_equal(out.module_x.view(np.int64), x.view(np.int64)) and
            np.array_equal(out.module_y.view(np.int64), y.view(np.int64)) and
            np.array_equal(out.module_orientation, orientation) and
            all(result[k] == theirs[k] for k in ("evaluated_windows", "evaluated_permutations",
                                                 "accepted_operations", "hpwl_after")))
    line = {
        "form": "detailed", "metric": "detailed placement seconds (two window-reorder passes)",
        "value": statistics.median(runs), "unit": "s", "n_gpus": 1, "higher_is_better": False,
        "runs_s": runs, "reference_cuda_runs_s": ref_runs, "reference_backend_used": used,
        "speedup_vs_reference_cuda": statistics.median(ref_runs) / statistics.median(runs),
        "identical_to_reference_cuda": bool(same),
        "windows": result["evaluated_windows"], "accepted": result["accepted_operations"],
        "hpwl_before": result["hpwl_before"], "hpwl_after": result["hpwl_after"],
        "data": f"synthetic: {args.workload} (seed {args.seed}) with its standard cells packed legally in "
                "shuffled order (packed_placement, seed 7)",
    }
    print(json.dumps(line))


def run_bookshelf(args) -> None:
    """Reading the workload written as BookShelf files (host only): seconds for the native reader on one
    and on all host threads, and for the reference reader (oracle/_ref/libref_cpu.so), and whether the
    two read the same design."""
    import os as _os
    import tempfile

    import numpy as np

    import myplacement_b200 as mp
    from oracle.ref import ReferenceLibrary

    design, _ = mp.workload(args.workload, seed=args.seed)
    x, y = mp.random_placement(design, args.seed)
    with tempfile.TemporaryDirectory() as directory:
        aux = mp.write_bookshelf(design.copy_with_positions(x, y), directory, args.workload)
        size = sum(f.stat().st_size for f in Path(directory).iterdir())
        timings = {}
        for threads in (1, 0):
            best = math.inf
            for _ in range(3):
                t0 = time.perf_counter()
                mine = mp.read_bookshelf(aux, threads)
                best = min(best, time.perf_counter() - t0)
            timings["one_thread" if threads == 1 else "all_threads"] = best
        t0 = time.perf_counter()
        theirs = ReferenceLibrary("cpu").read_bookshelf(aux)
        reference_seconds = time.perf_counter() - t0
    same = (np.array_equal(mine.module_x, theirs["modules"]["x"]) and
            np.array_equal(mine.pin_module, theirs["nets"]["pin_module"]) and
            np.array_equal(mine.pin_offset_x, theirs["nets"]["offset_x"]) and
            list(mine.bookshelf.net_names) == theirs["net_names"])
    line = {
        "form": "bookshelf", "metric": "BookShelf read seconds", "value": timings["all_threads"], "unit": "s",
        "higher_is_better": False, "threads": _os.cpu_count(), "one_thread_s": timings["one_thread"],
        "reference_reader_s": reference_seconds,
        "speedup_vs_reference": reference_seconds / timings["all_threads"], "bytes": size,
        "modules": mine.module_count, "nets": mine.net_count, "pins": mine.pin_count,
        "identical_to_reference": bool(same),
        "data": f"synthetic: {args.workload} (seed {args.seed}) written by write_bookshelf",
    }
    print(json.dumps(line))


def main() -> int:
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "batched":
        run_batched(args)
    elif args.form == "serving":
        run_serving(args)
    elif args.form == "detailed":
        run_detailed(args)
    elif args.form == "bookshelf":
        run_bookshelf(args)
    else:
        run_mine(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
