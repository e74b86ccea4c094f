"""Autotuner of the engine's work split, run on the GPU the engine serves.

    python -m myplacement_b200.tune [--sizes 128 256 512 1024] [--iterations 16] [--write]

The tcgen05 field contractions split each output tile's K range over a cluster
of 1 or 2 CTAs (dct_tc.cu).  Which is faster depends on the bin grid: a split
halves each CTA's K loop but adds an exchange of FP64 partial tiles, and it
doubles the CTAs a launch needs.  For every grid size this tuner runs the
adaptive controller on a synthetic design (the mid design's structure at about
16k cells) with that many bins per side, once with each split, times every
contraction launch with CUDA events (the engine's own profiler) and keeps the
split with the least device time per iteration.  With --write it stores the
table in csrc/tuned_splits.inc, which the library compiles in (rebuild after).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

PACKAGE = Path(__file__).resolve().parent
TABLE = PACKAGE / "csrc" / "tuned_splits.inc"
FAMILIES = ["dct_forward", "dct_inverse"]


def set_splits(table: dict[int, int]) -> None:
    from . import _abi, load_library

    lib = load_library()
    sizes = np.array(sorted(table), np.int32)
    splits = np.array([table[s] for s in sorted(table)], np.int32)
    _abi.check(lib.mpgp_tuning_set_splits(sizes.ctypes.data_as(C.POINTER(C.c_int32)),
                                          splits.ctypes.data_as(C.POINTER(C.c_int32)), len(sizes)))


def get_splits() -> dict[int, int]:
    from . import _abi, load_library

    lib = load_library()
    sizes = np.zeros(64, np.int32)
    splits = np.zeros(64, np.int32)
    count = C.c_int32()
    _abi.check(lib.mpgp_tuning_get_splits(sizes.ctypes.data_as(C.POINTER(C.c_int32)),
                                          splits.ctypes.data_as(C.POINTER(C.c_int32)), 64, C.byref(count)))
    return {int(sizes[i]): int(splits[i]) for i in range(min(count.value, 64))}


def contraction_us_per_iteration(design, bins: int, warmup: int, iterations: int) -> tuple[float, int]:
    """Device microseconds of the field contractions per controller iteration, and their launches."""
    from . import placer

    options = placer.default_options(bins_x=bins, bins_y=bins, target_density=0.9,
                                     iterations=warmup + iterations, feasible_refinement_iterations=10 ** 9)
    session = placer.Session(design, options)
    try:
        session.step(warmup)
        session.set_profiling(FAMILIES)
        session.step(iterations)
        stats = session.kernel_stats()
    finally:
        session.close()
    launches = sum(stats[f][0] for f in FAMILIES)
    return 1e3 * sum(stats[f][1] for f in FAMILIES) / iterations, launches


def tune(sizes: list[int], warmup: int, iterations: int, repeats: int) -> dict:
    from . import placer
    from .design import workload

    design, _ = workload("mid_210k", seed=2026, scale=16_000 / 210_000)
    x, y = placer.random_placement(design, 2026)
    design = design.copy_with_positions(x, y)
    start = get_splits()
    report = {}
    for bins in sizes:
        timings = {}
        for split in (1, 2):
            set_splits({**start, bins: split})
            runs = [contraction_us_per_iteration(design, bins, warmup, iterations)[0] for _ in range(repeats)]
            timings[split] = float(np.median(runs))
        best = min(timings, key=timings.get)
        report[bins] = {"split": best, "us_per_iteration": timings}
        print(f"{bins:5d} bins: split 1 {timings[1]:9.1f} us, split 2 {timings[2]:9.1f} us per iteration -> {best}",
              flush=True)
    set_splits(start)
    return report


def write_table(report: dict, device_name: str) -> None:
    lines = [
        "// K split of the tcgen05 field contractions per contracted length (bins along the",
        "// axis the contraction sums over): {bins, split}.  Written by myplacement_b200/tune.py,",
        "// which times the field contractions of a placement run at each size with every",
        "// split on the device it runs on; a size not listed takes the occupancy rule of tcPlan.",
        f"// Measured on: {device_name}.  Device microseconds of the contractions per iteration",
        "// (median of the repeats) for splits 1 and 2 are given beside each entry.",
    ]
    for bins in sorted(report):
        r = report[bins]
        t = r["us_per_iteration"]
        lines.append(f"{{{bins}, {r['split']}}},  // {t[1]:.1f} / {t[2]:.1f} us")
    TABLE.write_text("\n".join(lines) + "\n")


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--sizes", type=int, nargs="+", default=[128, 256, 512, 1024])
    parser.add_argument("--warmup", type=int, default=4)
    parser.add_argument("--iterations", type=int, default=16)
    parser.add_argument("--repeats", type=int, default=3)
    parser.add_argument("--write", action="store_true", help="store the table in csrc/tuned_splits.inc")
    args = parser.parse_args()
    report = tune(args.sizes, args.warmup, args.iterations, args.repeats)
    print(json.dumps({str(k): v for k, v in report.items()}))
    if args.write:
        import torch

        write_table(report, torch.cuda.get_device_name(0) if torch.cuda.is_available() else "unknown")
        print(f"wrote {TABLE}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
