"""Regenerates tests/golden/whole_runs.json (test infrastructure).

    python tests/golden/make_whole_runs.py [--seeds 12] [--nudges 6] [--workers 8]

Whole adaptive global-placement runs of the reference CPU path
(oracle/_ref/libref_cpu.so: AdaptiveGlobalPlacer with its default options, the
280-iteration budget and the early stop on) on the small synthetic design
(5,000 cells, 64 x 64 bins, target density 0.9), one run per seed from the
reference's randomPlacement (InitialPlacer.cpp:102-121), plus runs from the same
placement with every movable centre nudged by at most 1e-6 bin widths.  The
nudged runs measure how far the reference's own result moves under a
perturbation far below FP32 rounding: the whole-run parity test holds the
engine's final HPWL and overflow to that spread.

The design comes from the seeded generator in myplacement_b200/design.py; the
file records a fingerprint of it so the test can tell when the generator changed.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mpc
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

SEEDS = [2026, 7, 11, 3, 5, 13, 17, 19, 23, 29, 31, 37]
NUDGE_BASE = 1000


def design_fingerprint(design) -> str:
    """A short digest of the design arrays (float64 sums in a fixed order)."""
    parts = [design.module_width, design.module_height, design.module_x, design.module_y, design.pin_offset_x,
             design.pin_offset_y, design.pin_module.astype(np.float64), design.net_pin_start.astype(np.float64)]
    return ",".join(f"{float(np.sum(p * (1.0 + np.arange(p.size) % 7))):.10e}" for p in parts)


def nudged(design, bins: int, k: int):
    """The same placement with every movable centre moved by at most 1e-6 bin widths."""
    rng = np.random.default_rng(NUDGE_BASE + k)
    step = 1e-6 * (design.core[2] - design.core[0]) / bins
    x = design.module_x.copy()
    y = design.module_y.copy()
    movable = design.movable_mask
    x[movable] += step * rng.uniform(-1.0, 1.0, int(movable.sum()))
    y[movable] += step * rng.uniform(-1.0, 1.0, int(movable.sum()))
    return design.copy_with_positions(x, y)


def start_design(seed: int):
    import myplacement_b200 as mp
    from oracle.ref import ReferenceLibrary

    design, bins = mp.workload("small_5k")
    x, y = ReferenceLibrary("cpu").random_placement(design, seed)
    return design.copy_with_positions(x, y), bins


def run_case(case: tuple[int, int]) -> dict:
    """One reference run: nudge -1 is the un-nudged placement."""
    seed, k = case
    from oracle.ref import ReferenceLibrary, default_options

    design, bins = start_design(seed)
    if k >= 0:
        design = nudged(design, bins, k)
    options = default_options(bins_x=bins, bins_y=bins, target_density=0.9, compute_backend=0)
    _, _, result, _ = ReferenceLibrary("cpu").global_place(design, options)
    return {"seed": seed, "nudge": k, "hpwl_after": result.hpwl_after, "overflow_after": result.overflow_after,
            "completed_iterations": result.completed_iterations,
            "best_checkpoint_iteration": result.best_checkpoint_iteration, "hpwl_before": result.hpwl_before}


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--seeds", type=int, default=len(SEEDS))
    parser.add_argument("--nudges", type=int, default=6)
    parser.add_argument("--workers", type=int, default=8)
    args = parser.parse_args()
    seeds = SEEDS[:args.seeds]
    cases = [(s, k) for s in seeds for k in range(-1, args.nudges)]
    with mpc.get_context("spawn").Pool(args.workers) as pool:
        runs = pool.map(run_case, cases)
    out = {"design": "small_5k", "bins": 64, "target_density": 0.9, "options": "reference defaults "
           "(280-iteration budget, early stop on), compute_backend cpu", "nudge": "movable centres moved by "
           "U(-1, 1) x 1e-6 bin widths, numpy default_rng(1000 + k)", "seeds": {}}
    for seed in seeds:
        design, _ = start_design(seed)
        mine = [r for r in runs if r["seed"] == seed]
        base = next(r for r in mine if r["nudge"] == -1)
        out["seeds"][str(seed)] = {"fingerprint": design_fingerprint(design), "reference": base,
                                   "nudged": [r for r in mine if r["nudge"] >= 0]}
    (HERE / "whole_runs.json").write_text(json.dumps(out, indent=1) + "\n")
    gaps = [n["hpwl_after"] / v["reference"]["hpwl_after"] - 1.0 for v in out["seeds"].values() for n in v["nudged"]]
    print(f"wrote {HERE / 'whole_runs.json'}: {len(seeds)} seeds; nudged HPWL gaps mean {np.mean(gaps):+.4%}, "
          f"std {np.std(gaps):.4%}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
