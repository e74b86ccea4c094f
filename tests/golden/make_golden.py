"""Regenerates the committed golden fixtures (test infrastructure).

    python tests/golden/make_golden.py

Writes, next to this script:

``fixtures.npz``
    The reference's own BookShelf test designs ``tiny`` and ``mixed``
    (tests/fixtures/{tiny,mixed}.* in the reference tree), flattened into the
    Design arrays by the small reader below (.nodes/.nets/.pl/.scl/.wts).
``eval_small.npz``
    A seeded 1,000-cell synthetic design (2 fixed macros), random positions and
    the reference CPU path's outputs there: one GlobalPlacementSession
    evaluation (metrics, raw/preconditioned gradients) and the separated
    wire / density parts, layers and fields (oracle/_ref/libref_cpu.so).

Only this script reads the reference tree; the tests read the .npz files.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from myplacement_b200 import _abi  # noqa: E402
from myplacement_b200.design import Design, synthetic_design  # noqa: E402
from oracle.ref import ReferenceLibrary, default_options  # noqa: E402

# The reference tree this recipe reads (MPGP_REFERENCE_ROOT, as oracle/build_oracle.py takes it).
REFERENCE_FIXTURES = Path(os.environ.get("MPGP_REFERENCE_ROOT", "/root/reference")) / "tests" / "fixtures"


def _lines(path: Path):
    for raw in path.read_text().splitlines():
        line = raw.split("#", 1)[0].strip()
        if line and not line.startswith("UCLA"):
            yield line


def read_bookshelf(stem: str) -> Design:
    base = REFERENCE_FIXTURES / stem
    names, width, height, flags = [], [], [], []
    for line in _lines(base.with_suffix(".nodes")):
        if ":" in line:
            continue
        parts = line.split()
        names.append(parts[0])
        width.append(float(parts[1]))
        height.append(float(parts[2]))
        flags.append(_abi.MODULE_TERMINAL | _abi.MODULE_FIXED if "terminal" in parts[3:] else 0)
    index = {n: i for i, n in enumerate(names)}
    x = np.zeros(len(names))
    y = np.zeros(len(names))
    for line in _lines(base.with_suffix(".pl")):
        parts = line.split()
        i = index[parts[0]]
        x[i] = float(parts[1]) + width[i] * 0.5
        y[i] = float(parts[2]) + height[i] * 0.5
        if any("FIXED" in p.upper() for p in parts[3:]):
            flags[i] |= _abi.MODULE_FIXED
    weights = {}
    wts = base.with_suffix(".wts")
    if wts.exists():
        for line in _lines(wts):
            parts = line.split()
            if len(parts) >= 2:
                weights[parts[0]] = float(parts[1])
    net_weight, net_start, pin_module, pin_dx, pin_dy = [], [0], [], [], []
    lines = list(_lines(base.with_suffix(".nets")))
    k = 0
    while k < len(lines):
        line = lines[k]
        if line.startswith("NetDegree"):
            parts = line.replace(":", " ").split()
            degree = int(parts[1])
            name = parts[2] if len(parts) > 2 else f"net_{len(net_weight)}"
            for j in range(degree):
                pin = lines[k + 1 + j].replace(":", " ").split()
                pin_module.append(index[pin[0]])
                pin_dx.append(float(pin[2]) if len(pin) > 2 else 0.0)
                pin_dy.append(float(pin[3]) if len(pin) > 3 else 0.0)
            net_weight.append(weights.get(name, 1.0))
            net_start.append(len(pin_module))
            k += degree + 1
        else:
            k += 1
    rows = []
    current = {}
    for line in _lines(base.with_suffix(".scl")):
        if line.startswith("CoreRow"):
            current = {}
        elif line.startswith("End"):
            rows.append(current)
        else:
            parts = line.replace(":", " ").split()
            if parts[0] == "Coordinate":
                current["bottom"] = float(parts[1])
            elif parts[0] == "Height":
                current["height"] = float(parts[1])
            elif parts[0] == "Sitewidth":
                current["site_width"] = float(parts[1])
            elif parts[0] == "Sitespacing":
                current["site_spacing"] = float(parts[1])
            elif parts[0] == "SubrowOrigin":
                current["x_start"] = float(parts[1])
                current["site_count"] = int(parts[3])
    return Design(
        module_width=np.array(width), module_height=np.array(height), module_x=x, module_y=y,
        module_flags=np.array(flags), net_weight=np.array(net_weight), net_pin_start=np.array(net_start),
        pin_module=np.array(pin_module), pin_offset_x=np.array(pin_dx), pin_offset_y=np.array(pin_dy),
        row_bottom=np.array([r["bottom"] for r in rows]), row_height=np.array([r["height"] for r in rows]),
        row_site_width=np.array([r["site_width"] for r in rows]),
        row_site_spacing=np.array([r["site_spacing"] for r in rows]),
        row_x_start=np.array([r["x_start"] for r in rows]), row_site_count=np.array([r["site_count"] for r in rows]),
        name=stem)


def small_eval_case():
    design = synthetic_design(cells=1_000, nets=1_040, terminals=24, macros=2, utilization=0.6, tail_p=0.25,
                              seed=11, name="eval_small")
    ref = ReferenceLibrary("cpu")
    x, y = ref.random_placement(design, 3)
    design = design.copy_with_positions(x, y)
    options = default_options(bins_x=32, bins_y=32, target_density=0.9)
    session = ref.session(design, options)
    positions = session.positions
    smoothing, penalty, reference_penalty = 6.5, 0.37, 0.5
    ev = session.evaluate(positions, smoothing, penalty, reference_penalty, True)
    comp = session.components(positions, smoothing)
    fixed, dark = session.static_density()
    out = {f"dsg_{k}": v for k, v in _design_arrays(design).items()}
    out.update(
        positions=positions, smoothing=smoothing, penalty=penalty, reference_penalty=reference_penalty,
        bins=32, target_density=0.9,
        particle_width=session.width, particle_height=session.height, particle_layer=session.layer,
        particle_pin_count=session.pin_count, movable_count=session.movable_count,
        static_fixed=fixed, static_dark=dark,
        hpwl=ev["hpwl"], smooth_wirelength=ev["smooth_wirelength"], density_energy=ev["density_energy"],
        objective=ev["objective"], wire_gradient_l1=ev["wire_gradient_l1"],
        density_gradient_l1=ev["density_gradient_l1"], raw_gradient_norm=ev["raw_gradient_norm"],
        preconditioned_gradient_norm=ev["preconditioned_gradient_norm"],
        optimizer_density=np.array([ev["optimizer_density"][k] for k in _abi.DENSITY_METRIC_FIELDS]),
        design_density=np.array([ev["design_density"][k] for k in _abi.DENSITY_METRIC_FIELDS]),
        raw_gradient=ev["raw_gradient"], preconditioned_gradient=ev["preconditioned_gradient"],
        wire_gradient=comp["wire_gradient"], density_gradient=comp["density_gradient"],
        movable_layer=comp["movable"], macro_layer=comp["macro"], filler_layer=comp["filler"],
        potential=comp["potential"], field_x=comp["field_x"], field_y=comp["field_y"])
    return out


def _design_arrays(design: Design) -> dict:
    return {k: getattr(design, k) for k in design.__dataclass_fields__
            if not k.startswith("_") and k != "name" and getattr(design, k) is not None}


def main() -> int:
    arrays = {}
    for stem in ("tiny", "mixed"):
        design = read_bookshelf(stem)
        for k, v in _design_arrays(design).items():
            arrays[f"{stem}_{k}"] = v
    np.savez_compressed(HERE / "fixtures.npz", **arrays)
    np.savez_compressed(HERE / "eval_small.npz", **small_eval_case())
    print("wrote", HERE / "fixtures.npz", HERE / "eval_small.npz")
    return 0


if __name__ == "__main__":
    sys.exit(main())
