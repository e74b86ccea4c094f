"""Placement designs: the flattened PlacementDatabase and seeded synthetic generators.

A :class:`Design` holds exactly what the reference's PlacementDatabase holds
(include/myplacement/model/PlacementDatabase.hpp): modules with width, height,
centre, terminal/fixed flags and orientation; nets with weights and their pins
(module + offset from the module centre); and SiteRows.  Pins are stored net by
net, which is the order the BookShelf reader creates them in
(src/io/BookshelfParser.cpp parseNets).

The generators build the synthetic workloads the engine is measured on.  All
randomness comes from ``numpy.random.Generator(PCG64(seed))``; the same seed
always gives the same design.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _abi

ROW_HEIGHT = 12.0


@dataclass
class Design:
    module_width: np.ndarray
    module_height: np.ndarray
    module_x: np.ndarray
    module_y: np.ndarray
    module_flags: np.ndarray
    net_weight: np.ndarray
    net_pin_start: np.ndarray
    pin_module: np.ndarray
    pin_offset_x: np.ndarray
    pin_offset_y: np.ndarray
    row_bottom: np.ndarray
    row_height: np.ndarray
    row_site_width: np.ndarray
    row_site_spacing: np.ndarray
    row_x_start: np.ndarray
    row_site_count: np.ndarray
    module_orientation: np.ndarray | None = None
    name: str = "design"
    # Names, pin directions, row orientations and declared counts of a design
    # read from BookShelf files (myplacement_b200.bookshelf.BookshelfInfo).
    bookshelf: object | None = None
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self) -> None:
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        i64 = lambda a: np.ascontiguousarray(a, dtype=np.int64)
        for name in ("module_width", "module_height", "module_x", "module_y", "net_weight", "pin_offset_x",
                     "pin_offset_y", "row_bottom", "row_height", "row_site_width", "row_site_spacing",
                     "row_x_start"):
            setattr(self, name, f64(getattr(self, name)))
        for name in ("module_flags", "pin_module"):
            setattr(self, name, i32(getattr(self, name)))
        for name in ("net_pin_start", "row_site_count"):
            setattr(self, name, i64(getattr(self, name)))
        if self.module_orientation is not None:
            self.module_orientation = i32(self.module_orientation)

    # ---- sizes -------------------------------------------------------------------
    @property
    def module_count(self) -> int:
        return int(self.module_width.shape[0])

    @property
    def net_count(self) -> int:
        return int(self.net_weight.shape[0])

    @property
    def pin_count(self) -> int:
        return int(self.pin_module.shape[0])

    @property
    def movable_mask(self) -> np.ndarray:
        return (self.module_flags & (_abi.MODULE_TERMINAL | _abi.MODULE_FIXED)) == 0

    @property
    def core(self) -> tuple[float, float, float, float]:
        x_end = self.row_x_start + self.row_site_count * self.row_site_spacing
        return (float(self.row_x_start.min()), float(self.row_bottom.min()), float(x_end.max()),
                float((self.row_bottom + self.row_height).max()))

    def copy_with_positions(self, x: np.ndarray, y: np.ndarray) -> "Design":
        fields = {k: getattr(self, k) for k in self.__dataclass_fields__ if not k.startswith("_")}
        fields["module_x"] = np.array(x, dtype=np.float64)
        fields["module_y"] = np.array(y, dtype=np.float64)
        return Design(**fields)

    # ---- C view --------------------------------------------------------------------
    def as_c(self) -> _abi.Design:
        """A struct pointing into this design's arrays (valid while the design lives)."""
        d = C.POINTER(C.c_double)
        i32 = C.POINTER(C.c_int32)
        i64 = C.POINTER(C.c_int64)
        p = lambda a, t: a.ctypes.data_as(t)
        s = _abi.Design()
        s.module_count = self.module_count
        s.module_width = p(self.module_width, d)
        s.module_height = p(self.module_height, d)
        s.module_x = p(self.module_x, d)
        s.module_y = p(self.module_y, d)
        s.module_flags = p(self.module_flags, i32)
        s.module_orientation = p(self.module_orientation, i32) if self.module_orientation is not None else None
        s.net_count = self.net_count
        s.net_weight = p(self.net_weight, d)
        s.net_pin_start = p(self.net_pin_start, i64)
        s.pin_count = self.pin_count
        s.pin_module = p(self.pin_module, i32)
        s.pin_offset_x = p(self.pin_offset_x, d)
        s.pin_offset_y = p(self.pin_offset_y, d)
        s.row_count = int(self.row_bottom.shape[0])
        s.row_bottom = p(self.row_bottom, d)
        s.row_height = p(self.row_height, d)
        s.row_site_width = p(self.row_site_width, d)
        s.row_site_spacing = p(self.row_site_spacing, d)
        s.row_x_start = p(self.row_x_start, d)
        s.row_site_count = p(self.row_site_count, i64)
        return s

    # ---- persistence -----------------------------------------------------------------
    def save(self, path: str | Path) -> None:
        arrays = {k: getattr(self, k) for k in self.__dataclass_fields__
                  if not k.startswith("_") and isinstance(getattr(self, k), np.ndarray)}
        np.savez_compressed(path, name=np.array(self.name), **arrays)

    @staticmethod
    def load(path: str | Path) -> "Design":
        with np.load(path) as data:
            fields = {k: data[k] for k in data.files if k != "name"}
            fields["name"] = str(data["name"]) if "name" in data.files else Path(path).stem
        return Design(**fields)


# ---- synthetic generators ---------------------------------------------------------


def _degree_law(rng: np.random.Generator, count: int, tail_p: float) -> np.ndarray:
    """Net degrees: 2 w.p. 0.6, U{3..5} w.p. 0.3, 6 + Geometric(tail_p) capped at 64 w.p. 0.1."""
    kind = rng.random(count)
    degree = np.full(count, 2, dtype=np.int64)
    mid = (kind >= 0.6) & (kind < 0.9)
    degree[mid] = rng.integers(3, 6, size=int(mid.sum()))
    tail = kind >= 0.9
    failures = rng.geometric(tail_p, size=int(tail.sum())) - 1  # failures before the first success
    degree[tail] = np.minimum(6 + failures, 64)
    return degree


def _expected_degree(tail_p: float) -> float:
    k = np.arange(0, 59)
    pmf = tail_p * (1.0 - tail_p) ** k
    tail = np.minimum(6 + k, 64)
    mean_tail = float((pmf * tail).sum() + (1.0 - pmf.sum()) * 64)
    return 0.6 * 2 + 0.3 * 4 + 0.1 * mean_tail


def calibrate_tail(pins_per_net: float) -> float:
    """Geometric tail parameter whose degree law gives `pins_per_net` on average."""
    lo, hi = 0.01, 0.99
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if _expected_degree(mid) > pins_per_net:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def _pack_macros(rng: np.random.Generator, widths: np.ndarray, heights: np.ndarray, core_w: float,
                 core_h: float) -> tuple[np.ndarray, np.ndarray] | None:
    """Seeded non-overlapping shelf placement of macros (lower-left corners), or None if they do not fit.

    Macros are sorted by height and filled into horizontal shelves; the slack of
    each shelf and of the stack of shelves is spread as random gaps, so the
    layout varies with the seed while never overlapping.
    """
    order = np.argsort(-heights, kind="stable")
    shelves: list[list[int]] = []
    shelf_heights: list[float] = []
    current: list[int] = []
    used = 0.0
    for index in order:
        w = float(widths[index])
        if w > core_w:
            return None
        if current and used + w > core_w:
            shelves.append(current)
            current, used = [], 0.0
        if not current:
            shelf_heights.append(float(heights[index]))
        current.append(int(index))
        used += w
    if current:
        shelves.append(current)
    total_h = float(sum(shelf_heights))
    if total_h > core_h:
        return None
    llx = np.zeros(widths.shape[0])
    lly = np.zeros(widths.shape[0])
    gaps_y = rng.dirichlet(np.ones(len(shelves) + 1)) * (core_h - total_h)
    y = 0.0
    for s, members in enumerate(shelves):
        y += gaps_y[s]
        slack = core_w - float(sum(widths[m] for m in members))
        gaps_x = rng.dirichlet(np.ones(len(members) + 1)) * slack
        x = 0.0
        for k, m in enumerate(members):
            x += gaps_x[k]
            llx[m] = x
            # Shorter macros in a shelf are dropped to a random height inside it.
            lly[m] = y + rng.random() * (shelf_heights[s] - heights[m])
            x += widths[m]
        y += shelf_heights[s]
    # Snap to integer coordinates inside the core (BookShelf .pl coordinates are integral).
    llx = np.floor(llx)
    lly = np.floor(lly)
    return llx, lly


def _boundary_terminals(count: int, core_w: float, core_h: float) -> tuple[np.ndarray, np.ndarray]:
    """Centres of `count` terminals spaced evenly along the core perimeter."""
    perimeter = 2.0 * (core_w + core_h)
    s = (np.arange(count) + 0.5) * perimeter / count
    x = np.empty(count)
    y = np.empty(count)
    for i, t in enumerate(s):
        if t < core_w:
            x[i], y[i] = t, 0.0
        elif t < core_w + core_h:
            x[i], y[i] = core_w, t - core_w
        elif t < 2 * core_w + core_h:
            x[i], y[i] = core_w - (t - core_w - core_h), core_h
        else:
            x[i], y[i] = 0.0, core_h - (t - 2 * core_w - core_h)
    return x, y


def synthetic_design(*, cells: int, nets: int, terminals: int, macros: int = 0, rows: int | None = None,
                     sites: int | None = None, utilization: float = 0.70, tail_p: float = 0.25,
                     pins_per_net: float | None = None, terminal_net_fraction: float = 0.02,
                     locality_window: int = 1024, seed: int = 2026, name: str = "synthetic") -> Design:
    """A seeded row-based design with the degree law of the synthetic workloads.

    Cells are one row tall (12 units) with integer widths U{2..12}.  Terminals
    are 1x1 and sit on the core boundary.  Macros (fixed) are 12*U{8..60} tall
    with aspect U(0.5, 2) and are packed without overlap.  When `rows`/`sites`
    are not given, the core is square and sized so that
    cell area / (row area - macro area) equals `utilization`.  Each net picks
    distinct cells from a random window of `locality_window` consecutive cell
    indices; `terminal_net_fraction` of the nets also connect one terminal.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    cell_w = rng.integers(2, 13, size=cells).astype(np.float64)
    cell_h = np.full(cells, ROW_HEIGHT)
    macro_h = ROW_HEIGHT * rng.integers(8, 61, size=macros).astype(np.float64)
    macro_w = np.round(macro_h * rng.uniform(0.5, 2.0, size=macros))
    cell_area = float((cell_w * cell_h).sum())
    macro_area = float((macro_w * macro_h).sum())

    if rows is None or sites is None:
        core_area = cell_area / utilization + macro_area
        side = math.sqrt(core_area)
        rows = int(math.ceil(side / ROW_HEIGHT))
        sites = int(math.ceil(core_area / (rows * ROW_HEIGHT)))
    packed = None
    for _ in range(200):
        if macros == 0:
            packed = (np.zeros(0), np.zeros(0))
            break
        packed = _pack_macros(rng, macro_w, macro_h, float(sites), rows * ROW_HEIGHT)
        if packed is not None:
            break
        rows = int(math.ceil(rows * 1.01))
        sites = int(math.ceil(sites * 1.01))
    if packed is None:
        raise ValueError("macros do not fit the core")
    core_w = float(sites)
    core_h = rows * ROW_HEIGHT

    term_x, term_y = _boundary_terminals(terminals, core_w, core_h)
    module_w = np.concatenate([cell_w, macro_w, np.ones(terminals)])
    module_h = np.concatenate([cell_h, macro_h, np.ones(terminals)])
    module_x = np.concatenate([np.full(cells, core_w * 0.5), packed[0] + macro_w * 0.5, term_x])
    module_y = np.concatenate([np.full(cells, core_h * 0.5), packed[1] + macro_h * 0.5, term_y])
    flags = np.concatenate([np.zeros(cells, np.int32), np.full(macros, _abi.MODULE_FIXED, np.int32),
                            np.full(terminals, _abi.MODULE_TERMINAL | _abi.MODULE_FIXED, np.int32)])

    if pins_per_net is not None:
        tail_p = calibrate_tail(pins_per_net)
    degree = _degree_law(rng, nets, tail_p)
    degree = np.minimum(degree, cells)
    with_terminal = (rng.random(nets) < terminal_net_fraction) if terminals > 0 else np.zeros(nets, bool)
    cell_pins = degree - with_terminal.astype(np.int64)
    cell_pins = np.maximum(cell_pins, 1)
    degree = cell_pins + with_terminal
    window = min(locality_window, cells)
    starts = rng.integers(0, cells - window + 1, size=nets)
    net_of_cell_pin = np.repeat(np.arange(nets), cell_pins)
    chosen = starts[net_of_cell_pin] + rng.integers(0, window, size=int(cell_pins.sum()))
    # Make the cells of each net distinct: re-draw colliding picks.
    offsets = np.concatenate([[0], np.cumsum(cell_pins)])
    key = net_of_cell_pin * np.int64(cells) + chosen
    order = np.argsort(key, kind="stable")
    dup = np.zeros(chosen.shape[0], bool)
    dup[order[1:]] = key[order[1:]] == key[order[:-1]]
    for pin in np.nonzero(dup)[0]:
        net = net_of_cell_pin[pin]
        taken = set(chosen[offsets[net]:offsets[net + 1]].tolist())
        while True:
            candidate = int(starts[net] + rng.integers(0, window))
            if candidate not in taken:
                chosen[pin] = candidate
                break
    pin_module_parts = []
    pin_dx_parts = []
    pin_dy_parts = []
    net_pin_start = np.zeros(nets + 1, np.int64)
    net_pin_start[1:] = np.cumsum(degree)
    # Assemble net-major pin arrays: cell pins then (optionally) one terminal pin.
    total = int(degree.sum())
    pin_module = np.empty(total, np.int32)
    write = np.arange(int(cell_pins.sum())) - offsets[net_of_cell_pin] + net_pin_start[net_of_cell_pin]
    pin_module[write] = chosen
    term_nets = np.nonzero(with_terminal)[0]
    if term_nets.size:
        pin_module[net_pin_start[term_nets + 1] - 1] = cells + macros + rng.integers(0, terminals, size=term_nets.size)
    del pin_module_parts, pin_dx_parts, pin_dy_parts
    w = module_w[pin_module]
    h = module_h[pin_module]
    pin_dx = rng.uniform(-0.5, 0.5, size=total) * w
    pin_dy = rng.uniform(-0.5, 0.5, size=total) * h
    is_term = pin_module >= cells + macros
    pin_dx[is_term] = 0.0
    pin_dy[is_term] = 0.0

    return Design(
        module_width=module_w, module_height=module_h, module_x=module_x, module_y=module_y,
        module_flags=flags, net_weight=np.ones(nets), net_pin_start=net_pin_start, pin_module=pin_module,
        pin_offset_x=pin_dx, pin_offset_y=pin_dy,
        row_bottom=np.arange(rows) * ROW_HEIGHT, row_height=np.full(rows, ROW_HEIGHT),
        row_site_width=np.ones(rows), row_site_spacing=np.ones(rows), row_x_start=np.zeros(rows),
        row_site_count=np.full(rows, sites, np.int64), name=name)


# ---- the named workloads -------------------------------------------------------------

WORKLOADS = {
    # Plain method, small: 5,000 cells, 120 terminals, 100 rows x 600 sites, 5,200 nets, 64^2 bins.
    "small_5k": dict(cells=5_000, nets=5_200, terminals=120, rows=100, sites=600, tail_p=0.25, bins=64),
    # Plain GPU form, mid: 210k cells, 400 fixed macros, 1,200 terminals, 220k nets (~850k pins), 512^2 bins.
    "mid_210k": dict(cells=210_000, nets=220_000, terminals=1_200, macros=400, utilization=0.70,
                     pins_per_net=850_000 / 220_000, bins=512),
    # Precision form, large: 1.3M cells, 2,000 macros, 1.4M nets (~5.5M pins), 1024^2 bins.
    "large_1m3": dict(cells=1_300_000, nets=1_400_000, terminals=1_200, macros=2_000, utilization=0.70,
                      pins_per_net=5_500_000 / 1_400_000, bins=1024),
}


def workload(name: str, seed: int = 2026, scale: float = 1.0) -> tuple[Design, int]:
    """(design, bins) for a named workload; `scale` shrinks cell/net/macro/terminal counts for tests."""
    spec = dict(WORKLOADS[name])
    bins = spec.pop("bins")
    if scale != 1.0:
        for key in ("cells", "nets", "terminals", "macros"):
            if key in spec:
                spec[key] = max(1 if key != "macros" else 0, int(round(spec[key] * scale)))
        if "rows" in spec:
            spec.pop("rows")
            spec.pop("sites")
            spec["utilization"] = 0.58
        bins = max(8, int(2 ** round(math.log2(max(8.0, bins * math.sqrt(scale))))))
    design = synthetic_design(seed=seed, name=name, **spec)
    return design, bins


def packed_placement(design: Design, seed: int, gap_probability: float = 0.05) -> Design:
    """A seeded legal placement of the standard cells, the input detailed placement expects.

    Standard cells (neither fixed nor taller than the median row) are shuffled
    and packed left to right into the rows, bottom row first: each takes its
    width rounded up to whole sites (alignUp, as the detailed placer measures
    it), and with probability `gap_probability` one free site follows it.
    Other modules keep their positions.  Raises ValueError if the cells do not
    fit the rows.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    rows = np.argsort(design.row_bottom, kind="stable")
    nominal = float(np.sort(design.row_height)[design.row_height.shape[0] // 2])
    fixed = (design.module_flags & (_abi.MODULE_TERMINAL | _abi.MODULE_FIXED)) != 0
    standard = ~fixed & (np.abs(design.module_height - nominal) <= 1e-9)
    cells = rng.permutation(np.nonzero(standard)[0])
    gaps = rng.random(cells.shape[0]) < gap_probability
    x = design.module_x.copy()
    y = design.module_y.copy()
    r = 0
    cursor = float(design.row_x_start[rows[0]])
    for cell, gap in zip(cells.tolist(), gaps.tolist()):
        width = float(design.module_width[cell])
        while True:
            row = rows[r]
            spacing = float(design.row_site_spacing[row])
            taken = width if spacing <= 1e-9 else math.ceil((width - 1e-9) / spacing) * spacing
            end = float(design.row_x_start[row] + design.row_site_count[row] * spacing)
            if cursor + taken <= end + 1e-9:
                break
            r += 1
            if r == rows.shape[0]:
                raise ValueError("the standard cells do not fit the rows")
            cursor = float(design.row_x_start[rows[r]])
        x[cell] = cursor + width * 0.5
        y[cell] = float(design.row_bottom[row]) + float(design.module_height[cell]) * 0.5
        cursor += taken + (spacing if gap else 0.0)
    return design.copy_with_positions(x, y)


def small_instance(cells: int, seed: int) -> tuple[Design, int]:
    """A small-design-structured instance (no macros) of `cells` cells; bins = power of two nearest sqrt(cells)."""
    nets = int(round(cells * 5_200 / 5_000))
    terminals = max(8, int(round(cells * 120 / 5_000)))
    design = synthetic_design(cells=cells, nets=nets, terminals=terminals, utilization=0.58, tail_p=0.25,
                              seed=seed, name=f"inst{cells}")
    bins = int(2 ** round(math.log2(math.sqrt(cells))))
    return design, max(8, min(1024, bins))
