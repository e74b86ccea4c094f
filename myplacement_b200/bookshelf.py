"""BookShelf designs: the native reader and a writer.

``BookshelfParser().parse_aux(path)`` is the reference's
``myplacement::BookshelfParser::parseAux`` (include/myplacement/io/
BookshelfParser.hpp:16-19, src/io/BookshelfParser.cpp:313-348): it reads the
.aux file and the .nodes, .scl, .pl, .nets and .wts files it names through
libmpgp.so's multi-threaded reader (``mpgp_bookshelf_read``) and returns a
:class:`~myplacement_b200.design.Design` whose ``bookshelf`` field holds the
names, pin directions, row orientations and declared counts.  Malformed input
raises :class:`ParseError` (the reference's ParseError) or, for duplicate
names and negative sizes, :class:`EngineError` with status
MPGP_ERR_INVALID_ARGUMENT (the database's std::invalid_argument); the messages
are the reference's.

``write_bookshelf`` writes a Design as BookShelf files, so that the synthetic
designs can be read back by this reader or by the reference's.
"""
from __future__ import annotations

import ctypes as C
import os
from collections.abc import Sequence
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _abi
from ._abi import EngineError, ParseError, check, load_library
from .design import Design

__all__ = ["BookshelfInfo", "BookshelfParser", "EngineError", "Names", "ParseError", "read_bookshelf",
           "write_bookshelf"]

ORIENTATIONS = ("N", "S", "E", "W", "FN", "FS", "FE", "FW", "UNKNOWN")
DIRECTIONS = ("I", "O", "B", "B")  # PinDirection order; an unknown direction is written as B


class Names(Sequence):
    """Names stored back to back (one bytes object plus offsets), decoded on access."""

    def __init__(self, blob: bytes, start: np.ndarray):
        self._blob = blob
        self._start = np.asarray(start, dtype=np.int64)

    def __len__(self) -> int:
        return int(self._start.shape[0]) - 1

    def __getitem__(self, index):
        if isinstance(index, slice):
            return [self[i] for i in range(*index.indices(len(self)))]
        if index < 0:
            index += len(self)
        if not 0 <= index < len(self):
            raise IndexError(index)
        return self._blob[int(self._start[index]):int(self._start[index + 1])].decode("utf-8", "surrogateescape")

    def __eq__(self, other) -> bool:
        return list(self) == list(other)


@dataclass
class BookshelfInfo:
    module_names: Names
    net_names: Names
    pin_direction: np.ndarray    # int8, PinDirection order: input, output, bidirectional, unknown
    row_orientation: np.ndarray  # int32, Orientation order, 8 = unknown
    declared: dict               # NumNodes / NumTerminals / NumNets / NumPins -> int or None


def _array(pointer, count: int, dtype) -> np.ndarray:
    if count <= 0 or not pointer:
        return np.zeros(max(count, 0), dtype=dtype)
    return np.ctypeslib.as_array(pointer, shape=(count,)).astype(dtype, copy=True)


def _names(pointer, start: np.ndarray) -> Names:
    size = int(start[-1]) if start.shape[0] else 0
    blob = C.string_at(pointer, size) if size > 0 else b""
    return Names(blob, start)


class BookshelfParser:
    """myplacement::BookshelfParser over the native reader."""

    def __init__(self, threads: int = 0):
        self.threads = int(threads)

    def parse_aux(self, aux_path: str | os.PathLike) -> Design:
        lib = load_library()
        handle = C.c_void_p()
        check(lib.mpgp_bookshelf_read(os.fsencode(aux_path), self.threads, C.byref(handle)))
        try:
            view = _abi.BookshelfView()
            check(lib.mpgp_bookshelf_get(handle, C.byref(view)))
            d = view.design
            modules, nets, pins, rows = d.module_count, d.net_count, d.pin_count, d.row_count
            f64 = lambda ptr, n: _array(ptr, n, np.float64)
            info = BookshelfInfo(
                module_names=_names(view.module_names, _array(view.module_name_start, modules + 1, np.int64)),
                net_names=_names(view.net_names, _array(view.net_name_start, nets + 1, np.int64)),
                pin_direction=_array(view.pin_direction, pins, np.int8),
                row_orientation=_array(view.row_orientation, rows, np.int32),
                declared={key: (None if value < 0 else int(value)) for key, value in (
                    ("NumNodes", view.declared_nodes), ("NumTerminals", view.declared_terminals),
                    ("NumNets", view.declared_nets), ("NumPins", view.declared_pins))},
            )
            return Design(
                module_width=f64(d.module_width, modules), module_height=f64(d.module_height, modules),
                module_x=f64(d.module_x, modules), module_y=f64(d.module_y, modules),
                module_flags=_array(d.module_flags, modules, np.int32),
                module_orientation=_array(d.module_orientation, modules, np.int32),
                net_weight=f64(d.net_weight, nets), net_pin_start=_array(d.net_pin_start, nets + 1, np.int64),
                pin_module=_array(d.pin_module, pins, np.int32), pin_offset_x=f64(d.pin_offset_x, pins),
                pin_offset_y=f64(d.pin_offset_y, pins),
                row_bottom=f64(d.row_bottom, rows), row_height=f64(d.row_height, rows),
                row_site_width=f64(d.row_site_width, rows), row_site_spacing=f64(d.row_site_spacing, rows),
                row_x_start=f64(d.row_x_start, rows), row_site_count=_array(d.row_site_count, rows, np.int64),
                name=Path(aux_path).stem, bookshelf=info)
        finally:
            lib.mpgp_bookshelf_destroy(handle)


def read_bookshelf(aux_path: str | os.PathLike, threads: int = 0) -> Design:
    """BookshelfParser(threads).parse_aux(aux_path)."""
    return BookshelfParser(threads).parse_aux(aux_path)


def _number(value) -> str:
    return repr(float(value))  # shortest text that reads back to the same double


def write_bookshelf(design: Design, directory: str | os.PathLike, stem: str | None = None,
                    module_names: Sequence[str] | None = None, net_names: Sequence[str] | None = None) -> Path:
    """Writes `design` as <stem>.aux/.nodes/.nets/.wts/.pl/.scl; returns the .aux path.

    Modules are named ``o<i>`` and nets ``n<i>`` unless names are given (or the
    design was read from BookShelf).  Lower-left corners are written as
    centre - size / 2, so centres read back exactly when that is exact (integer
    corners, as in the synthetic designs).
    """
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    stem = stem or design.name
    info = design.bookshelf if isinstance(design.bookshelf, BookshelfInfo) else None
    if module_names is None:
        module_names = info.module_names if info else [f"o{i}" for i in range(design.module_count)]
    if net_names is None:
        net_names = info.net_names if info else [f"n{i}" for i in range(design.net_count)]
    module_names = list(module_names)
    net_names = list(net_names)
    terminal = (design.module_flags & _abi.MODULE_TERMINAL) != 0
    fixed = (design.module_flags & _abi.MODULE_FIXED) != 0
    orientation = (design.module_orientation if design.module_orientation is not None
                   else np.zeros(design.module_count, np.int32))
    direction = info.pin_direction if info else np.full(design.pin_count, 2, np.int8)

    def write(suffix: str, lines: list[str]) -> None:
        (directory / f"{stem}{suffix}").write_text("\n".join(lines) + "\n")

    write(".aux", [f"RowBasedPlacement : {stem}.nodes {stem}.nets {stem}.wts {stem}.pl {stem}.scl"])
    write(".nodes", ["UCLA nodes 1.0", "", f"NumNodes : {design.module_count}",
                     f"NumTerminals : {int(terminal.sum())}", ""] +
          [f"\t{module_names[m]}\t{_number(w)}\t{_number(h)}" + ("\tterminal" if t else "")
           for m, (w, h, t) in enumerate(zip(design.module_width, design.module_height, terminal))])
    write(".pl", ["UCLA pl 1.0", ""] +
          [f"{module_names[m]}\t{_number(x - w * 0.5)}\t{_number(y - h * 0.5)}\t: {ORIENTATIONS[o]}" +
           (" /FIXED" if f else "")
           for m, (x, y, w, h, o, f) in enumerate(zip(design.module_x, design.module_y, design.module_width,
                                                      design.module_height, orientation, fixed))])
    nets = ["UCLA nets 1.0", "", f"NumNets : {design.net_count}", f"NumPins : {design.pin_count}", ""]
    start = design.net_pin_start
    for n in range(design.net_count):
        nets.append(f"NetDegree : {int(start[n + 1] - start[n])}   {net_names[n]}")
        nets.extend(f"\t{module_names[design.pin_module[p]]} {DIRECTIONS[direction[p]]} : "
                    f"{_number(design.pin_offset_x[p])} {_number(design.pin_offset_y[p])}"
                    for p in range(int(start[n]), int(start[n + 1])))
    write(".nets", nets)
    write(".wts", ["UCLA wts 1.0", ""] + [f"{net_names[n]} {_number(w)}" for n, w in enumerate(design.net_weight)])
    rows = ["UCLA scl 1.0", "", f"NumRows : {design.row_bottom.shape[0]}", ""]
    row_orientation = info.row_orientation if info else np.zeros(design.row_bottom.shape[0], np.int32)
    for r in range(design.row_bottom.shape[0]):
        rows += ["CoreRow Horizontal", f"  Coordinate    : {_number(design.row_bottom[r])}",
                 f"  Height        : {_number(design.row_height[r])}",
                 f"  Sitewidth     : {_number(design.row_site_width[r])}",
                 f"  Sitespacing   : {_number(design.row_site_spacing[r])}",
                 f"  Siteorient    : {ORIENTATIONS[row_orientation[r]]}", "  Sitesymmetry  : Y",
                 f"  SubrowOrigin  : {_number(design.row_x_start[r])}  NumSites : {int(design.row_site_count[r])}",
                 "End"]
    write(".scl", rows)
    return directory / f"{stem}.aux"
