"""The native BookShelf reader against the reference's BookshelfParser (CPU only).

Three readers see the same files:
  * mine: libmpgp.so's mpgp_bookshelf_read (myplacement_b200.read_bookshelf);
  * theirs: the reference's src/io/BookshelfParser.cpp, compiled unmodified
    into oracle/_ref/libref_cpu.so;
  * the drop-in: the reference's BookshelfParser API served by
    myplacement_b200/adapter/mpgp_bookshelf_parser.cpp over libmpgp.so
    (oracle/_ref/libref_dropin.so).
Every value read must be bit-identical (sizes, centres, offsets, weights,
orientations, directions, rows, names, declared counts), and malformed input
must fail the same way: ParseError vs std::invalid_argument, and the same
message, naming the same line.  Each case runs with one thread and with
several, whose pieces split the files at many line boundaries.
"""
from __future__ import annotations

import random
from pathlib import Path

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi
from oracle.build_oracle import REF_ROOT
from oracle.ref import ReferenceFailure, ReferenceLibrary
from oracle.ref import default_options as ref_options

THREADS = (1, 5)


@pytest.fixture(scope="module")
def readers():
    return ReferenceLibrary("cpu"), ReferenceLibrary("dropin")


def _bits(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def _assert_same(mine: mp.Design, theirs: dict) -> None:
    m, n, r = theirs["modules"], theirs["nets"], theirs["rows"]
    for mine_key, their_key in (("module_width", "width"), ("module_height", "height"), ("module_x", "x"),
                                ("module_y", "y")):
        assert np.array_equal(_bits(getattr(mine, mine_key)), _bits(m[their_key])), mine_key
    assert np.array_equal(mine.module_flags, m["flags"] & 3)
    assert np.array_equal(mine.module_orientation, m["orientation"])
    assert np.array_equal(_bits(mine.net_weight), _bits(n["weight"]))
    assert np.array_equal(mine.net_pin_start, n["pin_start"])
    assert np.array_equal(n["pins"], np.arange(mine.pin_count))  # the reference lists pins net by net too
    assert np.array_equal(mine.pin_module, n["pin_module"])
    assert np.array_equal(np.repeat(np.arange(mine.net_count), np.diff(mine.net_pin_start)), n["pin_net"])
    assert np.array_equal(_bits(mine.pin_offset_x), _bits(n["offset_x"]))
    assert np.array_equal(_bits(mine.pin_offset_y), _bits(n["offset_y"]))
    assert np.array_equal(mine.bookshelf.pin_direction, n["direction"])
    for mine_key, their_key in (("row_bottom", "bottom"), ("row_height", "height"),
                                ("row_site_width", "site_width"), ("row_site_spacing", "site_spacing"),
                                ("row_x_start", "x_start")):
        assert np.array_equal(_bits(getattr(mine, mine_key)), _bits(r[their_key])), mine_key
    assert np.array_equal(mine.row_site_count, r["site_count"])
    assert np.array_equal(mine.bookshelf.row_orientation, r["orientation"])
    assert list(mine.bookshelf.module_names) == theirs["module_names"]
    assert list(mine.bookshelf.net_names) == theirs["net_names"]
    declared = [mine.bookshelf.declared[k] for k in ("NumNodes", "NumTerminals", "NumNets", "NumPins")]
    assert [-1 if v is None else v for v in declared] == theirs["declared"].tolist()


def _outcome(read):
    try:
        return "ok", read()
    except ReferenceFailure as failure:
        return failure.status, failure.message
    except mp.EngineError as error:
        return error.status, str(error).split(": ", 1)[1]


def _check(readers, aux: Path) -> str:
    """All readers agree on `aux`; returns "ok" or the reference's message."""
    ref, dropin = readers
    status, theirs = _outcome(lambda: ref.read_bookshelf(aux))
    for threads in THREADS:
        mine_status, mine = _outcome(lambda: mp.read_bookshelf(aux, threads))
        assert mine_status == status, (threads, mine_status, mine, status, theirs)
        if status == "ok":
            _assert_same(mine, theirs)
        else:
            assert mine == theirs, threads
    dropin_status, via_dropin = _outcome(lambda: dropin.read_bookshelf(aux))
    assert dropin_status == status
    if status == "ok":
        for part in ("modules", "nets", "rows"):
            for key in theirs[part]:
                assert np.array_equal(via_dropin[part][key], theirs[part][key]), (part, key)
        for key in ("module_names", "net_names", "movable_count"):
            assert via_dropin[key] == theirs[key]
        assert np.array_equal(via_dropin["declared"], theirs["declared"])
        assert np.array_equal(via_dropin["regions"], theirs["regions"])
        return "ok"
    assert via_dropin == theirs
    return theirs


def _write(directory: Path, stem: str, files: dict[str, str], aux: str | None = None) -> Path:
    directory.mkdir(parents=True, exist_ok=True)
    for suffix, text in files.items():
        (directory / f"{stem}{suffix}").write_text(text)
    names = " ".join(f"{stem}{s}" for s in (".nodes", ".nets", ".wts", ".pl", ".scl"))
    (directory / f"{stem}.aux").write_text(aux if aux is not None else f"RowBasedPlacement : {names}\n")
    return directory / f"{stem}.aux"


def _synthetic_files(tmp_path: Path, cells: int = 800, macros: int = 4, seed: int = 7) -> dict[str, list[str]]:
    design = mp.synthetic_design(cells=cells, nets=cells + cells // 20, terminals=24, macros=macros, seed=seed,
                                 name="base")
    aux = mp.write_bookshelf(design, tmp_path / "base", "base")
    return {s: (aux.parent / f"base{s}").read_text().splitlines() for s in (".nodes", ".nets", ".wts", ".pl", ".scl")}


# ---- well-formed designs -----------------------------------------------------------------


def test_reference_fixtures(readers, golden_dir):
    """The reference's own test designs (tests/fixtures/{tiny,mixed}) and the committed golden arrays."""
    fixtures = REF_ROOT / "tests" / "fixtures"
    if not fixtures.is_dir():
        pytest.skip("the reference tree is not present")
    golden = np.load(golden_dir / "fixtures.npz")
    for stem in ("tiny", "mixed"):
        assert _check(readers, fixtures / f"{stem}.aux") == "ok"
        mine = mp.read_bookshelf(fixtures / f"{stem}.aux")
        for key in (k for k in golden.files if k.startswith(stem + "_")):
            assert np.array_equal(golden[key], getattr(mine, key[len(stem) + 1:])), key


@pytest.mark.parametrize("name,scale", [("small_5k", 1.0), ("mid_210k", 0.02)])
def test_synthetic_round_trip(readers, tmp_path, name, scale):
    """Written synthetic designs read back exactly (integer corners), by every reader."""
    design, _ = mp.workload(name, scale=scale)
    aux = mp.write_bookshelf(design, tmp_path, name)
    assert _check(readers, aux) == "ok"
    mine = mp.read_bookshelf(aux)
    for key in ("module_width", "module_height", "module_x", "module_y", "module_flags", "net_weight",
                "net_pin_start", "pin_module", "pin_offset_x", "pin_offset_y", "row_bottom", "row_height",
                "row_x_start", "row_site_count"):
        assert np.array_equal(getattr(mine, key), getattr(design, key)), key
    assert mine.bookshelf.declared == {"NumNodes": design.module_count,
                                       "NumTerminals": int(((design.module_flags & _abi.MODULE_TERMINAL) != 0).sum()),
                                       "NumNets": design.net_count, "NumPins": design.pin_count}
    again = mp.read_bookshelf(mp.write_bookshelf(mine, tmp_path / "again", name))
    assert list(again.bookshelf.net_names) == list(mine.bookshelf.net_names)


QUIRKS_NODES = """UCLA nodes 1.0
# a comment line
NumNodes : 10\r
NumTerminals:2
   a1   4   12   \r
a2\t2.5\t12 # trailing comment
a3 +3 12.
a4 .5e1 1.2e1 extra words
M1 40 48
p1 1 1 terminal
p2 1 1 TERMINAL_NI
a5 1e-400 12
a6 3 12
NetDegree 2 12
"""
QUIRKS_PL = """UCLA pl 1.0

a1 0 0 : N
a2 10.5 0 :FS
a3 20 0 : E /FIXED
a4 30 0 /FIXED
a5 40 0 :
M1 100 100 : W /FIXED
p1 -1 5 : N /FIXED
p2 601 7
a6 5 5 : n
a6 6 6
bad line here
a2 x y
"""
QUIRKS_NETS = """UCLA nets 1.0
NumNets : 6
NumPins : 14

NetDegree : 3 net_a
  a1 I : 0.5 -0.5
# comment inside a net

  a2 O:1:2
  p1 B : 0 0
NetDegree : 2   net_b   extra
\ta3\tINPUT\t:\t-1.5\t+2
  a4 output : 1e-400 .25
NetDegree : 0 net_empty
NetDegree : 2 net_c
  M1 inout : -20 24
  NetDegree B : 0 0   # a pin line of net_c: its module is named NetDegree
NetDegree : 3 net_d
  a5 x : 0 0
  a6 I : 1e2 1E-2
  p2 b : 0 0
NumPins : 14
NetDegree : 4 net_e
  a1 I : 0 0
  a2 I : 0 0
  a3 I : 0 0
  a4 I : 0 0
"""
QUIRKS_WTS = """UCLA wts 1.0
net_a 2
net_b 0.5
unknown_net 9
net_c x
net_d 3 extra
net_a 4
"""
QUIRKS_SCL = """UCLA scl 1.0
NumRows : 3
Coordinate : 999
CoreRow Horizontal
  Coordinate    :   0
  Height        :   12
  Sitewidth     :    1
  Sitespacing   :    1
  Siteorient    :    FS
  Sitesymmetry  :    Y
  SubrowOrigin  :    0  NumSites  :  600
End
CoreRow Horizontal
  Coordinate : 12
  Height : 12
  Siteorient: N
  SubrowOrigin : 5 NumSites : 590
End
CoreRow Horizontal
  Coordinate : 24
  Height : 12
  Sitespacing : 2
  Siteorient : W
  SubrowOrigin : 0 NumSites : 300
End
"""


def _quirk_files(**changes) -> dict[str, str]:
    files = {".nodes": QUIRKS_NODES, ".pl": QUIRKS_PL, ".nets": QUIRKS_NETS, ".wts": QUIRKS_WTS,
             ".scl": QUIRKS_SCL}
    for suffix, text in changes.items():
        files["." + suffix] = text
    return {k: v for k, v in files.items() if v is not None}


def test_quirks_match_reference(readers, tmp_path):
    """Comments, CR, tabs, colons, signs and exponents, underflow, orientation and
    fixed tokens, a pin line whose module is named NetDegree, empty nets, unknown
    and repeated weights: every reader reads the same records."""
    aux = _write(tmp_path, "quirks", _quirk_files())
    assert _check(readers, aux) == "ok"
    mine = mp.read_bookshelf(aux)
    # Spot checks of the reference's reading of the quirks.
    names = list(mine.bookshelf.module_names)
    assert names[-1] == "NetDegree"
    orientation = dict(zip(names, mine.module_orientation.tolist()))
    assert orientation["a4"] == 8 and orientation["a5"] == 8 and orientation["a6"] == 0
    fixed = dict(zip(names, (mine.module_flags & _abi.MODULE_FIXED).tolist()))
    assert fixed["a3"] and not fixed["a4"] and fixed["p2"]
    assert mine.module_width[names.index("a5")] == 0.0
    assert mine.net_weight.tolist()[:2] == [4.0, 0.5]


def test_missing_weights_file_is_optional(readers, tmp_path):
    aux = _write(tmp_path, "nowts", _quirk_files(wts=None))
    assert _check(readers, aux) == "ok"
    assert np.all(mp.read_bookshelf(aux).net_weight == 1.0)


# ---- malformed designs ----------------------------------------------------------------------

ERROR_CASES = {
    "invalid node": dict(nodes=QUIRKS_NODES.replace("a6 3 12", "a6 3")),
    "invalid NumNodes": dict(nodes=QUIRKS_NODES.replace("NumNodes : 10", "NumNodes : nine")),
    "invalid NumTerminals": dict(nodes=QUIRKS_NODES.replace("NumTerminals:2", "NumTerminals")),
    "negative size": dict(nodes=QUIRKS_NODES.replace("a3 +3 12.", "a3 -3 12.")),
    "duplicate module": dict(nodes=QUIRKS_NODES.replace("a6 3 12", "a2 3 12")),
    "negative before duplicate": dict(nodes=QUIRKS_NODES.replace("a6 3 12", "a2 -3 12")),
    "duplicate before invalid node": dict(nodes=QUIRKS_NODES.replace("a6 3 12", "a1 3 12\nbroken")),
    "invalid node before duplicate": dict(nodes=QUIRKS_NODES.replace("M1 40 48", "M1 40\nM1 40 48")),
    "declared nodes": dict(nodes=QUIRKS_NODES.replace("NumNodes : 10", "NumNodes : 11")),
    "declared terminals": dict(nodes=QUIRKS_NODES.replace("NumTerminals:2", "NumTerminals : 3")),
    "invalid SubrowOrigin": dict(scl=QUIRKS_SCL.replace("SubrowOrigin : 5 NumSites : 590", "SubrowOrigin : 5")),
    "zero row height": dict(scl=QUIRKS_SCL.replace("Coordinate : 12\n  Height : 12", "Coordinate : 12")),
    "no rows": dict(scl="UCLA scl 1.0\nNumRows : 0\n"),
    "unknown module in pl": dict(pl=QUIRKS_PL.replace("p2 601 7", "p3 601 7")),
    "invalid NetDegree": dict(nets=QUIRKS_NETS.replace("NetDegree : 3 net_d", "NetDegree : 3")),
    "invalid NetDegree count": dict(nets=QUIRKS_NETS.replace("NetDegree : 3 net_d", "NetDegree : x net_d")),
    "invalid pin": dict(nets=QUIRKS_NETS.replace("a6 I : 1e2 1E-2", "a6 I : 1e2")),
    "unknown pin module": dict(nets=QUIRKS_NETS.replace("p2 b : 0 0", "p9 b : 0 0")),
    "end of file in a net": dict(nets=QUIRKS_NETS.replace("NetDegree : 4 net_e", "NetDegree : 5 net_e")),
    "negative degree": dict(nets=QUIRKS_NETS.replace("NetDegree : 4 net_e", "NetDegree : -1 net_e")),
    "duplicate net": dict(nets=QUIRKS_NETS.replace("net_d", "net_b")),
    "pin before duplicate net": dict(nets=QUIRKS_NETS.replace("net_e", "net_a").replace("a5 x : 0 0", "a5 x 0")),
    "duplicate net before pin": dict(nets=QUIRKS_NETS.replace("net_d", "net_a").replace("a1 I : 0 0", "zz I : 0 0")),
    "declared nets": dict(nets=QUIRKS_NETS.replace("NumNets : 6", "NumNets : 7")),
    "declared pins": dict(nets=QUIRKS_NETS.replace("NumPins : 14\nNetDegree : 4", "NumPins : 15\nNetDegree : 4")),
}


@pytest.mark.parametrize("case", list(ERROR_CASES))
def test_errors_match_reference(readers, tmp_path, case):
    aux = _write(tmp_path, "bad", _quirk_files(**ERROR_CASES[case]))
    message = _check(readers, aux)
    assert message != "ok", case
    status = _outcome(lambda: mp.read_bookshelf(aux))[0]
    expected = _abi.MPGP_ERR_INVALID_ARGUMENT if "uplicate" in message or "negative" in message else \
        _abi.MPGP_ERR_PARSE
    assert status == expected, message
    if expected == _abi.MPGP_ERR_PARSE:
        with pytest.raises(mp.ParseError):
            mp.read_bookshelf(aux)


def test_aux_errors_match_reference(readers, tmp_path):
    files = _quirk_files()
    assert _check(readers, tmp_path / "absent.aux").startswith("Unable to open BookShelf file")
    for suffix in (".nodes", ".scl", ".pl", ".nets"):
        named = " ".join(f"x{s}" for s in (".nodes", ".nets", ".wts", ".pl", ".scl") if s != suffix)
        aux = _write(tmp_path / suffix[1:], "x", files, aux=f"RowBasedPlacement : {named}\n")
        assert "missing required" in _check(readers, aux)
    aux = _write(tmp_path / "unopened", "x", {k: v for k, v in files.items() if k != ".pl"})
    assert _check(readers, aux).startswith("Unable to open BookShelf file")
    # The first file named for an extension wins; comments and colon-less lines are ignored.
    aux = _write(tmp_path / "twice", "x", files,
                 aux="# x.nodes\nRowBasedPlacement : x.nodes x.nets x.wts x.pl x.scl other.nodes\nno colon x.pl\n")
    assert _check(readers, aux) == "ok"


# ---- seeded mutations ---------------------------------------------------------------------------

JUNK_TOKENS = ["", "x", "-1", "1e", "1e400", "1e-400", "+5", ".5", "5.", ":", ":N", "/FIXED", "terminal", "#",
               "NetDegree", "UCLA", "0x10", "99999999999999999999", "-0", "nan", "inf", "FW", "\t"]
JUNK_LINES = ["", "   ", "# comment", "NumNets : 3", "NumPins :", "NetDegree : 2 extra_net", "NetDegree : x",
              "NetDegree : 1", "UCLA nets 1.0", "o1 B : 0 0", "o2 I : 1", "CoreRow Horizontal", "End",
              "NumNodes : 5", "o3 4 12", "o4 4", "n1 2.5", "o5 1 1 : FN /FIXED"]


def _mutate(lines: list[str], rng: random.Random) -> list[str]:
    lines = list(lines)
    for _ in range(rng.randint(1, 3)):
        if not lines:
            break
        at = rng.randrange(len(lines))
        kind = rng.randrange(6)
        if kind == 0:
            del lines[at]
        elif kind == 1:
            lines.insert(rng.randrange(len(lines) + 1), lines[at])
        elif kind == 2:
            tokens = lines[at].split(" ")
            tokens[rng.randrange(len(tokens))] = rng.choice(JUNK_TOKENS)
            lines[at] = " ".join(tokens)
        elif kind == 3:
            lines.insert(at, rng.choice(JUNK_LINES))
        elif kind == 4:
            other = rng.randrange(len(lines))
            lines[at], lines[other] = lines[other], lines[at]
        else:
            lines = lines[:at]
    return lines


JUNK_BYTES = [b"\x00", b"#", b":", b"\r", b"\t", b" ", b"\xff", b"\xc3\xa9", b"-", b"+", b".", b"e", b"\n", b"1"]


def _mutate_bytes(data: bytes, rng: random.Random) -> bytes:
    out = bytearray(data)
    for _ in range(rng.randint(1, 4)):
        if not out:
            break
        at = rng.randrange(len(out))
        kind = rng.randrange(3)
        if kind == 0:
            del out[at]
        elif kind == 1:
            out[at:at] = rng.choice(JUNK_BYTES)
        else:
            out[at:at + 1] = rng.choice(JUNK_BYTES)
    return bytes(out)


def test_seeded_byte_mutations_match_reference(readers, tmp_path):
    """100 seeded byte-level edits (NUL, '#', ':', CR, tabs, bytes above 0x7f,
    signs, points, exponents, newlines) of a written 300-cell design: the
    readers agree on each."""
    base = _synthetic_files(tmp_path, cells=300)
    outcomes = {"ok": 0, "error": 0}
    for case in range(100):
        rng = random.Random(70000 + case)
        suffix = rng.choice([".nets", ".nets", ".nodes", ".pl", ".wts", ".scl"])
        directory = tmp_path / f"b{case}"
        directory.mkdir()
        for s, lines in base.items():
            data = ("\n".join(lines) + "\n").encode()
            (directory / f"m{s}").write_bytes(_mutate_bytes(data, rng) if s == suffix else data)
        names = " ".join(f"m{s}" for s in (".nodes", ".nets", ".wts", ".pl", ".scl"))
        (directory / "m.aux").write_text(f"RowBasedPlacement : {names}\n")
        outcomes["ok" if _check(readers, directory / "m.aux") == "ok" else "error"] += 1
    assert outcomes["ok"] > 10 and outcomes["error"] > 10, outcomes


def test_seeded_mutations_match_reference(readers, tmp_path):
    """200 seeded edits of a written 800-cell design (deleted, repeated, swapped and
    junk lines and tokens, truncations, in every file): the readers agree on each."""
    base = _synthetic_files(tmp_path)
    weights = [(".nets", 5), (".nodes", 3), (".pl", 3), (".wts", 1), (".scl", 1)]
    outcomes = {"ok": 0, "error": 0}
    for case in range(200):
        rng = random.Random(1000 + case)
        suffix = rng.choices([w[0] for w in weights], [w[1] for w in weights])[0]
        files = {s: "\n".join(lines) + "\n" for s, lines in base.items()}
        files[suffix] = "\n".join(_mutate(base[suffix], rng)) + "\n"
        aux = _write(tmp_path / f"m{case}", "m", files)
        outcomes["ok" if _check(readers, aux) == "ok" else "error"] += 1
    assert outcomes["ok"] > 20 and outcomes["error"] > 20, outcomes


def test_view_layout_matches_header():
    import ctypes
    assert ctypes.sizeof(_abi.BookshelfView) == ctypes.sizeof(_abi.Design) + 10 * 8


# ---- read, then place on the device ------------------------------------------------------------------


def _design_from_reference(theirs: dict) -> mp.Design:
    m, n, r = theirs["modules"], theirs["nets"], theirs["rows"]
    return mp.Design(module_width=m["width"], module_height=m["height"], module_x=m["x"], module_y=m["y"],
                     module_flags=m["flags"] & 3, module_orientation=m["orientation"], net_weight=n["weight"],
                     net_pin_start=n["pin_start"], pin_module=n["pin_module"], pin_offset_x=n["offset_x"],
                     pin_offset_y=n["offset_y"], row_bottom=r["bottom"], row_height=r["height"],
                     row_site_width=r["site_width"], row_site_spacing=r["site_spacing"], row_x_start=r["x_start"],
                     row_site_count=r["site_count"])


@pytest.mark.gpu
def test_read_design_places_like_reference(gpu, readers, tmp_path):
    """BookShelf files -> native reader -> the engine on the device, against the
    same files -> the reference reader -> the reference CPU placer: the first 25
    iterations take the same accept / backtrack / restart decisions, with HPWL
    and overflow within 1e-4."""
    design, bins = mp.workload("small_5k")
    x, y = mp.random_placement(design, 2026)
    aux = mp.write_bookshelf(design.copy_with_positions(x, y), tmp_path, "placed")
    ref, _ = readers
    theirs = _design_from_reference(ref.read_bookshelf(aux))
    mine = mp.read_bookshelf(aux)
    fixed = dict(bins_x=bins, bins_y=bins, target_density=0.9, iterations=30, feasible_refinement_iterations=100000)
    _, _, ref_result, ref_history = ref.global_place(theirs, ref_options(**fixed))
    result = mp.GlobalPlacer().run(mine, mp.default_options(**fixed))
    assert result.completed_iterations == ref_result.completed_iterations == 30
    assert result.hpwl_before == pytest.approx(ref_result.hpwl_before, rel=1e-6)
    for row, ref_row in zip(result.history[:25], ref_history[:25]):
        for key in ("accepted", "backtracks", "momentum_restarted"):
            assert row[key] == ref_row[key], (row["iteration"], key)
        assert row["hpwl"] == pytest.approx(ref_row["hpwl"], rel=1e-4)
        assert row["overflow"] == pytest.approx(ref_row["overflow"], rel=1e-4)
