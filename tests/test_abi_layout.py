"""The ctypes mirrors in myplacement_b200/_abi.py have the exact layout of include/mpgp.h (CPU only).

A small C program compiled against the header prints sizeof and the offset of
every field the mirror declares; each must equal ctypes' own figure.
"""
from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

from myplacement_b200 import _abi

REPO = Path(__file__).resolve().parents[1]

MIRRORS = {
    "mpgp_design": _abi.Design,
    "mpgp_options": _abi.Options,
    "mpgp_density_metrics": _abi.DensityMetrics,
    "mpgp_evaluation": _abi.Evaluation,
    "mpgp_history_row": _abi.HistoryRow,
    "mpgp_result": _abi.Result,
    "mpgp_layout": _abi.Layout,
    "mpgp_bookshelf_view": _abi.BookshelfView,
    "mpgp_detailed_options": _abi.DetailedOptions,
    "mpgp_detailed_result": _abi.DetailedResult,
    "mpgp_job_stats": _abi.JobStats,
    "mpgp_server_stats": _abi.ServerStats,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_every_mirror_matches_the_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "mpgp.h"', "int main(void) {"]
    for name, mirror in MIRRORS.items():
        lines.append(f'    printf("{name} sizeof %zu\\n", sizeof({name}));')
        for field, _ in mirror._fields_:
            lines.append(f'    printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["    return 0;", "}"]
    source = tmp_path / "layout.c"
    source.write_text("\n".join(lines) + "\n")
    binary = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", f"-I{REPO / 'include'}", str(source), "-o", str(binary)], check=True)
    printed = subprocess.run([str(binary)], capture_output=True, text=True, check=True).stdout.split("\n")
    figures = {tuple(line.split()[:2]): int(line.split()[2]) for line in printed if line}
    for name, mirror in MIRRORS.items():
        assert figures[(name, "sizeof")] == ctypes.sizeof(mirror), name
        for field, _ in mirror._fields_:
            assert figures[(name, field)] == getattr(mirror, field).offset, (name, field)
