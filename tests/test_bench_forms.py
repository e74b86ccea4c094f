"""bench.py's host-only form runs and prints its line (CPU only)."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]


def test_bookshelf_form_reads_like_the_reference():
    out = subprocess.run([sys.executable, str(REPO / "bench.py"), "--form", "bookshelf", "--workload", "small_5k"],
                         capture_output=True, text=True, timeout=300, check=True)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["form"] == "bookshelf" and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["identical_to_reference"] is True
    assert line["modules"] == 5120 and line["pins"] > 0 and line["value"] > 0.0
    assert line["reference_reader_s"] > 0.0 and line["one_thread_s"] > 0.0
