"""The C-ABI library loads and exports every entry point declared in include/*.h (CPU only)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import myplacement_b200 as mp
from myplacement_b200 import _abi

from conftest import GPU_PRESENT

REPO = Path(__file__).resolve().parents[1]


def _declared_symbols() -> list[str]:
    names = []
    for header in (REPO / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        names += re.findall(r"\b(mpgp_\w+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(_abi.LIBRARY_PATH))
    declared = _declared_symbols()
    assert len(declared) >= 20
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing


def test_library_identity():
    lib = mp.load_library()
    assert lib.mpgp_compiled() == 1
    assert lib.mpgp_abi_version() == 1


def test_struct_sizes_match_header():
    """ctypes mirrors have the C layout (checked by the offsets of the last field)."""
    assert ctypes.sizeof(_abi.DensityMetrics) == 64
    assert ctypes.sizeof(_abi.Evaluation) == 24 + 128
    assert _abi.Options.maximum_cuda_memory_bytes.offset == ctypes.sizeof(_abi.Options) - 8
    assert ctypes.sizeof(_abi.HistoryRow) == 8 + 16 * 8 + 16


def test_errors_cross_the_boundary_as_status_codes():
    lib = mp.load_library()
    status = lib.mpgp_session_step(None, 1, None, None)
    assert status == _abi.MPGP_ERR_INVALID_ARGUMENT
    assert b"session" in lib.mpgp_last_error()


@pytest.mark.skipif(GPU_PRESENT, reason="checks the behaviour without a GPU")
def test_no_cpu_fallback_without_gpu(golden_dir):
    """Without a CUDA device the engine refuses to run instead of computing on the CPU."""
    f = np.load(golden_dir / "fixtures.npz")
    design = mp.Design(**{k[5:]: f[k] for k in f.files if k.startswith("tiny_")}, name="tiny")
    with pytest.raises(mp.EngineError) as error:
        mp.GlobalPlacer().run(design, mp.default_options(bins_x=8, bins_y=8, iterations=4))
    assert error.value.status in (_abi.MPGP_ERR_UNAVAILABLE, _abi.MPGP_ERR_CUDA)
    layout = mp.build_layout(design, np.ones(3), np.ones(3), np.zeros(3), np.ones(3), 3, 8, 8, 0.85,
                             np.zeros(64), np.zeros(64))
    backend, reason = mp.try_create_backend(layout, 0)
    assert backend is None and reason


def test_tuning_table_round_trip():
    """The autotuned contraction splits can be read, replaced and restored; bad splits are refused."""
    from myplacement_b200 import tune

    original = tune.get_splits()
    try:
        tune.set_splits({256: 2, 512: 1, 1024: 2})
        assert tune.get_splits() == {256: 2, 512: 1, 1024: 2}
        with pytest.raises(mp.EngineError) as error:
            tune.set_splits({512: 3})
        assert error.value.status == mp._abi.MPGP_ERR_INVALID_ARGUMENT
    finally:
        tune.set_splits(original)
    assert tune.get_splits() == original
