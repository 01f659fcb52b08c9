"""The C-ABI library: it loads without a GPU, exports every symbol the public
header declares, and fails loudly (no CPU fallback) when no B200 is present."""
import ctypes
import re

import pytest

import pawan_b200
from pawan_b200 import HEADER, LIB_PATH, load_library


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pawan_[a-z0-9_]+)\s*\(", text)))


def test_library_exists_and_loads():
    lib = load_library()
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(header_symbols()) == set(pawan_b200._SIGS)


def test_status_names():
    lib = load_library()
    assert lib.pawan_status_name(0) == b"ok"
    assert lib.pawan_status_name(5) == b"exceeds budget"
    assert lib.pawan_status_name(99) == b"unknown status"


def test_null_handles_are_rejected():
    lib = load_library()
    assert lib.pawan_ctx_synchronize(None) == 1
    assert lib.pawan_system_solve(None) == 1
    assert lib.pawan_batch_rk4(None, None, 0.1, 1, 0) == 1
    assert lib.pawan_server_poll(None, 1, None) == 1
    lib.pawan_ctx_destroy(None)
    lib.pawan_system_destroy(None)


def test_context_without_gpu_raises():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pawan_b200.PawanError):
        pawan_b200.Context(0)


def test_tile_candidates_listed_host_side():
    """The autotuner's candidate tilings and chunkings, without a GPU; the
    full-size parity tests (tests/test_gpu_pairs.py) run exactly these."""
    from test_gpu_pairs import DEFAULT_TILING, TIMED_TILING, TUNE_CANDIDATES
    keys = ("threads", "threads_per_target", "targets_per_thread", "unroll", "blocks_per_sm", "packed",
            "split_near")
    got = [tuple(c[k] for k in keys) for c in pawan_b200.tile_candidates("f32")]
    assert got == TUNE_CANDIDATES
    assert TIMED_TILING in got and DEFAULT_TILING in got
    assert pawan_b200.tile_chunkings() == [4, 8, 32, 64, 128]
    assert len(pawan_b200.tile_candidates("f64")) == 2
    assert len(pawan_b200.tile_candidates("f32", "gaussian")) >= 2
    lib = load_library()
    n = ctypes.c_size_t(0)
    assert lib.pawan_tile_candidates(9, 0, None, 0, ctypes.byref(n)) == 1
    assert lib.pawan_tile_candidates(0, 0, None, 0, None) == 1
