"""The C-ABI library loads on a CPU-only machine and exports every declared symbol."""

import re
from pathlib import Path

from tenet import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "tenet_b200.h"


def declared() -> set[str]:
    text = HEADER.read_text()
    return set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(tnb_\w+)\s*\(", text, re.M))


def test_every_declared_symbol_is_exported_and_bound():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 8
    for name in names:
        assert hasattr(lib, name), f"{name} is declared in tenet_b200.h but not exported"
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_version_and_error_string_need_no_gpu():
    lib = _lib.load()
    assert lib.tnb_version() >= 100
    assert isinstance(lib.tnb_last_error(), bytes)


def test_refusals_move_nothing_and_set_a_message():
    """Argument validation happens before any launch, so it runs without a device."""
    lib = _lib.load()
    assert lib.tnb_axpby(-1, 1.0, None, 1.0, None, None, None) == 1
    assert b"negative" in lib.tnb_last_error()
    assert lib.tnb_weighted_dot(None, None, 5, None, None, 1, None, None, None) == 1
    assert lib.tnb_block_gather(None, 1, None, 1, None, None, None, 0, None, 0, None, 0, None,
                                0, None, 0, None) == 1
    assert lib.tnb_grouped_gemm_f64(None, 1, None, 1, 7, None, 0, None, 0, None, 0, None, 0, 0,
                                    None) == 1


def test_launch_sequence_bookkeeping_needs_no_gpu():
    """Recording, appending and the refusals of the sequence API are host-only."""
    import ctypes

    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.tnb_seq_create(ctypes.byref(h)) == 0
    assert lib.tnb_seq_length(h) == 0
    # recording borrows pointers; nothing is dereferenced until a replay
    assert lib.tnb_seq_add_gather(h, 16, 1, 32, 1, 48, 64, 80, 1, 96, 4, 112, 4, None, 0, None,
                                  0) == 0
    assert lib.tnb_seq_add_gemm(h, 16, 1, 32, 1, 0, 48, 1, 64, 1, 80, 1, None, 0, 0) == 0
    assert lib.tnb_seq_length(h) == 2
    assert lib.tnb_seq_add_gemm(h, 16, -1, 32, 1, 0, 48, 1, 64, 1, 80, 1, None, 0, 0) == 1
    assert lib.tnb_seq_append(h, h) == 1
    h2 = ctypes.c_void_p()
    assert lib.tnb_seq_create(ctypes.byref(h2)) == 0
    assert lib.tnb_seq_append(h2, h) == 0 and lib.tnb_seq_append(h2, h) == 0
    assert lib.tnb_seq_length(h2) == 4
    assert lib.tnb_seq_run(h2, -1, None, None, None) == 1
    assert lib.tnb_seq_run(None, 0, None, None, None) == 1
    assert lib.tnb_lanczos_solve(None, None, None, 4, 2, 1e-13, 0, None, None, 4, None, None,
                                 None, None, None, None, None, 1, None, None, None) == 1
    assert lib.tnb_seq_length(None) == -1
    lib.tnb_seq_destroy(h)
    lib.tnb_seq_destroy(h2)
