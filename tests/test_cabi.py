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
