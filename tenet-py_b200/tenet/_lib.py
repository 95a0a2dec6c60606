"""ctypes binding of ``libtenet_b200.so``, the C ABI declared in ``include/tenet_b200.h``.

There is no fallback: if the library is missing, or no CUDA device is present when a
kernel is about to run, the call raises.  ``load()`` alone (symbol resolution) works on
a CPU-only machine, which is what the CPU test-suite checks.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_NAME = "libtenet_b200.so"
LIB_PATH = _HERE / LIB_NAME

_i64, _i32, _f64, _vp = ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_void_p

#: every exported entry point and its (restype, argtypes)
SIGNATURES = {
    "tnb_block_gather": (_i32, [_vp, _i64, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _vp,
                                _i64, _vp, _i64, _vp, _i64, _vp]),
    "tnb_block_gather_direct": (_i32, [_vp, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _vp, _i64,
                                       _vp, _i64, _vp, _i64, _vp]),
    "tnb_copy_f64": (_i32, [_i64, _vp, _vp, _vp]),
    "tnb_mapped_address": (_i32, [_vp, ctypes.POINTER(_vp)]),
    "tnb_block_gather_product": (_i32, [_vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp,
                                        _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp]),
    "tnb_grouped_gemm_f64": (_i32, [_vp, _i64, _vp, _i64, _i32, _vp, _i64, _vp, _i64, _vp,
                                    _i64, _vp, _i64, _i64, _vp]),
    "tnb_grouped_gemm_f64_rows": (_i32, [_vp, _i64, _i32, _vp, _i64, _vp, _i64, _vp, _i64, _vp,
                                         _i64, _i64, _vp]),
    "tnb_grouped_gemm_gather_a": (_i32, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _vp,
                                         _i64, _vp, _i64, _vp, _i64, _vp]),
    "tnb_seq_add_gemm_gather_a": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i64,
                                         _vp, _i64, _vp, _i64, _vp, _i64]),
    "tnb_dot_work_bytes": (_i64, [_i64]),
    "tnb_weighted_dot": (_i32, [_vp, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp]),
    "tnb_weighted_dot_noalloc": (_i32, [_vp, _vp, _i64, _vp, _vp, _i64, _vp, _vp]),
    "tnb_axpby": (_i32, [_i64, _f64, _vp, _f64, _vp, _vp, _vp]),
    "tnb_lincomb": (_i32, [_i64, _i64, _vp, _vp, _vp, _vp]),
    "tnb_lanczos_update": (_i32, [_i64, _vp, _vp, _vp, _vp, _i32, _i32, _vp]),
    "tnb_lanczos_next": (_i32, [_i64, _vp, _vp, _vp, _i32, _i32, _f64, _vp]),
    "tnb_scale_rsqrt": (_i32, [_i64, _vp, _vp, _vp, _vp]),
    "tnb_lanczos_step_max_n": (_i64, []),
    "tnb_lanczos_step": (_i32, [_i64, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _f64, _vp, _vp, _i64,
                                _vp]),
    "tnb_multi_dot_work_bytes": (_i64, [_i64, _i64]),
    "tnb_multi_dot": (_i32, [_i64, _i64, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp]),
    "tnb_lanczos_reorth": (_i32, [_i64, _i64, _vp, _vp, _vp, _vp, _i32, _vp]),
    "tnb_seq_create": (_i32, [ctypes.POINTER(_vp)]),
    "tnb_seq_destroy": (None, [_vp]),
    "tnb_seq_length": (_i64, [_vp]),
    "tnb_seq_add_gather_product": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i64,
                                          _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64]),
    "tnb_seq_add_gather": (_i32, [_vp, _vp, _i64, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _i64,
                                  _vp, _i64, _vp, _i64, _vp, _i64]),
    "tnb_seq_add_gather_direct": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _i64, _vp,
                                         _i64, _vp, _i64, _vp, _i64]),
    "tnb_seq_add_gemm": (_i32, [_vp, _vp, _i64, _vp, _i64, _i32, _vp, _i64, _vp, _i64, _vp,
                                _i64, _vp, _i64, _i64]),
    "tnb_seq_append": (_i32, [_vp, _vp]),
    "tnb_seq_fuse": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "tnb_seq_fuse_cluster": (_i32, [_vp, _vp, _vp, _i32, ctypes.POINTER(_i32), _vp]),
    "tnb_seq_run": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "tnb_lanczos_solve": (_i32, [_vp, _vp, _vp, _i64, _i32, _f64, _i32, _vp, _vp, _i64, _vp,
                                 _vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp]),
    "tnb_lanczos_ritz": (_i32, [_vp, _vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                _i64, _vp, _vp]),
    "tnb_plan_gather_table": (_i32, [_i64, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64, _vp,
                                     _vp, _vp, _vp, _vp, _i32, _vp, _i64, _vp, _vp, _vp, _vp,
                                     _vp]),
    "tnb_plan_gather_rows": (_i32, [_i64, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i64,
                                    _vp]),
    "tnb_plan_compose": (_i64, [_i64, _vp, _i64, _vp, _vp, _i64]),
    "tnb_block_svd_smem_doubles": (_i64, []),
    "tnb_block_svd": (_i32, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64,
                             _vp, _i64, _vp]),
    "tnb_truncate_decide": (_i32, [_vp, _vp, _i64, _vp, _i64, _f64, _i32, _f64, _i32, _vp, _vp,
                                   _vp, _vp, _vp]),
    "tnb_svd_compact": (_i32, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _f64, _vp, _i64,
                               _vp, _i64, _vp, _i64, _vp]),
    "tnb_block_lq": (_i32, [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _vp]),
    "tnb_set_pdl": (_i32, [_i32]),
    "tnb_version": (_i32, []),
    "tnb_last_error": (ctypes.c_char_p, []),
    "tnb_device_error": (_i32, [ctypes.POINTER(ctypes.c_int), _vp]),
}

_lib = None


class TenetCudaError(RuntimeError):
    """A library call returned a nonzero status."""


def load():
    """Load the library (once) and bind every signature; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("TENET_B200_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"tenet_b200: the CUDA library {path} is not built; run __graft_entry__.build() "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    status = getattr(load(), name)(*args)
    if status != 0:
        msg = load().tnb_last_error().decode(errors="replace")
        raise TenetCudaError(f"{name} failed with status {status}: {msg}")


def device_error(stream) -> int:
    out = ctypes.c_int(0)
    call("tnb_device_error", ctypes.byref(out), stream)
    return int(out.value)


def mapped_address(p: int) -> int:
    """The address kernels use for ``p`` (``tnb_mapped_address``): pinned host memory
    through its mapped device pointer; raises for pageable memory."""
    out = _vp()
    call("tnb_mapped_address", p, ctypes.byref(out))
    return int(out.value)
