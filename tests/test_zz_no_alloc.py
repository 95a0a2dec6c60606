"""The allocation-free weighted dot, called through the C ABI.

Some callers of this library cannot allocate device memory: code being captured into a
CUDA graph under the global capture mode (where cudaMalloc is an error), a serving loop
that has admitted its work against a fixed HBM budget and must not grow its footprint
mid-request, and foreign-language hosts that hold only borrowed buffers.  For them
``tnb_weighted_dot_noalloc`` keeps its scratch in a static device array instead of a
caller buffer.  This test checks it against the allocating entry point,
``tnb_weighted_dot``, on two calls in a row (the shared array keeps the last call's
contents, so the second call must not depend on them), and that an n beyond the array's
limit is refused on the host.  The file is named to be collected last.
"""

import ctypes

import pytest
import torch

from tenet import _lib

pytestmark = pytest.mark.gpu

MAX_N = 2_097_152  # TNB_DOT_NOALLOC_MAX_N in include/tenet_b200.h


def _dot(lib, fn, x, y, starts, w, stream, work=None):
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    n = x.numel()
    if fn == "noalloc":
        st = lib.tnb_weighted_dot_noalloc(x.data_ptr(), y.data_ptr(), n, starts.data_ptr(),
                                          w.data_ptr(), w.numel(), out.data_ptr(), stream)
    else:
        st = lib.tnb_weighted_dot(x.data_ptr(), y.data_ptr(), n, starts.data_ptr(),
                                  w.data_ptr(), w.numel(), work.data_ptr(), out.data_ptr(), stream)
    assert st == 0, lib.tnb_last_error()
    torch.cuda.synchronize()
    return out.item()


@pytest.mark.parametrize("n", [1, 2047, 40_540, 387_756, MAX_N])
def test_noalloc_dot_matches_allocating_dot_twice(n):
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    cuts = sorted({0, n // 5, n // 2, n})
    starts = torch.tensor(cuts, dtype=torch.int64, device="cuda")
    w = torch.tensor([float(k + 1) for k in range(len(cuts) - 1)], dtype=torch.float64,
                     device="cuda")
    work = torch.zeros(lib.tnb_dot_work_bytes(n), dtype=torch.uint8, device="cuda")
    want = _dot(lib, "alloc", x, y, starts, w, stream, work)
    for _ in range(2):
        got = _dot(lib, "noalloc", x, y, starts, w, stream)
        assert got == pytest.approx(want, rel=1e-12, abs=1e-12)
    # after a different call in between, the shared scratch still starts clean
    got = _dot(lib, "noalloc", y, x, starts, w, stream)
    assert got == pytest.approx(want, rel=1e-12, abs=1e-12)


def test_noalloc_dot_refuses_n_beyond_its_scratch():
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    starts = torch.tensor([0, 1], dtype=torch.int64, device="cuda")
    # refused on the host before any launch, so the pointers are never dereferenced
    st = lib.tnb_weighted_dot_noalloc(one.data_ptr(), one.data_ptr(), MAX_N + 1,
                                      starts.data_ptr(), one.data_ptr(), 1, out.data_ptr(),
                                      stream)
    assert st == 1
    assert b"exceeds the allocation-free maximum" in lib.tnb_last_error()
