"""The allocation-free inner product, me_dot_re_noalloc, against me_dot_re.

me_dot_re_noalloc exists for callers that cannot allocate device memory (a host runtime that
owns all GPU memory, or a serving process that may not allocate once it is running): its
partial sums live in a static array inside libmotionest.so.  This file is
collected last so that, if it fails, a run that stops at the first failure has already run
every other test.  It passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _dot_pair(lib, a, b, work):
    ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = a.numel()
    assert lib.me_dot_re(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                         ctypes.c_void_p(ref.data_ptr()), n, ctypes.c_void_p(work.data_ptr()),
                         st) == 0
    assert lib.me_dot_re_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                                 ctypes.c_void_p(got.data_ptr()), n, st) == 0
    torch.cuda.synchronize()
    return float(ref.item()), float(got.item())


def test_noalloc_dot_matches_allocating_dot_twice():
    from motionest import _lib
    lib = _lib.load()
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(7)
    work = torch.empty(lib.me_cg_workspace_bytes(1 << 22), dtype=torch.uint8, device="cuda")
    # two calls in a row with different sizes: the second must not see the first's partials
    for n in (3_000_001, 70_000):
        a = torch.randn(n, dtype=torch.complex64, device="cuda", generator=g)
        b = torch.randn(n, dtype=torch.complex64, device="cuda", generator=g)
        ref, got = _dot_pair(lib, a, b, work)
        exact = float(np.vdot(a.cpu().numpy().astype(np.complex128),
                              b.cpu().numpy().astype(np.complex128)).real)
        assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (n, got, ref)
        assert abs(got - exact) <= 1e-9 * max(1.0, abs(exact)), (n, got, exact)


def test_noalloc_dot_rejects_oversize():
    from motionest import _lib
    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    a = torch.zeros(4, dtype=torch.complex64, device="cuda")
    n = (1 << 28) + 1
    rc = lib.me_dot_re_noalloc(ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(a.data_ptr()),
                               ctypes.c_void_p(out.data_ptr()), n, None)
    assert rc == 1
    assert b"ME_NOALLOC_DOT_MAX_N" in lib.me_last_error()
