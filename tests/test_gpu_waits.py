"""Bounded barrier waits: a wait that nothing completes gives up, records its fault bit, and
the context stays usable."""
import ctypes
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_selftest_wait_runs_out_and_context_survives():
    from motionest import _lib
    lib = _lib.load()
    torch.cuda.init()
    assert _lib.wait_status() == 0
    _lib.check(lib.me_wait_selftest(1 << 20, _lib.stream_ptr()))
    assert _lib.wait_status() == _lib.ME_WAIT_SELFTEST
    assert _lib.wait_status() == 0  # read-and-clear
    # the device still computes: an FFT along y against torch's
    x = torch.randn(4, 6, 8, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    lay = _lib.layout_of(x)
    _lib.call("me_fft_axis", _lib.ptr(x), 0, _lib.ptr(y), 0, 1, 4, 6, 8, lay, 1, 0,
              _lib.stream_ptr())
    ref = torch.fft.fft(x, dim=1, norm="ortho")
    torch.testing.assert_close(y, ref, rtol=1e-5, atol=1e-5)


def test_selftest_rejects_bad_limit():
    from motionest import _lib
    with pytest.raises(ValueError):
        _lib.check(_lib.load().me_wait_selftest(0, _lib.stream_ptr()))
