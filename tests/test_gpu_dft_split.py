"""The split-precision tensor-core row DFT (me_dft_rows_split) against FP64 (numpy) and the
register FFT (me_fft_axis along the contiguous axis): relative L2 error per transform <= 2e-6
against FP64, forward and inverse, for the line lengths it supports."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [192, 224, 256])
@pytest.mark.parametrize("inverse", [0, 1])
def test_split_dft_vs_fp64(n, inverse):
    from motionest import _lib
    rows = 1000  # not a multiple of the 8-row tile
    rng = np.random.default_rng(n + inverse)
    x = (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))).astype(np.complex64)
    xd = torch.tensor(x, device="cuda")
    out = torch.empty_like(xd)
    _lib.call("me_dft_rows_split", _lib.ptr(xd), _lib.ptr(out), rows, n, inverse,
              _lib.stream_ptr())
    ref = (np.fft.ifft if inverse else np.fft.fft)(x.astype(np.complex128), axis=1, norm="ortho")
    err = np.linalg.norm(out.cpu().numpy() - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() <= 2e-6, err.max()
    # the register FFT on the same rows (one volume of rows x n x 1, FFT along y)
    fo = torch.empty_like(xd)
    lay = _lib.MeLayout(n, 1, 1)
    _lib.call("me_fft_axis", _lib.ptr(xd), 0, _lib.ptr(fo), 0, 1, rows, n, 1, lay, 1, inverse,
              _lib.stream_ptr())
    err_reg = np.linalg.norm(fo.cpu().numpy() - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err_reg.max() <= 2e-6


def test_split_dft_rejects_other_lengths():
    from motionest import _lib
    x = torch.zeros(16 * 176, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    rc = _lib.load().me_dft_rows_split(_lib.ptr(x), _lib.ptr(y), 16, 176, 0, _lib.stream_ptr())
    assert rc == 3  # ME_ERR_UNSUPPORTED
