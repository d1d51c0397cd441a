"""Minimal SigPy stand-in (test support only).

Restates, from SigPy's documented behaviour, only what the reference's hot path calls:
get_array_module, centred orthonormal fft/ifft, centred resize, and stubs for the Linop
base class and the Device objects that are touched at import time.
"""
import sys as _sys

import numpy as _np

from . import linop, mri, plot  # noqa: F401


def get_array_module(*args):
    return _sys.modules["cupy"]


class Device:
    def __init__(self, device_id=-1):
        self.id = device_id
        self.xp = _np

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


cpu_device = Device(-1)


def to_device(x, device=None):
    return _np.asarray(x)


def _norm_axes(axes, ndim):
    if axes is None:
        return tuple(range(ndim))
    return tuple(a % ndim for a in axes)


def resize(input, oshape, ishift=None, oshift=None):
    """Centred crop / zero-pad: input offset max(i//2 - o//2, 0), output offset max(o//2 - i//2, 0)."""
    ishape = input.shape
    if tuple(ishape) == tuple(oshape):
        return input
    ishift = [max(i // 2 - o // 2, 0) for i, o in zip(ishape, oshape)] if ishift is None else ishift
    oshift = [max(o // 2 - i // 2, 0) for i, o in zip(ishape, oshape)] if oshift is None else oshift
    copy = [min(i - si, o - so) for i, si, o, so in zip(ishape, ishift, oshape, oshift)]
    out = _np.zeros(oshape, dtype=input.dtype)
    islc = tuple(slice(s, s + c) for s, c in zip(ishift, copy))
    oslc = tuple(slice(s, s + c) for s, c in zip(oshift, copy))
    out[oslc] = input[islc]
    return out


def _as_complex(x):
    x = _np.asarray(x)
    if not _np.iscomplexobj(x):
        x = x.astype(_np.complex64)
    return x


def fft(input, oshape=None, axes=None, center=True, norm="ortho"):
    x = _as_complex(input)
    ax = _norm_axes(axes, x.ndim)
    if oshape is not None:
        x = resize(x, oshape)
    if center:
        y = _np.fft.fftshift(_np.fft.fftn(_np.fft.ifftshift(x, axes=ax), axes=ax, norm=norm), axes=ax)
    else:
        y = _np.fft.fftn(x, axes=ax, norm=norm)
    return y.astype(x.dtype, copy=False)


def ifft(input, oshape=None, axes=None, center=True, norm="ortho"):
    x = _as_complex(input)
    ax = _norm_axes(axes, x.ndim)
    if oshape is not None:
        x = resize(x, oshape)
    if center:
        y = _np.fft.fftshift(_np.fft.ifftn(_np.fft.ifftshift(x, axes=ax), axes=ax, norm=norm), axes=ax)
    else:
        y = _np.fft.ifftn(x, axes=ax, norm=norm)
    return y.astype(x.dtype, copy=False)
