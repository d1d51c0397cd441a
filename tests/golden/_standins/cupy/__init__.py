"""NumPy-backed stand-in for the parts of CuPy the reference calls (test support only)."""
import sys as _sys

import numpy as _np
from numpy import *  # noqa: F401,F403
from numpy import fft, linalg, random  # noqa: F401

ndarray = _np.ndarray


def get_array_module(*args):
    # Returning this module (not numpy) makes `xp is cp` true inside the reference,
    # which routes its FFTs through cupyx.scipy.fft (the stand-in below).
    return _sys.modules[__name__]


def asnumpy(a, *args, **kwargs):
    return _np.asarray(a)


def asarray(a, dtype=None):
    return _np.asarray(a, dtype=dtype)
