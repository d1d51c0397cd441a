"""cupyx.scipy.fft stand-in: forwards to scipy.fft (test support only)."""
from scipy.fft import fft, fftn, ifft, ifftn  # noqa: F401
