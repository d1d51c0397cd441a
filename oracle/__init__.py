"""CPU oracle (test infrastructure only): a NumPy restatement of the reference's path.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this package.
"""
from .oracle import Oracle, centred_fft, centred_ifft, resize, transform_grids  # noqa: F401
