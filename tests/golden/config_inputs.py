"""Inputs of the 64x64x48 / 8-coil / 16-shot JointRecon fixture (``config0.npz``).

The fixture pins the CUDA reconstruction against the reference's own JointRecon on the small
workload it runs on CPU: a seeded phantom of 10 ellipsoids, 8 Gaussian-bump coils on a ring
normalised to unit root-sum-of-squares, 16 shots of DISORDER 4x4 tiles at accel 1, uniform
random motion (rotations U[-3, 3] degrees, translations U[-2, 2] voxels) and complex Gaussian
noise of 1e-3 max|k|, reconstructed with 10 outer iterations of 5 CG iterations and one LM step.

What is stored and what is rebuilt:
- k-space is stored (it comes from the reference's forward model plus noise), quantised to
  float16 real and imaginary parts with a power-of-two scale, so that the stored values ARE the
  input: both the reference run and the tests read exactly these numbers;
- the coil maps are rebuilt by ``coil_maps`` below, which uses only IEEE-754 basic operations
  (+, -, *, /, sqrt, floor) in float64 and an explicit summation order, so it gives the same
  bits on every machine; the fixture keeps a SHA-256 of the maps to prove it;
- the masks are the reference's DISORDER masks (stored packed).
"""
import hashlib

import numpy as np

SHAPE = (64, 64, 48)
NCOILS = 8
NSHOTS = 16
TILE = (4, 4)
ACCEL = 1
CG_ITERS = 5
OUTER_ITERS = 10
TWO_PI = 6.283185307179586


def _exp(u):
    """exp(u) for float64 arrays with |u| <= 64, by exp(u / 2^10)^(2^10) with a 12-term
    Taylor series for the reduced argument (basic operations only)."""
    v = u / 1024.0
    term = np.ones_like(v)
    acc = np.ones_like(v)
    for n in range(1, 13):
        term = term * v / float(n)
        acc = acc + term
    for _ in range(10):
        acc = acc * acc
    return acc


def _cos_sin(theta):
    """(cos, sin) of float64 arrays: reduce to [-pi, pi], halve 8 times, Taylor series, then
    the double-angle formulas (basic operations only)."""
    th = theta - TWO_PI * np.floor(theta / TWO_PI + 0.5)
    v = th / 256.0
    v2 = v * v
    c = 1.0 - v2 / 2.0 + v2 * v2 / 24.0 - v2 * v2 * v2 / 720.0
    s = v - v * v2 / 6.0 + v * v2 * v2 / 120.0 - v * v2 * v2 * v2 / 5040.0
    for _ in range(8):
        c, s = c * c - s * s, 2.0 * s * c
    return c, s


def _grid(n):
    return -1.0 + 2.0 * np.arange(n, dtype=np.float64) / float(n - 1)


def coil_maps(shape=SHAPE, ncoils=NCOILS):
    """Centred [C, X, Y, Z] complex64 Gaussian-bump sensitivities centred on a ring of radius
    1.2 in the x-y plane, width 0.9, with the ring angle plus 0.4 z as phase, normalised to
    unit root-sum-of-squares."""
    X, Y, Z = shape
    gx = _grid(X).reshape(X, 1, 1)
    gy = _grid(Y).reshape(1, Y, 1)
    gz = _grid(Z).reshape(1, 1, Z)
    re, im = [], []
    for c in range(ncoils):
        a = np.array(TWO_PI * c / ncoils)
        ca, sa = _cos_sin(a)
        cx, cy = 1.2 * float(ca), 1.2 * float(sa)
        d2 = (gx - cx) * (gx - cx) + (gy - cy) * (gy - cy) + 0.6 * gz * gz
        mag = _exp(-d2 / 0.9) * np.ones((1, 1, Z))
        pc, ps = _cos_sin(float(a) + 0.4 * gz)
        re.append(mag * pc)
        im.append(mag * ps)
    rss = re[0] * re[0] + im[0] * im[0]
    for c in range(1, ncoils):
        rss = rss + (re[c] * re[c] + im[c] * im[c])
    rss = np.sqrt(rss)
    out = np.empty((ncoils,) + tuple(shape), np.complex64)
    for c in range(ncoils):
        out[c].real = (re[c] / rss).astype(np.float32)
        out[c].imag = (im[c] / rss).astype(np.float32)
    return out


def digest(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def quantise_kspace(ksp):
    """(float16 [C, X, Y, Z, 2], power-of-two scale): ksp / scale rounded to float16."""
    peak = float(np.max(np.abs(ksp.view(np.float32))))
    scale = 2.0 ** np.ceil(np.log2(peak / 32768.0))
    q = (ksp.view(np.float32).reshape(ksp.shape + (2,)) / np.float32(scale)).astype(np.float16)
    return q, np.float32(scale)


def dequantise_kspace(q, scale):
    """The complex64 k-space the fixture stands for (exact: scale is a power of two)."""
    f = q.astype(np.float32) * np.float32(scale)
    return np.ascontiguousarray(f).view(np.complex64).reshape(q.shape[:-1])


def load(golden_dir):
    """(ksp, mps, masks [S, X, Y, 1], fixture dict) with the maps rebuilt and checked."""
    d = dict(np.load(golden_dir / "config0.npz"))
    mps = coil_maps()
    if not np.array_equal(digest(mps), d["mps_sha256"]):
        raise RuntimeError("rebuilt coil maps differ from the ones the reference ran on")
    ksp = dequantise_kspace(d["ksp_f16"], d["ksp_scale"])
    S, X, Y = NSHOTS, SHAPE[0], SHAPE[1]
    masks = np.unpackbits(d["mask_packed"])[:S * X * Y].reshape(S, X, Y, 1).astype(bool)
    return ksp, mps, masks, d
