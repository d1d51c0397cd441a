"""Rigid-transform operators with the reference's interface (transform.py:243-504).

RigidTransformCudaOptimzied(parameters, kgrid, rkgrid, inverse=False).apply(x, out=None) /
.adjoint(x, out=None) and RigidTransformDerivativeCuda(shape, parameters, kgrid, rkgrid)
.apply(x, p_idx), on hand-written sm_100a kernels (libmotionest.so).  Inputs are uncentred
[X, Y, Z] complex64 volumes (NumPy, torch CUDA or any __dlpack__ CUDA array); results come
back as the caller's array kind.
"""
import numpy as np
import torch

from . import _lib
from ._arrays import as_float64_host, is_numpy, like_input, to_device
from .utils import device_grid

_JAC_MODES = {"reference": _lib.ME_JAC_REFERENCE, "exact": _lib.ME_JAC_EXACT}


def _params_dev(parameters):
    p = as_float64_host(parameters).reshape(-1)
    if p.size != 6:
        raise ValueError("rigid parameters must have 6 entries (tx, ty, tz, rx, ry, rz)")
    return torch.as_tensor(p, dtype=torch.float64).cuda()


def _volume(x):
    t = to_device(x, torch.complex64)
    if t.dim() != 3:
        raise ValueError(f"expected an [X, Y, Z] volume, got shape {tuple(t.shape)}")
    return t


class RigidTransformCudaOptimzied:
    """Rigid-body 3-D transform: three-shear rotations about x, y, z then a translation.

    apply: T x = Tr . Rz . Ry . Rx x (transform.py:263-318).  adjoint: T^H (transform.py:320-377).
    As in the reference, `inverse` conjugates only the translation ramp, and passing `out`
    transforms `out` in place and ignores `x` (transform.py:265)."""

    def __init__(self, parameters, kgrid, rkgrid, inverse=False):
        self.params = parameters
        self.kgrid = kgrid
        self.rkgrid = rkgrid
        self.inverse = inverse

    def _run(self, x, out, adjoint):
        _lib.require_cuda()
        src = _volume(out if out is not None else x)
        grid = device_grid(self.kgrid, self.rkgrid, src.shape)
        prm = _params_dev(self.params)
        if out is not None and isinstance(out, torch.Tensor) and out.is_cuda and \
                out.dtype == torch.complex64 and out.is_contiguous():
            dst = out
        else:
            dst = torch.empty_like(src)
        st = _lib.stream_ptr()
        if adjoint:
            _lib.call("me_rigid_adjoint", _lib.ptr(src), 0, _lib.ptr(dst), 0, 1,
                      _lib.layout_of(src), grid.ref, _lib.ptr(prm), 0, 0, st)
        else:
            _lib.call("me_rigid_apply", _lib.ptr(src), 0, _lib.ptr(dst), 0, 1,
                      _lib.layout_of(src), grid.ref, _lib.ptr(prm), 0, int(bool(self.inverse)),
                      st)
        ref = out if out is not None else x
        if is_numpy(ref) and out is not None:
            np.copyto(out, dst.cpu().numpy())
            return out
        return like_input(dst, ref)

    def apply(self, x, out=None):
        return self._run(x, out, adjoint=False)

    def adjoint(self, x, out=None):
        return self._run(x, out, adjoint=True)


class RigidTransformDerivativeCuda:
    """Partial derivatives of the rigid transform (transform.py:379-504).

    apply(x, p_idx) returns dT/dparams[p_idx] x.  With jacobian='reference' (the default) this is
    the reference's convention, the derivative of Tr . Rx . Ry . Rz (z rotated first,
    transform.py:480-502), which is NOT the derivative of RigidTransformCudaOptimzied.apply;
    jacobian='exact' differentiates the operator apply implements.  p_idx outside 0..5 returns a
    copy of x, as the reference does."""

    def __init__(self, shape, parameters, kgrid, rkgrid, jacobian="reference"):
        if jacobian not in _JAC_MODES:
            raise ValueError("jacobian must be 'reference' or 'exact'")
        self.shape = tuple(shape)
        self.parameters = parameters
        self.kgrid = kgrid
        self.rkgrid = rkgrid
        self.mode = _JAC_MODES[jacobian]
        self._work = None

    def _workspace(self, dev):
        nbytes = _lib.load().me_rigid_jacobian_workspace_bytes(*self.shape)
        if self._work is None or self._work.numel() < nbytes:
            self._work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        return self._work

    def apply(self, input, p_idx):
        _lib.require_cuda()
        src = _volume(input)
        if tuple(src.shape) != self.shape:
            raise ValueError(f"input shape {tuple(src.shape)} != operator shape {self.shape}")
        grid = device_grid(self.kgrid, self.rkgrid, src.shape)
        prm = _params_dev(self.parameters)
        dst = torch.empty_like(src)
        _lib.call("me_rigid_derivative", _lib.ptr(src), _lib.ptr(dst), _lib.layout_of(src),
                  grid.ref, _lib.ptr(prm), int(p_idx), self.mode,
                  _lib.ptr(self._workspace(src.device)), _lib.stream_ptr())
        return like_input(dst, input)

    def jacobian(self, input):
        """[7, X, Y, Z]: T x followed by the six partials (one sweep sharing the rotation
        prefixes)."""
        _lib.require_cuda()
        src = _volume(input)
        grid = device_grid(self.kgrid, self.rkgrid, src.shape)
        prm = _params_dev(self.parameters)
        dst = torch.empty((7,) + tuple(src.shape), dtype=torch.complex64, device=src.device)
        _lib.call("me_rigid_jacobian", _lib.ptr(src), _lib.ptr(dst), src.numel(),
                  _lib.layout_of(src), grid.ref, _lib.ptr(prm), self.mode,
                  _lib.ptr(self._workspace(src.device)), _lib.stream_ptr())
        return like_input(dst, input)
