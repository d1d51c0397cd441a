"""Levenberg-Marquardt motion step with the reference's interface
(transform_estimation.py:7-151)."""
import numpy as np
import torch

from . import _lib
from ._arrays import like_input, to_device
from ._lib import ptr
from .image_estimation import _host_mask
from .problem import SenseProblem, xyz_to_zxy, zxy_to_xyz

_JAC = {"reference": _lib.ME_JAC_REFERENCE, "exact": _lib.ME_JAC_EXACT}


class LMState:
    """Device buffers of the per-shot LM step (float64 transforms, damping, flags)."""

    def __init__(self, nshots, device):
        self.stats = torch.empty((nshots, 28), dtype=torch.float64, device=device)
        self.t_next = torch.empty((nshots, 6), dtype=torch.float64, device=device)
        self.e1 = torch.empty(nshots, dtype=torch.float64, device=device)
        self.mean = torch.empty(6, dtype=torch.float64, device=device)


def lm_step(pb, x, t, damp, flags, state, jacobian="reference", tol=1e-6, out=None):
    """One sweep of estimate_transform over all shots (shots are independent given the image,
    so they are processed as a batch), then mean removal.  Updates t, damp, flags in place and
    returns T(mean) x (zxy).  No host synchronisation."""
    mode = _JAC[jacobian]
    pb.set_transforms(t)
    pb.lm_stats(x, mode, out=state.stats)
    st = _lib.stream_ptr()
    _lib.call("me_lm_propose", ptr(state.stats), ptr(damp), ptr(t), ptr(state.t_next),
              pb.nshots, st)
    pb.residual_norms(x, state.t_next, out=state.e1)
    _lib.call("me_lm_accept", ptr(state.stats), ptr(state.e1), ptr(t), ptr(state.t_next),
              ptr(damp), ptr(flags), float(tol), ptr(state.mean), pb.nshots, st)
    out = torch.empty_like(x) if out is None else out
    pb.apply_transform(x, state.mean, out=out)
    return out


def estimate_transform(ksp, mps, shot_mask, image, kgrid, rkgrid, damp, convergence_flags,
                       residual_buf=None, partial_buf=None, gradient_buf=None, hessian_buf=None,
                       transforms=None, max_iter=10, tol=1e-6, use_ga=False,
                       jacobian="reference", lm_batch=None):
    """Estimate each shot's rigid transform by one damped Gauss-Newton (LM) step.

    Same contract as the reference: `transforms`, `damp` and `convergence_flags` are updated in
    place, and the image transformed by the mean transform is returned (the mean is removed
    from `transforms`).  The reference's scratch buffers (residual_buf, partial_buf,
    gradient_buf, hessian_buf) are accepted and unused: nothing of size [6, C, X, Y, Z] is
    materialised.  Like the reference, max_iter does not repeat the sweep.  jacobian='exact'
    (extra) uses the true derivative of the applied transform instead of the reference's."""
    if use_ga:
        raise NotImplementedError("geodesic acceleration (use_ga=True) is not implemented")
    _lib.require_cuda()
    ksp_t = to_device(ksp, torch.complex64)
    mps_t = to_device(mps, torch.complex64)
    planes = _host_mask(shot_mask)
    S = planes.shape[0]
    dev = ksp_t.device
    t_host = transforms
    if transforms is None:
        transforms = np.zeros((S, 6))
    t = to_device(np.asarray(transforms, dtype=np.float64) if not isinstance(transforms, torch.Tensor)
                  else transforms, torch.float64).clone()
    d = to_device(np.asarray(damp, dtype=np.float64) if not isinstance(damp, torch.Tensor)
                  else damp, torch.float64).clone()
    f = to_device(np.asarray(convergence_flags).astype(np.uint8)
                  if not isinstance(convergence_flags, torch.Tensor)
                  else convergence_flags.to(torch.uint8), torch.uint8).clone()
    pb = SenseProblem(ksp_t, mps_t, planes, kgrid, rkgrid, t, lm_batch=lm_batch)
    x = xyz_to_zxy(to_device(image, torch.complex64))
    out = lm_step(pb, x, t, d, f, LMState(S, dev), jacobian=jacobian, tol=tol)
    _write_back(transforms if t_host is not None else None, t)
    _write_back(damp, d)
    _write_back(convergence_flags, f.to(torch.bool))
    return like_input(zxy_to_xyz(out), image)


def _write_back(dst, src):
    if dst is None:
        return
    if isinstance(dst, np.ndarray):
        np.copyto(dst, src.cpu().numpy().astype(dst.dtype))
    elif isinstance(dst, torch.Tensor):
        dst.copy_(src.to(dst.dtype))
    elif hasattr(dst, "set"):  # CuPy
        dst.set(src.cpu().numpy().astype(dst.dtype))
    else:
        dst[...] = src.cpu().numpy()
