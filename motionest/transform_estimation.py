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


_GA = {"reference": _lib.ME_GA_REFERENCE, "intended": _lib.ME_GA_INTENDED}
GA_EPS = 1e-4  # the finite-difference step of transform_estimation.py:77


class LMState:
    """Device buffers of the per-shot LM step (float64 transforms, damping, flags)."""

    def __init__(self, nshots, device):
        self.stats = torch.empty((nshots, 28), dtype=torch.float64, device=device)
        self.t_next = torch.empty((nshots, 6), dtype=torch.float64, device=device)
        self.e1 = torch.empty(nshots, dtype=torch.float64, device=device)
        self.mean = torch.empty(6, dtype=torch.float64, device=device)


def geodesic_step(pb, x, t, damp, state, jac_mode, ga_mode, eps=GA_EPS):
    """Replace the LM proposal in state.t_next by its geodesic-accelerated form
    (transform_estimation.py:75-121): with v = t_next - t, a = (H + damp I)^-1 rhs where
    rhs = -J^T (J(t + eps v) v - J(t) v) / eps, and the step v + a / 2 when |a| <= |v|
    (else v).  ga_mode 'reference' forms J(t + eps v) v as the reference's loop leaves it (see
    me_lm_ga_rhs); 'intended' as the sum over the six partials."""
    v = state.t_next - t
    t_eps = (t + eps * v).contiguous()
    lib = _lib.load()
    need = lib.me_lm_ga_workspace_bytes(pb.ref, pb.lm_batch)
    if need < 0:
        raise ValueError(lib.me_last_error().decode())
    work = torch.empty(int(need), dtype=torch.uint8, device=x.device)
    rhs = torch.empty((pb.nshots, 6), dtype=torch.float64, device=x.device)
    st = _lib.stream_ptr()
    _lib.call("me_lm_ga_rhs", pb.ref, ptr(x), int(jac_mode), _GA[ga_mode], ptr(t_eps),
              ptr(v.contiguous()), float(eps), ptr(rhs), pb.lm_batch, ptr(work), st)
    del work
    # a = (H + damp I)^-1 rhs with the same damped LU solve as the proposal: propose from
    # t = 0 with g = -rhs gives 0 - (H + damp I)^-1 (-rhs)
    st_a = state.stats.clone()
    st_a[:, 1:7] = -rhs
    zeros = torch.zeros_like(t)
    a = torch.empty_like(t)
    _lib.call("me_lm_propose", ptr(st_a), ptr(damp), ptr(zeros), ptr(a), pb.nshots, st)
    keep = torch.linalg.vector_norm(a, dim=1) <= torch.linalg.vector_norm(v, dim=1)
    v_ga = torch.where(keep[:, None], v + 0.5 * a, v)
    state.t_next.copy_(t + v_ga)
    return keep


def lm_step(pb, x, t, damp, flags, state, jacobian="reference", tol=1e-6, out=None,
            use_ga=False, ga_mode="reference"):
    """One sweep of estimate_transform over all shots (shots are independent given the image,
    so they are processed as a batch), then mean removal.  Updates t, damp, flags in place and
    returns T(mean) x (zxy).  No host synchronisation.  use_ga adds the geodesic acceleration
    of transform_estimation.py:75-121 to every shot's proposal."""
    mode = _JAC[jacobian]
    pb.set_transforms(t)
    pb.lm_stats(x, mode, out=state.stats)
    st = _lib.stream_ptr()
    _lib.call("me_lm_propose", ptr(state.stats), ptr(damp), ptr(t), ptr(state.t_next),
              pb.nshots, st)
    if use_ga:
        geodesic_step(pb, x, t, damp, state, mode, ga_mode)
    pb.residual_norms(x, state.t_next, out=state.e1)
    _lib.call("me_lm_accept", ptr(state.stats), ptr(state.e1), ptr(t), ptr(state.t_next),
              ptr(damp), ptr(flags), float(tol), ptr(state.mean), pb.nshots, st)
    out = torch.empty_like(x) if out is None else out
    pb.apply_transform(x, state.mean, out=out)
    return out


def estimate_transform(ksp, mps, shot_mask, image, kgrid, rkgrid, damp, convergence_flags,
                       residual_buf=None, partial_buf=None, gradient_buf=None, hessian_buf=None,
                       transforms=None, max_iter=10, tol=1e-6, use_ga=False,
                       jacobian="reference", lm_batch=None, ga_mode="reference"):
    """Estimate each shot's rigid transform by one damped Gauss-Newton (LM) step.

    Same contract as the reference: `transforms`, `damp` and `convergence_flags` are updated in
    place, and the image transformed by the mean transform is returned (the mean is removed
    from `transforms`).  The reference's scratch buffers (residual_buf, partial_buf,
    gradient_buf, hessian_buf) are accepted and unused: nothing of size [6, C, X, Y, Z] is
    materialised.  Like the reference, max_iter does not repeat the sweep.  jacobian='exact'
    (extra) uses the true derivative of the applied transform instead of the reference's.

    use_ga=True adds geodesic acceleration (transform_estimation.py:75-121).  ga_mode='reference'
    (default) reproduces the reference's branch as written, including its accumulator that each
    partial overwrites; ga_mode='intended' (extra) sums J(t + eps v) v over all six partials."""
    if ga_mode not in _GA:
        raise ValueError("ga_mode must be 'reference' or 'intended'")
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
    out = lm_step(pb, x, t, d, f, LMState(S, dev), jacobian=jacobian, tol=tol, use_ga=use_ga,
                  ga_mode=ga_mode)
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
