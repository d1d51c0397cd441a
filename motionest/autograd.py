"""Differentiable forward-model loss on the CUDA kernels.

    loss(x, theta) = 0.5 * sum_s || M_s F C T(theta_s) x - y_s ||^2

the data term of the reference's joint objective (joint_recon.py:108-115, halved), as a
torch.autograd.Function.  Backward is hand-written on the same kernels the solvers use:

  * d loss / d theta_{s,p} = Re<r_s, J_{s,p}> with r_s = M_s (F C T_s x - y_s) and
    J_{s,p} = M_s F C dT_s/dtheta_p x, computed gradient-only (me_lm_gradient) as
    Re<C^H F^H M_s r_s, dT_s/dtheta_p x> in image space: one SENSE forward and one adjoint per
    shot, no forward of the partials and no Gram matrix.  The rotation partials are
    recomputed from x and theta by the shared-prefix Jacobian sweep; nothing from the forward
    pass is stored per shot.
  * d loss / d conj(x) (torch's convention for a complex leaf: the returned gradient is
    A^H (A x - y)) = sum_s T_s^H C^H F^H M_s F C T_s x - sum_s T_s^H C^H F^H M_s y, the SENSE
    normal operator and right-hand side without the support mask.

jacobian='exact' (default) gives the true gradient of the loss; jacobian='reference' uses the
reference's RigidTransformDerivativeCuda convention (the derivative of Tr.Rx.Ry.Rz), which is
what the reference's own motion step differentiates.
"""
import numpy as np
import torch

from . import _lib
from ._arrays import to_device
from .image_estimation import _host_mask
from .problem import SenseProblem, xyz_to_zxy, zxy_to_xyz

_MODES = {"reference": _lib.ME_JAC_REFERENCE, "exact": _lib.ME_JAC_EXACT}


class _ForwardModelLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x_zxy, theta, pb, mode):
        t = theta.detach().to(torch.float64).contiguous()
        e = pb.residual_norms(x_zxy.detach(), t)
        ctx.save_for_backward(x_zxy.detach(), t)
        ctx.pb = pb
        ctx.mode = mode
        ctx.theta_dtype = theta.dtype
        return (0.5 * e.sum()).to(torch.float64)

    @staticmethod
    def backward(ctx, gout):
        x, t = ctx.saved_tensors
        pb = ctx.pb
        gx = gt = None
        if ctx.needs_input_grad[1]:
            pb.set_transforms(t)
            grad = pb.lm_gradient(x, ctx.mode)
            gt = (grad[:, 1:7] * gout).to(ctx.theta_dtype)
        if ctx.needs_input_grad[0]:
            pb.set_transforms(t)
            ax = pb.normal(x, pb.empty_image(), masked=False)
            b = pb.rhs(pb.empty_image(), masked=False)
            gx = (ax - b) * gout.to(torch.float32)
        return gx, gt, None, None


class ForwardModel:
    """The motion-corrupted SENSE forward model of one acquisition, for autograd.

    ksp, mps: uncentred [C, X, Y, Z] complex64 (as the reference's operators take them);
    shot_mask: [S, X, Y, 1] bool (uncentred); kgrid/rkgrid from compute_transform_grids_voxel."""

    def __init__(self, ksp, mps, shot_mask, kgrid, rkgrid, jacobian="exact"):
        _lib.require_cuda()
        if jacobian not in _MODES:
            raise ValueError("jacobian must be 'reference' or 'exact'")
        ksp_t = to_device(ksp, torch.complex64)
        mps_t = to_device(mps, torch.complex64)
        planes = _host_mask(shot_mask)
        self.nshots = planes.shape[0]
        t0 = torch.zeros((self.nshots, 6), dtype=torch.float64, device=ksp_t.device)
        self.pb = SenseProblem(ksp_t, mps_t, planes, kgrid, rkgrid, t0)
        self.mode = _MODES[jacobian]

    def loss(self, x, theta):
        """0.5 sum_s ||M_s F C T(theta_s) x - y_s||^2 (float64 scalar tensor).

        x: [X, Y, Z] complex64 CUDA tensor (uncentred), theta: [S, 6] CUDA tensor (radians for
        rotations); either may require grad."""
        if x.dim() != 3 or tuple(x.shape) != self.pb.shape:
            raise ValueError(f"x must be {self.pb.shape}, got {tuple(x.shape)}")
        if tuple(theta.shape) != (self.nshots, 6):
            raise ValueError(f"theta must be [{self.nshots}, 6], got {tuple(theta.shape)}")
        return _ForwardModelLoss.apply(_ToZxy.apply(x), theta, self.pb, self.mode)


class _ToZxy(torch.autograd.Function):
    """[X, Y, Z] -> the kernels' [Z, X, Y] layout, with the inverse permutation in backward."""

    @staticmethod
    def forward(ctx, x):
        return xyz_to_zxy(x.to(torch.complex64))

    @staticmethod
    def backward(ctx, g):
        return zxy_to_xyz(g)


def forward_model_loss(x, theta, ksp, mps, shot_mask, kgrid, rkgrid, jacobian="exact"):
    """One-shot convenience wrapper around ForwardModel(...).loss(x, theta)."""
    return ForwardModel(ksp, mps, shot_mask, kgrid, rkgrid, jacobian).loss(x, theta)
