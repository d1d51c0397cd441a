"""Autograd of the forward-model loss 0.5 sum_s ||M_s F C T(theta_s) x - y_s||^2 on the CUDA
kernels, checked against FP64 central finite differences of the oracle (h = 1e-3 degree for
rotations, 1e-3 voxel for translations) and, for jacobian='reference', against the oracle's
restatement of the reference's RigidTransformDerivativeCuda."""
import numpy as np
import pytest
import torch

from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O64 = Oracle(np.complex128)


def _case(seed=3):
    from motionest.sampling import disorder_masks
    from motionest.simulation import coil_maps, phantom
    shape = (24, 20, 12)
    rng = np.random.default_rng(seed)
    mps = np.fft.ifftshift(coil_maps(shape, 3, seed=seed, unit_rss=False).cpu().numpy(),
                           axes=(-3, -2, -1))
    planes = np.fft.ifftshift(disorder_masks(24, 20, (4, 4), 1, 4)[..., 0], axes=(-2, -1))
    mask = planes[..., None]
    x_true = np.fft.ifftshift(phantom(shape, 5, seed=seed).cpu().numpy())
    t_true = np.zeros((4, 6))
    t_true[:, :3] = rng.uniform(-1.5, 1.5, (4, 3))
    t_true[:, 3:] = np.deg2rad(rng.uniform(-4, 4, (4, 3)))
    kg, rk = transform_grids(shape, [1, 1, 1])
    ksp = sum(O64.fft(mps * O64.rigid_apply(x_true, t_true[s], kg, rk), (-3, -2, -1)) * mask[s]
              for s in range(4)).astype(np.complex64)
    x = (x_true + 0.05 * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)))
    t = t_true + np.concatenate([rng.normal(0, 0.3, (4, 3)),
                                 np.deg2rad(rng.normal(0, 1.0, (4, 3)))], axis=1)
    return dict(shape=shape, mps=mps, mask=mask, ksp=ksp, x=x.astype(np.complex64), t=t,
                kg=kg, rk=rk)


def _oracle_loss(c, x, t):
    return 0.5 * sum(float(np.vdot(r, r).real) for r in (
        O64.forward_residual(c["ksp"].astype(np.complex128), c["mps"].astype(np.complex128),
                             c["mask"][s], x, t[s], c["kg"], c["rk"]) for s in range(4)))


def _grads(c, jacobian):
    from motionest.autograd import ForwardModel
    fm = ForwardModel(c["ksp"], c["mps"], c["mask"], c["kg"], c["rk"], jacobian=jacobian)
    x = torch.tensor(c["x"], device="cuda", requires_grad=True)
    t = torch.tensor(c["t"], device="cuda", requires_grad=True)
    loss = fm.loss(x, t)
    loss.backward()
    return float(loss.item()), x.grad.cpu().numpy(), t.grad.cpu().numpy()


def test_loss_matches_fp64_oracle():
    c = _case()
    loss, _, _ = _grads(c, "exact")
    ref = _oracle_loss(c, c["x"].astype(np.complex128), c["t"])
    assert abs(loss - ref) / ref < 1e-5


def test_theta_gradient_vs_fp64_central_differences():
    c = _case()
    _, _, gt = _grads(c, "exact")
    x = c["x"].astype(np.complex128)
    for s in range(4):
        for p in range(6):
            h = 1e-3 if p < 3 else np.deg2rad(1e-3)
            tp, tm = c["t"].copy(), c["t"].copy()
            tp[s, p] += h
            tm[s, p] -= h
            fd = (_oracle_loss(c, x, tp) - _oracle_loss(c, x, tm)) / (2 * h)
            scale = np.abs(gt[s]).max()
            assert abs(gt[s, p] - fd) <= 2e-3 * scale + 1e-6, (s, p, gt[s, p], fd)


def test_image_gradient_vs_fp64_central_differences():
    c = _case()
    _, gx, _ = _grads(c, "exact")
    rng = np.random.default_rng(11)
    x = c["x"].astype(np.complex128)
    for _ in range(3):
        v = rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)
        eps = 1e-4
        fd = (_oracle_loss(c, x + eps * v, c["t"]) - _oracle_loss(c, x - eps * v, c["t"])) / (2 * eps)
        an = float(np.vdot(gx.astype(np.complex128), v).real)
        assert abs(an - fd) <= 1e-4 * abs(fd) + 1e-6, (an, fd)


def test_reference_convention_gradient_vs_reference_derivative():
    """jacobian='reference' gives Re<r, M F C dT_ref/dp x> with the reference's derivative."""
    c = _case()
    _, _, gt = _grads(c, "reference")
    x = c["x"].astype(np.complex128)
    ksp = c["ksp"].astype(np.complex128)
    mps = c["mps"].astype(np.complex128)
    for s in range(4):
        r = O64.forward_residual(ksp, mps, c["mask"][s], x, c["t"][s], c["kg"], c["rk"])
        J = O64.jacobian(ksp.shape, mps, c["mask"][s], x, c["t"][s], c["kg"], c["rk"],
                         "reference")
        g = np.array([np.vdot(r, J[p]).real for p in range(6)])
        np.testing.assert_allclose(gt[s], g, rtol=1e-4, atol=1e-4 * np.abs(g).max())


@pytest.mark.parametrize("jacobian", ["reference", "exact"])
def test_gradient_only_statistics_match_full_statistics(jacobian):
    """me_lm_gradient (image-space <C^H F^H M r, dT/dp x>) against the gradient entries of the
    full Gauss-Newton statistics (k-space <r, M F C dT/dp x>): the same numbers by adjointness,
    to FP32 rounding."""
    from motionest.autograd import _MODES, ForwardModel
    c = _case()
    fm = ForwardModel(c["ksp"], c["mps"], c["mask"], c["kg"], c["rk"], jacobian=jacobian)
    pb = fm.pb
    pb.set_transforms(torch.tensor(c["t"], device="cuda"))
    x = torch.tensor(c["x"], device="cuda").permute(2, 0, 1).contiguous()
    full = pb.lm_stats(x, _MODES[jacobian]).cpu().numpy()
    grad = pb.lm_gradient(x, _MODES[jacobian]).cpu().numpy()
    np.testing.assert_allclose(grad[:, 0], full[:, 0], rtol=1e-6)
    scale = np.abs(full[:, 1:7]).max()
    np.testing.assert_allclose(grad[:, 1:7], full[:, 1:7], rtol=1e-4, atol=1e-5 * scale)
