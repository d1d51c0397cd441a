"""Autograd of the forward-model loss at full differentiation-workload size: 128x128x96, 16
coils, 32 shots of DISORDER 8x8 tiles (the reference's order chunked into 32 shots).

    loss(x, theta) = 0.5 sum_s ||M_s F C T(theta_s) x - y_s||^2

Checks, all against the FP64 oracle on the CPU:
- d loss / d theta on 12 sampled (shot, parameter) pairs against FP64 central differences with
  h = 1e-3 degree (rotations) and 1e-3 voxel (translations), |err| <= 2e-3 of the shot's
  largest gradient entry;
- d loss / d conj(x) along a random direction: the loss is exactly quadratic in x, so
  (L(x + e v) - L(x - e v)) / (2 e) equals Re<grad, v> for any e and no truncation error
  enters; relative error <= 1e-4;
- jacobian='reference' against the gradient built from the oracle's restatement of the
  reference's RigidTransformDerivativeCuda (explicit, materialised [6, C, X, Y, Z] columns);
- the LM statistics from Jacobian-vector products contracted in registers (no per-shot
  Jacobian volume in k-space) against the explicit-Jacobian statistics of
  transform_estimation.py:50-68 (g and the Gram matrix H), and the damped proposal of
  :60-71 from both, for sampled shots.
"""
import numpy as np
import pytest
import torch

from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

SHAPE = (128, 128, 96)
C, S = 16, 32
O64 = Oracle(np.complex128, workers=-1)


@pytest.fixture(scope="module")
def case():
    from motionest.sampling import disorder_masks
    from motionest.simulation import (add_noise, coil_maps, generate_corrupted_kspace,
                                      motion_uniform, phantom)
    X, Y, Z = SHAPE
    gt = phantom(SHAPE, 20, seed=2)
    mps = coil_maps(SHAPE, C, seed=2, unit_rss=True)
    masks = disorder_masks(X, Y, (8, 8), 1, S)
    t_true = motion_uniform(S, 3.0, 2.0, seed=2)
    ksp = add_noise(generate_corrupted_kspace(gt, mps, masks, t_true), 1e-3, seed=2)
    ax = (-3, -2, -1)
    ksp_u = np.fft.ifftshift(ksp.cpu().numpy(), axes=ax)
    mps_u = np.fft.ifftshift(mps.cpu().numpy(), axes=ax)
    mask_u = np.fft.ifftshift(masks, axes=(1, 2))
    rng = np.random.default_rng(5)
    x = np.fft.ifftshift(gt.cpu().numpy())
    x = (x + 0.05 * (rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE))).astype(
        np.complex64)
    t = t_true + np.concatenate([rng.normal(0, 0.3, (S, 3)),
                                 np.deg2rad(rng.normal(0, 1.0, (S, 3)))], axis=1)
    kg, rk = transform_grids(SHAPE, [1, 1, 1])
    return dict(ksp=ksp_u, mps=mps_u, mask=mask_u, x=x, t=t, kg=kg, rk=rk,
                ksp64=ksp_u.astype(np.complex128), mps64=mps_u.astype(np.complex128))


def _shot_loss(c, x, t_s, s):
    r = O64.forward_residual(c["ksp64"], c["mps64"], c["mask"][s], x, t_s, c["kg"], c["rk"])
    return 0.5 * float(np.vdot(r, r).real)


def _grads(c, jacobian):
    from motionest.autograd import ForwardModel
    fm = ForwardModel(c["ksp"], c["mps"], c["mask"], c["kg"], c["rk"], jacobian=jacobian)
    x = torch.tensor(c["x"], device="cuda", requires_grad=True)
    t = torch.tensor(c["t"], device="cuda", requires_grad=True)
    loss = fm.loss(x, t)
    loss.backward()
    return fm, float(loss.item()), x.grad.cpu().numpy(), t.grad.cpu().numpy()


PAIRS = [(0, 0), (5, 1), (9, 2), (13, 3), (17, 4), (21, 5),
         (24, 3), (27, 4), (31, 5), (2, 2), (11, 0), (30, 1)]


def test_theta_gradient_vs_fp64_central_differences(case):
    c = case
    _, _, _, gt = _grads(c, "exact")
    x = c["x"].astype(np.complex128)
    for s, p in PAIRS:
        h = 1e-3 if p < 3 else np.deg2rad(1e-3)
        tp, tm = c["t"][s].copy(), c["t"][s].copy()
        tp[p] += h
        tm[p] -= h
        fd = (_shot_loss(c, x, tp, s) - _shot_loss(c, x, tm, s)) / (2 * h)
        scale = np.abs(gt[s]).max()
        assert abs(gt[s, p] - fd) <= 2e-3 * scale, (s, p, gt[s, p], fd)


def test_image_gradient_directional_vs_fp64(case):
    c = case
    _, loss, gx, _ = _grads(c, "exact")
    rng = np.random.default_rng(17)
    x = c["x"].astype(np.complex128)
    v = rng.standard_normal(SHAPE) + 1j * rng.standard_normal(SHAPE)
    eps = 0.1 * np.linalg.norm(x) / np.linalg.norm(v)
    lp = sum(_shot_loss(c, x + eps * v, c["t"][s], s) for s in range(S))
    lm = sum(_shot_loss(c, x - eps * v, c["t"][s], s) for s in range(S))
    fd = (lp - lm) / (2 * eps)
    an = float(np.vdot(gx.astype(np.complex128), v).real)
    assert abs(an - fd) <= 1e-4 * abs(fd), (an, fd)


SHOTS = (4, 26)


def test_reference_gradient_and_lm_statistics_vs_explicit_jacobian(case):
    """Gradient in the reference's derivative convention, and the LM normal equations formed
    from JVPs, against the explicit [6, C, X, Y, Z] Jacobian of transform_estimation.py:50-68."""
    c = case
    fm, _, _, gt = _grads(c, "reference")
    pb = fm.pb
    pb.set_transforms(torch.tensor(c["t"], device="cuda"))
    x_zxy = torch.tensor(c["x"], device="cuda").permute(2, 0, 1).contiguous()
    stats = pb.lm_stats(x_zxy, fm.mode).cpu().numpy()
    x = c["x"].astype(np.complex128)
    iu = np.triu_indices(6)
    for s in SHOTS:
        r = O64.forward_residual(c["ksp64"], c["mps64"], c["mask"][s], x, c["t"][s], c["kg"],
                                 c["rk"])
        J = O64.jacobian(c["ksp64"].shape, c["mps64"], c["mask"][s], x, c["t"][s], c["kg"],
                         c["rk"], "reference")
        g = np.array([np.vdot(r, J[p]).real for p in range(6)])
        H = np.array([[np.vdot(J[i], J[j]).real for j in range(6)] for i in range(6)])
        np.testing.assert_allclose(gt[s], g, rtol=1e-4, atol=1e-4 * np.abs(g).max())
        np.testing.assert_allclose(stats[s, 1:7], g, rtol=1e-4, atol=1e-4 * np.abs(g).max())
        np.testing.assert_allclose(stats[s, 7:], H[iu], rtol=1e-4, atol=1e-4 * np.abs(H).max())
        assert abs(stats[s, 0] - np.vdot(r, r).real) <= 1e-5 * np.vdot(r, r).real
        # the damped proposal of transform_estimation.py:60-71 from either set of statistics
        Hs = np.zeros((6, 6))
        Hs[iu] = stats[s, 7:]
        Hs = Hs + np.triu(Hs, 1).T
        for damp in (1.0, 1e-2):
            d_jvp = np.linalg.solve(Hs + damp * np.eye(6), stats[s, 1:7])
            d_exp = np.linalg.solve(H + damp * np.eye(6), g)
            assert np.abs(d_jvp - d_exp).max() <= 1e-4 * max(np.abs(d_exp).max(), 1e-3), s
