"""Parity at the bench workload's line lengths (256, 224, 176) on thin volumes, so that the
FP64 oracle stays fast: the compile-time FFT kernels for exactly these lengths, the sparse
x-DFT over 256 rows, 448 samples per shot (the 256x224 DISORDER 16x16 accel-2 order chunked
into 64 shots, with its cross-shot duplicates), and the 1,792-samples-per-shot variant."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O64 = Oracle(np.complex128)


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


@pytest.mark.parametrize("shape", [(256, 224, 4), (8, 6, 176), (224, 176, 2), (176, 256, 2)])
def test_transform_bench_lengths(shape):
    import motionest
    rng = np.random.default_rng(sum(shape))
    x = _rand(rng, shape)
    p = np.array([2.1, -1.4, 0.8, 0.09, -0.13, 0.11])
    kg, rk = transform_grids(shape, [1, 1, 1])
    T = motionest.RigidTransformCudaOptimzied(p, kg, rk)
    assert rel_l2(T.apply(x), O64.rigid_apply(x, p, kg, rk)) < 2e-6
    assert rel_l2(T.adjoint(x), O64.rigid_adjoint(x, p, kg, rk)) < 2e-6
    dT = motionest.RigidTransformDerivativeCuda(shape, p, kg, rk)
    J = dT.jacobian(x)
    for q in range(6):
        assert rel_l2(J[1 + q], O64.rigid_derivative(x, p, q, kg, rk)) < 2e-5, q


@pytest.mark.parametrize("nshots", [64, 16])
def test_sense_operators_bench_planes(nshots):
    """256 x 224 planes, DISORDER 16x16 accel 2 chunked into `nshots` shots (448 or 1,792
    samples per shot), 2 coils, 2 readout points."""
    from motionest.problem import SenseProblem, xyz_to_zxy, zxy_to_xyz
    from motionest.sampling import disorder_masks
    shape = (256, 224, 2)
    rng = np.random.default_rng(nshots)
    planes = np.fft.ifftshift(disorder_masks(256, 224, (16, 16), 2, nshots)[..., 0], axes=(-2, -1))
    assert (planes.sum(0) > 1).any()  # the order revisits points across shots
    mps = 0.5 * _rand(rng, (2,) + shape)
    ksp = _rand(rng, (2,) + shape)
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-3, 3, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-6, 6, (nshots, 3)))
    kg, rk = transform_grids(shape, [1, 1, 1])
    pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk,
                      torch.as_tensor(t).cuda())
    mask = planes[..., None]
    M = zxy_to_xyz(pb.M).cpu().numpy().astype(bool)
    x = _rand(rng, shape)
    xd = xyz_to_zxy(torch.as_tensor(x).cuda())
    got = zxy_to_xyz(pb.normal(xd, pb.empty_image())).cpu().numpy()
    assert rel_l2(got, O64.normal_op(x, mps, mask, t, kg, rk, M)) < 2e-5
    b = zxy_to_xyz(pb.rhs(pb.empty_image())).cpu().numpy()
    assert rel_l2(b, O64.cg_rhs(ksp, mps, mask, t, kg, rk, M)) < 2e-5
    e = pb.residual_norms(xd, torch.as_tensor(t).cuda()).cpu().numpy()
    for s in (0, nshots // 2, nshots - 1):
        r = O64.forward_residual(ksp, mps, mask[s], x, t[s], kg, rk)
        np.testing.assert_allclose(e[s], np.vdot(r, r).real, rtol=2e-5)
    stats = pb.lm_stats(xd, 0).cpu().numpy()
    for s in (0, nshots - 1):
        r = O64.forward_residual(ksp, mps, mask[s], x, t[s], kg, rk)
        J = O64.jacobian(ksp.shape, mps, mask[s], x, t[s], kg, rk, "reference")
        g = np.array([np.vdot(r, J[p]).real for p in range(6)])
        np.testing.assert_allclose(stats[s, 1:7], g, rtol=2e-4, atol=2e-4 * np.abs(g).max())
