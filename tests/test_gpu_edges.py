"""Edge cases of the CUDA path against the oracle: an empty shot, a single shot, line lengths
the compile-time kernels do not cover (runtime-plan FFT), a single-plane volume (lines of
length 1), non-separable rk grids (per-element chirps), duplicate samples across shots, and the
CG early exit."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O32 = Oracle(np.complex64)
O64 = Oracle(np.complex128)


def _problem(shape, ncoils, planes, seed, rot=3.0, trans=1.0, unit_rss=False):
    """Centred (ksp, mps, masks, t) with the oracle's FP32 forward model."""
    rng = np.random.default_rng(seed)
    X, Y, Z = shape
    gx, gy, gz = np.meshgrid(*(np.linspace(-1, 1, n) for n in shape), indexing="ij")
    img = sum(rng.uniform(0.2, 1) / (1 + np.exp(6 * (((gx - c[0]) / 0.4) ** 2 + ((gy - c[1]) / 0.3) ** 2
                                                   + ((gz - c[2]) / 0.5) ** 2 - 1)))
              for c in rng.uniform(-0.3, 0.3, (3, 3)))
    gt = (img * np.exp(0.4j * gx)).astype(np.complex64)
    maps = []
    for c in range(ncoils):
        a = 2 * np.pi * c / ncoils
        maps.append(np.exp(-((gx - np.cos(a)) ** 2 + (gy - np.sin(a)) ** 2) / 1.2) * np.exp(1j * a))
    mps = np.stack(maps)
    mps = (mps / np.sqrt((np.abs(mps) ** 2).sum(0)) if unit_rss else 1.6 * mps).astype(np.complex64)
    S = planes.shape[0]
    t = np.zeros((S, 6))
    t[:, :3] = rng.uniform(-trans, trans, (S, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-rot, rot, (S, 3)))
    masks = planes[..., None]
    ksp = O32.corrupted_kspace(gt, mps, masks, t).astype(np.complex64)
    return ksp, mps, masks, t


def _joint(me, ksp, mps, masks, iters=2, cg=3):
    kg, rk = transform_grids(ksp.shape[1:], [1, 1, 1])
    app = me.JointRecon(ksp, mps, masks, kg, rk, max_cg_iter=cg, max_joint_iter=iters)
    x, t = app.run()
    ox, ot, oh, _ = O32.joint_recon(ksp, mps, masks, kg, rk, max_cg_iter=cg, max_joint_iter=iters)
    return x.cpu().numpy(), t.cpu().numpy(), app, ox, ot, oh


@pytest.fixture(scope="module")
def me():
    import motionest
    from motionest.joint_recon import JointRecon
    motionest.JointRecon = JointRecon
    return motionest


def test_joint_recon_with_an_empty_shot(me):
    from motionest.sampling import disorder_masks
    planes = disorder_masks(16, 12, (4, 4), 1, 4)[..., 0].copy()
    planes[2] = False
    ksp, mps, masks, _ = _problem((16, 12, 10), 3, planes, 1)
    x, t, app, ox, ot, oh = _joint(me, ksp, mps, masks)
    assert rel_l2(x, ox) < 1e-4
    np.testing.assert_allclose(t, ot, atol=1e-5)
    np.testing.assert_allclose(app.objective_history, oh, rtol=1e-4)


def test_joint_recon_single_shot(me):
    planes = np.ones((1, 12, 8), bool)
    ksp, mps, masks, _ = _problem((12, 8, 6), 2, planes, 2)
    x, t, app, ox, ot, oh = _joint(me, ksp, mps, masks)
    assert rel_l2(x, ox) < 1e-4
    np.testing.assert_allclose(t, ot, atol=1e-5)


def test_joint_recon_runtime_plan_lengths(me):
    """12 x 10 x 7: no compile-time kernel for 12, 10 or 7, so the runtime-plan passes and the
    generic SENSE kernels run."""
    from motionest.sampling import disorder_masks
    planes = disorder_masks(12, 10, (2, 2), 1, 4)[..., 0]
    ksp, mps, masks, _ = _problem((12, 10, 7), 3, planes, 3)
    x, t, app, ox, ot, oh = _joint(me, ksp, mps, masks)
    assert rel_l2(x, ox) < 1e-4
    np.testing.assert_allclose(t, ot, atol=1e-5)


def test_joint_recon_single_plane_volume(me):
    """16 x 12 x 1 (a 2-D acquisition): the shears and the ramp along z act on lines of length
    1, and the hybrid k-space has one plane."""
    from motionest.sampling import disorder_masks
    planes = disorder_masks(16, 12, (4, 4), 1, 4)[..., 0]
    ksp, mps, masks, _ = _problem((16, 12, 1), 3, planes, 8)
    x, t, app, ox, ot, oh = _joint(me, ksp, mps, masks)
    assert rel_l2(x, ox) < 1e-4
    np.testing.assert_allclose(t, ot, atol=1e-5)
    np.testing.assert_allclose(app.objective_history, oh, rtol=1e-4)


@pytest.mark.parametrize("shape", [(9, 8, 7), (16, 12, 1), (32, 28, 22)])
def test_identity_transform(me, shape):
    """T(0) = I and T(0)^H = I, on runtime-plan and compile-time line lengths."""
    rng = np.random.default_rng(len(shape) + sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    kg, rk = transform_grids(shape, [1, 1, 1])
    T = me.RigidTransformCudaOptimzied(np.zeros(6), kg, rk)
    assert rel_l2(T.apply(x), x) < 1e-6
    assert rel_l2(T.adjoint(x), x) < 1e-6


def test_non_separable_grid_uses_per_element_chirps(me):
    shape = (16, 14, 12)
    rng = np.random.default_rng(4)
    kg, rk = transform_grids(shape, [1, 1, 1])
    # perturb every rk plane so it is no longer an outer product r * k
    rk = {m: {a: v + 0.3 * rng.standard_normal(v.shape) for a, v in d.items()}
          for m, d in rk.items()}
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    p = np.array([0.7, -1.1, 0.4, 0.06, -0.05, 0.08])
    T = me.RigidTransformCudaOptimzied(p, kg, rk)
    assert rel_l2(T.apply(x), O64.rigid_apply(x, p, kg, rk)) < 2e-6
    assert rel_l2(T.adjoint(x), O64.rigid_adjoint(x, p, kg, rk)) < 2e-6
    dT = me.RigidTransformDerivativeCuda(shape, p, kg, rk)
    for q in (0, 3, 5):
        assert rel_l2(dT.apply(x, q), O64.rigid_derivative(x, p, q, kg, rk)) < 2e-5


def test_forward_model_with_duplicate_samples_across_shots(me):
    """96x96 with 8x8 tiles revisits 1,536 k-space points across shots; the reference adds the
    shots' contributions there (simulation.py:82), and so must the scatter."""
    from motionest.sampling import disorder_masks
    from motionest.simulation import generate_corrupted_kspace
    planes = disorder_masks(96, 96, (8, 8), 1, 16)[..., 0]
    assert (planes.sum(0) > 1).any()
    rng = np.random.default_rng(5)
    shape = (96, 96, 4)
    gt = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    mps = (rng.standard_normal((2,) + shape) + 1j * rng.standard_normal((2,) + shape)).astype(np.complex64)
    t = np.zeros((16, 6))
    t[:, 3:] = np.deg2rad(rng.uniform(-2, 2, (16, 3)))
    t[:, :3] = rng.uniform(-1, 1, (16, 3))
    got = generate_corrupted_kspace(gt, mps, planes[..., None], t).cpu().numpy()
    ref = O32.corrupted_kspace(gt, mps, planes[..., None], t)
    assert rel_l2(got, ref) < 1e-5


def test_cg_trip_count_matches_reference_rule(me):
    """The stopping rule sqrt|<r, P r>| < tol (image_estimation.py:156).  Unit-RSS coils, no
    motion and full coverage make the normal operator ~I, so one step solves the system and
    the residual drops to rounding (~1e-7 |b|); with tol = 1e-4 |b| both implementations stop
    after exactly one iteration, with three orders of magnitude of margin.  With motion the
    residual stays far above tol and all iterations run."""
    from motionest.image_estimation import cg_solve
    from motionest.problem import SenseProblem
    planes = np.ones((2, 16, 12), bool)
    planes[0, :, ::2] = False
    planes[1, :, 1::2] = False
    for rot, trans, expect_early in ((0.0, 0.0, True), (4.0, 1.5, False)):
        ksp, mps, masks, t = _problem((16, 12, 8), 4, planes, 6, rot=rot, trans=trans,
                                      unit_rss=True)
        kg, rk = transform_grids(ksp.shape[1:], [1, 1, 1])
        ks, ms, mk, mx, P, M = O32.joint_setup(ksp, mps, masks)
        b = O64.cg_rhs(ks, ms, mk, t, kg, rk, M)
        tol = 1e-4 * float(np.sqrt(np.vdot(b, P * b).real))
        _, oiters = O32.estimate_image_cg(ks, ms, mk, t, kg, rk, P, M, max_iter=6, tol=tol,
                                          return_iters=True)
        pb = SenseProblem(torch.as_tensor(ks).cuda(), torch.as_tensor(ms).cuda(), mk[..., 0],
                          kg, rk, torch.as_tensor(t).cuda())
        x = pb.empty_image().zero_()
        iters = cg_solve(pb, x, 6, tol)
        assert iters == oiters
        assert (iters == 1) if expect_early else (iters == 6)
