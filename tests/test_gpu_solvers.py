"""CUDA SENSE / CG / LM / JointRecon / pyramid vs the reference's outputs (golden fixtures)
and the FP64 oracle.  Tolerances: image relative L2 <= 1e-4 against the reference's FP32 path,
motion parameters within 1e-5 (rad / voxel) of it -- well inside the 0.01 deg / 0.01 voxel
parity target -- and bit-equal damping / convergence decisions."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O32 = Oracle(np.complex64)
O64 = Oracle(np.complex128)


@pytest.fixture(scope="module")
def me():
    import motionest
    import motionest.image_estimation
    import motionest.joint_recon
    import motionest.pyramid
    import motionest.simulation
    import motionest.transform_estimation
    return motionest


def _np(a):
    return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)


def test_forward_model_vs_reference(me):
    d = load_golden("forward")
    ksp = me.simulation.generate_corrupted_kspace(d["gt"], d["mps"], d["mask"], d["transforms"])
    assert rel_l2(_np(ksp), d["ksp"]) < 1e-5


@pytest.mark.parametrize("case", range(3))
def test_cg_vs_reference(me, case):
    d = load_golden("cg")
    g = lambda k: d[f"c{case}_{k}"]  # noqa: E731
    kg, rk = me.compute_transform_grids_voxel(g("x").shape, [1, 1, 1])
    x = me.image_estimation.estimate_image_cg(g("ksp"), g("mps"), g("mask"), g("transforms"), kg,
                                              rk, g("P"), g("M"), x0=g("x0"),
                                              max_iter=int(g("max_iter")))
    assert isinstance(x, np.ndarray)
    assert rel_l2(x, g("x")) < 1e-4


@pytest.mark.parametrize("case", range(3))
def test_lm_vs_reference(me, case):
    d = load_golden("lm")
    g = lambda k: d[f"c{case}_{k}"]  # noqa: E731
    kg, rk = me.compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    t = g("t0").copy()
    damp = g("damp0").copy()
    flags = np.zeros(len(damp), bool)
    out = me.transform_estimation.estimate_transform(d["ksp"], d["mps"], d["mask"], g("image"), kg,
                                                     rk, damp, flags, None, None, None, None,
                                                     transforms=t)
    np.testing.assert_array_equal(damp, g("damp"))
    np.testing.assert_array_equal(flags, g("flags"))
    np.testing.assert_allclose(t, g("t"), atol=1e-5)
    assert rel_l2(out, g("image_out")) < 1e-4


def test_joint_recon_vs_reference(me):
    d = load_golden("joint")
    kg, rk = me.compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    app = me.joint_recon.JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk,
                                    max_cg_iter=int(d["max_cg_iter"]),
                                    max_nm_iter=int(d["max_nm_iter"]),
                                    max_joint_iter=int(d["max_joint_iter"]))
    x, t = app.run()
    assert rel_l2(_np(x), d["x"]) < 1e-4
    np.testing.assert_allclose(_np(t), d["t"], atol=1e-5)
    np.testing.assert_allclose(app.objective_history, d["objective_history"], rtol=1e-4)
    np.testing.assert_allclose(app.transform_history, d["transform_history"], atol=1e-5)


def test_pyramid_vs_reference(me):
    d = load_golden("pyramid")
    x, t = me.pyramid.pyramid_reconstruction(d["ksp"], d["mps"], d["mask"], d["mask"].shape[0],
                                             n_joint_iters=int(d["n_joint_iters"]), verbose=False)
    assert rel_l2(x, d["x"]) < 1e-4
    np.testing.assert_allclose(t, d["t"], atol=1e-5)


def _problem(me, shape, ncoils, nshots, tile, accel, seed, unit_rss=False):
    from motionest.problem import SenseProblem
    from motionest.sampling import disorder_masks
    X, Y, Z = shape
    rng = np.random.default_rng(seed)
    mps = (rng.standard_normal((ncoils,) + shape) + 1j * rng.standard_normal((ncoils,) + shape))
    mps = (0.5 * mps).astype(np.complex64)
    ksp = (rng.standard_normal((ncoils,) + shape) + 1j * rng.standard_normal((ncoils,) + shape))
    ksp = ksp.astype(np.complex64)
    planes = disorder_masks(X, Y, tile, accel, nshots)[..., 0]
    planes = np.fft.ifftshift(planes, axes=(-2, -1))
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-2, 2, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-5, 5, (nshots, 3)))
    kg, rk = transform_grids(shape, [1, 1, 1])
    tt = torch.as_tensor(t).cuda()
    pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk, tt)
    return pb, ksp, mps, planes, t, kg, rk


@pytest.mark.parametrize("shape,ncoils,nshots,tile,accel", [
    ((32, 28, 20), 6, 8, (4, 4), 1),
    ((48, 40, 22), 4, 16, (8, 8), 2),
    ((30, 21, 15), 3, 5, (3, 3), 1),
])
def test_sense_operators_vs_fp64_oracle(me, shape, ncoils, nshots, tile, accel):
    from motionest.problem import xyz_to_zxy, zxy_to_xyz
    pb, ksp, mps, planes, t, kg, rk = _problem(me, shape, ncoils, nshots, tile, accel, 11)
    mask = planes[..., None]
    M = _np(zxy_to_xyz(pb.M)).astype(bool)
    rng = np.random.default_rng(5)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    xd = xyz_to_zxy(torch.as_tensor(x).cuda())
    # normal operator, plain (one shot per launch) and batched
    ref = O64.normal_op(x, mps, mask, t, kg, rk, M)
    for batch in (1, 3, nshots):
        got = _np(zxy_to_xyz(pb.normal(xd, pb.empty_image(), batch=batch)))
        assert rel_l2(got, ref) < 2e-5, batch
    # right-hand side
    b = _np(zxy_to_xyz(pb.rhs(pb.empty_image())))
    assert rel_l2(b, O64.cg_rhs(ksp, mps, mask, t, kg, rk, M)) < 2e-5
    # residual energies
    e = _np(pb.residual_norms(xd, torch.as_tensor(t).cuda()))
    ref_e = [float(np.vdot(r, r).real) for r in
             (O64.forward_residual(ksp, mps, mask[s], x, t[s], kg, rk) for s in range(nshots))]
    np.testing.assert_allclose(e, ref_e, rtol=2e-5)


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_lm_statistics_vs_fp64_oracle(me, mode):
    shape, nshots = (24, 20, 12), 4
    pb, ksp, mps, planes, t, kg, rk = _problem(me, shape, 3, nshots, (4, 4), 1, 3)
    from motionest.problem import xyz_to_zxy
    mask = planes[..., None]
    x = me.simulation.phantom(shape, 6, seed=2).cpu().numpy()
    x = np.fft.ifftshift(x)
    stats = _np(pb.lm_stats(xyz_to_zxy(torch.as_tensor(x).cuda()), 0 if mode == "reference" else 1))
    for s in range(nshots):
        r = O64.forward_residual(ksp, mps, mask[s], x, t[s], kg, rk)
        J = O64.jacobian(ksp.shape, mps, mask[s], x, t[s], kg, rk, mode)
        g = np.array([np.vdot(r, J[p]).real for p in range(6)])
        H = np.array([[np.vdot(J[p], J[q]).real for q in range(6)] for p in range(6)])
        np.testing.assert_allclose(stats[s, 0], np.vdot(r, r).real, rtol=2e-5)
        np.testing.assert_allclose(stats[s, 1:7], g, rtol=1e-4, atol=1e-4 * np.abs(g).max())
        iu = np.triu_indices(6)
        np.testing.assert_allclose(stats[s, 7:], H[iu], rtol=1e-4, atol=1e-5 * np.abs(H).max())


def test_joint_recon_exact_jacobian_runs(me):
    d = load_golden("joint")
    kg, rk = me.compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    app = me.joint_recon.JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3,
                                    max_joint_iter=3, jacobian="exact")
    x, t = app.run()
    assert np.isfinite(app.objective_history).all()
    assert app.objective_history[-1] <= app.objective_history[0]


def test_pyramid_temporal_levels_vs_oracle(me):
    """pyramid_reconstruction(temporal=True): at the coarsest spatial level, 2 and then 1 shot
    per motion state before the per-shot level (the reference's disabled sketch, completed),
    against the oracle's restatement of the same schedule."""
    d = load_golden("pyramid")
    S = d["mask"].shape[0]
    x, t = me.pyramid.pyramid_reconstruction(d["ksp"], d["mps"], d["mask"], S,
                                             n_temporal_levels=2, n_joint_iters=2,
                                             verbose=False, temporal=True)
    ox, ot = O32.pyramid_reconstruction(d["ksp"], d["mps"], d["mask"], S, n_joint_iters=2,
                                        n_temporal_levels=2, temporal=True)
    assert rel_l2(x, ox) < 1e-4
    np.testing.assert_allclose(t, ot, atol=1e-5)
    assert np.abs(t - d["t"]).max() > 1e-6  # the extra level changed the estimate


def test_continuous_motion_forward_model_vs_oracle(me):
    """k-space corrupted by intra-shot motion (4 segments per shot, each its own corruption
    state, as simulation.py:372-373,404-410 builds it) against the oracle's forward model."""
    from motionest.sampling import disorder_masks
    from motionest.simulation import coil_maps, motion_continuous, phantom
    shape, S, K = (16, 16, 8), 4, 4
    gt = phantom(shape, 4, seed=9).cpu().numpy()
    mps = coil_maps(shape, 3, seed=9).cpu().numpy()
    cor = disorder_masks(16, 16, (4, 4), 1, S * K)
    t = motion_continuous(S, K, seed=9)
    ksp = me.simulation.generate_corrupted_kspace(gt, mps, cor, t)
    ref = O32.corrupted_kspace(gt, mps, cor, t)
    assert rel_l2(_np(ksp), ref) < 1e-5


def test_precision_size_operators_vs_fp64(me):
    """The FP32 path's error against FP64 at the precision workload's size, 256x256x192 (line
    lengths 256, 256 and 192): the normal operator and the per-shot residual energies for two
    of its 64 DISORDER 16x16 (accel 2) shots with 4 coils, against the FP64 oracle.  The same
    bounds as at the small sizes: relative L2 <= 2e-5."""
    from motionest.problem import SenseProblem, xyz_to_zxy, zxy_to_xyz
    from motionest.sampling import disorder_masks
    from motionest.simulation import coil_maps, phantom
    shape = (256, 256, 192)
    planes = np.fft.ifftshift(disorder_masks(256, 256, (16, 16), 2, 64)[[0, 31], ..., 0],
                              axes=(-2, -1))
    mps = np.fft.ifftshift(coil_maps(shape, 4, seed=5, unit_rss=False).cpu().numpy(),
                           axes=(-3, -2, -1))
    x = np.fft.ifftshift(phantom(shape, 12, seed=5).cpu().numpy())
    rng = np.random.default_rng(6)
    ksp = (0.01 * (rng.standard_normal((4,) + shape) + 1j * rng.standard_normal((4,) + shape))
           ).astype(np.complex64)
    t = np.array([[1.5, -0.7, 2.2, 0.04, -0.06, 0.08], [-2.1, 0.9, -0.4, -0.09, 0.03, -0.05]])
    kg, rk = transform_grids(shape, [1, 1, 1])
    pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk,
                      torch.as_tensor(t).cuda())
    M = _np(zxy_to_xyz(pb.M)).astype(bool)
    xd = xyz_to_zxy(torch.as_tensor(x).cuda())
    got = _np(zxy_to_xyz(pb.normal(xd, pb.empty_image())))
    ref = O64.normal_op(x.astype(np.complex128), mps.astype(np.complex128), planes[..., None], t,
                        kg, rk, M)
    assert rel_l2(got, ref) < 2e-5
    e = _np(pb.residual_norms(xd, torch.as_tensor(t).cuda()))
    ref_e = [float(np.vdot(r, r).real) for r in (
        O64.forward_residual(ksp.astype(np.complex128), mps.astype(np.complex128),
                             planes[s][..., None], x.astype(np.complex128), t[s], kg, rk)
        for s in range(2))]
    np.testing.assert_allclose(e, ref_e, rtol=2e-5)
