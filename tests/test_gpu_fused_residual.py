"""The CG's initial residual b - A x from one pass over the shots (me_sense_residual) and the
objective pass that leaves it for the next solve.

- me_sense_residual against the FP64 oracle's b - A x (image_estimation.py:93-103, :133-134)
  and against the library's own right-hand side minus normal operator, on the compile-time
  SENSE kernels (y = 32) and the run-time ones (y = 28); its energies against
  me_sense_residual_norms and the oracle's forward residuals.
- JointRecon with the residual left by each objective pass is bit-identical to JointRecon
  forming every solve's residual itself (host-loop CG and CUDA-graph CG), and within rounding
  of the reference's order of operations (fused_residual=False).
- A change of the image or the transforms between the objective and the next step makes the
  step form the residual again."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O64 = Oracle(np.complex128)


def _np(a):
    return a.detach().cpu().numpy()


def _problem(shape, ncoils, nshots, tile, accel, seed):
    from motionest.problem import SenseProblem
    from motionest.sampling import disorder_masks
    X, Y, Z = shape
    rng = np.random.default_rng(seed)
    mps = (0.5 * (rng.standard_normal((ncoils,) + shape)
                  + 1j * rng.standard_normal((ncoils,) + shape))).astype(np.complex64)
    ksp = (rng.standard_normal((ncoils,) + shape)
           + 1j * rng.standard_normal((ncoils,) + shape)).astype(np.complex64)
    planes = np.fft.ifftshift(disorder_masks(X, Y, tile, accel, nshots)[..., 0], axes=(-2, -1))
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-2, 2, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-5, 5, (nshots, 3)))
    kg, rk = transform_grids(shape, [1, 1, 1])
    pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk,
                      torch.as_tensor(t).cuda())
    return pb, ksp, mps, planes, t, kg, rk


@pytest.mark.parametrize("shape,ncoils,nshots,tile,accel", [
    ((32, 32, 16), 4, 8, (4, 4), 2),   # compile-time SENSE kernels (y = 32)
    ((32, 28, 20), 6, 8, (4, 4), 1),   # run-time SENSE kernels (y = 28)
])
def test_residual_vs_fp64_oracle_and_two_pass_form(shape, ncoils, nshots, tile, accel):
    from motionest.problem import xyz_to_zxy, zxy_to_xyz
    pb, ksp, mps, planes, t, kg, rk = _problem(shape, ncoils, nshots, tile, accel, 21)
    mask = planes[..., None]
    M = _np(zxy_to_xyz(pb.M)).astype(bool)
    rng = np.random.default_rng(4)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    xd = xyz_to_zxy(torch.as_tensor(x).cuda())
    ref = O64.cg_rhs(ksp, mps, mask, t, kg, rk, M) - O64.normal_op(x, mps, mask, t, kg, rk, M)
    for batch in (1, 3, nshots):
        e = torch.empty(nshots, dtype=torch.float64, device="cuda")
        r = pb.residual(xd, pb.empty_image(), energies=e, batch=batch)
        assert rel_l2(_np(zxy_to_xyz(r)), ref) < 2e-5, batch
        # the library's two-pass form of the same vector
        two = pb.rhs(pb.empty_image(), batch=batch) - pb.normal(xd, pb.empty_image(), batch=batch)
        assert rel_l2(_np(r), _np(two)) < 1e-5, batch
        # energies: as me_sense_residual_norms (which may round scale * acc - y once, where
        # this pass stores K first) and as the oracle's forward residuals
        en = _np(pb.residual_norms(xd, pb.transforms, batch=batch))
        np.testing.assert_allclose(_np(e), en, rtol=1e-6)
        ref_e = [float(np.vdot(q, q).real) for q in
                 (O64.forward_residual(ksp, mps, mask[s], x, t[s], kg, rk) for s in range(nshots))]
        np.testing.assert_allclose(_np(e), ref_e, rtol=2e-5)
    # with a zero image the residual is the right-hand side itself, bit for bit
    z = pb.empty_image().zero_()
    np.testing.assert_array_equal(_np(pb.residual(z, pb.empty_image())),
                                  _np(pb.rhs(pb.empty_image())))


def _recon(d, kg, rk, graph, reuse, fused=True):
    from motionest.joint_recon import JointRecon
    app = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=4, max_joint_iter=3,
                     cg_graph=graph, fused_residual=fused)
    objs = []
    for _ in range(3):
        app.step()
        objs.append(app._compute_objective())
        if not reuse:
            app._r0_key = None  # the next step forms its residual itself
    return _np(app.x), _np(app.t), list(app.cg_iterations), objs


@pytest.mark.parametrize("graph", [False, True])
def test_objective_residual_reuse_is_bit_identical(graph):
    from motionest.utils import compute_transform_grids_voxel
    d = dict(load_golden("joint"))
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    xa, ta, ca, oa = _recon(d, kg, rk, graph, reuse=True)
    xb, tb, cb, ob = _recon(d, kg, rk, graph, reuse=False)
    assert ca == cb
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(ta, tb)
    assert oa == ob
    # the reference's order of operations: the same iterates up to rounding
    xc, tc, cc, oc = _recon(d, kg, rk, graph, reuse=True, fused=False)
    assert cc == ca
    assert rel_l2(xa, xc) < 1e-5
    np.testing.assert_allclose(ta, tc, atol=1e-6)
    np.testing.assert_allclose(oa, oc, rtol=1e-5)


def test_changed_state_forms_the_residual_again():
    from motionest.joint_recon import JointRecon
    from motionest.utils import compute_transform_grids_voxel
    d = dict(load_golden("joint"))
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    app = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=2)
    app.step()
    app._compute_objective()
    assert app._r0_ready()
    app.x.mul_(1.0)  # an in-place write, even of the same values
    assert not app._r0_ready()
    app._compute_objective()
    assert app._r0_ready()
    app.t[0, 0] *= 1.0
    assert not app._r0_ready()
    app._compute_objective()
    app.step()  # consumes it
    assert not app._r0_ready()
    # a fresh residual after a state change gives the same step as without the objective
    ref = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=2)
    ref.step()
    ref.step()
    np.testing.assert_array_equal(_np(app.x), _np(ref.x))
    np.testing.assert_array_equal(_np(app.t), _np(ref.t))
