"""JointRecon on the CUDA kernels against the reference's own run on the 64x64x48 / 8-coil /
16-shot DISORDER workload (tests/golden/config0.npz: 10 outer iterations of 5 CG iterations and
one LM step, inputs rebuilt by tests/golden/config_inputs.py).

Tolerances: image relative L2 <= 1e-4; every outer iteration's transforms within 0.01 degree and
0.01 voxel (in practice far closer); damping and convergence flags bit-equal; the objective
history to 1e-4 relative.  The reference accumulates its CG and LM inner products in float32
and this build in float64, which is where the small differences come from."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

sys.path.insert(0, str(GOLDEN))
import config_inputs as ci  # noqa: E402

pytestmark = pytest.mark.gpu

DEG = np.deg2rad(0.01)


def test_joint_recon_config0_matches_reference():
    from motionest.joint_recon import JointRecon
    from motionest.utils import compute_transform_grids_voxel
    ksp, mps, masks, d = ci.load(GOLDEN)
    kg, rk = compute_transform_grids_voxel(ci.SHAPE, [1, 1, 1])
    app = JointRecon(ksp, mps, masks, kg, rk, max_cg_iter=ci.CG_ITERS, max_nm_iter=1,
                     max_joint_iter=ci.OUTER_ITERS)
    x, t = app.run()
    x = x.cpu().numpy()
    err = rel_l2(x, d["x"])
    assert err <= 1e-4, err
    th = app.transform_history
    assert th.shape == d["transform_history"].shape
    dtr = np.abs(th[:, :, :3] - d["transform_history"][:, :, :3]).max()
    drot = np.abs(th[:, :, 3:] - d["transform_history"][:, :, 3:]).max()
    assert dtr <= 0.01 and drot <= DEG, (dtr, np.rad2deg(drot))
    np.testing.assert_array_equal(app.damp.cpu().numpy(), d["damp"])
    np.testing.assert_array_equal(app.convergence_flags.cpu().numpy().astype(bool), d["flags"])
    np.testing.assert_allclose(app.objective_history, d["objective_history"], rtol=1e-4)
    print(f"config0: image rel L2 {err:.2e}, max |dt| {dtr:.2e} voxel, "
          f"max |drot| {np.rad2deg(drot):.2e} deg")


def test_pyramid_config0_matches_reference():
    """pyramid_reconstruction on the same inputs against the reference's own run
    (tests/golden/config0_pyramid.npz: 3 spatial levels, n_joint_iters=2, i.e. 8 outer
    iterations at x0.25, 4 at x0.5, then image-only CG at full size, which the reference's
    tolerance test stopped after 45 iterations): image relative L2 <= 1e-4 and transforms within
    0.01 voxel / 0.01 degree."""
    from motionest.pyramid import pyramid_reconstruction
    ksp, mps, masks, _ = ci.load(GOLDEN)
    d = np.load(GOLDEN / "config0_pyramid.npz")
    x, t = pyramid_reconstruction(ksp, mps, masks, ci.NSHOTS, n_spatial_levels=3,
                                  n_joint_iters=2, verbose=False)
    err = rel_l2(x, d["x"])
    assert err <= 1e-4, err
    assert np.abs(t[:, :3] - d["t"][:, :3]).max() <= 0.01
    assert np.abs(t[:, 3:] - d["t"][:, 3:]).max() <= DEG
    print(f"config0 pyramid: image rel L2 {err:.2e}")
