"""The 64x64x48 / 8-coil / 16-shot JointRecon fixture (tests/golden/config0.npz), on CPU:
its inputs rebuild bit for bit, its masks are the DISORDER masks motionest builds, and the
oracle's first outer iteration reproduces the reference's (the GPU run of all ten iterations is
tests/test_gpu_config0.py)."""
import sys

import numpy as np

from conftest import GOLDEN, rel_l2

sys.path.insert(0, str(GOLDEN))
import config_inputs as ci  # noqa: E402


def test_inputs_rebuild_and_masks_match_motionest():
    from motionest.sampling import disorder_masks
    ksp, mps, masks, d = ci.load(GOLDEN)  # raises if the rebuilt maps differ
    assert ksp.shape == (ci.NCOILS,) + ci.SHAPE and ksp.dtype == np.complex64
    rss = np.sqrt(np.sum(np.abs(mps.astype(np.complex128)) ** 2, axis=0))
    assert np.abs(rss - 1).max() < 1e-6
    X, Y, _ = ci.SHAPE
    np.testing.assert_array_equal(masks, disorder_masks(X, Y, ci.TILE, ci.ACCEL, ci.NSHOTS))
    assert masks.sum() == X * Y  # 4x4 tiles at accel 1: every (kx, ky) once


def test_oracle_first_outer_iteration_matches_reference():
    from oracle import Oracle, transform_grids
    ksp, mps, masks, d = ci.load(GOLDEN)
    kg, rk = transform_grids(ci.SHAPE, [1, 1, 1])
    x, t, oh, th = Oracle(np.complex64, workers=-1).joint_recon(
        ksp, mps, masks, kg, rk, max_cg_iter=ci.CG_ITERS, max_nm_iter=1, max_joint_iter=1)
    np.testing.assert_allclose(th[0], d["transform_history"][0], atol=1e-6)
    assert abs(oh[0] - d["objective_history"][0]) <= 1e-5 * d["objective_history"][0]
