"""CG-SENSE as one CUDA graph (me_cg_graph_create: a conditional WHILE node with the stopping
test on the device) against the host-driven CG loop: the same kernels in the same order, so the
images, transforms, CG iteration counts and objective histories must be bit-identical, both
when CG runs all its iterations and when the reference's tolerance test stops it early."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

sys.path.insert(0, str(GOLDEN))
import config_inputs as ci  # noqa: E402

pytestmark = pytest.mark.gpu


def _pair(ksp, mps, mask, shape, **kw):
    from motionest.joint_recon import JointRecon
    from motionest.utils import compute_transform_grids_voxel
    kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
    out = []
    for graph in (False, True):
        app = JointRecon(ksp, mps, mask, kg, rk, cg_graph=graph, **kw)
        x, t = app.run()
        out.append((x.cpu().numpy(), t.cpu().numpy(), list(app.cg_iterations),
                    app.objective_history))
    return out


def test_graph_cg_matches_host_loop_joint_fixture():
    d = load_golden("joint")
    (xa, ta, ca, oa), (xb, tb, cb, ob) = _pair(d["ksp"], d["mps"], d["mask"], d["ksp"].shape[1:],
                                               max_cg_iter=4, max_joint_iter=3)
    assert ca == cb
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(ta, tb)
    np.testing.assert_array_equal(oa, ob)


def test_graph_cg_stops_early_like_the_host_loop():
    """Unit-RSS coils and no motion estimate yet: the first CG solve meets the tolerance after
    one or two iterations; the device-side test must stop at the same iteration."""
    ksp, mps, masks, _ = ci.load(GOLDEN)
    (xa, ta, ca, oa), (xb, tb, cb, ob) = _pair(ksp, mps, masks, ci.SHAPE, max_cg_iter=5,
                                               max_joint_iter=2)
    assert ca == cb
    assert ca[0] < 5, ca  # the early stop happened
    np.testing.assert_array_equal(xa, xb)
    np.testing.assert_array_equal(ta, tb)
