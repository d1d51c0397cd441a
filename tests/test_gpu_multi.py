"""MultiRecon: reconstructions of uneven size advanced together, each on its own stream with its
CG solves as CUDA graphs, against the same reconstructions run one at a time: bit-identical
images, transforms, CG counts and objectives (the instances do not interact)."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

sys.path.insert(0, str(GOLDEN))
import config_inputs as ci  # noqa: E402

pytestmark = pytest.mark.gpu


def _problems():
    from motionest.simulation import make_workload
    from motionest.utils import compute_transform_grids_voxel
    d = load_golden("joint")
    ksp0, mps0, masks0, _ = ci.load(GOLDEN)
    wl = make_workload((32, 24, 16), 4, 8, (4, 4), 1, motion="continuous", seed=4)
    out = []
    for ksp, mps, masks in ((d["ksp"], d["mps"], d["mask"]), (ksp0, mps0, masks0),
                            (wl["ksp"], wl["mps"], wl["masks"])):
        shape = tuple(ksp.shape[1:])
        kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
        out.append(dict(ksp=ksp, mps=mps, masks=masks, kgrid=kg, rkgrid=rk))
    return out


def test_multi_recon_matches_one_at_a_time():
    from motionest.joint_recon import JointRecon
    from motionest.multi import MultiRecon
    probs = _problems()
    mr = MultiRecon(probs, max_cg_iter=4, max_nm_iter=1, batch=None)
    res = mr.run(3)
    for p, (x, t), oh, app in zip(probs, res, mr.objective_history, mr.apps):
        ref = JointRecon(p["ksp"], p["mps"], p["masks"], p["kgrid"], p["rkgrid"], max_cg_iter=4,
                         max_joint_iter=3, cg_graph=True)
        xr, tr = ref.run()
        np.testing.assert_array_equal(x.cpu().numpy(), xr.cpu().numpy())
        np.testing.assert_array_equal(t.cpu().numpy(), tr.cpu().numpy())
        assert app.cg_iterations == ref.cg_iterations
        np.testing.assert_array_equal(np.array(oh), ref.objective_history)
    mr.close()
