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


@pytest.mark.parametrize("sizes", [
    (((16, 24, 32), 3), ((32, 16, 48), 5), ((64, 56, 24), 2), ((24, 24, 24), 4)),
    (((64, 64, 32), 3), ((96, 96, 48), 2), ((128, 64, 64), 2), ((64, 96, 96), 2)),
])
def test_multi_job_transform_matches_one_job_at_a_time(sizes):
    """me_rigid_apply_multi over reconstructions of uneven size (each shear step one persistent
    launch per line length over all jobs' volumes and line tiles) against one me_rigid_apply
    per job: bit-identical.  In the first set no line row divides into whole tiles, so every
    step takes the cp.async kernels; in the second every one does, so every step moves its
    tiles by tensor copies (16-line tiles for 96 and 128 points, 32-line tiles for 32 and 64,
    strided along x and z, contiguous along y)."""
    import torch
    from motionest import _lib
    from motionest.multi import apply_transforms
    from motionest.utils import DeviceGrid, compute_transform_grids_voxel
    rng = np.random.default_rng(12)
    jobs, refs = [], []
    for shape, nvol in sizes:
        X, Y, Z = shape
        kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
        grid = DeviceGrid(kg, rk, shape)
        x = torch.tensor((rng.standard_normal((Z, X, Y)) + 1j * rng.standard_normal((Z, X, Y)))
                         .astype(np.complex64), device="cuda")
        t = np.zeros((nvol, 6))
        t[:, :3] = rng.uniform(-2, 2, (nvol, 3))
        t[:, 3:] = np.deg2rad(rng.uniform(-6, 6, (nvol, 3)))
        params = torch.tensor(t, device="cuda")
        out = torch.empty((nvol, Z, X, Y), dtype=torch.complex64, device="cuda")
        ref = torch.empty_like(out)
        _lib.call("me_rigid_apply", _lib.ptr(x), 0, _lib.ptr(ref), X * Y * Z, nvol,
                  _lib.MeLayout(Y, 1, X * Y), grid.ref, _lib.ptr(params), 6, 0,
                  _lib.stream_ptr())
        jobs.append(dict(x=x, out=out, params=params, grid=grid))
        refs.append(ref)
    apply_transforms(jobs)
    for jb, ref in zip(jobs, refs):
        assert torch.equal(jb["out"], ref)
