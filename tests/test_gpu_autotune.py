"""The launch-shape autotuner: it picks a shots-per-launch batch by timing, caches the choice by
problem shape and GPU, and the reconstruction does not depend on the batch it picks."""
import json

import numpy as np
import pytest
import torch

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_auto_batch_is_cached_and_result_invariant(tmp_path, monkeypatch):
    monkeypatch.setenv("MOTIONEST_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    import motionest.autotune as at
    at._CACHE = None
    from motionest.joint_recon import JointRecon
    from motionest.utils import compute_transform_grids_voxel
    d = load_golden("joint")
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    ref = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=2)
    xr, tr = ref.run()
    auto = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=2,
                      batch="auto")
    cache = json.loads((tmp_path / "tune.json").read_text())
    (entry,) = cache.values()
    assert auto.pb.batch == entry["batch"] and auto.pb.lm_batch == entry["lm_batch"]
    assert entry["timings"]["normal_ms"]
    xa, ta = auto.run()
    # every batch size adds the shots' contributions in the same order: bit-identical results
    assert torch.equal(xa, xr)
    assert torch.equal(ta, tr)
    # a second problem of the same shape reuses the cached choice without timing
    at._CACHE = None
    again = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_joint_iter=1, batch="auto")
    assert again.pb.batch == entry["batch"]
