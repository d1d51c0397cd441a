"""Geodesic-accelerated LM (estimate_transform(use_ga=True), transform_estimation.py:75-121) on
the CUDA kernels.

- ga_mode='reference' against the reference's own use_ga=True run (tests/golden/lm_ga.npz):
  damping and flags bit-equal, transforms within 1e-5, image relative L2 <= 1e-4.  As written,
  the reference's branch never keeps its acceleration on these cases (its accumulator is
  overwritten by each partial), so these results equal the plain LM step's.
- ga_mode='intended' (the sum over all six partials) against the FP64 oracle's restatement of
  the same, where the acceleration is kept: damping and flags bit-equal, transforms within the
  parity target of 0.01 voxel / 0.01 degree.  The acceleration's right-hand side is a finite
  difference with step 1e-4 of two nearly equal FP32 vectors (transform_estimation.py:105-106),
  so in FP32 it carries a relative error near 1e-3 in any implementation, the reference's
  included; the tolerance is the parity target, not FP32 rounding."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O32 = Oracle(np.complex64)
O64 = Oracle(np.complex128)


def _run(d, case, ga_mode):
    from motionest.transform_estimation import estimate_transform
    from motionest.utils import compute_transform_grids_voxel
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    t = d[f"c{case}_t0"].copy()
    damp = d[f"c{case}_damp0"].copy()
    flags = np.zeros(len(damp), bool)
    out = estimate_transform(d["ksp"], d["mps"], d["mask"], d[f"c{case}_image"], kg, rk, damp,
                             flags, transforms=t, use_ga=True, ga_mode=ga_mode)
    return t, damp, flags, out


@pytest.mark.parametrize("case", range(3))
def test_geodesic_lm_reference_mode_vs_reference(case):
    d = load_golden("lm")
    g = load_golden("lm_ga")
    t, damp, flags, out = _run(d, case, "reference")
    np.testing.assert_array_equal(damp, g[f"c{case}_damp"])
    np.testing.assert_array_equal(flags, g[f"c{case}_flags"])
    np.testing.assert_allclose(t, g[f"c{case}_t"], atol=1e-5)
    assert rel_l2(out, g[f"c{case}_image_out"]) < 1e-4


@pytest.mark.parametrize("case", range(3))
def test_geodesic_lm_intended_mode_vs_oracle(case):
    d = load_golden("lm")
    t, damp, flags, out = _run(d, case, "intended")
    kg, rk = transform_grids(d["ksp"].shape[1:], [1, 1, 1])
    t_o = d[f"c{case}_t0"].copy()
    damp_o = d[f"c{case}_damp0"].copy()
    flags_o = np.zeros(len(damp_o), bool)
    out_o = O64.estimate_transform(d["ksp"].astype(np.complex128),
                                   d["mps"].astype(np.complex128), d["mask"],
                                   d[f"c{case}_image"].astype(np.complex128), kg, rk, damp_o,
                                   flags_o, t_o, use_ga=True, ga_mode="intended")
    np.testing.assert_array_equal(damp, damp_o)
    np.testing.assert_array_equal(flags, flags_o)
    assert np.abs(t[:, :3] - t_o[:, :3]).max() <= 0.01
    assert np.abs(t[:, 3:] - t_o[:, 3:]).max() <= np.deg2rad(0.01)
    assert rel_l2(out, out_o) < 1e-3
    assert np.abs(t - d[f"c{case}_t"]).max() > 1e-3  # the acceleration was kept
