"""Pin the CPU oracle against fixtures produced by the reference itself (tests/golden)."""
import numpy as np
import pytest

from conftest import grids_from_golden, load_golden, rel_l2
from oracle import Oracle, transform_grids

O32 = Oracle(np.complex64)
O64 = Oracle(np.complex128)


def test_grids_match_reference():
    d = load_golden("grids")
    for i in range(int(d["ncases"])):
        shape = tuple(int(v) for v in d[f"c{i}_shape"])
        ds = tuple(int(v) for v in d[f"c{i}_ds"])
        kg, rk = transform_grids(shape, list(d[f"c{i}_vox"]), ds)
        ref_kg, ref_rk = grids_from_golden(d, i)
        for a in "xyz":
            np.testing.assert_array_equal(kg[a], ref_kg[a])
            np.testing.assert_array_equal(rk["tan"][a], ref_rk["tan"][a])
            np.testing.assert_array_equal(rk["sin"][a], ref_rk["sin"][a])


@pytest.mark.parametrize("case", range(4))
def test_transform_apply_adjoint_derivative(case):
    d = load_golden("transform")
    x = d[f"c{case}_x"]
    p = d[f"c{case}_params"]
    kg, rk = transform_grids(x.shape, [1, 1, 1])
    assert rel_l2(O32.rigid_apply(x, p, kg, rk), d[f"c{case}_apply"]) < 2e-6
    assert rel_l2(O32.rigid_apply(x, p, kg, rk, inverse=True), d[f"c{case}_apply_inv"]) < 2e-6
    assert rel_l2(O32.rigid_adjoint(x, p, kg, rk), d[f"c{case}_adjoint"]) < 2e-6
    for q in range(6):
        ref = d[f"c{case}_deriv"][q]
        got = O32.rigid_derivative(x, p, q, kg, rk, mode="reference")
        assert rel_l2(got, ref) < 5e-6, q
    # the FP64 oracle agrees with the reference to FP32 accuracy
    assert rel_l2(O64.rigid_apply(x, p, kg, rk), d[f"c{case}_apply"]) < 5e-6


def test_forward_model():
    d = load_golden("forward")
    ksp = O32.corrupted_kspace(d["gt"], d["mps"], d["mask"], d["transforms"])
    assert rel_l2(ksp, d["ksp"]) < 2e-6


@pytest.mark.parametrize("case", range(3))
def test_cg(case):
    d = load_golden("cg")
    g = lambda k: d[f"c{case}_{k}"]  # noqa: E731
    kg, rk = transform_grids(g("x").shape, [1, 1, 1])
    x = O32.estimate_image_cg(g("ksp"), g("mps"), g("mask"), g("transforms"), kg, rk, g("P"),
                              g("M"), x0=g("x0"), max_iter=int(g("max_iter")))
    assert rel_l2(x, g("x")) < 1e-5


@pytest.mark.parametrize("case", range(3))
def test_lm(case):
    d = load_golden("lm")
    g = lambda k: d[f"c{case}_{k}"]  # noqa: E731
    kg, rk = transform_grids(d["ksp"].shape[1:], [1, 1, 1])
    t = g("t0").copy()
    damp = g("damp0").copy()
    flags = np.zeros(len(damp), bool)
    out = O32.estimate_transform(d["ksp"], d["mps"], d["mask"], g("image"), kg, rk, damp, flags, t)
    np.testing.assert_array_equal(damp, g("damp"))
    np.testing.assert_array_equal(flags, g("flags"))
    np.testing.assert_allclose(t, g("t"), atol=1e-6)
    assert rel_l2(out, g("image_out")) < 1e-5


def test_joint_recon():
    d = load_golden("joint")
    kg, rk = transform_grids(d["ksp"].shape[1:], [1, 1, 1])
    x, t, oh, th = O32.joint_recon(d["ksp"], d["mps"], d["mask"], kg, rk,
                                   max_cg_iter=int(d["max_cg_iter"]),
                                   max_nm_iter=int(d["max_nm_iter"]),
                                   max_joint_iter=int(d["max_joint_iter"]))
    assert rel_l2(x, d["x"]) < 1e-4
    np.testing.assert_allclose(t, d["t"], atol=1e-5)
    np.testing.assert_allclose(oh, d["objective_history"], rtol=1e-4)


def test_pyramid():
    d = load_golden("pyramid")
    x, t = O32.pyramid_reconstruction(d["ksp"], d["mps"], d["mask"], d["mask"].shape[0],
                                      n_joint_iters=int(d["n_joint_iters"]))
    assert rel_l2(x, d["x"]) < 1e-4
    np.testing.assert_allclose(t, d["t"], atol=1e-5)


def test_reference_jacobian_is_reversed_order():
    """The reference derivative differentiates Tr.Rx.Ry.Rz, not the applied Tr.Rz.Ry.Rx."""
    d = load_golden("transform")
    x = d["c0_x"].astype(np.complex128)
    p = d["c0_params"]
    kg, rk = transform_grids(x.shape, [1, 1, 1])
    h = 1e-5
    for q in (3, 4, 5):
        e = np.zeros(6)
        e[q] = h
        fd = (O64.rigid_apply(x, p + e, kg, rk) - O64.rigid_apply(x, p - e, kg, rk)) / (2 * h)
        exact = O64.rigid_derivative(x, p, q, kg, rk, mode="exact")
        assert rel_l2(exact, fd) < 1e-6
        refmode = O64.rigid_derivative(x, p, q, kg, rk, mode="reference")
        assert rel_l2(refmode, fd) > 1e-2


def test_product_grids_are_bit_equal_to_reference():
    """motionest.utils.compute_transform_grids_voxel (the product's grid builder, not the
    oracle's) against every reference case, odd sizes and downsampled grids included."""
    from motionest.utils import compute_transform_grids_voxel
    d = load_golden("grids")
    for i in range(int(d["ncases"])):
        shape = tuple(int(v) for v in d[f"c{i}_shape"])
        ds = tuple(int(v) for v in d[f"c{i}_ds"])
        kg, rk = compute_transform_grids_voxel(shape, list(d[f"c{i}_vox"]), ds)
        ref_kg, ref_rk = grids_from_golden(d, i)
        for a in "xyz":
            assert kg[a].dtype == np.float64 and kg[a].shape == ref_kg[a].shape
            np.testing.assert_array_equal(kg[a], ref_kg[a])
            for m in ("tan", "sin"):
                assert rk[m][a].shape == ref_rk[m][a].shape
                np.testing.assert_array_equal(rk[m][a], ref_rk[m][a])


@pytest.mark.parametrize("case", range(3))
def test_geodesic_lm_matches_reference(case):
    """use_ga=True (transform_estimation.py:75-121) as written: the oracle's 'reference' mode
    reproduces the reference's results, which equal the plain LM step's (its overwritten
    accumulator makes the acceleration fail the |a| <= |v| gate), while the 'intended' mode
    keeps the acceleration and moves the transforms."""
    d = load_golden("lm")
    g = load_golden("lm_ga")
    kg, rk = transform_grids(d["ksp"].shape[1:], [1, 1, 1])
    t = d[f"c{case}_t0"].copy()
    damp = d[f"c{case}_damp0"].copy()
    flags = np.zeros(4, dtype=bool)
    out = O32.estimate_transform(d["ksp"], d["mps"], d["mask"], d[f"c{case}_image"], kg, rk,
                                 damp, flags, t, use_ga=True, ga_mode="reference")
    np.testing.assert_allclose(t, g[f"c{case}_t"], atol=1e-6)
    np.testing.assert_array_equal(damp, g[f"c{case}_damp"])
    np.testing.assert_array_equal(flags, g[f"c{case}_flags"])
    assert rel_l2(out, g[f"c{case}_image_out"]) < 1e-5
    np.testing.assert_array_equal(g[f"c{case}_t"], d[f"c{case}_t"])  # = the plain LM step
    t2 = d[f"c{case}_t0"].copy()
    O32.estimate_transform(d["ksp"], d["mps"], d["mask"], d[f"c{case}_image"], kg, rk,
                           d[f"c{case}_damp0"].copy(), np.zeros(4, dtype=bool), t2, use_ga=True,
                           ga_mode="intended")
    assert np.abs(t2 - g[f"c{case}_t"]).max() > 1e-3
