"""CUDA rigid-transform operators vs the reference's outputs (golden) and the FP64 oracle."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import Oracle, transform_grids

pytestmark = pytest.mark.gpu

O64 = Oracle(np.complex128)


@pytest.fixture(scope="module")
def me():
    import motionest
    return motionest


@pytest.mark.parametrize("case", range(4))
def test_apply_adjoint_vs_reference(me, case):
    d = load_golden("transform")
    x, p = d[f"c{case}_x"], d[f"c{case}_params"]
    kg, rk = me.compute_transform_grids_voxel(x.shape, [1, 1, 1])
    T = me.RigidTransformCudaOptimzied(p, kg, rk)
    assert rel_l2(T.apply(x), d[f"c{case}_apply"]) < 1e-5
    assert rel_l2(T.adjoint(x), d[f"c{case}_adjoint"]) < 1e-5
    Ti = me.RigidTransformCudaOptimzied(p, kg, rk, inverse=True)
    assert rel_l2(Ti.apply(x), d[f"c{case}_apply_inv"]) < 1e-5


@pytest.mark.parametrize("case", range(4))
def test_reference_derivative_vs_reference(me, case):
    d = load_golden("transform")
    x, p = d[f"c{case}_x"], d[f"c{case}_params"]
    kg, rk = me.compute_transform_grids_voxel(x.shape, [1, 1, 1])
    dT = me.RigidTransformDerivativeCuda(x.shape, p, kg, rk)
    for q in range(6):
        ref = d[f"c{case}_deriv"][q]
        got = dT.apply(x, q)
        assert rel_l2(got, ref) < 2e-5, q
    np.testing.assert_array_equal(dT.apply(x, 7), x)
    J = dT.jacobian(x)
    for q in range(6):
        assert rel_l2(J[1 + q], d[f"c{case}_deriv"][q]) < 2e-5, q
    assert rel_l2(J[0], d[f"c{case}_apply"]) < 1e-5


# (64, 64, 32) and (96, 48, 32): in the API's x-y-z layout the rows of lines divide into whole
# tiles, so the passes move their tiles by TMA tensor copies (32-line tiles for 32 and 64
# points, 16-line tiles for 48 and 96); the other shapes take the cp.async kernels
@pytest.mark.parametrize("shape", [(32, 28, 22), (24, 20, 18), (20, 14, 12), (12, 10, 8),
                                   (64, 56, 44), (30, 21, 15), (64, 64, 32), (96, 48, 32)])
def test_apply_adjoint_vs_fp64_oracle(me, shape):
    rng = np.random.default_rng(sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    p = np.array([1.7, -2.3, 0.9, 0.12, -0.09, 0.14])
    kg, rk = transform_grids(shape, [1, 1, 1])
    T = me.RigidTransformCudaOptimzied(p, kg, rk)
    assert rel_l2(T.apply(x), O64.rigid_apply(x, p, kg, rk)) < 2e-6
    assert rel_l2(T.adjoint(x), O64.rigid_adjoint(x, p, kg, rk)) < 2e-6
    # unitarity and adjoint dot test
    y = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    lhs = np.vdot(T.apply(x).astype(np.complex128), y)
    rhs = np.vdot(x.astype(np.complex128), T.adjoint(y))
    assert abs(lhs - rhs) / abs(lhs) < 1e-5
    assert rel_l2(T.adjoint(T.apply(x)), x) < 2e-6


@pytest.mark.parametrize("shape", [(24, 20, 18), (64, 64, 32)])
@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_jacobian_vs_fp64_oracle(me, mode, shape):
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    p = np.array([0.7, 1.3, -0.4, 0.07, 0.11, -0.05])
    kg, rk = transform_grids(shape, [1, 1, 1])
    dT = me.RigidTransformDerivativeCuda(shape, p, kg, rk, jacobian=mode)
    J = dT.jacobian(x)
    for q in range(6):
        ref = O64.rigid_derivative(x, p, q, kg, rk, mode=mode)
        assert rel_l2(J[1 + q], ref) < 1e-5, q
        assert rel_l2(dT.apply(x, q), ref) < 1e-5, q


def test_torch_inputs_stay_on_device(me):
    shape = (16, 12, 10)
    x = torch.randn(shape, dtype=torch.complex64, device="cuda")
    kg, rk = me.compute_transform_grids_voxel(shape, [1, 1, 1])
    y = me.RigidTransformCudaOptimzied(np.zeros(6), kg, rk).apply(x)
    assert isinstance(y, torch.Tensor) and y.is_cuda
    assert rel_l2(y.cpu().numpy(), x.cpu().numpy()) < 1e-6
