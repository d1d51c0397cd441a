"""The SENSE kernels alone on caller-transformed volumes (me_sense_forward_volumes,
me_sense_adjoint_volumes; A_func's coil/FFT/mask steps, image_estimation.py:115-128, without the
rigid transform): the forward is bit-identical to me_sense_forward's K, the adjoint is the
forward's adjoint (<C^H F^H M K, u> = <K, M F C u>), the two together with the rigid transforms
reproduce the normal operator, and bad shot ranges and strides are rejected."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import transform_grids

pytestmark = pytest.mark.gpu


def _problem(shape, ncoils, nshots, seed):
    from motionest.problem import SenseProblem
    from motionest.sampling import disorder_masks
    X, Y, Z = shape
    rng = np.random.default_rng(seed)
    mps = (0.5 * (rng.standard_normal((ncoils,) + shape)
                  + 1j * rng.standard_normal((ncoils,) + shape))).astype(np.complex64)
    ksp = (rng.standard_normal((ncoils,) + shape)
           + 1j * rng.standard_normal((ncoils,) + shape)).astype(np.complex64)
    planes = np.fft.ifftshift(disorder_masks(X, Y, (4, 4), 2, nshots)[..., 0], axes=(-2, -1))
    t = np.zeros((nshots, 6))
    t[:, :3] = rng.uniform(-2, 2, (nshots, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-5, 5, (nshots, 3)))
    kg, rk = transform_grids(shape, [1, 1, 1])
    return SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk,
                        torch.as_tensor(t).cuda())


def _cdot(a, b):
    return complex(torch.sum(torch.conj(a.to(torch.complex128)) * b.to(torch.complex128)).item())


@pytest.mark.parametrize("shape", [(32, 32, 16), (32, 28, 20)])
def test_sense_volumes_match_forward_and_normal(shape):
    from motionest import _lib
    from motionest._lib import ptr
    S = 6
    pb = _problem(shape, 4, S, 9)
    X, Y, Z = shape
    V = X * Y * Z
    rng = np.random.default_rng(3)
    x = torch.as_tensor((rng.standard_normal((Z, X, Y)) + 1j * rng.standard_normal((Z, X, Y))
                         ).astype(np.complex64)).cuda()
    st = _lib.stream_ptr()
    lay = _lib.MeLayout(Y, 1, X * Y)
    U = torch.empty((S, Z, X, Y), dtype=torch.complex64, device="cuda")
    _lib.call("me_rigid_apply", ptr(x), 0, ptr(U), V, S, lay, pb.grid.ref, ptr(pb.transforms), 6,
              0, st)
    K = torch.empty_like(pb.ydat)
    _lib.call("me_sense_forward_volumes", pb.ref, ptr(U), V, 0, S, ptr(K), st)
    np.testing.assert_array_equal(K.cpu().numpy(), pb.forward(x, pb.transforms).cpu().numpy())
    # the adjoint of the forward, per shot volume
    W = torch.empty_like(U)
    Kr = torch.as_tensor((rng.standard_normal(K.shape) + 1j * rng.standard_normal(K.shape)
                          ).astype(np.complex64)).cuda()
    _lib.call("me_sense_adjoint_volumes", pb.ref, ptr(Kr), 0, S, ptr(W), V, st)
    lhs = _cdot(W, U)
    rhs = _cdot(Kr, K)
    assert abs(lhs - rhs) <= 1e-5 * abs(rhs)
    # T^H of the adjoint of the forward, summed over shots and masked: the normal operator
    _lib.call("me_sense_adjoint_volumes", pb.ref, ptr(K), 0, S, ptr(W), V, st)
    _lib.call("me_rigid_adjoint", ptr(W), V, ptr(U), V, S, lay, pb.grid.ref, ptr(pb.transforms),
              6, 0, st)
    got = (U.sum(0) * pb.M).cpu().numpy()
    ref = pb.normal(x, pb.empty_image()).cpu().numpy()
    assert rel_l2(got, ref) < 1e-6
    # a sub-range of shots starts at that shot's first sample
    K2 = torch.empty_like(pb.ydat)
    _lib.call("me_sense_forward_volumes", pb.ref, ptr(U[2]), V, 2, 3, ptr(K2), st)
    _lib.call("me_sense_forward_volumes", pb.ref, ptr(U), V, 0, S, ptr(K), st)
    off = pb.shot_off.cpu().numpy()
    n = (off[5] - off[2]) * 4 * Z
    a = (off[2] - off[0]) * 4 * Z
    np.testing.assert_array_equal(K2[:n].cpu().numpy(), K[a:a + n].cpu().numpy())


def test_sense_volumes_reject_bad_ranges():
    """Shot ranges outside the problem and strides below one volume are refused on the host,
    before any launch."""
    from motionest import _lib
    from motionest._lib import ptr
    pb = _problem((32, 32, 16), 2, 4, 1)
    lib = _lib.load()
    V = 32 * 32 * 16
    U = torch.zeros((4, 16, 32, 32), dtype=torch.complex64, device="cuda")
    K = torch.empty_like(pb.ydat)
    st = _lib.stream_ptr()
    assert lib.me_sense_forward_volumes(pb.ref, ptr(U), V, 2, 3, ptr(K), st) != 0
    assert lib.me_sense_forward_volumes(pb.ref, ptr(U), V - 1, 0, 4, ptr(K), st) != 0
    assert lib.me_sense_adjoint_volumes(pb.ref, ptr(K), 0, 4, ptr(U), 0, st) != 0
    assert lib.me_sense_adjoint_volumes(pb.ref, ptr(K), -1, 1, ptr(U), V, st) != 0
    assert lib.me_sense_adjoint_volumes(pb.ref, ptr(K), 0, 0, ptr(U), V, st) != 0
