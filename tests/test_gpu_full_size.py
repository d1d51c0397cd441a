"""Size-independent properties at the benchmark's full size (256 x 224 x 176, 32 coils, 64
DISORDER shots of 448 samples), where the FP64 oracle would take hours: unitarity and the
adjoint dot test of the rigid transform, a Hermitian positive normal operator, batch
invariance of the normal operator (every shots-per-launch batch sums the shots in the same
order, so they agree bit for bit), the residual energies against the sampled
forward model, and the LM statistics' residual energy against the separately computed one."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

SHAPE = (256, 224, 176)
C, S = 32, 64


def _dot(a, b):
    return torch.vdot(a.reshape(-1).to(torch.complex128), b.reshape(-1).to(torch.complex128))


@pytest.fixture(scope="module")
def full():
    from motionest.problem import SenseProblem
    from motionest.sampling import disorder_masks
    from motionest.utils import compute_transform_grids_voxel
    X, Y, Z = SHAPE
    g = torch.Generator(device="cuda").manual_seed(7)
    mps = 0.2 * torch.randn((C,) + SHAPE, dtype=torch.complex64, device="cuda", generator=g)
    ksp = torch.randn((C,) + SHAPE, dtype=torch.complex64, device="cuda", generator=g)
    planes = np.fft.ifftshift(disorder_masks(X, Y, (16, 16), 2, S)[..., 0], axes=(-2, -1))
    rng = np.random.default_rng(7)
    t = np.zeros((S, 6))
    t[:, :3] = rng.uniform(-3, 3, (S, 3))
    t[:, 3:] = np.deg2rad(rng.uniform(-6, 6, (S, 3)))
    t = torch.as_tensor(t, device="cuda")
    kg, rk = compute_transform_grids_voxel(SHAPE, [1, 1, 1])
    pb = SenseProblem(ksp, mps, planes, kg, rk, t, batch=S, lm_batch=8)
    del ksp, mps
    x = torch.randn((Z, X, Y), dtype=torch.complex64, device="cuda", generator=g)
    y = torch.randn((Z, X, Y), dtype=torch.complex64, device="cuda", generator=g)
    yield pb, x, y, t
    del pb
    torch.cuda.empty_cache()


def test_transform_unitary_and_adjoint_at_full_size(full):
    from motionest import _lib
    from motionest._lib import ptr
    pb, x, y, t = full
    X, Y, Z = SHAPE
    lay = _lib.MeLayout(Y, 1, X * Y)
    st = _lib.stream_ptr()
    for s in (0, 31, 63):
        p = t[s].contiguous()
        tx = torch.empty_like(x)
        thy = torch.empty_like(y)
        back = torch.empty_like(x)
        _lib.call("me_rigid_apply", ptr(x), 0, ptr(tx), 0, 1, lay, pb.grid.ref, ptr(p), 0, 0, st)
        _lib.call("me_rigid_adjoint", ptr(y), 0, ptr(thy), 0, 1, lay, pb.grid.ref, ptr(p), 0, 0,
                  st)
        _lib.call("me_rigid_adjoint", ptr(tx), 0, ptr(back), 0, 1, lay, pb.grid.ref, ptr(p), 0, 0,
                  st)
        rel = float(torch.linalg.vector_norm(back - x) / torch.linalg.vector_norm(x))
        assert rel < 2e-5, (s, rel)  # T^H T = I (the transform is unitary)
        lhs, rhs = _dot(tx, y), _dot(x, thy)
        assert abs(lhs - rhs) <= 1e-5 * abs(lhs), s  # <T x, y> = <x, T^H y>


def test_normal_operator_hermitian_positive_and_batch_invariant(full):
    pb, x, y, _ = full
    ax = pb.normal(x, pb.empty_image())
    ay = pb.normal(y, pb.empty_image())
    lhs, rhs = _dot(ax, y), _dot(x, ay)
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    q = _dot(x, ax)
    assert q.real > 0 and abs(q.imag) <= 1e-5 * q.real
    # every shots-per-launch batch adds the shots into the output in the same order, so the
    # results agree bit for bit
    for b in (1, 7, 24):
        assert torch.equal(pb.normal(x, pb.empty_image(), batch=b), ax), b


def test_residual_energies_at_full_size(full):
    pb, x, _, t = full
    e = pb.residual_norms(x, t)
    k = pb.forward(x, t)
    off = pb.samples.shot_off
    zc = SHAPE[2] * C
    for s in (0, 17, 63):
        a, b = int(off[s]) * zc, int(off[s + 1]) * zc
        r = (k.reshape(-1)[a:b] - pb.ydat.reshape(-1)[a:b]).to(torch.complex128)
        ref = float(torch.vdot(r, r).real)
        np.testing.assert_allclose(float(e[s]), ref, rtol=1e-6)


def test_lm_statistics_energy_matches_residual_at_full_size(full):
    from motionest import _lib
    pb, x, _, t = full
    stats = pb.lm_stats(x, _lib.ME_JAC_REFERENCE)
    e = pb.residual_norms(x, t)
    # The same transform and forward arithmetic and the same FP64 reduction order; the residual
    # kernel forms scale * acc - y with one fused multiply-add, the statistics start from the
    # stored (rounded) scale * acc, so the energies differ at the 1e-10 level only.
    torch.testing.assert_close(stats[:, 0], e, rtol=1e-9, atol=0)
    # Gauss-Newton Hessian diagonals are energies of the Jacobian columns
    diag = stats[:, [7, 13, 18, 22, 25, 27]]
    assert bool((diag > 0).all())
