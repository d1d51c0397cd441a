"""Equivalent kernel variants give bit-identical results: staging by the TMA engine (bulk copies
in the SENSE kernels, tiled tensor loads and stores in the line passes) against cp.async
staging, and the fused seven-volume LM statistics kernel against the forward kernel writing
seven K regions followed by the statistics kernel.  Each variant runs in its own process
(the switches are read once per process), and no bounded wait may run out."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.gpu

_CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from motionest import _lib
from motionest.problem import SenseProblem, xyz_to_zxy
from motionest.sampling import disorder_masks
from motionest.utils import compute_transform_grids_voxel
shape, C, S = tuple(int(v) for v in sys.argv[3].split("x")), 3, 64
rng = np.random.default_rng(7)
def rnd(sh):
    return (rng.standard_normal(sh) + 1j * rng.standard_normal(sh)).astype(np.complex64)
planes = np.fft.ifftshift(disorder_masks(shape[0], shape[1], (16, 16), 2, S)[..., 0],
                         axes=(-2, -1))
mps, ksp = 0.5 * rnd((C,) + shape), rnd((C,) + shape)
t = np.zeros((S, 6))
t[:, :3] = rng.uniform(-3, 3, (S, 3))
t[:, 3:] = np.deg2rad(rng.uniform(-6, 6, (S, 3)))
kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
td = torch.as_tensor(t).cuda()
pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk, td)
xd = xyz_to_zxy(torch.as_tensor(rnd(shape)).cuda())
res = [pb.normal(xd, pb.empty_image()), pb.rhs(pb.empty_image()),
       pb.apply_transform(xd, td[3], out=pb.empty_image())]
res = [r.cpu().numpy().ravel() for r in res]
res.append(pb.residual_norms(xd, td).cpu().numpy().astype(np.complex128))
res.append(pb.lm_stats(xd, 0).cpu().numpy().ravel().astype(np.complex128))
assert _lib.wait_status() == 0
np.save(sys.argv[2], np.concatenate([r.astype(np.complex128) for r in res]))
"""


def _run_child(tmp_path, env_extra, name, shape):
    out = tmp_path / f"{name}.npy"
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT), str(out), shape], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


@pytest.mark.parametrize("shape", ["256x224x3", "96x224x48", "64x64x32"])
def test_staging_and_fused_lm_variants(tmp_path, shape):
    """The normal operator, right-hand side, one rigid transform, the residual energies and the
    LM statistics (whose Jacobian uses the two-input and two-output passes) are bit-identical
    whether the SENSE kernels stage rows by bulk copies and the line passes move tiles by
    tensor loads and stores, or both use cp.async (ME_NO_BULK=1, ME_NO_TMA=1).  256x224 planes
    carry 448 samples per shot; at 96x224x48 every axis (96, 224, 48) has 16-line tiles, so
    passes along all three run on the tensor-map kernel: strided lines along x and z, contiguous
    lines along y.  At 64x64x32 the lines (64, 64, 32 points) take 8 threads each, so the
    tensor-map kernel moves tiles of 32 lines (two 16-line sub-tiles when strided).  The LM statistics also run once as the forward kernel writing seven K
    regions followed by the statistics kernel (ME_LM_TWO_PASS=1) instead of the fused kernel
    (448, 168 and 32 samples per shot, at most two per thread)."""
    a = _run_child(tmp_path, {}, "default", shape)
    b = _run_child(tmp_path, {"ME_NO_BULK": "1", "ME_NO_TMA": "1"}, "cpasync", shape)
    c = _run_child(tmp_path, {"ME_LM_TWO_PASS": "1"}, "twopass", shape)
    for other, name in ((b, "cp.async staging"), (c, "two-kernel LM statistics")):
        bad = np.flatnonzero(a != other)
        assert bad.size == 0, (f"{name}: {bad.size} of {a.size} values differ, first at {bad[:5]}"
                               f" (of {a.size}), max |diff| {np.abs(a - other).max():.3e}")


def test_misaligned_volumes_take_the_cp_async_kernel():
    """A volume whose base is 8-byte but not 16-byte aligned cannot be described by a tensor
    map: the pass falls back to the cp.async kernel (in the same process) and gives the same
    result as the aligned copy on TMA tiles."""
    import torch
    from motionest import _lib
    from motionest.utils import DeviceGrid, compute_transform_grids_voxel
    shape = (64, 96, 48)
    X, Y, Z = shape
    n = X * Y * Z
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
    grid = DeviceGrid(kg, rk, shape)
    params = torch.tensor([1.3, -0.7, 2.1, 0.05, -0.08, 0.11], dtype=torch.float64, device="cuda")
    outs = []
    for off in (0, 1):  # element offset 1: 8 bytes past a 256-byte aligned allocation
        buf = torch.zeros(n + 2, dtype=torch.complex64, device="cuda")
        x = buf[off:off + n]
        x.copy_(torch.as_tensor(v, device="cuda"))
        ob = torch.zeros(n + 2, dtype=torch.complex64, device="cuda")
        out = ob[off:off + n]
        _lib.call("me_rigid_apply", _lib.ptr(x), 0, _lib.ptr(out), 0, 1,
                  _lib.MeLayout(Y, 1, X * Y), grid.ref, _lib.ptr(params), 0, 0,
                  _lib.stream_ptr())
        outs.append(out.cpu().numpy())
    assert _lib.wait_status() == 0
    assert np.array_equal(outs[0], outs[1])
