"""Bounded barrier waits: a wait that nothing completes gives up, records its fault bit, and
the context stays usable; the bulk-copy (TMA engine) staging of the SENSE kernels gives the
same results as the cp.async staging and records no fault."""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]

pytestmark = pytest.mark.gpu


def test_selftest_wait_runs_out_and_context_survives():
    from motionest import _lib
    lib = _lib.load()
    torch.cuda.init()
    assert _lib.wait_status() == 0
    _lib.check(lib.me_wait_selftest(1 << 20, _lib.stream_ptr()))
    assert _lib.wait_status() == _lib.ME_WAIT_SELFTEST
    assert _lib.wait_status() == 0  # read-and-clear
    # the device still computes: an FFT along y against torch's
    x = torch.randn(4, 6, 8, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    lay = _lib.layout_of(x)
    _lib.call("me_fft_axis", _lib.ptr(x), 0, _lib.ptr(y), 0, 1, 4, 6, 8, lay, 1, 0,
              _lib.stream_ptr())
    ref = torch.fft.fft(x, dim=1, norm="ortho")
    torch.testing.assert_close(y, ref, rtol=1e-5, atol=1e-5)


def test_selftest_rejects_bad_limit():
    from motionest import _lib
    with pytest.raises(ValueError):
        _lib.check(_lib.load().me_wait_selftest(0, _lib.stream_ptr()))


_CHILD = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from motionest import _lib
from motionest.problem import SenseProblem, xyz_to_zxy
from motionest.sampling import disorder_masks
from motionest.utils import compute_transform_grids_voxel
shape, C, S = (256, 224, 3), 3, 16
rng = np.random.default_rng(7)
def rnd(sh):
    return (rng.standard_normal(sh) + 1j * rng.standard_normal(sh)).astype(np.complex64)
planes = np.fft.ifftshift(disorder_masks(256, 224, (16, 16), 2, S)[..., 0], axes=(-2, -1))
mps, ksp = 0.5 * rnd((C,) + shape), rnd((C,) + shape)
t = np.zeros((S, 6))
t[:, :3] = rng.uniform(-3, 3, (S, 3))
t[:, 3:] = np.deg2rad(rng.uniform(-6, 6, (S, 3)))
kg, rk = compute_transform_grids_voxel(shape, [1, 1, 1])
td = torch.as_tensor(t).cuda()
pb = SenseProblem(torch.as_tensor(ksp).cuda(), torch.as_tensor(mps).cuda(), planes, kg, rk, td)
xd = xyz_to_zxy(torch.as_tensor(rnd(shape)).cuda())
res = [pb.normal(xd, pb.empty_image()), pb.rhs(pb.empty_image())]
res = [r.cpu().numpy().ravel() for r in res]
res.append(pb.residual_norms(xd, td).cpu().numpy().astype(np.complex128))
res.append(pb.lm_stats(xd, 0).cpu().numpy().ravel().astype(np.complex128))
assert _lib.wait_status() == 0
np.save(sys.argv[2], np.concatenate([r.astype(np.complex128) for r in res]))
"""


def _run_child(tmp_path, env_extra, name):
    out = tmp_path / f"{name}.npy"
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT), str(out)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return np.load(out)


def test_bulk_staging_matches_cp_async(tmp_path):
    """The normal operator, right-hand side, residual energies and LM statistics with the SENSE
    kernels' rows staged by bulk copies are bit-identical to the same kernels staging by
    cp.async (ME_NO_BULK=1), on 256 x 224 planes with 448 samples per shot."""
    a = _run_child(tmp_path, {"ME_NO_BULK": "0"}, "bulk")
    b = _run_child(tmp_path, {"ME_NO_BULK": "1"}, "cpasync")
    assert np.array_equal(a, b)
