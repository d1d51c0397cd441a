"""Coil preprocessing on the GPU against the reference's own outputs (tests/golden/preprocess.npz,
written by running coil_compression.py and espirit.py unmodified):
- coil_compression: the same number of virtual coils, and the compressed maps and k-space
  compared through quantities that do not depend on the basis of the kept subspace -- each
  voxel's energy sum_i |cc_i|^2 and the spectrum of the virtual coils' Gram matrix -- to
  relative 1e-4: coils on a ring give pairs of nearly equal singular values, whose singular
  vectors any SVD may rotate within their pair;
- rx_espirit_3d: the same support mask on >= 99.5% of voxels (voxels whose largest eigenvalue
  sits at the threshold may fall either way in FP32) and, where both are non-zero, the maps to
  relative L2 <= 1e-3 (the calibration SVD and the eigensolver are different libraries' FP32
  routines; the maps are fixed up to phase by the rotation to coil 0's phase)."""
import numpy as np
import pytest

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


def test_coil_compression_vs_reference():
    from motionest.preprocess import coil_compression
    d = load_golden("preprocess")
    cm, ck = coil_compression(d["mps"], d["ksp"], perc=0.95)
    assert cm.shape == d["cc_mps"].shape
    for got, ref in ((cm.cpu().numpy(), d["cc_mps"]), (ck.cpu().numpy(), d["cc_ksp"])):
        g = got.reshape(got.shape[0], -1).astype(np.complex128)
        r = ref.reshape(ref.shape[0], -1).astype(np.complex128)
        assert rel_l2(np.sum(np.abs(g) ** 2, axis=0), np.sum(np.abs(r) ** 2, axis=0)) <= 1e-4
        sg = np.linalg.eigvalsh(g @ g.conj().T)
        sr = np.linalg.eigvalsh(r @ r.conj().T)
        np.testing.assert_allclose(sg, sr, rtol=1e-4)


def test_espirit_vs_reference():
    from motionest.preprocess import rx_espirit_3d
    d = load_golden("preprocess")
    ref = d["sens"]
    got = rx_espirit_3d(d["calib"], ref.shape[:3], kernel_size=(3, 3, 3), eig_thresh=0.02,
                        mask_thresh=0.99).cpu().numpy()
    m_ref = np.abs(ref).sum(-1) > 0
    m_got = np.abs(got).sum(-1) > 0
    assert (m_ref == m_got).mean() >= 0.995
    both = m_ref & m_got
    assert both.sum() > 0
    assert rel_l2(got[both], ref[both]) <= 1e-3
