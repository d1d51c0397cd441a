"""DISORDER ordering, shot masks and per-shot sample lists (host integer work, CPU).

The order and masks must be bit-identical to the reference's make_disorder_order and shot
binning (simulation.py:201-245, 397-402); the fixtures were produced by the reference itself."""
import hashlib

import numpy as np
import pytest

from conftest import load_golden
from motionest.sampling import (DisorderConfig, SampleLists, bin_order, disorder_masks,
                                disorder_order, make_disorder_order, plane_masks,
                                sequential_masks)


def _cases():
    d = load_golden("disorder")
    return [(i, d) for i in range(int(d["ncases"]))]


@pytest.mark.parametrize("i", range(8))
def test_disorder_order_and_masks_bit_exact(i):
    d = load_golden("disorder")
    X, Y, tp, tl, accel, nshots = (int(v) for v in d[f"c{i}_case"])
    order = disorder_order(X, Y, (tp, tl), accel)
    np.testing.assert_array_equal(order, d[f"c{i}_order"].astype(np.int64))
    cfg = DisorderConfig(Y - 1, X - 1, Y // accel, tl, tp)
    _, LP = make_disorder_order(cfg)
    assert tuple(LP) == tuple(int(v) for v in d[f"c{i}_LP"])
    A = bin_order(order, nshots, X, Y)
    assert hashlib.sha256(np.ascontiguousarray(A).tobytes()).digest() == \
        bytes(d[f"c{i}_mask_sha256"])
    if f"c{i}_mask_packed" in d:
        np.testing.assert_array_equal(np.packbits(A.ravel()), d[f"c{i}_mask_packed"])
    assert disorder_masks(X, Y, (tp, tl), accel, nshots).shape == (nshots, X, Y, 1)


def test_known_overlap_counts():
    """The 256x224 16x16 R2 order revisits 1,699 (partition, line) points and never samples
    lines 198-223, as the reference's line formula does (documented, reproduced)."""
    order = disorder_order(256, 224, (16, 16), 2)
    pts = order[:, 1] * 224 + order[:, 0]
    assert order.shape[0] - np.unique(pts).size == 1699
    assert order[:, 0].max() == 197


def test_sequential_masks_partition():
    A = sequential_masks(8, 6, 2, 4)[..., 0]
    assert A.shape == (4, 8, 6)
    assert A.sum() == 4 * 6 and (A.sum(axis=0) <= 1).all()


def test_sample_lists_csr():
    rng = np.random.default_rng(0)
    planes = rng.random((5, 12, 10)) < 0.2
    planes[2] = False  # an empty shot
    sl = SampleLists(planes)
    assert sl.shot_off[-1] == planes.sum()
    assert sl.max_per_shot == planes.sum(axis=(1, 2)).max()
    for s in range(5):
        a, b = sl.shot_off[s], sl.shot_off[s + 1]
        kx, ky = sl.kx[a:b], sl.ky[a:b]
        got = np.zeros((12, 10), bool)
        got[kx, ky] = True
        np.testing.assert_array_equal(got, planes[s])
        assert (np.diff(ky) >= 0).all()
        off = sl.ky_off[s * 11:(s + 1) * 11]
        for v in range(10):
            assert (ky[off[v]:off[v + 1]] == v).all()


def test_masks_must_be_constant_along_z():
    m = np.zeros((2, 4, 4, 3), bool)
    m[0, 1, 1, :] = True
    assert plane_masks(m).shape == (2, 4, 4)
    m[1, 2, 2, 1] = True
    with pytest.raises(ValueError):
        plane_masks(m)


def test_continuous_motion_segments():
    """Intra-shot motion: nshots * segments poses, each shot's segments on a straight line
    through its pose with a drift of at most 2 degrees / 2 voxels, zero mean overall; the
    corruption masks bin the same DISORDER order into nshots * segments states, each the
    union of 4 consecutive states being one reconstruction shot's mask."""
    from motionest.sampling import disorder_masks
    from motionest.simulation import motion_continuous
    S, K = 16, 4
    t = motion_continuous(S, K, seed=3)
    assert t.shape == (S * K, 6)
    np.testing.assert_allclose(t.mean(axis=0), 0.0, atol=1e-12)
    seg = t.reshape(S, K, 6)
    d = seg[:, 1:] - seg[:, :-1]
    np.testing.assert_allclose(d, d[:, :1].repeat(K - 1, axis=1), atol=1e-12)  # linear
    total = seg[:, -1] - seg[:, 0]
    assert np.abs(total[:, :3]).max() <= 2.0 and np.abs(np.rad2deg(total[:, 3:])).max() <= 2.0
    rec = disorder_masks(64, 64, (4, 4), 1, S)
    cor = disorder_masks(64, 64, (4, 4), 1, S * K)
    np.testing.assert_array_equal(cor.reshape(S, K, 64, 64, 1).any(axis=1), rec)


def test_adjoint_bin_order_keeps_counts_and_spreads_residues():
    """Each shot's ky_order is a permutation of its bins by non-increasing sample count (the
    adjoint's load balance), with equal-count bins spread over residues mod 16 (the bank of a
    half warp's H-row store): fewer collisions over all windows than the plain stable sort."""
    from motionest.sampling import SampleLists, disorder_masks
    for X, Y, tile, accel, S in ((256, 224, (16, 16), 2, 64), (64, 48, (4, 4), 1, 16),
                                 (30, 21, (3, 3), 1, 5)):
        planes = np.fft.ifftshift(disorder_masks(X, Y, tile, accel, S)[..., 0], axes=(-2, -1))
        sl = SampleLists(planes)
        bins = np.diff(sl.ky_off.reshape(S, Y + 1), axis=1)
        order = sl.ky_order.reshape(S, Y)
        plain = np.argsort(-bins, axis=1, kind="stable")
        split = 256 - Y if 128 < Y < 256 else 0
        new = old = 0
        for s in range(S):
            assert sorted(order[s].tolist()) == list(range(Y))
            np.testing.assert_array_equal(bins[s][order[s]], bins[s][plain[s]])
            # the bins built as two half walks are the same ones
            assert set(order[s][:split].tolist()) == set(plain[s][:split].tolist())
            for w in range(0, Y, 16):
                new += np.bincount(order[s][w:w + 16] % 16, minlength=16).max()
                old += np.bincount(plain[s][w:w + 16] % 16, minlength=16).max()
        assert new <= old, (X, Y, new, old)
