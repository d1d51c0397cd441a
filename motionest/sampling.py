"""DISORDER sampling and per-shot sample lists (host side, integer work).

make_disorder_order restates simulation.py:192-245 of the reference (tile shuffle by Python's
random.Random(seed), interleave out_pos = j*num_groups + linG*num_par_groups + parG);
disorder_masks restates the shot binning of simulation.py:396-410.  Both must stay in Python:
the order depends on random.Random's shuffle, which the tests pin bit for bit against the
reference's own output.
"""
import random
from dataclasses import dataclass
from math import ceil

import numpy as np


@dataclass
class DisorderConfig:
    max_line_number: int
    max_partition_number: int
    pat_lines_to_measure: int
    block_lin: int
    block_par: int
    seed: int = 123456


def make_disorder_order(cfg):
    """(line, partition) reorder list of length indices_per_group*num_groups, and (L, P)."""
    L = ceil((cfg.max_line_number + 1) / cfg.block_lin) * cfg.block_lin
    P = ceil((cfg.max_partition_number + 1) / cfg.block_par) * cfg.block_par
    max_line = L - 1
    n_reorder = cfg.pat_lines_to_measure * P
    per_tile = cfg.block_lin * cfg.block_par
    n_lin_groups = L // cfg.block_lin
    n_par_groups = P // cfg.block_par
    n_groups = n_lin_groups * n_par_groups
    per_group = n_reorder // n_groups
    rng = random.Random(cfg.seed)
    base = list(range(per_tile))
    out = [None] * (per_group * n_groups)
    for lin_g in range(n_lin_groups):
        for par_g in range(n_par_groups):
            idx = base[:]
            rng.shuffle(idx)
            line_base = (lin_g % cfg.block_par) * (max_line + 1) // cfg.block_par \
                + (lin_g // cfg.block_par) * cfg.block_lin
            for j in range(per_group):
                local = idx[j]
                line = local % cfg.block_lin + line_base
                part = local // cfg.block_lin + par_g * cfg.block_par
                out[j * n_groups + lin_g * n_par_groups + par_g] = (line, part)
    return out, (L, P)


def disorder_order(nx, ny, tile, accel, seed=123456):
    """DISORDER order for an [nx partitions, ny lines] plane with tile = (partitions, lines),
    configured as simulation.py:385-392 does."""
    cfg = DisorderConfig(max_line_number=ny - 1, max_partition_number=nx - 1,
                         pat_lines_to_measure=ny // accel, block_lin=tile[1], block_par=tile[0],
                         seed=seed)
    order, _ = make_disorder_order(cfg)
    return np.array(order, dtype=np.int64)


def bin_order(order, nshots, nx, ny):
    """Masks [nshots, nx, ny] bool: consecutive chunks of the order (simulation.py:397-402)."""
    A = np.zeros((nshots, nx, ny), dtype=bool)
    sps = order.shape[0] // nshots
    for s in range(nshots):
        chunk = order[s * sps:(s + 1) * sps]
        A[s, chunk[:, 1], chunk[:, 0]] = True
    return A


def disorder_masks(nx, ny, tile, accel, nshots, seed=123456):
    """Centred DISORDER shot masks [nshots, nx, ny, 1] bool."""
    return bin_order(disorder_order(nx, ny, tile, accel, seed), nshots, nx, ny)[..., None]


def sequential_masks(nx, ny, accel, nshots):
    """Line-by-line masks as simulation.py:412-424 builds them."""
    y = np.repeat(np.arange(0, nx, accel), ny)
    x = np.tile(np.arange(ny), nx // accel)
    A = np.zeros((nshots, nx, ny), dtype=bool)
    sps = y.shape[0] // nshots
    for s in range(nshots):
        A[s, y[s * sps:(s + 1) * sps], x[s * sps:(s + 1) * sps]] = True
    return A[..., None]


def plane_masks(mask):
    """[S, X, Y] bool plane masks from a [S, X, Y, Z|1] mask that is constant along z."""
    m = np.asarray(mask)
    if m.ndim == 3:
        return m.astype(bool)
    if m.ndim != 4:
        raise ValueError(f"shot masks must be [nshots, X, Y, 1] (or [nshots, X, Y, Z]); got {m.shape}")
    m = m.astype(bool)
    if m.shape[3] > 1 and not (m == m[..., :1]).all():
        raise ValueError("shot masks must be constant along the readout (z) axis, as the "
                         "reference's DISORDER and sequential masks are")
    return m[..., 0]


class SampleLists:
    """Per-shot sampled (kx, ky) points of uncentred plane masks, grouped by ky (CSR), as the
    me_samples struct of the C ABI describes them."""

    def __init__(self, planes):
        planes = np.asarray(planes, dtype=bool)
        S, X, Y = planes.shape
        kx_all, ky_all, off, kyoff = [], [], [0], []
        for s in range(S):
            kx, ky = np.nonzero(planes[s])
            order = np.lexsort((kx, ky))
            kx, ky = kx[order], ky[order]
            kx_all.append(kx)
            ky_all.append(ky)
            off.append(off[-1] + kx.size)
            kyoff.append(np.searchsorted(ky, np.arange(Y + 1), side="left"))
        self.nshots, self.nx, self.ny = S, X, Y
        self.shot_off = np.asarray(off, dtype=np.int32)
        self.kx = np.concatenate(kx_all).astype(np.int32) if S else np.zeros(0, np.int32)
        self.ky = np.concatenate(ky_all).astype(np.int32) if S else np.zeros(0, np.int32)
        self.ky_off = np.stack(kyoff).astype(np.int32).reshape(-1)
        counts = np.diff(self.shot_off)
        self.max_per_shot = int(counts.max()) if S else 0
        self.total = int(self.shot_off[-1])
        # bins of each shot by decreasing sample count (stable), for load-balanced adjoints,
        # spread over bank residues within each run of equal counts
        bins = np.diff(self.ky_off.reshape(S, Y + 1), axis=1)
        # With 128 < Y < 256 the adjoint's 256 threads hold one bin each and the 256 - Y spare
        # threads take the second halves of the first 256 - Y bins of this order, which are
        # then built as two halves of 8 rows.
        split = 256 - Y if 128 < Y < 256 else 0
        order = np.argsort(-bins, axis=1, kind="stable")
        self.ky_order = np.stack([spread_residues(o, b[o], split=split)
                                  for o, b in zip(order, bins)]
                                 ).astype(np.int32).reshape(-1) if S else order.reshape(-1)


def spread_residues(order, counts, width=16, split=0):
    """Reorder bins that have the same sample count so that each window of `width`
    consecutive positions holds bins of distinct residues mod `width` where it can.

    The adjoint kernel gives the bin at position i of this order to thread i, and the 16 lanes
    of a half warp store their bins' H values (8-byte elements, one row at a time) in one
    shared-memory request: bins of equal residue mod 16 fall in the same banks.  Only bins of
    equal count trade places, and none across position `split` (the bins before it are built
    as two half-row walks, the others as one), so every position keeps its sample count (each
    warp's walk lengths, and so the balance between warps, are unchanged) and every bin is
    built exactly as in the plain order: the H values are bit-identical."""
    order = np.asarray(order)
    counts = np.asarray(counts)
    out = order.copy()
    start = 0
    n = order.size
    while start < n:
        stop = start
        while stop < n and counts[stop] == counts[start] and (stop != split or stop == start):
            stop += 1
        pool = list(order[start:stop])
        for i in range(start, stop):
            w0 = i - i % width
            used = {int(out[k]) % width for k in range(w0, i)}
            pick = next((j for j, b in enumerate(pool) if int(b) % width not in used), 0)
            out[i] = pool.pop(pick)
        start = stop
    return out
